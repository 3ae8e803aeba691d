// march_m2.cu -- the fused step for M = 2 (see march_m.cuh).
#define FOMO_MARCH_M 2
#include "march_m.cuh"
