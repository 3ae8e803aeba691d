// march_m1.cu -- the fused step for M = 1 (see march_m.cuh).
#define FOMO_MARCH_M 1
#include "march_m.cuh"
