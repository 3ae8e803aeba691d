// march_m4.cu -- the fused step for M = 4 (see march_m.cuh).
#define FOMO_MARCH_M 4
#include "march_m.cuh"
