// march_m3.cu -- the fused step for M = 3 (see march_m.cuh).
#define FOMO_MARCH_M 3
#include "march_m.cuh"
