// sweep_m1.cu -- the swept time step for M = 1 (see sweep_m.cuh).
#define FOMO_SWEEP_M 1
#include "sweep_m.cuh"
