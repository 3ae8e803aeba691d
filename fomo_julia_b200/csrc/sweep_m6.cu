// sweep_m6.cu -- the swept time step for M = 6 (see sweep_m.cuh).
#define FOMO_SWEEP_M 6
#include "sweep_m.cuh"
