// sweep_m4.cu -- the swept time step for M = 4 (see sweep_m.cuh).
#define FOMO_SWEEP_M 4
#include "sweep_m.cuh"
