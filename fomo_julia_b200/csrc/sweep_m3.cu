// sweep_m3.cu -- the swept time step for M = 3 (see sweep_m.cuh).
#define FOMO_SWEEP_M 3
#include "sweep_m.cuh"
