// sweep_m5.cu -- the swept time step for M = 5 (see sweep_m.cuh).
#define FOMO_SWEEP_M 5
#include "sweep_m.cuh"
