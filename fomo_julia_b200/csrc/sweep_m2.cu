// sweep_m2.cu -- the swept time step for M = 2 (see sweep_m.cuh).
#define FOMO_SWEEP_M 2
#include "sweep_m.cuh"
