// sweep_m.cuh -- body of the translation units sweep_m1.cu .. sweep_m6.cu:
// instantiates sweep_kernel<FOMO_SWEEP_M> and its host entry points.
#pragma once

#include "step_sweep.cuh"
#include "sweep_launch.h"

namespace fomo {

template <>
cudaError_t sweep_launch<FOMO_SWEEP_M>(int blocks, size_t smem, cudaStream_t st, const SweepLaunch& L) {
    sweep_kernel<FOMO_SWEEP_M><<<blocks, kThreads, smem, st>>>(L);
    return cudaGetLastError();
}

template <>
const void* sweep_kernel_fn<FOMO_SWEEP_M>() {
    return reinterpret_cast<const void*>(&sweep_kernel<FOMO_SWEEP_M>);
}

}  // namespace fomo
