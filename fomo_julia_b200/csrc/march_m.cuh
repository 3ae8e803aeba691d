// march_m.cuh -- body of the translation units march_m1.cu .. march_m4.cu:
// instantiates march_kernel<FOMO_MARCH_M> and its host entry points.
#pragma once

#include "march_launch.h"
#include "step_march.cuh"

namespace fomo {

template <>
cudaError_t march_launch<FOMO_MARCH_M>(int blocks, cudaStream_t st, const StepParams& P, const MarchArgs& A,
                                       const MarchMaps& mp) {
    march_kernel<FOMO_MARCH_M><<<blocks, kMThreads, march_smem_bytes<FOMO_MARCH_M>(), st>>>(P, A, mp);
    return cudaGetLastError();
}

template <>
const void* march_kernel_fn<FOMO_MARCH_M>() {
    return reinterpret_cast<const void*>(&march_kernel<FOMO_MARCH_M>);
}

template <>
cudaError_t batch_march_launch<FOMO_MARCH_M>(int blocks, cudaStream_t st, const BatchMarchLaunch& L) {
    batch_march_kernel<FOMO_MARCH_M><<<blocks, kMThreads, march_smem_bytes<FOMO_MARCH_M>(), st>>>(L);
    return cudaGetLastError();
}

template <>
const void* batch_march_kernel_fn<FOMO_MARCH_M>() {
    return reinterpret_cast<const void*>(&batch_march_kernel<FOMO_MARCH_M>);
}

}  // namespace fomo
