// march_launch.h -- host entry points of the fused-step kernels.  Each
// march_kernel<M> is compiled in its own translation unit (march_m<M>.cu,
// through march_m.cuh), so the library builds them in parallel; the runtime
// launches them through these functions only.
#pragma once

#include <cuda_runtime.h>

namespace fomo {

struct StepParams;
struct MarchArgs;
struct MarchMaps;
struct BatchMarchLaunch;

// Launches march_kernel<M> with `blocks` blocks on `st`.
template <int M>
cudaError_t march_launch(int blocks, cudaStream_t st, const StepParams& P, const MarchArgs& A, const MarchMaps& mp);

// The kernel's host stub, for cudaFuncSetAttribute and occupancy queries.
template <int M>
const void* march_kernel_fn();

// Launches batch_march_kernel<M> (many shots per launch) with `blocks` blocks.
template <int M>
cudaError_t batch_march_launch(int blocks, cudaStream_t st, const BatchMarchLaunch& L);
template <int M>
const void* batch_march_kernel_fn();

#define FOMO_MARCH_DECLARE(M)                                                                              \
    template <>                                                                                            \
    cudaError_t march_launch<M>(int, cudaStream_t, const StepParams&, const MarchArgs&, const MarchMaps&); \
    template <>                                                                                            \
    const void* march_kernel_fn<M>();                                                                      \
    template <>                                                                                            \
    cudaError_t batch_march_launch<M>(int, cudaStream_t, const BatchMarchLaunch&);                         \
    template <>                                                                                            \
    const void* batch_march_kernel_fn<M>();
FOMO_MARCH_DECLARE(1)
FOMO_MARCH_DECLARE(2)
FOMO_MARCH_DECLARE(3)
FOMO_MARCH_DECLARE(4)
#undef FOMO_MARCH_DECLARE

}  // namespace fomo
