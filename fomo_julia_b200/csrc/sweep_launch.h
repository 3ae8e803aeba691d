// sweep_launch.h -- host entry points of the swept time step.  Each
// sweep_kernel<M> is compiled in its own translation unit (sweep_m<M>.cu,
// through sweep_m.cuh), so the library builds them in parallel; the runtime
// launches them through these functions only.
#pragma once

#include <cuda_runtime.h>

namespace fomo {

struct SweepLaunch;

// Launches sweep_kernel<M> with `blocks` blocks and `smem` bytes of dynamic
// shared memory on `st`.
template <int M>
cudaError_t sweep_launch(int blocks, size_t smem, cudaStream_t st, const SweepLaunch& L);

// The kernel's host stub, for cudaFuncSetAttribute and occupancy queries.
template <int M>
const void* sweep_kernel_fn();

#define FOMO_SWEEP_DECLARE(M)                                                          \
    template <>                                                                        \
    cudaError_t sweep_launch<M>(int, size_t, cudaStream_t, const SweepLaunch&);        \
    template <>                                                                        \
    const void* sweep_kernel_fn<M>();
FOMO_SWEEP_DECLARE(1)
FOMO_SWEEP_DECLARE(2)
FOMO_SWEEP_DECLARE(3)
FOMO_SWEEP_DECLARE(4)
FOMO_SWEEP_DECLARE(5)
FOMO_SWEEP_DECLARE(6)
#undef FOMO_SWEEP_DECLARE

}  // namespace fomo
