// step_batch.cuh -- time-step kernels over many shots per launch.
//
// The single-shot kernels (step_tiled.cuh) take one shot's parameters by
// value.  The batch kernels take a table of shots in device memory and read
// the batch step from a device counter, so every launch of a batch has the
// same arguments: a run of K time steps (velocity, stress, counter advance)
// can be captured once into a CUDA graph and replayed.
//
// Shots are grouped by medium (same nx, nz, hence the same block counts).
// A tile launch holds, for every shot s whose local step ks = k - start_s + 1
// lies in 1..nt_s (k = batch step):
//   tile blocks   all groups, then
//   receivers     (velocity launch only) the receivers of step ks-1;
// the band launch that follows it holds the band-pass warps of every group.
// Inside a group, tile and band blocks are interleaved tile-major
// (block = local * n + shot), so the n shots' copies of one tile run side by
// side and the medium tile is read from HBM once and from L2 by the others.
// A block whose shot is outside its step range returns at once; that is how
// shots join and leave a running batch at step boundaries.
//
// Every block runs the single-shot code (edge_tile, fast_vel, fast_str,
// record_block, band_march) on its shot's parameters, so a batched shot's
// results are bit-identical to the same shot run alone.
#pragma once

#include "step_tiled.cuh"

namespace fomo {

// One shot of a batch (device memory, written by the host).
struct alignas(64) ShotDev {
    VelMaps vmap[2];        // by input copy a: tau(a) halo boxes, v(a), buoyancy
    StrMaps smap[2];        // by input copy a: v(1-a) halo boxes, tau(a), moduli
    StepParams P;           // static part; in/out, src_w and rec_k are set per launch
    TiledArgs T;            // block counts, buoyancy, status word
    float* field[2][5];     // the two copies of the five fields
    const float* wavelet;   // n_wavelet samples
    int n_wavelet;
    int start;              // batch step of the shot's step 1 (>= 1)
    int nt;
    int pad_;
};

// Shots first..first+n-1 of the table share a medium.
struct GroupDev {
    int first, n;
    int n_band, n_tile;     // band-pass and tile blocks per shot
    int band_off, tile_off; // first band / tile block of the group in its launch
};

struct BatchArgs {
    const ShotDev* shots;
    const GroupDev* groups;
    const int* rec_off;     // [n_shots + 1]: first receiver block of each shot
    const int* step;        // batch step of this launch (1-based)
    int n_shots, n_groups;
    int total_band, total_tile;
};

struct BatchItem {
    int role;   // 0 band pass, 1 tile, 2 receivers, -1 none
    int shot, local;
};

// Group of block b of one role: the last group whose offset is <= b.
template <bool TILE>
__device__ __forceinline__ BatchItem in_groups(const BatchArgs& B, int b) {
    int g = 0;
    for (int h = 1; h < B.n_groups; ++h) {
        const int off = TILE ? B.groups[h].tile_off : B.groups[h].band_off;
        if (off <= b) g = h;
    }
    const GroupDev G = B.groups[g];
    const int r = b - (TILE ? G.tile_off : G.band_off);
    BatchItem it;
    it.role = TILE ? 1 : 0;
    it.shot = G.first + r % G.n;
    it.local = r / G.n;
    return it;
}

// Block bid of a tile launch (band == false) or of a band launch.
__device__ __forceinline__ BatchItem decode(const BatchArgs& B, int bid, bool vel, bool band) {
    if (band) return in_groups<false>(B, bid);
    if (bid < B.total_tile) return in_groups<true>(B, bid);
    bid -= B.total_tile;
    BatchItem it{-1, 0, 0};
    if (!vel || bid >= B.rec_off[B.n_shots]) return it;
    int lo = 0, hi = B.n_shots;  // rec_off[lo] <= bid < rec_off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (B.rec_off[mid] <= bid) lo = mid;
        else hi = mid;
    }
    it.role = 2;
    it.shot = lo;
    it.local = bid - B.rec_off[lo];
    return it;
}

// Shared-memory copy of a block's shot parameters for this launch.
struct BatchBlock {
    StepParams P;
    TiledArgs T;
    BatchItem it;
    int a;       // input copy
    int ks;      // local step (0 = block idle)
};

// Orders the host's copy of a shot table entry before the TMA unit reads the
// descriptor from global memory (issued by the thread that issues the loads).
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* m) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(m) : "memory");
}

// Thread 0 decodes the block; all threads copy the shot's parameters; thread 0
// then sets the per-step fields.  Returns false for an idle block.
template <bool VEL, bool BAND>
__device__ __forceinline__ bool setup_block(const BatchArgs& B, BatchBlock& bb) {
    if (threadIdx.x == 0) {
        bb.ks = 0;
        bb.it = decode(B, blockIdx.x, VEL, BAND);
        if (bb.it.role >= 0) {
            const ShotDev& sd = B.shots[bb.it.shot];
            const int ks = *B.step - sd.start + 1;
            const bool run = bb.it.role == 2 ? (ks >= 2 && ks <= sd.nt + 1) : (ks >= 1 && ks <= sd.nt);
            if (run) bb.ks = ks;
        }
    }
    __syncthreads();
    if (bb.ks == 0) return false;
    const ShotDev& sd = B.shots[bb.it.shot];
    static_assert(sizeof(StepParams) % 4 == 0 && sizeof(TiledArgs) % 4 == 0, "word copies");
    {
        const int* src = reinterpret_cast<const int*>(&sd.P);
        int* dst = reinterpret_cast<int*>(&bb.P);
        for (int w = threadIdx.x; w < (int)(sizeof(StepParams) / 4); w += blockDim.x) dst[w] = src[w];
        const int* srt = reinterpret_cast<const int*>(&sd.T);
        int* dtt = reinterpret_cast<int*>(&bb.T);
        for (int w = threadIdx.x; w < (int)(sizeof(TiledArgs) / 4); w += blockDim.x) dtt[w] = srt[w];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int ks = bb.ks;
        const int a = (ks - 1) & 1, b = 1 - a;
        bb.a = a;
        bb.P.src_w = (ks <= sd.n_wavelet) ? sd.wavelet[ks - 1] : 0.f;
        for (int q = 0; q < 5; ++q) bb.P.in[q] = sd.field[a][q];
        for (int q = 0; q < 5; ++q) bb.P.out[q] = nullptr;
        if (bb.it.role == 1) {
            const CUtensorMap* m = VEL ? reinterpret_cast<const CUtensorMap*>(&sd.vmap[a])
                                       : reinterpret_cast<const CUtensorMap*>(&sd.smap[a]);
            const int n = VEL ? (int)(sizeof(VelMaps) / sizeof(CUtensorMap)) : (int)(sizeof(StrMaps) / sizeof(CUtensorMap));
            for (int t = 0; t < n; ++t) tensormap_acquire(m + t);
        }
        if (VEL) {
            // reads v(a), tau(a); writes v(b); records step ks-1 from copy a
            bb.P.out[VX] = sd.field[b][VX];
            bb.P.out[VZ] = sd.field[b][VZ];
            bb.P.rec_k = ks - 1;
        } else {
            // reads v(b) (new), tau(a); writes tau(b)
            bb.P.in[VX] = sd.field[b][VX];
            bb.P.in[VZ] = sd.field[b][VZ];
            for (int q = 2; q < 5; ++q) bb.P.out[q] = sd.field[b][q];
            bb.P.rec_k = 0;
        }
    }
    __syncthreads();
    return true;
}

template <int M>
__global__ void __launch_bounds__(kThreads, 5) batch_velocity_kernel(const __grid_constant__ BatchArgs B) {
    extern __shared__ __align__(128) float smem[];
    __shared__ BatchBlock bb;
    if (!setup_block<true, false>(B, bb)) return;
    const StepParams& P = bb.P;
    const TiledArgs& T = bb.T;
    if (bb.it.role == 1) {
        const TileKind k = classify(P, T, bb.it.local);
        if (k.generic) edge_tile<M, true>(P, T, k.x0, k.z0, k.x_end, smem);
        else fast_vel<M>(P, T, B.shots[bb.it.shot].vmap[bb.a], k.x0, k.z0, k.x_end, k.band, k.rim, smem);
    } else {
        record_block(P, bb.it.local);
    }
}

template <int M>
__global__ void __launch_bounds__(kThreads, 5) batch_stress_kernel(const __grid_constant__ BatchArgs B) {
    extern __shared__ __align__(128) float smem[];
    __shared__ BatchBlock bb;
    if (!setup_block<false, false>(B, bb)) return;
    const StepParams& P = bb.P;
    const TiledArgs& T = bb.T;
    {
        const TileKind k = classify(P, T, bb.it.local);
        if (k.generic) edge_tile<M, false>(P, T, k.x0, k.z0, k.x_end, smem);
        else fast_str<M>(P, T, B.shots[bb.it.shot].smap[bb.a], k.x0, k.z0, k.x_end, k.band, k.rim, smem);
    }
}

// Band pass of every shot in flight (after the tile launch of the same half
// step): one warp per (shot, strip, field).
template <bool VEL>
__global__ void __launch_bounds__(32) batch_band_kernel(const __grid_constant__ BatchArgs B) {
    __shared__ __align__(16) float stage[kMarchStage];
    __shared__ float stab[kMaxBandTab];
    __shared__ BatchBlock bb;
    if (!setup_block<VEL, true>(B, bb)) return;
    band_march<VEL>(bb.P, bb.T, bb.it.local, stage, stab);
}

// Advances the batch step counter; launched once per step after the stress
// launches of every order.
__global__ void batch_advance_kernel(int* step) { *step += 1; }

// Static shared memory of a batch block (beyond the dynamic part).
constexpr size_t kBatchStaticSmem = sizeof(BatchBlock);

}  // namespace fomo
