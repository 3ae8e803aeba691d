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
// results are bit-identical to the same shot run alone.  The TMA descriptors
// of a launch's shots travel in its kernel parameters (BatchVelMaps,
// BatchStrMaps): descriptors kept in global memory would need a proxy fence
// per descriptor in every block.
#pragma once

#include <cstddef>

#include "step_tiled.cuh"

namespace fomo {

// One shot of a batch (device memory, written by the host).
struct ShotDev {
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

// Per-shot state of the current batch step, written by batch_prep_kernel.
struct ShotStep {
    int ks;        // local step (may lie outside 1..nt)
    float src_w;   // wavelet sample of step ks (0 outside the wavelet)
    int pad_[2];
};

constexpr int kMaxGroups = 16;       // media per launch
constexpr int kShotsPerLaunch = 16;  // shots per launch (the host splits larger batches)

// TMA descriptors of a launch's shots, passed as kernel parameters (by
// shot s of the launch and wavefield copy c).
struct BatchVelMaps {
    CUtensorMap tau[kShotsPerLaunch][2][3];  // halo boxes of txx, tzz, txz
    CUtensorMap v[kShotsPerLaunch][2][2];    // tile boxes of vx, vz
    CUtensorMap b[kShotsPerLaunch][4];       // tile boxes of the four buoyancy arrays
};
struct BatchStrMaps {
    CUtensorMap v[kShotsPerLaunch][2][2];    // halo boxes of vx, vz
    CUtensorMap tau[kShotsPerLaunch][2][3];  // tile boxes of txx, tzz, txz
    CUtensorMap mod[kShotsPerLaunch][3];     // tile boxes of lam, mu_txx, mu_txz
};

struct BatchArgs {
    const ShotDev* shots;
    ShotStep* steps;        // [n_shots]
    const int* rec_off;     // [n_shots + 1]: first receiver block of each shot
    const int* step;        // batch step of this launch (1-based)
    int n_shots, n_groups;
    int total_band, total_tile;
    GroupDev groups[kMaxGroups];  // by value: decoded from the constant bank
};

struct BatchItem {
    int role;   // 0 band pass, 1 tile, 2 receivers, -1 none
    int shot, local;
};

// Group of block b of one role: the last group whose offset is <= b.
template <bool TILE>
__device__ __forceinline__ BatchItem in_groups(const BatchArgs& B, int b) {
    int g = 0;
#pragma unroll 1
    for (int h = 1; h < B.n_groups; ++h) {
        const int off = TILE ? B.groups[h].tile_off : B.groups[h].band_off;
        if (off <= b) g = h;
    }
    const int r = b - (TILE ? B.groups[g].tile_off : B.groups[g].band_off);
    const int n = B.groups[g].n;
    BatchItem it;
    it.role = TILE ? 1 : 0;
    it.shot = B.groups[g].first + r % n;
    it.local = r / n;
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
    float* field[2][5];
    ShotStep st;
    int a;       // input copy
};

// Every thread decodes the block from the kernel parameters; thread 0 reads
// the shot's step record while all threads copy its parameters (one round
// trip to memory); thread 0 then sets the per-step fields.  Returns false for
// an idle block.
template <bool VEL, bool BAND>
__device__ __forceinline__ bool setup_block(const BatchArgs& B, BatchBlock& bb, BatchItem& it) {
    it = decode(B, blockIdx.x, VEL, BAND);
    if (it.role < 0) return false;  // block-uniform
    const ShotDev& sd = B.shots[it.shot];
    static_assert(offsetof(ShotDev, T) == offsetof(ShotDev, P) + sizeof(StepParams) &&
                      offsetof(ShotDev, field) == offsetof(ShotDev, T) + sizeof(TiledArgs) &&
                      offsetof(BatchBlock, T) == sizeof(StepParams) &&
                      offsetof(BatchBlock, field) == sizeof(StepParams) + sizeof(TiledArgs),
                  "contiguous parameter copy");
    constexpr int W = (int)((sizeof(StepParams) + sizeof(TiledArgs) + sizeof(sd.field)) / 4);
    const int* src = reinterpret_cast<const int*>(&sd.P);
    int* dst = reinterpret_cast<int*>(&bb.P);
    if (threadIdx.x == 0) bb.st = B.steps[it.shot];
    for (int w = threadIdx.x; w < W; w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    const int ks = bb.st.ks;
    const bool run = it.role == 2 ? (ks >= 2 && ks <= bb.P.nt + 1) : (ks >= 1 && ks <= bb.P.nt);
    if (!run) return false;  // block-uniform
    if (threadIdx.x == 0) {
        const int a = (ks - 1) & 1, b = 1 - a;
        bb.a = a;
        bb.P.src_w = bb.st.src_w;
        for (int q = 0; q < 5; ++q) bb.P.in[q] = bb.field[a][q];
        for (int q = 0; q < 5; ++q) bb.P.out[q] = nullptr;
        if (VEL) {
            // reads v(a), tau(a); writes v(b); records step ks-1 from copy a
            bb.P.out[VX] = bb.field[b][VX];
            bb.P.out[VZ] = bb.field[b][VZ];
            bb.P.rec_k = ks - 1;
        } else {
            // reads v(b) (new), tau(a); writes tau(b)
            bb.P.in[VX] = bb.field[b][VX];
            bb.P.in[VZ] = bb.field[b][VZ];
            for (int q = 2; q < 5; ++q) bb.P.out[q] = bb.field[b][q];
            bb.P.rec_k = 0;
        }
    }
    __syncthreads();
    return true;
}

// Step records of every shot for the batch step *B.step (one thread each);
// launched before the step's first launch.
__global__ void batch_prep_kernel(const __grid_constant__ BatchArgs B) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B.n_shots) return;
    const ShotDev& sd = B.shots[s];
    ShotStep st;
    st.ks = *B.step - sd.start + 1;
    st.src_w = (st.ks >= 1 && st.ks <= sd.n_wavelet) ? sd.wavelet[st.ks - 1] : 0.f;
    st.pad_[0] = st.pad_[1] = 0;
    B.steps[s] = st;
}

template <int M>
__global__ void __launch_bounds__(kThreads, 5) batch_velocity_kernel(const __grid_constant__ BatchArgs B,
                                                                  const __grid_constant__ BatchVelMaps MV) {
    extern __shared__ __align__(128) float smem[];
    __shared__ BatchBlock bb;
    BatchItem it;
    if (!setup_block<true, false>(B, bb, it)) return;
    const StepParams& P = bb.P;
    const TiledArgs& T = bb.T;
    if (it.role == 1) {
        const TileKind k = classify(P, T, it.local);
        if (k.generic) edge_tile<M, true>(P, T, k.x0, k.z0, k.x_end, smem);
        else {
            const int s = it.shot, a = bb.a;
            const VelMapRefs mp{&MV.tau[s][a][0], &MV.tau[s][a][1], &MV.tau[s][a][2], &MV.v[s][a][0], &MV.v[s][a][1],
                                &MV.b[s][0],      &MV.b[s][1],      &MV.b[s][2],      &MV.b[s][3]};
            fast_vel<M>(P, T, mp, k.x0, k.z0, k.x_end, k.band, k.rim, smem);
        }
    } else {
        record_block(P, it.local);
    }
}

template <int M>
__global__ void __launch_bounds__(kThreads, 5) batch_stress_kernel(const __grid_constant__ BatchArgs B,
                                                                const __grid_constant__ BatchStrMaps MS) {
    extern __shared__ __align__(128) float smem[];
    __shared__ BatchBlock bb;
    BatchItem it;
    if (!setup_block<false, false>(B, bb, it)) return;
    const StepParams& P = bb.P;
    const TiledArgs& T = bb.T;
    const TileKind k = classify(P, T, it.local);
    if (k.generic) edge_tile<M, false>(P, T, k.x0, k.z0, k.x_end, smem);
    else {
        const int s = it.shot, a = bb.a, b = 1 - a;
        const StrMapRefs mp{&MS.v[s][b][0],   &MS.v[s][b][1],   &MS.tau[s][a][0], &MS.tau[s][a][1],
                            &MS.tau[s][a][2], &MS.mod[s][0],    &MS.mod[s][1],    &MS.mod[s][2]};
        fast_str<M>(P, T, mp, k.x0, k.z0, k.x_end, k.band, k.rim, smem);
    }
}

// Band pass of every shot in flight (after the tile launch of the same half
// step): one warp per (shot, strip, field).
template <bool VEL>
__global__ void __launch_bounds__(32) batch_band_kernel(const __grid_constant__ BatchArgs B) {
    __shared__ __align__(16) float stage[kMarchStage];
    __shared__ float stab[kMaxBandTab];
    __shared__ BatchBlock bb;
    BatchItem it;
    if (!setup_block<VEL, true>(B, bb, it)) return;
    band_march<VEL>(bb.P, bb.T, it.local, stage, stab);
}

// Advances the batch step counter; launched once per step after the stress
// launches of every order.
__global__ void batch_advance_kernel(int* step) { *step += 1; }

static_assert(sizeof(BatchArgs) + sizeof(BatchVelMaps) <= 32764 && sizeof(BatchArgs) + sizeof(BatchStrMaps) <= 32764,
              "kernel parameters above the 32764-byte limit");

// Static shared memory of a batch block (beyond the dynamic part).
constexpr size_t kBatchStaticSmem = sizeof(BatchBlock);

}  // namespace fomo
