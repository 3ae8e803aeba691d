// step_batch.cuh -- time-step kernels over many shots per launch.
//
// A batch launch covers up to kShotsPerLaunch shots.  Everything a block
// needs travels in the kernel parameters (__grid_constant__, read through the
// constant cache): for every shot, its StepParams for both wavefield copies
// it may read (in/out pointers differ by the parity of the local step), its
// TiledArgs, its start step and wavelet, and its TMA descriptors.  The batch
// step comes from device counters, so every launch of a batch has the same
// arguments and a run of K time steps (tile and band launches of velocity
// and stress) can be captured once into a CUDA graph and replayed.
//
// A launch set (up to kShotsPerLaunch shots) runs velocity tiles, velocity
// band pass, stress tiles, stress band pass, then the next set; every tile
// launch may start beside the band pass just before it (programmatic
// dependent launch), so each set has two counters: its velocity launches
// (tiles and band) read the velocity counter, its stress launches the
// stress counter.  Block 0 of the velocity tile launch waits for the launch
// before it and advances the stress counter to the step; block 0 of the
// stress tile launch waits for the velocity band pass and advances the
// velocity counter to the next step.  Nothing reads a counter while it is
// advanced: a tile launch overlaps only the band pass just before it, which
// block 0 has waited for, and the launches that read the counter next start
// after the advancing launch has completed.
//
// Shots are grouped by medium (same nx, nz, hence the same block counts).  A
// tile launch holds, for every shot s whose local step ks = k - start_s + 1
// lies in 1..nt_s (k = batch step):
//   tile blocks   all groups, then
//   receivers     (velocity launch only) the receivers of step ks-1;
// the band launch that follows it holds the band-pass warps of every group.
// Inside a group, tile and band blocks are interleaved tile-major
// (block = local * n + shot), so the n shots' copies of one tile run side by
// side and the medium tile is read from HBM once and from L2 by the others.
// A tile block takes its shot's wavefield copy from the launch's step parity
// (BatchHead::kpar), so its TMA loads start at once, and reads the step
// counter beside them; a block whose shot is outside its step range stores
// nothing (receiver and generic-tile blocks return at once).  That is how
// shots join and leave a running batch at step boundaries.  Thread 0 of a
// fast tile also prefetches into L2 the boxes of the block pf_ahead later.
//
// Every block runs the single-shot code (edge_tile, fast_vel, fast_str,
// record_block, band_march) on its shot's parameters, so a batched shot's
// results are bit-identical to the same shot run alone.  Descriptors in
// kernel parameters need no proxy fence (descriptors kept in global memory
// would need one per descriptor in every block).
#pragma once

#include "step_tiled.cuh"

namespace fomo {

constexpr int kMaxGroups = 16;       // media per launch
constexpr int kShotsPerLaunch = 12;  // shots per launch (the host splits larger batches)

// Shots first..first+n-1 of a launch share a medium.
struct GroupDev {
    int first, n;
    int n_band, n_tile;     // band-pass and tile blocks per shot
    int band_off, tile_off; // first band / tile block of the group in its launch
};

struct BatchHead {
    const int* step;                  // batch step (1-based) of the launch's half step
    int* advance;                     // the other half step's counter of the set (block 0 advances it)
    int kpar;                         // parity of that batch step (the host knows it when it launches)
    int pf_ahead;                     // tile blocks between a block and the one whose boxes it prefetches
    int n_shots, n_groups;
    int total_band, total_tile;
    int rec_off[kShotsPerLaunch + 1]; // first receiver block of each shot
    GroupDev groups[kMaxGroups];
};

// One shot of a launch.  P[c] is the half step's StepParams when the step
// reads copy c: velocity: in = copy c, out vx/vz = copy 1-c; stress: in
// vx/vz = copy 1-c (the new velocities), in tau = copy c, out tau = copy 1-c.
struct BatchShot {
    StepParams P[2];
    TiledArgs T;
    const float* wavelet;
    int n_wavelet;
    int start;              // batch step of the shot's step 1 (>= 1)
    int nt;
    int pad_;
};

struct BatchVelLaunch {
    BatchHead H;
    BatchShot shot[kShotsPerLaunch];
    CUtensorMap tau[kShotsPerLaunch][2][3];  // halo boxes of txx, tzz, txz of copy c
    CUtensorMap v[kShotsPerLaunch][2][2];    // tile boxes of vx, vz of copy c
    CUtensorMap b[kShotsPerLaunch][4];       // tile boxes of the buoyancy arrays
};

struct BatchStrLaunch {
    BatchHead H;
    BatchShot shot[kShotsPerLaunch];
    CUtensorMap v[kShotsPerLaunch][2][2];    // halo boxes of vx, vz of copy c
    CUtensorMap tau[kShotsPerLaunch][2][3];  // tile boxes of txx, tzz, txz of copy c
    CUtensorMap mod[kShotsPerLaunch][3];     // tile boxes of lam, mu_txx, mu_txz
};

static_assert(sizeof(BatchVelLaunch) <= 32764 && sizeof(BatchStrLaunch) <= 32764,
              "kernel parameters above the 32764-byte limit");

struct BatchItem {
    int role;   // 0 band pass, 1 tile, 2 receivers, -1 none
    int shot, local;
};

// Group of block b of one role: the last group whose offset is <= b.
template <bool TILE>
__device__ __forceinline__ BatchItem in_groups(const BatchHead& H, int b) {
    int g = 0;
#pragma unroll 1
    for (int h = 1; h < H.n_groups; ++h) {
        const int off = TILE ? H.groups[h].tile_off : H.groups[h].band_off;
        if (off <= b) g = h;
    }
    const int r = b - (TILE ? H.groups[g].tile_off : H.groups[g].band_off);
    const int n = H.groups[g].n;
    BatchItem it;
    it.role = TILE ? 1 : 0;
    it.shot = H.groups[g].first + r % n;
    it.local = r / n;
    return it;
}

// Block bid of a tile launch (band == false) or of a band launch.
__device__ __forceinline__ BatchItem decode(const BatchHead& H, int bid, bool vel, bool band) {
    if (band) return in_groups<false>(H, bid);
    if (bid < H.total_tile) return in_groups<true>(H, bid);
    bid -= H.total_tile;
    BatchItem it{-1, 0, 0};
    if (!vel || bid >= H.rec_off[H.n_shots]) return it;
    int s = 0;
#pragma unroll 1
    while (H.rec_off[s + 1] <= bid) ++s;
    it.role = 2;
    it.shot = s;
    it.local = bid - H.rec_off[s];
    return it;
}

// Local step of a block's shot (every thread computes it: one broadcast load).
__device__ __forceinline__ int local_step(const BatchHead& H, const BatchShot& S) {
    return *H.step - S.start + 1;
}

// The wavefield copy a shot's step reads, (ks - 1) & 1, from the launch's
// step parity alone: no memory access stands between a tile block's start
// and its TMA loads.  A block whose local step disagrees flags an error.
__device__ __forceinline__ int read_copy(const BatchHead& H, const BatchShot& S) { return (H.kpar ^ S.start) & 1; }
constexpr int kErrBatchParity = 3;

__device__ __forceinline__ float wavelet_at(const BatchShot& S, int ks) {
    return (ks >= 1 && ks <= S.n_wavelet) ? __ldg(S.wavelet + ks - 1) : 0.f;
}

// Block 0 of a tile launch: waits for the launches before it (always, so
// the launch cannot complete before them) and advances the other counter.
__device__ __forceinline__ void block0_advance(const BatchHead& H) {
    if (blockIdx.x != 0) return;
    grid_dep_wait();
    if (threadIdx.x == 0 && H.advance) *H.advance += 1;
}

// Sets the counters of n launch sets when the host rebuilds its tables:
// velocity counter of set i (counters[2i]) to `step`, stress counter
// (counters[2i+1]) to step - 1.
__global__ void batch_counters_kernel(int* counters, int n, int step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        counters[2 * i] = step;
        counters[2 * i + 1] = step - 1;
    }
}

// L2 prefetch of the boxes of tile block `b` of a launch (thread 0, right
// after its own tile's copies): the shot's own boxes, and the medium boxes
// only for the group's first shot (its other shots read the same ones).
// The copy comes from the launch's parity, so nothing is loaded first.
template <int M, bool VEL, class LaunchT>
struct BatchPrefetch {
    const LaunchT& L;
    int b;
    __device__ void operator()() const {
        const BatchHead& H = L.H;
        if (b >= H.total_tile) return;
        const BatchItem it = in_groups<true>(H, b);
        const BatchShot& S = L.shot[it.shot];
        if (it.local >= S.T.n_tile_blocks) return;
        const TileKind k = classify(S.P[0], S.T, it.local);
        if (k.generic) return;
        int g = 0;
#pragma unroll 1
        for (int h = 1; h < H.n_groups; ++h)
            if (H.groups[h].tile_off <= b) g = h;
        const bool medium = it.shot == H.groups[g].first;
        const int s = it.shot, c = read_copy(H, S);
        using G = Geo<M>;
        if constexpr (VEL) {
            for (int f = 0; f < 3; ++f) tma_prefetch_2d(&L.tau[s][c][f], k.x0 - G::HX, k.z0 - M);
            for (int f = 0; f < 2; ++f) tma_prefetch_2d(&L.v[s][c][f], k.x0, k.z0);
            if (medium)
                for (int q = 0; q < (S.T.iso ? 3 : 4); q += (S.T.iso ? 2 : 1)) tma_prefetch_2d(&L.b[s][q], k.x0, k.z0);
        } else {
            for (int f = 0; f < 2; ++f) tma_prefetch_2d(&L.v[s][1 - c][f], k.x0 - G::HX, k.z0 - M);
            for (int f = 0; f < 3; ++f) tma_prefetch_2d(&L.tau[s][c][f], k.x0, k.z0);
            if (medium)
                for (int q = 0; q < 3; ++q) tma_prefetch_2d(&L.mod[s][q], k.x0, k.z0);
        }
    }
};

template <int M>
__global__ void __launch_bounds__(kThreads, kTileBlocks<M>) batch_velocity_kernel(const __grid_constant__ BatchVelLaunch L) {
    extern __shared__ __align__(128) float smem[];
    block0_advance(L.H);
    const BatchItem it = decode(L.H, blockIdx.x, true, false);
    if (it.role < 0) return;
    const BatchShot& S = L.shot[it.shot];
    const int ks = local_step(L.H, S);
    if (it.role == 2) {
        const int a = (ks - 1) & 1;
        grid_dep_wait();  // receivers may sit in the band rows
        if (ks >= 2 && ks <= S.nt + 1) record_block(S.P[a], it.local, ks - 1);  // state after step ks-1: copy a
        return;
    }
    // the tile path: the copy from the launch's parity, the step's range
    // checked once the boxes are on their way (live)
    const int c = read_copy(L.H, S);
    const bool live = ks >= 1 && ks <= S.nt;
    const StepParams& P = S.P[c];
    const TileKind k = classify(P, S.T, it.local);
    if (reads_band_rows(P, k.z0)) grid_dep_wait();
    if (k.generic) {
        if (!live) return;
        edge_tile<M, true>(P, S.T, k.x0, k.z0, k.x_end, smem, wavelet_at(S, ks));
    } else {
        const int s = it.shot;
        const VelMapRefs mp{&L.tau[s][c][0], &L.tau[s][c][1], &L.tau[s][c][2], &L.v[s][c][0], &L.v[s][c][1],
                            &L.b[s][0],      &L.b[s][1],      &L.b[s][2],      &L.b[s][3]};
        const BatchPrefetch<M, true, BatchVelLaunch> pf{L, L.H.pf_ahead > 0 ? (int)blockIdx.x + L.H.pf_ahead : 1 << 30};
        fast_vel<M>(P, S.T, mp, k.x0, k.z0, k.x_end, k.band, k.rim, smem, wavelet_at(S, ks), -1, live, pf);
    }
    if (threadIdx.x == 0 && live && ((ks - 1) & 1) != c) atomicCAS(S.T.status, 0, kErrBatchParity);
}

template <int M>
__global__ void __launch_bounds__(kThreads, kTileBlocks<M>) batch_stress_kernel(const __grid_constant__ BatchStrLaunch L) {
    extern __shared__ __align__(128) float smem[];
    block0_advance(L.H);
    const BatchItem it = decode(L.H, blockIdx.x, false, false);
    if (it.role < 0) return;
    const BatchShot& S = L.shot[it.shot];
    const int ks = local_step(L.H, S);
    const int a = read_copy(L.H, S), b = 1 - a;  // as in the velocity launch
    const bool live = ks >= 1 && ks <= S.nt;
    const StepParams& P = S.P[a];
    const TileKind k = classify(P, S.T, it.local);
    if (reads_band_rows(P, k.z0)) grid_dep_wait();
    if (k.generic) {
        if (!live) return;
        edge_tile<M, false>(P, S.T, k.x0, k.z0, k.x_end, smem, wavelet_at(S, ks));
    } else {
        const int s = it.shot;
        const StrMapRefs mp{&L.v[s][b][0],   &L.v[s][b][1],   &L.tau[s][a][0], &L.tau[s][a][1],
                            &L.tau[s][a][2], &L.mod[s][0],    &L.mod[s][1],    &L.mod[s][2]};
        const BatchPrefetch<M, false, BatchStrLaunch> pf{L, L.H.pf_ahead > 0 ? (int)blockIdx.x + L.H.pf_ahead : 1 << 30};
        fast_str<M>(P, S.T, mp, k.x0, k.z0, k.x_end, k.band, k.rim, smem, wavelet_at(S, ks), -1, live, pf);
    }
    if (threadIdx.x == 0 && live && ((ks - 1) & 1) != a) atomicCAS(S.T.status, 0, kErrBatchParity);
}

// Band pass of every shot in flight (after the tile launch of the same half
// step): one warp per (shot, strip, field).  LaunchT is the half step's
// launch type (its StepParams images; the descriptors are not used).
template <bool VEL, class LaunchT>
__global__ void __launch_bounds__(32) batch_band_kernel(const __grid_constant__ LaunchT L) {
    __shared__ __align__(16) float stage[kMarchStage];
    __shared__ float stab[kMaxBandTab];
    grid_dep_trigger();
    const BatchItem it = decode(L.H, blockIdx.x, VEL, true);
    const BatchShot& S = L.shot[it.shot];
    const int ks = local_step(L.H, S);
    if (ks < 1 || ks > S.nt) return;
    band_march<VEL>(S.P[(ks - 1) & 1], S.T, it.local, stage, stab);
}

}  // namespace fomo
