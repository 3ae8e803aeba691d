// step_sweep.cuh -- the swept time step: one persistent launch per step over
// the split launches' tiles.
//
// The split launches read tau and the new v from HBM twice per step (the
// velocity tiles read tau, the stress tiles read it again with the v the
// velocity tiles just wrote): 80 bytes per cell against the 60 the step must
// move.  Here one launch runs the velocity tiles, the stress tiles and both
// bottom-band passes of a step, taken from a work queue whose order keeps
// those re-reads in L2: velocity tile rows from the bottom of the grid up,
// each stress tile row a few rows (the lag) behind the velocity rows it
// reads.  Between a velocity row and the stress row that re-reads it, about
// 2 x lag tile rows of traffic pass through L2 (a few tens of MB on a
// 4552-column grid), far less than its 126 MB.
//
// Items, in queue order (a schedule the host builds; every item's inputs are
// produced by items earlier in the queue):
//   receivers of step rec_k (read the step's input copy only);
//   velocity tile rows, bottom to top; the velocity band pass (the bottom
//   HABC recurrence of vx, vz) right after the last velocity row it reads;
//   stress tile rows, bottom to top, row r once velocity rows r-1 .. r+1
//   (and the velocity band pass, if the row reads band rows) are queued; the
//   stress band pass right after the last stress row it reads.
// A block takes the next item, waits (bounded, thread 0) until the items it
// reads are complete, runs it with the same tile code as the split launches
// (fast_vel / fast_str / edge_tile / band_march, so the results are the same
// bit for bit), then publishes its completion.  A block only ever waits for
// items taken before its own, by blocks that are running, so the queue
// always drains.
//
// Completion counters are cumulative over the launches of a run (launch e
// waits for (e+1) x the per-launch count).  Publication: the block's stores,
// a block barrier, then thread 0 orders them for the async proxy and the
// GPU (fence.proxy.async, __threadfence) before its atomicAdd; the consumer's
// thread 0 reads the counter with ld.acquire.gpu and a proxy fence before
// its TMA loads, and a block barrier hands the order on to its other
// threads.  Data written inside the launch (the new v, the band scratch) is
// read only by TMA, plain loads or cp.async, never through the read-only
// data cache.
#pragma once

#include "step_tiled.cuh"

namespace fomo {

enum SweepKind { kSweepRecv = 0, kSweepVRow = 1, kSweepSRow = 2, kSweepVBand = 3, kSweepSBand = 4 };
constexpr int kErrDepTimeout = 2;
constexpr int kSweepPolls = 1 << 21;  // about 0.2 s of polling before a wait gives up
constexpr int kBandWarpsPerItem = kThreads / 32;

struct SweepArgs {
    int* queue;            // [0] next item, [1] blocks that left (both zero between launches)
    int* done;             // completion counters: [0, tz) velocity rows, [tz, 2tz) stress rows,
                           // [2tz] velocity band items, [2tz+1] stress band items
    const int4* sched;     // {kind, tile row, first item, items}, ascending first item
    int n_entries, n_items;
    int epoch;             // launches of this run before this one
    int tiles_z, band_row0;  // tile rows; first tile row holding row nz-nbc-2 (the band passes read it)
    int n_vband, n_sband;  // band items (kBandWarpsPerItem band warps each) per launch
    int prefetch_ahead;    // items between a tile and the item whose DRAM boxes it prefetches (0 = none)
};

struct SweepLaunch {
    StepParams Pv;         // velocity half step: reads copy a, writes v of copy b
    StepParams Ps;         // stress half step: reads v of copy b and tau of copy a, writes tau of copy b
    TiledArgs T;
    VelMaps vm;
    StrMaps sm;
    SweepArgs S;
};
static_assert(sizeof(SweepLaunch) <= 32764, "kernel parameters above the 32764-byte limit");

// Shared memory of the swept step: the larger tile layout, or the band
// warps' staging (two chunks and a weight table per warp).
__host__ __device__ constexpr int sweep_band_tab(int nbc) { return (nbc + 2 + 31) / 32 * 32; }
__host__ inline size_t sweep_band_smem(int nbc) {
    return (size_t)kBandWarpsPerItem * (kMarchStage + sweep_band_tab(nbc)) * 4;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// The two mbarriers a fast tile initialises (after its boxes: see fast_vel
// and fast_str).  A persistent block invalidates them once the tile is done,
// before the memory serves the next item.
template <int M>
__device__ __forceinline__ uint64_t* fast_tile_bars(float* smem, bool vel, bool iso) {
    constexpr int BOX = Geo<M>::BOXS;
    return reinterpret_cast<uint64_t*>(smem + (vel ? 3 * BOX + (iso ? 4 : 6) * kPBox : 2 * BOX + 6 * kPBox));
}

// Thread 0: waits until counter *c reaches `target`; false (status set) if
// it does not within kSweepPolls polls or another block has failed.
__device__ __forceinline__ bool sweep_wait(const int* c, int target, int* status) {
    if (ld_acquire(c) >= target) return true;
    for (int it = 0; it < kSweepPolls; ++it) {
        __nanosleep(64);
        if (ld_acquire(c) >= target) return true;
        if (*reinterpret_cast<volatile int*>(status)) return false;
    }
    atomicCAS(status, 0, kErrDepTimeout);
    return false;
}

// Thread 0: waits for the items a (kind, row) item reads.  A stress row
// whose inputs reach the bottom band rows (the split stress launch's
// reads_band_rows) also waits for the velocity band pass.
__device__ inline bool sweep_deps(const SweepLaunch& L, int kind, int row) {
    const SweepArgs& S = L.S;
    const int tz = S.tiles_z, e1 = S.epoch + 1;
    int* st = L.T.status;
    if (kind == kSweepSRow) {
        const int tx = L.T.tiles_x;
        for (int r = max(row - 1, 0); r <= min(row + 1, tz - 1); ++r)
            if (!sweep_wait(S.done + r, e1 * tx, st)) return false;
        if (reads_band_rows(L.Ps, row * kTZ) && !sweep_wait(S.done + 2 * tz, e1 * S.n_vband, st)) return false;
    } else if (kind == kSweepVBand || kind == kSweepSBand) {
        const int tx = L.T.tiles_x, base = kind == kSweepVBand ? 0 : tz;
        for (int r = S.band_row0; r < tz; ++r)
            if (!sweep_wait(S.done + base + r, e1 * tx, st)) return false;
    }
    return true;
}

// The entry of queue item `item` (thread 0).
__device__ __forceinline__ int4 sweep_entry(const SweepArgs& S, int item) {
    int lo = 0, hi = S.n_entries - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&S.sched[mid].z) <= item) lo = mid;
        else hi = mid - 1;
    }
    return __ldg(S.sched + lo);
}

// The DRAM boxes of item `item` into L2: a velocity tile's boxes, or the
// medium boxes of a stress tile (its tau and v boxes come from L2 already).
template <int M>
__device__ void sweep_prefetch(const SweepLaunch& L, int item) {
    if (item >= L.S.n_items) return;
    const int4 e = sweep_entry(L.S, item);
    const int tile = e.y * L.T.tiles_x + (item - e.z);
    if (e.x == kSweepVRow) {
        prefetch_vel<M>(L.Pv, L.T, refs_of(L.vm), tile);
    } else if (e.x == kSweepSRow) {
        const TileKind k = classify(L.Ps, L.T, tile);
        if (k.generic) return;
        tma_prefetch_2d(&L.sm.lam, k.x0, k.z0);
        tma_prefetch_2d(&L.sm.mu, k.x0, k.z0);
        tma_prefetch_2d(&L.sm.mxz, k.x0, k.z0);
    }
}

template <int M>
__global__ void __launch_bounds__(kThreads, kTileBlocks<M>) sweep_kernel(const __grid_constant__ SweepLaunch L) {
    extern __shared__ __align__(128) float smem[];
    __shared__ int s_job[3];  // kind (-1: leave), tile row, index in the entry
    const SweepArgs& S = L.S;
    for (;;) {
        if (threadIdx.x == 0) {
            int kind = -1, row = 0, idx = 0;
            const int item = atomicAdd(S.queue, 1);
            if (item < S.n_items && *reinterpret_cast<volatile int*>(L.T.status) == 0) {
                const int4 e = sweep_entry(S, item);
                if (sweep_deps(L, e.x, e.y)) {
                    kind = e.x;
                    row = e.y;
                    idx = item - e.z;
                    fence_proxy_async_global();  // the waited-for stores before this item's TMA loads
                    if (S.prefetch_ahead > 0 && (kind == kSweepVRow || kind == kSweepSRow))
                        sweep_prefetch<M>(L, item + S.prefetch_ahead);
                }
            }
            s_job[0] = kind;
            s_job[1] = row;
            s_job[2] = idx;
        }
        __syncthreads();
        const int kind = s_job[0], row = s_job[1], idx = s_job[2];
        if (kind < 0) break;
        uint64_t* bars = nullptr;  // a fast tile's mbarriers
        if (kind == kSweepVRow || kind == kSweepSRow) {
            const int tile = row * L.T.tiles_x + idx;
            if (kind == kSweepVRow) {
                const TileKind k = classify(L.Pv, L.T, tile);
                if (k.generic) {
                    edge_tile<M, true>(L.Pv, L.T, k.x0, k.z0, k.x_end, smem, L.Pv.src_w);
                } else {
                    fast_vel<M>(L.Pv, L.T, refs_of(L.vm), k.x0, k.z0, k.x_end, k.band, k.rim, smem, L.Pv.src_w);
                    bars = fast_tile_bars<M>(smem, true, L.T.iso != 0);
                }
            } else {
                const TileKind k = classify(L.Ps, L.T, tile);
                if (k.generic) {
                    edge_tile<M, false>(L.Ps, L.T, k.x0, k.z0, k.x_end, smem, L.Ps.src_w);
                } else {
                    fast_str<M>(L.Ps, L.T, refs_of(L.sm), k.x0, k.z0, k.x_end, k.band, k.rim, smem, L.Ps.src_w);
                    bars = fast_tile_bars<M>(smem, false, true);
                }
            }
        } else if (kind == kSweepVBand || kind == kSweepSBand) {
            // one band warp per (strip, field): vx, vz of each strip, or txx, tzz, txz
            const int w = threadIdx.x >> 5, bi = idx * kBandWarpsPerItem + w;
            float* stage = smem + w * (kMarchStage + sweep_band_tab(L.Pv.nbc));
            float* stab = stage + kMarchStage;
            const int n_strips = band_block_count(L.Pv.nx);
            if (kind == kSweepVBand) {
                if (bi < 2 * n_strips) band_march<true>(L.Pv, L.T, (bi >> 1) * 3 + (bi & 1), stage, stab);
            } else {
                if (bi < 3 * n_strips) band_march<false>(L.Ps, L.T, bi, stage, stab);
            }
        } else {
            record_block(L.Pv, idx, L.Pv.rec_k);
        }
        __syncthreads();  // the item's stores are done and its shared memory is free
        if (threadIdx.x == 0 && bars) {
            mbar_inval(bars);
            mbar_inval(bars + 1);
        }
        if (threadIdx.x == 0 && kind != kSweepRecv) {
            const int tz = S.tiles_z;
            const int c = kind == kSweepVRow ? row : kind == kSweepSRow ? tz + row : kind == kSweepVBand ? 2 * tz : 2 * tz + 1;
            fence_proxy_async_global();
            __threadfence();
            atomicAdd(S.done + c, 1);
        }
    }
    // the last block to leave resets the queue for the next launch
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(S.queue + 1, 1) == (int)gridDim.x - 1) {
            S.queue[0] = 0;
            S.queue[1] = 0;
            __threadfence();
        }
    }
}

}  // namespace fomo
