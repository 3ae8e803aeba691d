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
// waits for (e+1) x the per-launch count).  Publication: the item's stores,
// a block barrier, then warp 1 orders them for the async proxy
// (fence.proxy.async) and releases them with red.release.gpu; the consumer's
// thread 0 reads the counters (ld.relaxed.gpu), then fence.acq_rel.gpu and
// a proxy fence before its TMA loads, and a block barrier hands the order on
// to its other threads.  Data written inside the launch (the new v, the band
// scratch) is read only by TMA, plain loads or cp.async, never through the
// read-only data cache.  A row item is a chunk of consecutive tiles of one
// tile row, so the queue, the wait and the publication are paid once per
// chunk.
#pragma once

#include "step_tiled.cuh"

namespace fomo {

enum SweepKind { kSweepRecv = 0, kSweepVRow = 1, kSweepSRow = 2, kSweepVBand = 3, kSweepSBand = 4 };
constexpr int kErrDepTimeout = 2;
constexpr int kSweepPolls = 1 << 21;  // about 0.2 s of polling before a wait gives up
constexpr int kBandWarpsPerItem = kThreads / 32;
constexpr int kSweepMaxRows = 2048;   // row entries (velocity and stress rows): tile grids up to 1024 rows

struct SweepArgs {
    int* queue;            // [0] next item, [1] blocks that left (both zero between launches)
    int* done;             // completion counters: [0, tz) velocity rows, [tz, 2tz) stress rows,
                           // [2tz] velocity band items, [2tz+1] stress band items
    int n_items, n_rec;    // items per launch; receiver items (the first ones)
    int vb0, sb0;          // first velocity / stress band item, counted after the receiver items
    int epoch;             // launches of this run before this one
    int tiles_z, band_row0;  // tile rows; first tile row holding row nz-nbc-2 (the band passes read it)
    int n_vband, n_sband;  // band items (kBandWarpsPerItem band warps each) per launch
    int prefetch_ahead;    // items between an item and the item whose DRAM boxes it prefetches (0 = none)
    int chunk, n_chunks;   // tiles per row item; row items per tile row (the last may be shorter)
    // Row entries in queue order, n_chunks items each: the tile row, plus
    // 0x8000 for a stress row.  The band items sit at vb0 and sb0 between them.
    uint16_t rows[kSweepMaxRows];
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

// Item -> (kind, tile row, chunk of the row or item of the band pass), from the kernel
// parameters alone (no memory access on the way to an item's loads).
struct SweepJob {
    int kind, row, idx;
};
__device__ __forceinline__ SweepJob sweep_decode(const SweepArgs& S, int tiles_x, int item) {
    int i = item - S.n_rec;
    if (i < 0) return {kSweepRecv, 0, item};
    if (i >= S.vb0 && i < S.vb0 + S.n_vband) return {kSweepVBand, 0, i - S.vb0};
    if (i >= S.sb0 && i < S.sb0 + S.n_sband) return {kSweepSBand, 0, i - S.sb0};
    if (i >= S.sb0) i -= S.n_sband;
    if (i >= S.vb0) i -= S.n_vband;
    const int e = i / S.n_chunks;
    const int code = S.rows[e];
    return {(code & 0x8000) ? kSweepSRow : kSweepVRow, code & 0x7fff, i - e * S.n_chunks};
}

// Shared memory of the swept step: the larger tile layout, or the band
// warps' staging (two chunks and a weight table per warp).
__host__ __device__ constexpr int sweep_band_tab(int nbc) { return (nbc + 2 + 31) / 32 * 32; }
__host__ inline size_t sweep_band_smem(int nbc) {
    return (size_t)kBandWarpsPerItem * (kMarchStage + sweep_band_tab(nbc)) * 4;
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

__device__ __forceinline__ int ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void red_release_add(int* p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread 0: waits for the items a job reads -- up to four counters read
// together, then one acquire fence.  False (status set) if they are not
// complete within kSweepPolls polls or another block has failed.
static __device__ inline bool sweep_deps(const SweepLaunch& L, const SweepJob& j) {
    const SweepArgs& S = L.S;
    const int tz = S.tiles_z, e1 = S.epoch + 1, tx = L.T.tiles_x;
    if (j.kind == kSweepVBand || j.kind == kSweepSBand) {
        // the band pass reads rows band_row0 .. tz-1: wait for each (a few)
        const int base = j.kind == kSweepVBand ? 0 : tz;
        for (int r = S.band_row0; r < tz; ++r) {
            bool ok = ld_relaxed(S.done + base + r) >= e1 * tx;
            for (int it = 0; !ok && it < kSweepPolls; ++it) {
                __nanosleep(64);
                ok = ld_relaxed(S.done + base + r) >= e1 * tx;
                if (!ok && *reinterpret_cast<volatile int*>(L.T.status)) return false;
            }
            if (!ok) {
                atomicCAS(L.T.status, 0, kErrDepTimeout);
                return false;
            }
        }
        fence_acq_rel_gpu();
        return true;
    }
    if (j.kind != kSweepSRow) return true;
    // velocity rows row-1 .. row+1 (clamped; repeats are harmless) and, for a
    // row whose inputs reach the bottom band, the velocity band pass
    const int r0 = max(j.row - 1, 0), r2 = min(j.row + 1, tz - 1), r1 = min(r0 + 1, r2);
    const bool band = reads_band_rows(L.Ps, j.row * kTZ);
    const int* c3 = band ? S.done + 2 * tz : S.done + r2;
    const int t = e1 * tx, t3 = band ? e1 * S.n_vband : t;
    for (int it = 0;; ++it) {
        const int v0 = ld_relaxed(S.done + r0), v1 = ld_relaxed(S.done + r1), v2 = ld_relaxed(S.done + r2),
                  v3 = ld_relaxed(c3);
        if (v0 >= t && v1 >= t && v2 >= t && v3 >= t3) break;
        if (it >= kSweepPolls) {
            atomicCAS(L.T.status, 0, kErrDepTimeout);
            return false;
        }
        if (*reinterpret_cast<volatile int*>(L.T.status)) return false;
        __nanosleep(64);
    }
    fence_acq_rel_gpu();
    return true;
}

// The DRAM boxes of tile `tile` of a row item into L2: a velocity tile's
// boxes, or the medium boxes of a stress tile (its tau and v boxes come from
// L2 already).
template <int M>
__device__ void sweep_prefetch_tile(const SweepLaunch& L, bool vel, int tile) {
    if (vel) {
        prefetch_vel<M>(L.Pv, L.T, refs_of(L.vm), tile);
    } else {
        if (tile >= L.T.n_tile_blocks) return;
        const TileKind k = classify(L.Ps, L.T, tile);
        if (k.generic) return;
        tma_prefetch_2d(&L.sm.lam, k.x0, k.z0);
        tma_prefetch_2d(&L.sm.mu, k.x0, k.z0);
        tma_prefetch_2d(&L.sm.mxz, k.x0, k.z0);
    }
}

// The first tile of item `item`, if it is a row item.
template <int M>
__device__ void sweep_prefetch(const SweepLaunch& L, int item) {
    if (item >= L.S.n_items) return;
    const SweepJob j = sweep_decode(L.S, L.T.tiles_x, item);
    if (j.kind == kSweepVRow || j.kind == kSweepSRow)
        sweep_prefetch_tile<M>(L, j.kind == kSweepVRow, j.row * L.T.tiles_x + j.idx * L.S.chunk);
}

// The rare items out of line, so the loop over fast tiles stays compact in
// the instruction cache.
template <int M, bool VEL>
__device__ __noinline__ void sweep_edge_tile(const SweepLaunch& L, const TileKind& k, float* smem) {
    edge_tile<M, VEL>(VEL ? L.Pv : L.Ps, L.T, k.x0, k.z0, k.x_end, smem, L.Pv.src_w);
}
static __device__ __noinline__ void sweep_band_item(const SweepLaunch& L, int kind, int idx, float* smem) {
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
}

// Persistent blocks: thread 0 takes an item and waits for its inputs; warp 1
// publishes the finished item; a row item's tiles run one after the other,
// each prefetching the next one's DRAM boxes into L2.
template <int M>
__global__ void __launch_bounds__(kThreads, kTileBlocks<M>) sweep_kernel(const __grid_constant__ SweepLaunch L) {
    extern __shared__ __align__(128) float smem[];
    __shared__ int s_job[3];  // kind (-1: leave), tile row, chunk or band item
    const SweepArgs& S = L.S;
    const int tx = L.T.tiles_x;
    for (;;) {
        if (threadIdx.x == 0) {
            SweepJob j{-1, 0, 0};
            const int item = atomicAdd(S.queue, 1);
            if (item < S.n_items && *reinterpret_cast<volatile int*>(L.T.status) == 0) {
                j = sweep_decode(S, tx, item);
                if (sweep_deps(L, j)) {
                    fence_proxy_async_global();  // the waited-for stores before this item's TMA loads
                    if (S.prefetch_ahead > 0) sweep_prefetch<M>(L, item + S.prefetch_ahead);
                } else {
                    j.kind = -1;
                }
            }
            s_job[0] = j.kind;
            s_job[1] = j.row;
            s_job[2] = j.idx;
        }
        __syncthreads();
        const int kind = s_job[0], row = s_job[1], idx = s_job[2];
        if (kind < 0) break;
        int n_done = 1;  // what the item adds to its counter
        if (kind == kSweepVRow || kind == kSweepSRow) {
            const bool vel = kind == kSweepVRow;
            const int t0 = idx * S.chunk, t1 = min(t0 + S.chunk, tx);
            n_done = t1 - t0;
            for (int t = t0; t < t1; ++t) {
                const int tile = row * tx + t;
                if (threadIdx.x == 0 && t + 1 < t1) sweep_prefetch_tile<M>(L, vel, tile + 1);
                uint64_t* bars = nullptr;  // a fast tile's mbarriers
                if (vel) {
                    const TileKind k = classify(L.Pv, L.T, tile);
                    if (k.generic) {
                        sweep_edge_tile<M, true>(L, k, smem);
                    } else {
                        fast_vel<M>(L.Pv, L.T, refs_of(L.vm), k.x0, k.z0, k.x_end, k.band, k.rim, smem, L.Pv.src_w);
                        bars = fast_tile_bars<M>(smem, true, L.T.iso != 0);
                    }
                } else {
                    const TileKind k = classify(L.Ps, L.T, tile);
                    if (k.generic) {
                        sweep_edge_tile<M, false>(L, k, smem);
                    } else {
                        fast_str<M>(L.Ps, L.T, refs_of(L.sm), k.x0, k.z0, k.x_end, k.band, k.rim, smem, L.Ps.src_w);
                        bars = fast_tile_bars<M>(smem, false, true);
                    }
                }
                __syncthreads();  // the tile's stores are done and its shared memory is free
                if (threadIdx.x == 0 && bars) {
                    mbar_inval(bars);
                    mbar_inval(bars + 1);
                }
            }
        } else {
            if (kind == kSweepVBand || kind == kSweepSBand) {
                sweep_band_item(L, kind, idx, smem);
            } else {
                record_block(L.Pv, idx, L.Pv.rec_k);
            }
            __syncthreads();  // the item's stores are done and its shared memory is free
        }
        if (threadIdx.x == 32 && kind != kSweepRecv) {
            const int tz = S.tiles_z;
            const int c = kind == kSweepVRow ? row : kind == kSweepSRow ? tz + row : kind == kSweepVBand ? 2 * tz : 2 * tz + 1;
            fence_proxy_async_global();
            red_release_add(S.done + c, n_done);
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
