// step_march.cuh -- the fused time step: one launch per step computes the
// velocity and the stress update of every cell (time_stepper.jl:39-63), so
// each field and medium array crosses HBM once per step (read five fields and
// five medium arrays, write five fields: 60 B per cell with dx == dz).
//
// Work split.  The grid is cut into column strips of W output columns (W = 56
// for M <= 4) and each strip into row segments; one block owns one
// (strip, segment) and marches down it in blocks of kMR = 16 rows.  At
// iteration t it computes
//   velocity block t   rows za - M + 16t .. +16, over the strip plus an
//                      HV-column halo on each side (64 columns: the stress
//                      of the strip's edge columns reads them), and
//   stress block t-1   rows za + 16(t-1) .. +16, over the strip's own columns,
// from velocity blocks t-1 and t, which stay in a shared-memory ring of three
// blocks.  New velocities never go back to HBM before the stress reads them;
// the velocity halo and the rows above a segment are recomputed, and the tau
// boxes' overlap is served by L2.
//
// Data movement.  Thread 0 loads each iteration's tau box (txx, tzz, txz over
// 72 x (16 + 2M) cells: the velocity stencil's inputs and the stress's
// step-start values) by TMA into a four-stage ring, two iterations ahead, and
// prefetches into L2 the boxes of the pointwise operands (vx, vz, buoyancy,
// lam, mu, mu_xz), which the threads read with 128-bit loads.  Stage t is
// read by velocity block t and stress block t-1, so stage t+2 is loaded into
// the slot of stage t-2 once every thread has passed iteration t's barrier.
//
// Boundary rules, all inside the march:
//   left/right HABC (boundary.jl:76-85): strips whose columns reach a band
//     exchange their pre-HABC values through shared memory and apply the
//     rules of step_common.cuh; the host's plan (march_plan) admits a layout
//     only if every rule a strip needs reads columns the strip computes;
//   bottom band and corners (boundary.jl:88-132): a recurrence along j; the
//     blocks that hold band rows march them in order, one warp per 28-column
//     strip and field, with band_march's lane rules and shuffles;
//   free surface (boundary.jl:168-181): tzz = txz = 0 in rows pad-5..pad;
//   source (source_receiver.jl:18-30): added to the smem copy of a tau box;
//   receivers (source_receiver.jl:65-77): record blocks appended to the grid
//     read the step-start copy, as in the split launches.
// The fused step needs a free surface (no top HABC band) and M <= 4; other
// configurations run the split launches.
#pragma once

#include "step_tiled.cuh"

namespace fomo {

constexpr int kMR = 16;            // rows per block
constexpr int kMVW = 64;           // velocity columns of a strip, halo included
constexpr int kMRowsPerThread = 1;  // rows of a 16-row block each thread updates (4 columns each; 2 measured slower)
constexpr int kMThreads = 16 * kMR / kMRowsPerThread;  // 16 column groups x 16 rows
constexpr int kMStages = 4;        // tau box stages
constexpr int kMRing = 3;          // velocity blocks kept
constexpr int kMMaxSegs = 64;

template <int M>
struct MGeo {
    static_assert(M >= 1 && M <= 4, "the fused step covers M <= 4");
    static constexpr int HV = 4;                    // velocity halo columns (>= M, 16-byte aligned)
    static constexpr int W = kMVW - 2 * HV;         // output columns of a strip
    static constexpr int TW = kMVW + 2 * HV;        // tau box width
    static constexpr int TH = kMR + 2 * M;          // tau box rows
    static constexpr int TAU = (TW * TH + 31) / 32 * 32;  // floats of one field's box (128-byte multiple)
    static constexpr int STAGE = 3 * TAU;
    static constexpr int RING_ROWS = kMRing * kMR;  // 48 rows of the ring proper
    // The first 2M rows are mirrored after the ring, so a stress window (2M+1
    // rows from any ring row) never wraps.
    static constexpr int RING = (RING_ROWS + 2 * M) * kMVW;  // floats of one field's ring
};

// Launch-wide parameters of the fused step (besides StepParams).
struct MarchArgs {
    const float* b[4];     // buoyancy dtx/rho_vx, dtz/rho_vx, dtx/rho_vz, dtz/rho_vz
    int iso;
    int* status;
    int* queue;            // [0] next item, [1] blocks that left (both zero between launches)
    int n_rec_items;       // receiver items after the strip-segment items
    int n_strips, n_segs, n_items;
    int x_last;            // first output column of the last (right-aligned) strip
    int n_edge, n_segs_e;  // edge strips (the first and the last: HABC side rules) and their segments
    int seg_z[kMMaxSegs + 1];   // interior strips' segment s: stress rows [seg_z[s], seg_z[s+1])
    int seg_ze[kMMaxSegs + 1];  // edge strips' segments (finer: their items cost more)
};

// Descriptors: tau boxes (TW x TH) of the step-start copy; L2-prefetch boxes
// (64 x 16) of the pointwise operands.
struct MarchMaps {
    CUtensorMap xx, zz, xz;        // halo boxes of txx, tzz, txz (copy a)
    CUtensorMap vx, vz;            // tile boxes of vx, vz (copy a)
    CUtensorMap b0, b1, b2, b3;    // tile boxes of the buoyancy arrays
    CUtensorMap lam, mu, mxz;      // tile boxes of the medium
};

template <int M>
__host__ __device__ constexpr size_t march_smem_floats() {
    using G = MGeo<M>;
    return (size_t)kMStages * G::STAGE + 2 * (size_t)G::RING + 3 * kMVW;
}
template <int M>
__host__ __device__ constexpr size_t march_smem_bytes() {
    return march_smem_floats<M>() * 4 + kMStages * 8 + 16;
}

__device__ __forceinline__ bool mbar_wait_parity(uint64_t* bar, uint32_t parity, int* status) {
    for (int it = 0; it < kWaitPolls; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicCAS(status, 0, kErrTmaTimeout);
    return false;
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// d = sum_l a_l (w[M+l-1] - w[M-l]) over a 2M-row window (one row per thread),
// in the reference's accumulation order.
template <int M>
__device__ __forceinline__ float4 zderiv1(const StepParams& P, const float4 (&w)[2 * M]) {
    float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int l = 1; l <= M; ++l) {
        const float al = P.a[l - 1];
        d.x = fadd(fmul(al, fsub(w[M + l - 1].x, w[M - l].x)), d.x);
        d.y = fadd(fmul(al, fsub(w[M + l - 1].y, w[M - l].y)), d.y);
        d.z = fadd(fmul(al, fsub(w[M + l - 1].z, w[M - l].z)), d.z);
        d.w = fadd(fmul(al, fsub(w[M + l - 1].w, w[M - l].w)), d.w);
    }
    return d;
}

// x-derivative of 4 columns from a 12-wide window starting HV = 4 cells left
// of the first column; S = 0: f[i+l-1] - f[i-l], S = 1: f[i+l] - f[i-l+1].
template <int M, int S>
__device__ __forceinline__ float4 xderiv1(const StepParams& P, const float* row) {
    float w[12];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const float4 v = lds4(row + 4 * q);
        w[4 * q] = v.x;
        w[4 * q + 1] = v.y;
        w[4 * q + 2] = v.z;
        w[4 * q + 3] = v.w;
    }
    float d[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float acc = 0.f;
#pragma unroll
        for (int l = 1; l <= M; ++l) acc = fadd(fmul(P.a[l - 1], fsub(w[4 + c + l - 1 + S], w[4 + c - l + S])), acc);
        d[c] = acc;
    }
    return make_float4(d[0], d[1], d[2], d[3]);
}

__device__ __forceinline__ float4 add4(float4 a, float4 b) {
    return make_float4(fadd(a.x, b.x), fadd(a.y, b.y), fadd(a.z, b.z), fadd(a.w, b.w));
}
__device__ __forceinline__ float4 mul4(float4 a, float4 b) {
    return make_float4(fmul(a.x, b.x), fmul(a.y, b.y), fmul(a.z, b.z), fmul(a.w, b.w));
}
__device__ __forceinline__ float4 mul4s(float4 a, float s) {
    return make_float4(fmul(a.x, s), fmul(a.y, s), fmul(a.z, s), fmul(a.w, s));
}

// Values of one field over a shared-memory row-major region whose row r0
// holds grid row z0 and whose column 0 is grid column xs (rows wrap after
// `rows`).
struct SmemRows {
    const float* base;
    int xs, z0, r0, rows, pitch;
    __device__ float operator()(int i, int j) const {
        int r = r0 + (j - z0);
        r = r >= rows ? r - rows : (r < 0 ? r + rows : r);
        return base[r * pitch + (i - xs)];
    }
};


// The bottom-band recurrence (rows nz-nbc-1 .. nz-2) of one field over the
// band rows [ja, jb) of one block: `pre` holds the block's values after the
// stencil update (band rows) and final values (rows above), and receives the
// finals in place.  One warp per 28-column strip: lane l holds column
// xs - 2 + l; lanes 2..29 write back, and store their own columns
// [own_lo, own_hi).  Columns [c_lo, c_hi) hold values.  `prev` (column 0 =
// pre_xs), when given, holds the finals of row ja - 1; otherwise that row is
// read from `pre`.  The n_warps warps of one field (its strips) call it
// together: they meet at a named barrier between reading and writing back.
// The lane rules are band_march's.
__device__ __forceinline__ void march_band_rows(const StepParams& P, const float* tab, const float* oin, float* oout,
                                                float* pre, int pre_pitch, int pre_xs, int pre_z0, int pre_r0,
                                                int pre_rows, int c_lo, int c_hi, int own_lo, int own_hi, int xs,
                                                int ja, int jb, const float* prev, int n_warps) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int b = P.nbc, nx = P.nx, nz = P.nz, r0 = nx - b - 1;
    const int i = xs - 2 + lane;
    const bool have = i >= c_lo && i < c_hi && i >= 0 && i < nx;  // the lane's column holds a value
    const bool rim = i <= 0 || i >= nx - 1;
    const bool left = i >= 1 && i <= b;
    const bool corner = left || (i >= r0 && i <= nx - 2);
    const bool redo = i == b || (i > r0 - 1 && i <= nx - 2 && right_chunk_start(nx, b, i));
    const int nb = min(max(lane + (left ? 1 : -1), 0), 31);
    const int dxi = max(min(i, nx - 1 - i), 0);
    auto at = [&](int j) -> float* {
        int r = pre_r0 + (j - pre_z0);
        r = r >= pre_rows ? r - pre_rows : (r < 0 ? r + pre_rows : r);
        return pre + r * pre_pitch + (i - pre_xs);
    };
    float fprev = have ? (prev ? prev[i - pre_xs] : *at(ja - 1)) : 0.f;
    float ovp = have ? __ldg(oin + cell(P, i, ja - 1)) : 0.f;
    const bool store = have && lane >= 2 && lane < 30;
    const bool own = store && i >= own_lo && i < own_hi;
    // Every lane reads its column's values of the block's band rows before any
    // warp writes a final back: the margin lanes read columns that the
    // neighbouring warp stores.
    float pvs[kMR];
#pragma unroll
    for (int r = 0; r < kMR; ++r) pvs[r] = (have && ja + r < jb) ? *at(ja + r) : 0.f;
    asm volatile("bar.sync 1, %0;" ::"r"(n_warps * 32) : "memory");  // the n_warps warps of this round
#pragma unroll
    for (int r = 0; r < kMR; ++r) {
        const int j = ja + r;
        if (j >= jb) break;
        const float pv = pvs[r];
        const float ov = have ? __ldg(oin + cell(P, i, j)) : 0.f;
        const float w = __ldg(tab + min(min(dxi, nz - 1 - j), b + 1));
        const float pv_nb = __shfl_sync(FULL, pv, nb);
        const float ov_nb = __shfl_sync(FULL, ov, nb);
        const float sz = edge_sum(P.qz, P.qt_z, P.qxt, fprev, ov, ovp);
        const float fc = blend_corner(w, pv, edge_sum(P.qx, P.qt_x, P.qxt, pv_nb, ov, ov_nb), sz);
        const float fe = blend_edge(w, pv, sz);
        const float fa = rim ? pv : (corner ? fc : fe);
        const float fa_nb = __shfl_sync(FULL, fa, nb);
        const float fb = blend_corner(w, pv, edge_sum(P.qx, P.qt_x, P.qxt, fa_nb, ov, ov_nb), sz);
        const float fin = redo ? fb : fa;
        if (store) *at(j) = fin;
        if (own) oout[cell(P, i, j)] = fin;
        fprev = fin;
        ovp = ov;
    }
}

// The descriptors one item uses: its shot's tau boxes and, when the item
// prefetches, the L2-prefetch boxes (pf == false: none are read).
struct MarchMapRefs {
    const CUtensorMap *xx, *zz, *xz;
    const CUtensorMap *vx, *vz, *b0, *b1, *b2, *b3, *lam, *mu, *mxz;
    bool pf;
};
__device__ __forceinline__ MarchMapRefs refs_of(const MarchMaps& m) {
    return {&m.xx, &m.zz, &m.xz, &m.vx, &m.vz, &m.b0, &m.b1, &m.b2, &m.b3, &m.lam, &m.mu, &m.mxz, true};
}

// Item `item` of a shot's fused step: the edge strips' items first (they
// apply the side rules), then the interior strips'; bottom segments first in
// each (they march the band).
__device__ __forceinline__ void march_item_of(const MarchArgs& A, int item, int* strip, int* seg, bool* edge) {
    const int ne = A.n_edge * A.n_segs_e;
    if (item < ne) {
        *edge = true;
        *seg = A.n_segs_e - 1 - item / A.n_edge;
        *strip = item % A.n_edge == 0 ? 0 : A.n_strips - 1;
    } else {
        item -= ne;
        const int ni = A.n_strips - A.n_edge;
        *edge = false;
        *seg = A.n_segs - 1 - item / ni;
        *strip = 1 + item % ni;
    }
}

// Thread 0: TMA loads of the tau boxes of iteration t (the block's stage
// number g: slot g % kMStages) and, with mp.pf, L2 prefetches of the
// pointwise operands' boxes.
template <int M>
__device__ __forceinline__ void march_issue(const MarchArgs& A, const MarchMapRefs& mp, float* stage, uint64_t* full,
                                            int x0, int za, int t, int g) {
    using G = MGeo<M>;
    const int s = g % kMStages;
    float* dst = stage + s * G::STAGE;
    const int vr0 = za - M + t * kMR, xa = x0 - G::HV;
    mbar_expect_tx(full + s, 3 * G::TW * G::TH * 4);  // the bytes of the three boxes
    tma_load_2d(dst, mp.xx, x0 - 2 * G::HV, vr0 - M, full + s);
    tma_load_2d(dst + G::TAU, mp.zz, x0 - 2 * G::HV, vr0 - M, full + s);
    tma_load_2d(dst + 2 * G::TAU, mp.xz, x0 - 2 * G::HV, vr0 - M, full + s);
    if (mp.pf) {
        tma_prefetch_2d(mp.vx, xa, vr0);
        tma_prefetch_2d(mp.vz, xa, vr0);
        tma_prefetch_2d(mp.b0, xa, vr0);
        tma_prefetch_2d(mp.b2, xa, vr0);
        if (!A.iso) {
            tma_prefetch_2d(mp.b1, xa, vr0);
            tma_prefetch_2d(mp.b3, xa, vr0);
        }
        tma_prefetch_2d(mp.lam, x0, vr0 + M);
        tma_prefetch_2d(mp.mu, x0, vr0 + M);
        tma_prefetch_2d(mp.mxz, x0, vr0 + M);
    }
}

// Rows of a segment's velocity block t that its stress reads (the last
// block feeds only 2M stress rows): [vr0, march_v_hi).
template <int M>
__device__ __forceinline__ int march_v_hi(int vr0, int t, int n_it, int zb) {
    return min(vr0 + (t < n_it - 1 ? kMR : 2 * M), zb + M);
}

// z-derivatives of RT consecutive rows from a (2M + RT - 1)-row window:
// d[rr] = sum_l a_l (w[rr+M+l-1] - w[rr+M-l]), in the reference's order.
template <int M, int RT>
__device__ __forceinline__ void zderivR(const StepParams& P, const float4 (&w)[2 * M + RT - 1], float4 (&d)[RT]) {
#pragma unroll
    for (int rr = 0; rr < RT; ++rr) {
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int l = 1; l <= M; ++l) {
            const float al = P.a[l - 1];
            a.x = fadd(fmul(al, fsub(w[rr + M + l - 1].x, w[rr + M - l].x)), a.x);
            a.y = fadd(fmul(al, fsub(w[rr + M + l - 1].y, w[rr + M - l].y)), a.y);
            a.z = fadd(fmul(al, fsub(w[rr + M + l - 1].z, w[rr + M - l].z)), a.z);
            a.w = fadd(fmul(al, fsub(w[rr + M + l - 1].w, w[rr + M - l].w)), a.w);
        }
        d[rr] = a;
    }
}

// One (strip, segment) of a shot's time step; src_w is the wavelet sample
// added to txx and tzz at the source cell this step.  g is the block's
// running stage number (stage slots and mbarrier phases continue across the
// items a block runs); it advances by the item's iterations.  The caller
// has synchronised the block since its previous item.  Returns false (all
// threads alike) if a TMA load did not land: the status word holds the error.
// s_err: two shared words for the block's flag.  Each thread updates 4
// columns x kMRowsPerThread rows of every 16-row block.
template <int M>
__device__ __forceinline__ bool march_item(const StepParams& P, const MarchArgs& A, const MarchMapRefs& mp,
                                           int strip, int seg, bool edge, float src_w, int& g, int* s_err) {
    using G = MGeo<M>;
    constexpr int RT = kMRowsPerThread;
    extern __shared__ __align__(128) float smem[];
    const bool last_strip = strip == A.n_strips - 1;
    const int x0 = last_strip ? A.x_last : strip * G::W;
    const int x_end = last_strip ? min(x0 + G::W, (P.nx + 3) / 4 * 4) : min(x0 + G::W, A.x_last);
    const int xa = x0 - G::HV;
    const int* segz = edge ? A.seg_ze : A.seg_z;
    const int za = segz[seg], zb = segz[seg + 1];
    const int n_it = (zb - za + kMR - 1) / kMR + 1;  // velocity blocks 0..n_it-1; stress blocks 0..n_it-2
    const int nx = P.nx, nz = P.nz, b = P.nbc, pitch = P.pitch;
    const int j0 = nz - b - 1;                        // first bottom-band row
    const int ecols = max(b + 2, M);
    const bool side = xa < ecols || xa + kMVW > nx - ecols;  // block-uniform: side HABC or rim columns
    const int g0 = g;
    g += n_it;

    float* stage = smem;
    float* ring = smem + kMStages * G::STAGE;          // [2 fields][48 rows + mirror][64]
    float* s_last = ring + 2 * G::RING;                // [3][64] stress finals of a block's last row
    uint64_t* full = reinterpret_cast<uint64_t*>(s_last + 3 * kMVW);

    const int tx = threadIdx.x & 15, rp = threadIdx.x >> 4;
    const int ty = rp * RT;              // the thread's first row within a 16-row block
    const int xv = xa + 4 * tx;          // first column of the thread's velocity cells
    const int xs = x0 + 4 * tx;          // first column of the thread's stress cells (tx < W/4)
    const bool s_col = tx < G::W / 4;
    const bool v_own = xv >= x0 && xv < x_end;
    const bool s_own = s_col && xs < x_end;
    const bool v_in = xv >= 0 && xv < nx;
    const bool s_in = s_col && xs < nx;
    const int warp = threadIdx.x >> 5;

    if (threadIdx.x == 0) {
        fence_proxy_async_smem();  // the previous item's generic accesses of the slots before the TMA refills them
        for (int t = 0; t < min(kMStages, n_it); ++t) march_issue<M>(A, mp, stage, full, x0, za, t, g0 + t);
        s_err[0] = mbar_wait_parity(full + g0 % kMStages, (g0 / kMStages) & 1, A.status) ? 0 : 1;
    }
    // Pointwise operands of velocity block t, loaded one phase before they are used.
    float4 pvx[RT], pvz[RT], pb0[RT], pb1[RT], pb2[RT], pb3[RT];
    auto load_v = [&](int t) {
        const int vr = za - M + t * kMR;
        const int hi = march_v_hi<M>(vr, t, n_it, zb);
#pragma unroll
        for (int rr = 0; rr < RT; ++rr) {
            const int j = vr + ty + rr;
            pvx[rr] = pvz[rr] = pb0[rr] = pb1[rr] = pb2[rr] = pb3[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (v_in && j >= 0 && j < nz && j < hi) {
                const int c = xv + j * pitch;  // 32-bit offsets (march_plan: pitch * nz < 2^31)
                pvx[rr] = ldg4(P.in[VX] + c);
                pvz[rr] = ldg4(P.in[VZ] + c);
                pb0[rr] = ldg4(A.b[0] + c);
                pb2[rr] = ldg4(A.b[2] + c);
                pb1[rr] = A.iso ? pb0[rr] : ldg4(A.b[1] + c);
                pb3[rr] = A.iso ? pb2[rr] : ldg4(A.b[3] + c);
            }
        }
    };
    load_v(0);
    __syncthreads();
    if (s_err[0]) return false;

    for (int t = 0; t < n_it; ++t) {
        const int gt = g0 + t;
        float* tau = stage + (gt % kMStages) * G::STAGE;
        const int vr0 = za - M + t * kMR;
        const int slot = t % kMRing;
        // medium of stress block t-1, loaded now and used after the velocity
        const int sr0 = za + (t - 1) * kMR;
        float4 mlam[RT], mmu[RT], mmxz[RT];
        bool s_row[RT];
#pragma unroll
        for (int rr = 0; rr < RT; ++rr) {
            const int js = sr0 + ty + rr;
            s_row[rr] = t >= 1 && js < zb && js < nz;
            mlam[rr] = mmu[rr] = mmxz[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (s_row[rr] && s_in) {
                const int c = xs + js * pitch;
                mlam[rr] = ldg4(P.lam + c);
                mmu[rr] = ldg4(P.mu_txx + c);
                mmxz[rr] = ldg4(P.mu_txz + c);
            }
        }
        // ------------------------------------------------ the source, into this stage's copy
        {
            const int si = P.src_i - (x0 - 2 * G::HV), sj = P.src_j - (vr0 - M);
            if (si >= 0 && si < G::TW && sj >= 0 && sj < G::TH) {  // block-uniform
                if (threadIdx.x == 0) {
                    tau[sj * G::TW + si] = fadd(tau[sj * G::TW + si], src_w);
                    tau[G::TAU + sj * G::TW + si] = fadd(tau[G::TAU + sj * G::TW + si], src_w);
                }
                __syncthreads();
            }
        }
        // ------------------------------------------------ velocity block t
        {
            const int v_hi = march_v_hi<M>(vr0, t, n_it, zb);
            float4 ox[RT], oz[RT];
            bool row_ok[RT];
            bool any = false;
#pragma unroll
            for (int rr = 0; rr < RT; ++rr) {
                const int j = vr0 + ty + rr;
                row_ok[rr] = j < v_hi && j >= 0 && j < nz;
                any = any || row_ok[rr];
                ox[rr] = oz[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            if (any && v_in) {
                float4 d1[RT], d3[RT];
#pragma unroll
                for (int rr = 0; rr < RT; ++rr) {
                    const float* rxx = tau + (ty + rr + M) * G::TW + 4 * tx;  // windows from column xv - 4
                    const float* rxz = tau + 2 * G::TAU + (ty + rr + M) * G::TW + 4 * tx;
                    d1[rr] = xderiv1<M, 0>(P, rxx);   // dtxx/dx: txx[i+l-1] - txx[i-l]
                    d3[rr] = xderiv1<M, 1>(P, rxz);   // dtxz/dx: txz[i+l] - txz[i-l+1]
                }
                float4 wz[2 * M + RT - 1], d2[RT], d4[RT];
#pragma unroll
                for (int q = 0; q < 2 * M + RT - 1; ++q)
                    wz[q] = lds4(tau + 2 * G::TAU + (ty + q) * G::TW + 4 * tx + G::HV);
                zderivR<M, RT>(P, wz, d2);        // dtxz/dz: txz[j+l-1] - txz[j-l]
#pragma unroll
                for (int q = 0; q < 2 * M + RT - 1; ++q)
                    wz[q] = lds4(tau + G::TAU + (ty + 1 + q) * G::TW + 4 * tx + G::HV);
                zderivR<M, RT>(P, wz, d4);        // dtzz/dz: tzz[j+l] - tzz[j-l+1]
#pragma unroll
                for (int rr = 0; rr < RT; ++rr) {
                    const int j = vr0 + ty + rr;
                    ox[rr] = add4(pvx[rr], add4(mul4(pb0[rr], d1[rr]), mul4(pb1[rr], d2[rr])));
                    oz[rr] = add4(pvz[rr], add4(mul4(pb2[rr], d3[rr]), mul4(pb3[rr], d4[rr])));
                    if (side || j < M || j > nz - 1 - M) {
#pragma unroll
                        for (int c4 = 0; c4 < 4; ++c4)
                            if (!in_stencil(P, xv + c4, j)) {
                                set_comp(ox[rr], c4, comp(pvx[rr], c4));
                                set_comp(oz[rr], c4, comp(pvz[rr], c4));
                            }
                    }
                }
            }
            float* rvx = ring + (slot * kMR + ty) * kMVW + 4 * tx;  // ring row of the thread's first row
            float* rvz = rvx + G::RING;
#pragma unroll
            for (int rr = 0; rr < RT; ++rr) {
                *reinterpret_cast<float4*>(rvx + rr * kMVW) = ox[rr];
                *reinterpret_cast<float4*>(rvz + rr * kMVW) = oz[rr];
            }
            const bool band_rows = v_hi > j0 && vr0 <= nz - 2;  // block-uniform
            if (side || band_rows) {
                __syncthreads();  // pre values of the block in the ring
                if (side) {  // left/right HABC (free surface: rows nbc .. nz-nbc-2)
                    const SmemRows pre_x{ring, xa, vr0, slot * kMR, G::RING_ROWS, kMVW};
                    const SmemRows pre_z{ring + G::RING, xa, vr0, slot * kMR, G::RING_ROWS, kMVW};
                    const HabcPoint<SmemRows> hx{P, pre_x, P.in[VX], P.w_tab[0]};
                    const HabcPoint<SmemRows> hz{P, pre_z, P.in[VZ], P.w_tab[1]};
#pragma unroll
                    for (int rr = 0; rr < RT; ++rr) {
                        const int j = vr0 + ty + rr;
                        if (!row_ok[rr] || j < b || j > j0 - 1) continue;
#pragma unroll
                        for (int c4 = 0; c4 < 4; ++c4) {
                            const int i = xv + c4;
                            // the rule's neighbours (left: i+1; right: i-1, i-2) lie in the strip's
                            // columns for every cell the stress reads (march_plan checks it)
                            if (lr_band_cell(P, i, j) && (i <= b ? i + 1 < xa + kMVW : i - 2 >= xa)) {
                                set_comp(ox[rr], c4, hx.final_value(i, j));
                                set_comp(oz[rr], c4, hz.final_value(i, j));
                            }
                        }
                    }
                }
                __syncthreads();
#pragma unroll
                for (int rr = 0; rr < RT; ++rr) {
                    *reinterpret_cast<float4*>(rvx + rr * kMVW) = ox[rr];
                    *reinterpret_cast<float4*>(rvz + rr * kMVW) = oz[rr];
                }
                if (band_rows) {
                    __syncthreads();
                    // one round per field, one warp per 28-column strip
                    for (int f = 0; f < 2; ++f)
                        if (warp < 3)
                            march_band_rows(P, w_table(P, f), in_field(P, VX + f), out_field(P, VX + f),
                                            ring + f * G::RING, kMVW, xa, vr0, slot * kMR, G::RING_ROWS, xa,
                                            xa + kMVW, x0, x_end, xa + 28 * warp, max(vr0, j0), min(v_hi, nz - 1),
                                            nullptr, 3);
                    __syncthreads();
#pragma unroll
                    for (int rr = 0; rr < RT; ++rr) {
                        ox[rr] = *reinterpret_cast<const float4*>(rvx + rr * kMVW);
                        oz[rr] = *reinterpret_cast<const float4*>(rvz + rr * kMVW);
                    }
                }
            }
#pragma unroll
            for (int rr = 0; rr < RT; ++rr) {
                const int j = vr0 + ty + rr;
                if (slot == 0 && ty + rr < 2 * M) {  // the mirror of the ring's first rows
                    *reinterpret_cast<float4*>(rvx + (rr + G::RING_ROWS) * kMVW) = ox[rr];
                    *reinterpret_cast<float4*>(rvz + (rr + G::RING_ROWS) * kMVW) = oz[rr];
                }
                // the segment's own rows (the rows above are the previous segment's); band rows were
                // stored by the march
                if (row_ok[rr] && v_own && j >= za && j < zb && !(j >= j0 && j <= nz - 2)) {
                    stg4(P.out[VX] + (xv + j * pitch), ox[rr]);
                    stg4(P.out[VZ] + (xv + j * pitch), oz[rr]);
                }
            }
        }
        // velocity block t in the ring; every thread is done with iteration t-1.  Thread 0
        // waits for the next iteration's tau boxes here, so the other threads sleep in the
        // barrier instead of polling.  The flag alternates between two words, so a thread
        // that reads it late still reads the word written before this barrier (thread 0
        // rewrites it only two barriers later).
        if (threadIdx.x == 0)
            s_err[(t + 1) & 1] =
                t + 1 < n_it && !mbar_wait_parity(full + (gt + 1) % kMStages, ((gt + 1) / kMStages) & 1, A.status);
        __syncthreads();
        if (s_err[(t + 1) & 1]) return false;
        if (threadIdx.x == 0 && t >= 2 && t + 2 < n_it) {
            fence_proxy_async_smem();  // generic accesses of the slot before the TMA overwrites it
            march_issue<M>(A, mp, stage, full, x0, za, t + 2, gt + 2);
        }
        if (t + 1 < n_it) load_v(t + 1);  // velocity block t is done with the current ones
        // ------------------------------------------------ stress block t-1
        if (t >= 1) {
            const float* told = stage + ((gt - 1) % kMStages) * G::STAGE;  // stage t-1: rows from sr0 - 2M
            float4 oxx[RT], ozz[RT], oxz[RT];
            bool any = false;
#pragma unroll
            for (int rr = 0; rr < RT; ++rr) {
                oxx[rr] = ozz[rr] = oxz[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
                any = any || s_row[rr];
            }
            if (any && s_in) {
                float4 txx[RT], tzz[RT], txz[RT], dxx[RT], dzx[RT];
                // ring row of grid row j - M + q for the thread's first row j: r + q (rows past the
                // ring are its mirror)
                const int r = ((t - 1) % kMRing) * kMR + ty;
                const float* rvx = ring + r * kMVW + 4 * tx;
                const float* rvz = rvx + G::RING;
#pragma unroll
                for (int rr = 0; rr < RT; ++rr) {
                    const int bo = (ty + rr + 2 * M) * G::TW + 2 * G::HV + 4 * tx;
                    txx[rr] = lds4(told + bo);
                    tzz[rr] = lds4(told + G::TAU + bo);
                    txz[rr] = lds4(told + 2 * G::TAU + bo);
                    dxx[rr] = xderiv1<M, 1>(P, rvx + (rr + M) * kMVW);  // vx[i+l] - vx[i-l+1]
                    dzx[rr] = xderiv1<M, 0>(P, rvz + (rr + M) * kMVW);  // vz[i+l-1] - vz[i-l]
                }
                float4 wz[2 * M + RT - 1], dzz[RT], dxz[RT];
#pragma unroll
                for (int q = 0; q < 2 * M + RT - 1; ++q) wz[q] = lds4(rvz + q * kMVW + G::HV);
                zderivR<M, RT>(P, wz, dzz);       // vz[j+l-1] - vz[j-l]
#pragma unroll
                for (int q = 0; q < 2 * M + RT - 1; ++q) wz[q] = lds4(rvx + (q + 1) * kMVW + G::HV);
                zderivR<M, RT>(P, wz, dxz);       // vx[j+l] - vx[j-l+1]
#pragma unroll
                for (int rr = 0; rr < RT; ++rr) {
                    const int j = sr0 + ty + rr;
                    const float4 l2m = add4(mlam[rr], mul4s(mmu[rr], 2.f));
                    const float4 ex = mul4s(dxx[rr], P.dtx), ez = mul4s(dzz[rr], P.dtz);
                    oxx[rr] = add4(txx[rr], add4(mul4(l2m, ex), mul4(mlam[rr], ez)));
                    ozz[rr] = add4(tzz[rr], add4(mul4(mlam[rr], ex), mul4(l2m, ez)));
                    oxz[rr] = add4(txz[rr], mul4(mmxz[rr], add4(mul4s(dxz[rr], P.dtz), mul4s(dzx[rr], P.dtx))));
                    if (side || j < M || j > nz - 1 - M) {
#pragma unroll
                        for (int c4 = 0; c4 < 4; ++c4)
                            if (!in_stencil(P, xs + c4, j)) {
                                set_comp(oxx[rr], c4, comp(txx[rr], c4));
                                set_comp(ozz[rr], c4, comp(tzz[rr], c4));
                                set_comp(oxz[rr], c4, comp(txz[rr], c4));
                            }
                    }
                }
            }
            const bool band_rows = sr0 + kMR > j0 && sr0 <= nz - 2 && sr0 < zb;  // block-uniform
            if (side || band_rows) {
                // exchange through the slot of stage t-1 once every thread has read it
                __syncthreads();
                float* sp = stage + ((gt - 1) % kMStages) * G::STAGE;  // [3][16][64], column 0 = x0
                float* sq = sp + ty * kMVW + 4 * tx;
                if (s_col) {
#pragma unroll
                    for (int rr = 0; rr < RT; ++rr) {
                        *reinterpret_cast<float4*>(sq + rr * kMVW) = oxx[rr];
                        *reinterpret_cast<float4*>(sq + kMR * kMVW + rr * kMVW) = ozz[rr];
                        *reinterpret_cast<float4*>(sq + 2 * kMR * kMVW + rr * kMVW) = oxz[rr];
                    }
                }
                __syncthreads();
                if (side && s_in) {
                    const SmemRows p0{sp, x0, sr0, 0, kMR, kMVW};
                    const SmemRows p1{sp + kMR * kMVW, x0, sr0, 0, kMR, kMVW};
                    const SmemRows p2{sp + 2 * kMR * kMVW, x0, sr0, 0, kMR, kMVW};
                    const HabcPoint<SmemRows> h0{P, p0, P.in[TXX], P.w_tab[2]};
                    const HabcPoint<SmemRows> h1{P, p1, P.in[TZZ], P.w_tab[2]};
                    const HabcPoint<SmemRows> h2{P, p2, P.in[TXZ], P.w_tab[2]};
#pragma unroll
                    for (int rr = 0; rr < RT; ++rr) {
                        const int j = sr0 + ty + rr;
                        if (!s_row[rr] || j < b || j > j0 - 1) continue;
#pragma unroll
                        for (int c4 = 0; c4 < 4; ++c4) {
                            const int i = xs + c4;
                            if (lr_band_cell(P, i, j) && (i <= b ? i + 1 < x0 + G::W : i - 2 >= x0)) {
                                set_comp(oxx[rr], c4, h0.final_value(i, j));
                                set_comp(ozz[rr], c4, h1.final_value(i, j));
                                set_comp(oxz[rr], c4, h2.final_value(i, j));
                            }
                        }
                    }
                }
                __syncthreads();
                if (s_col) {
#pragma unroll
                    for (int rr = 0; rr < RT; ++rr) {
                        *reinterpret_cast<float4*>(sq + rr * kMVW) = oxx[rr];
                        *reinterpret_cast<float4*>(sq + kMR * kMVW + rr * kMVW) = ozz[rr];
                        *reinterpret_cast<float4*>(sq + 2 * kMR * kMVW + rr * kMVW) = oxz[rr];
                    }
                }
                if (band_rows) {
                    const int ja = max(sr0, j0), jb = min(min(sr0 + kMR, nz - 1), zb);
                    __syncthreads();
                    // one round per field, one warp per 28-column strip; the row above the first
                    // band row is in this block, or the previous block's last row
                    for (int f = 0; f < 3; ++f)
                        if (warp < 2)
                            march_band_rows(P, P.w_tab[2], in_field(P, TXX + f), out_field(P, TXX + f),
                                            sp + f * kMR * kMVW, kMVW, x0, sr0, 0, kMR, x0, x0 + G::W, x0, x_end,
                                            x0 + 28 * warp, ja, jb, ja == sr0 ? s_last + f * kMVW : nullptr, 2);
                    __syncthreads();
                    if (s_col) {
#pragma unroll
                        for (int rr = 0; rr < RT; ++rr) {
                            oxx[rr] = *reinterpret_cast<const float4*>(sq + rr * kMVW);
                            ozz[rr] = *reinterpret_cast<const float4*>(sq + kMR * kMVW + rr * kMVW);
                            oxz[rr] = *reinterpret_cast<const float4*>(sq + 2 * kMR * kMVW + rr * kMVW);
                        }
                    }
                }
            }
            if (ty + RT == kMR && s_col) {  // the block's last row, read by the next block's band march
                *reinterpret_cast<float4*>(s_last + 4 * tx) = oxx[RT - 1];
                *reinterpret_cast<float4*>(s_last + kMVW + 4 * tx) = ozz[RT - 1];
                *reinterpret_cast<float4*>(s_last + 2 * kMVW + 4 * tx) = oxz[RT - 1];
            }
#pragma unroll
            for (int rr = 0; rr < RT; ++rr) {
                const int j = sr0 + ty + rr;
                if (s_row[rr] && s_own && !(j >= j0 && j <= nz - 2)) {  // band rows were stored by the march
                    if (in_free_surface_rows(P, j)) {
                        ozz[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
                        oxz[rr] = ozz[rr];
                    }
                    stg4(P.out[TXX] + (xs + j * pitch), oxx[rr]);
                    stg4(P.out[TZZ] + (xs + j * pitch), ozz[rr]);
                    stg4(P.out[TXZ] + (xs + j * pitch), oxz[rr]);
                }
            }
        }
    }
    return true;
}

// Thread 0 initialises the block's stage mbarriers once, before its first
// item (their phases then run on across items: march_item's stage numbers);
// the caller's next barrier publishes them.
template <int M>
__device__ __forceinline__ void march_init_barriers() {
    using G = MGeo<M>;
    extern __shared__ __align__(128) float smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kMStages * G::STAGE + 2 * G::RING + 3 * kMVW);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kMStages; ++s) mbar_init(full + s, 1);
        fence_barrier_init();
    }
}

// Work queue of a fused-step launch: a block takes items until none are
// left; the last block to leave resets the queue for the next launch.
__device__ __forceinline__ int march_next(int* queue, int* s_item) {
    if (threadIdx.x == 0) *s_item = atomicAdd(queue, 1);
    __syncthreads();
    return *s_item;
}
__device__ __forceinline__ bool march_leave(int* queue) {  // true in thread 0 of the last block
    if (threadIdx.x != 0) return false;
    __threadfence();
    if (atomicAdd(queue + 1, 1) != (int)gridDim.x - 1) return false;
    queue[0] = 0;
    queue[1] = 0;
    __threadfence();
    return true;
}

// The fused step of one shot: persistent blocks take items from the queue
// A.queue -- the (strip, segment) items, then the receiver blocks of step
// P.rec_k.
template <int M>
__global__ void __launch_bounds__(kMThreads, 2)
    march_kernel(const __grid_constant__ StepParams P, const __grid_constant__ MarchArgs A,
                 const __grid_constant__ MarchMaps mp) {
    __shared__ int s_item, s_err[2];
    int g = 0;
    march_init_barriers<M>();  // published by march_next's barrier
    for (;;) {
        const int item = march_next(A.queue, &s_item);
        if (item >= A.n_items + A.n_rec_items) break;
        if (item < A.n_items) {
            int strip, seg;
            bool edge;
            march_item_of(A, item, &strip, &seg, &edge);
            if (!march_item<M>(P, A, refs_of(mp), strip, seg, edge, P.src_w, g, s_err)) break;
        } else {
            record_block(P, item - A.n_items, P.rec_k);
        }
        __syncthreads();  // the block is done with the item's shared memory and s_item
    }
    march_leave(A.queue);
}

// ---------------------------------------------------------------- many shots per launch
// The batched fused step: one launch per batch step covers up to
// kMarchShots shots, grouped by medium (and HABC width: one layout per
// group).  Inside a group the shots' items are interleaved item-major
// (item = strip-segment item * n + shot), so the shots' copies of one
// (strip, segment) run side by side and the medium's rows come from HBM
// once and from L2 for the others.  The batch step comes from a device
// counter, so every launch of a batch has the same parameters and a run of
// K steps can be captured once into a CUDA graph: each block reads the step
// first, and the last block to leave advances it for the next launch.
// Items of shots outside their step range are skipped; the receiver items
// record step ks-1 of each shot, including the shot's last step one batch
// step later, exactly like the split batch launches.
constexpr int kMarchShots = 12;
constexpr int kMarchGroups = 8;

struct MarchShot {
    StepParams P[2];        // the step reads copy c (P[c].in) and writes copy 1-c (P[c].out), all five fields
    const float* wavelet;
    int n_wavelet;
    int start;              // batch step of the shot's step 1 (>= 1)
    int nt;
    int pad_;
};

struct MarchGroup {
    MarchArgs A;            // the group's layout, buoyancy and status word
    int first, n;           // shots first .. first+n-1
    int item_off;           // the group's first item
    int pad_;
};

struct BatchMarchLaunch {
    int* step;              // step[0]: batch step (1-based) of this launch; step[1]: next item;
                            // step[2]: blocks that left (both zero between launches)
    int n_shots, n_groups, total_items, n_rec_items;
    int rec_off[kMarchShots + 1];  // first receiver item of each shot (after the strip-segment items)
    MarchGroup groups[kMarchGroups];
    MarchShot shot[kMarchShots];
    CUtensorMap tau[kMarchShots][2][3];  // tau boxes (TW x TH) of copy c
};

static_assert(sizeof(BatchMarchLaunch) <= 32764, "kernel parameters above the 32764-byte limit");

template <int M>
__global__ void __launch_bounds__(kMThreads, 2) batch_march_kernel(const __grid_constant__ BatchMarchLaunch L) {
    __shared__ int s_item, s_err[2];
    const int step = *reinterpret_cast<volatile const int*>(L.step);
    int* queue = L.step + 1;  // [0] next item, [1] blocks that left
    int g = 0;
    march_init_barriers<M>();  // published by march_next's barrier
    for (;;) {
        const int item = march_next(queue, &s_item);
        if (item >= L.total_items + L.n_rec_items) break;
        if (item < L.total_items) {
            int gi = 0;
#pragma unroll 1
            for (int h = 1; h < L.n_groups; ++h)
                if (L.groups[h].item_off <= item) gi = h;
            const MarchGroup& G = L.groups[gi];
            const int r = item - G.item_off;
            const int s = G.first + r % G.n;
            const MarchShot& S = L.shot[s];
            const int ks = step - S.start + 1;
            if (ks >= 1 && ks <= S.nt) {
                const int a = (ks - 1) & 1;
                int strip, seg;
                bool edge;
                march_item_of(G.A, r / G.n, &strip, &seg, &edge);
                const MarchMapRefs mp{&L.tau[s][a][0], &L.tau[s][a][1], &L.tau[s][a][2], nullptr, nullptr,
                                      nullptr,         nullptr,         nullptr,         nullptr, nullptr,
                                      nullptr,         nullptr,         false};
                const float src_w = ks <= S.n_wavelet ? __ldg(S.wavelet + ks - 1) : 0.f;
                if (!march_item<M>(S.P[a], G.A, mp, strip, seg, edge, src_w, g, s_err)) break;
            }
        } else {
            const int rb = item - L.total_items;
            int s = 0;
#pragma unroll 1
            while (L.rec_off[s + 1] <= rb) ++s;
            const MarchShot& S = L.shot[s];
            const int ks = step - S.start + 1;
            if (ks >= 2 && ks <= S.nt + 1) record_block(S.P[(ks - 1) & 1], rb - L.rec_off[s], ks - 1);
        }
        __syncthreads();
    }
    // every block has read the step and taken its items once the last one leaves
    if (march_leave(queue)) *reinterpret_cast<volatile int*>(L.step) = step + 1;
}

// Counters of n batched fused-step sets at a table rebuild: set i holds
// counters[4i] = `step`, then its block count and its next item (zero).
static __global__ void march_counters_kernel(int* counters, int n, int step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        counters[4 * i] = step;
        counters[4 * i + 1] = 0;
        counters[4 * i + 2] = 0;
        counters[4 * i + 3] = 0;
    }
}

}  // namespace fomo
