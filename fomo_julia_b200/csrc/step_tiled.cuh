// step_tiled.cuh -- the sm_100a time-step kernels (one launch per half step).
//
// Data flow per half step (velocity: reads tau, writes v; stress: reads the
// new v, writes tau).  The step reads the five fields from one copy of the
// wavefield and writes the other copy, so every written cell is a pure
// function of read-only inputs and no ordering is needed inside a launch.
// Block roles of one launch, in launch order:
//
//   [0, n_tiles)             64 x 16 cell tiles in raster order; the last tile
//                            of a row is aligned to the right edge of the grid
//                            so that the right HABC band and the two columns
//                            its rules read lie in one tile, as the left band
//                            does in the first tile.
//       fast tiles: the stencil fields of the tile plus an M-cell halo and
//         the tile's pointwise operands arrive by TMA (cp.async.bulk.tensor.2d;
//         one mbarrier for the halo boxes, one for the tile boxes; each tile
//         also prefetches into L2 the boxes of the tile prefetch_ahead blocks
//         later); each thread owns 4 columns x 2 rows, forms
//         x-derivatives from 128-bit shared-memory row windows and
//         z-derivatives from a (2M+1)-row register window.  Tiles
//         holding left/right HABC cells park their stencil values in shared
//         memory and apply the HABC rules of step_common.cuh to them.
//       generic tiles (top HABC band without a free surface, or HABC bands
//         wider than a tile allows): stencil values of the tile plus a 4 x 2
//         margin are computed into shared memory cell by cell, then the rules.
//   [.., +record blocks)     receivers of step rec_k (velocity launch only).
//
// Rows nz-nbc-1 .. nz-2 (the bottom HABC band) are stored by the tiles
// before their HABC, into a band scratch; a second launch per half step, the
// band pass (band_kernel), runs the band's recurrence along j and writes the
// final values.
#pragma once

#include <cuda.h>

#include "step_common.cuh"

namespace fomo {

constexpr int kTX = 64, kTZ = 16, kThreads = 128;
constexpr int kCG = kTX / 4;   // float4 column groups of a tile row
// Tile blocks per SM the register allocation is sized for.  Six blocks
// (80 registers) for M <= 4 were measured no faster than five.
template <int M>
constexpr int kTileBlocks = 5;
constexpr int kStripW = 28;     // columns a band-pass warp stores
constexpr int kMarchRows = 16;  // band rows staged per chunk by the band pass

// Band-pass strips over a grid nx cells wide.
__host__ __device__ constexpr int band_block_count(int nx) { return (nx + kStripW - 1) / kStripW; }
constexpr int kEdgeX = 4, kEdgeZ = 2;  // margin of stencil values around an edge tile

template <int M>
struct Geo {
    static constexpr int HQ = (M + 3) / 4;          // float4s of x halo on each side
    static constexpr int HX = 4 * HQ;               // x halo of the TMA box (16-byte aligned)
    static constexpr int BOXW = kTX + 2 * HX;
    static constexpr int BOXH = kTZ + 2 * M;
    static constexpr int NQ = 1 + 2 * HQ;           // float4s of an x window
    static constexpr int BOXS = (BOXW * BOXH + 31) / 32 * 32;  // floats per box in smem (128-byte multiple)
    static constexpr int RW = kTX + 2 * kEdgeX, RH = kTZ + 2 * kEdgeZ;  // edge-tile value region
};
constexpr int kPBox = kTX * kTZ;  // floats of a pointwise box (the tile itself, no halo)

// Device-side parameters beyond StepParams.
struct TiledArgs {
    const float* b[4];   // buoyancy dtx/rho_vx, dtz/rho_vx, dtx/rho_vz, dtz/rho_vz
    int iso;             // dtx == dtz: b[1] == b[0] and b[3] == b[2]
    int* status;         // first nonzero error code of the launch (0 = ok)
    float* band_pre;     // pre-HABC values of the bottom band rows (see band_pre_at)
    int n_tile_blocks, tiles_x;
    int x_last;          // first column of the last tile of a row (a multiple of 4)
    int prefetch_ahead;  // tile blocks between a fast tile and the tile it prefetches (0 = none)
};

__device__ __forceinline__ int tile_x0(const TiledArgs& T, int tx) {
    return tx == T.tiles_x - 1 ? T.x_last : tx * kTX;
}

// Column-pair arithmetic: two scalar IEEE round-to-nearest operations.  The
// sm_100a paired FP32 instructions (add/mul/sub.rn.f32x2, and the
// __fadd2_rn/__fmul2_rn intrinsics) were measured to give results that are
// not bit-identical to these scalar operations on this path, so the kernels
// keep the scalar forms and stay bit-identical to the CPU evaluation.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(fadd(a.x, b.x), fadd(a.y, b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return make_float2(fmul(a.x, b.x), fmul(a.y, b.y)); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(fsub(a.x, b.x), fsub(a.y, b.y)); }
__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }

// TMA descriptors of one launch.  Velocity: halo boxes of txx, tzz, txz;
// tile boxes of vx, vz, b0..b3.  Stress: halo boxes of vx, vz; tile boxes of
// txx, tzz, txz, lam, mu_txx, mu_txz.
struct VelMaps {
    CUtensorMap xx, zz, xz, vx, vz, b0, b1, b2, b3;
};
struct StrMaps {
    CUtensorMap vx, vz, txx, tzz, txz, lam, mu, mxz;
};
// The descriptors a tile uses, wherever they live (kernel parameters only:
// the TMA unit may cache descriptors, and parameter space needs no proxy
// fence).
struct VelMapRefs {
    const CUtensorMap *xx, *zz, *xz, *vx, *vz, *b0, *b1, *b2, *b3;
};
struct StrMapRefs {
    const CUtensorMap *vx, *vz, *txx, *tzz, *txz, *lam, *mu, *mxz;
};
__device__ __forceinline__ VelMapRefs refs_of(const VelMaps& m) {
    return {&m.xx, &m.zz, &m.xz, &m.vx, &m.vz, &m.b0, &m.b1, &m.b2, &m.b3};
}
__device__ __forceinline__ StrMapRefs refs_of(const StrMaps& m) {
    return {&m.vx, &m.vz, &m.txx, &m.tzz, &m.txz, &m.lam, &m.mu, &m.mxz};
}

constexpr int kErrTmaTimeout = 1;

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// 2-D tiled TMA load of box (x, z) of `map` into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(float* dst, const CUtensorMap* map, int x, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(x), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// L2 prefetch of a box (nothing reaches shared memory, nothing to wait for).
__device__ __forceinline__ void tma_prefetch_2d(const CUtensorMap* map, int x, int z) {
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"((uint64_t)map), "r"(x), "r"(z)
                 : "memory");
}

// 4-byte asynchronous global -> shared copy; valid == false writes zero.
__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(valid ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// Programmatic dependent launch.  A band pass lets the tile launch that
// follows it start at once (grid_dep_trigger); a tile block that reads what
// the band pass writes waits for the whole pass to complete and its stores to
// be visible (grid_dep_wait).  Without the launch attribute the wait returns
// at once and the trigger does nothing.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ void stg4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }

__device__ __forceinline__ float comp(const float4& v, int c) {
    return c == 0 ? v.x : (c == 1 ? v.y : (c == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_comp(float4& v, int c, float x) {
    if (c == 0) v.x = x; else if (c == 1) v.y = x; else if (c == 2) v.z = x; else v.w = x;
}

// Bounded wait on phase 0 of an mbarrier: false (and kErrTmaTimeout in the
// status word) after `limit` unsuccessful polls, so a load that never lands
// ends the block with an error the host reads instead of hanging the GPU.
constexpr int kWaitPolls = 1 << 24;
__device__ __forceinline__ bool bounded_wait(uint64_t* bar, int* status, int limit) {
    for (int it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, 0)) return true;
    atomicCAS(status, 0, kErrTmaTimeout);
    return false;
}

// Waits for the TMA boxes of this block; false (and status set) on timeout.
__device__ __forceinline__ bool wait_tma(uint64_t* bar, const TiledArgs& T) {
    return bounded_wait(bar, T.status, kWaitPolls);
}

// Self-test of the bounded wait: thread 0 arms an mbarrier for a byte count
// that no copy delivers and waits `limit` polls on it, exactly as a tile
// waits for its TMA boxes; no memory operation is outstanding.
static __global__ void wait_selftest_kernel(int* status, int limit) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    fence_barrier_init();
    mbar_expect_tx(&bar, 16);
    bounded_wait(&bar, status, limit);
}

// Rows a tile stores: every row of the grid.  Rows nz-nbc-1 .. nz-2 (the
// bottom band) are stored before their HABC, into the band scratch, for the
// band pass to finish.
__device__ __forceinline__ bool row_stored(const StepParams& P, int j) { return j < P.nz; }

// Band scratch: plane f of band row jb = j - (nz-nbc-1), planes of nbc rows
// with the grid's row pitch.  txx, tzz, txz use planes 0-2 and vx, vz planes
// kBandVelPlane + 0, 1, so a band pass never shares a plane with the tiles of
// the next half step, which may run beside it.
constexpr int kBandPlanes = 5;
constexpr int kBandVelPlane = 3;
__device__ __forceinline__ float* band_pre_at(const StepParams& P, const TiledArgs& T, int f, int jb, int i) {
    return T.band_pre + ((size_t)f * P.nbc + jb) * P.pitch + i;
}

// Where a tile stores output field f (pointer `out`) of cell (i, j).
__device__ __forceinline__ float* store_at(const StepParams& P, const TiledArgs& T, float* out, int f, int i, int j) {
    const int jb = j - (P.nz - P.nbc - 1);
    if (jb >= 0 && jb < P.nbc) return band_pre_at(P, T, f, jb, i);
    return out + cell(P, i, j);
}

__device__ __forceinline__ bool lr_band_cell(const StepParams& P, int i, int j) {
    const int js0 = P.fs ? P.nbc : 1;
    return (i <= P.nbc || i >= P.nx - P.nbc - 1) && j >= js0 && j <= P.nz - P.nbc - 2;
}

// ---------------------------------------------------------------- shared-memory stencil values
// Stencil input fields of one half step over [xa-M, xa+W+M) x [za-M, za+H+M)
// into `sin` (field-major, row-major), zero outside the grid.  Velocity:
// txx, tzz, txz with the source injected; stress: vx, vz.
template <int M, bool VEL>
__device__ void load_region_inputs(const StepParams& P, int xa, int za, int W, int H, float* sin, float src_w) {
    const int IW = W + 2 * M, IH = H + 2 * M;
    constexpr int NF = VEL ? 3 : 2;
    const int n = NF * IW * IH;
    for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
        const int f = idx / (IW * IH), r = idx - f * (IW * IH);
        const int zz = r / IW, xx = r - zz * IW;
        const int i = xa - M + xx, j = za - M + zz;
        float v = 0.f;
        if (i >= 0 && i < P.nx && j >= 0 && j < P.nz)
            v = VEL ? tau_in(P, TXX + f, i, j, src_w) : __ldg(in_field(P, VX + f) + cell(P, i, j));
        sin[idx] = v;
    }
}

// Values after the stencil update (before the HABC) of the half step's
// output fields over [xa, xa+W) x [za, za+H) into `spre` (field-major).
template <int M, bool VEL>
__device__ void compute_region_pre(const StepParams& P, const TiledArgs& T, int xa, int za, int W, int H,
                                   const float* sin, float* spre, float src_w) {
    const int IW = W + 2 * M, IH = H + 2 * M;
    auto S = [&](int f, int i, int j) -> float { return sin[(f * IH + (j - za + M)) * IW + (i - xa + M)]; };
    for (int idx = threadIdx.x; idx < W * H; idx += blockDim.x) {
        const int zz = idx / W, xx = idx - zz * W;
        const int i = xa + xx, j = za + zz;
        if (i < 0 || i >= P.nx || j < 0 || j >= P.nz) {
            spre[idx] = 0.f;
            spre[W * H + idx] = 0.f;
            if (!VEL) spre[2 * W * H + idx] = 0.f;
            continue;
        }
        const size_t c = cell(P, i, j);
        if (VEL) {
            float vx = __ldg(P.in[VX] + c), vz = __ldg(P.in[VZ] + c);
            if (in_stencil(P, i, j)) {
                float d1 = 0.f, d2 = 0.f, d3 = 0.f, d4 = 0.f;
#pragma unroll
                for (int l = 1; l <= M; ++l) {
                    const float al = P.a[l - 1];
                    d1 = fadd(fmul(al, fsub(S(0, i + l - 1, j), S(0, i - l, j))), d1);
                    d2 = fadd(fmul(al, fsub(S(2, i, j + l - 1), S(2, i, j - l))), d2);
                    d3 = fadd(fmul(al, fsub(S(2, i + l, j), S(2, i - l + 1, j))), d3);
                    d4 = fadd(fmul(al, fsub(S(1, i, j + l), S(1, i, j - l + 1))), d4);
                }
                vx = fadd(vx, fadd(fmul(__ldg(T.b[0] + c), d1), fmul(__ldg(T.b[1] + c), d2)));
                vz = fadd(vz, fadd(fmul(__ldg(T.b[2] + c), d3), fmul(__ldg(T.b[3] + c), d4)));
            }
            spre[idx] = vx;
            spre[W * H + idx] = vz;
        } else {
            float txx = tau_in(P, TXX, i, j, src_w), tzz = tau_in(P, TZZ, i, j, src_w), txz = __ldg(P.in[TXZ] + c);
            if (in_stencil(P, i, j)) {
                float dvxdx = 0.f, dvzdz = 0.f, dvxdz = 0.f, dvzdx = 0.f;
#pragma unroll
                for (int l = 1; l <= M; ++l) {
                    const float al = P.a[l - 1];
                    dvxdx = fadd(fmul(al, fsub(S(0, i + l, j), S(0, i - l + 1, j))), dvxdx);
                    dvzdz = fadd(fmul(al, fsub(S(1, i, j + l - 1), S(1, i, j - l))), dvzdz);
                    dvxdz = fadd(fmul(al, fsub(S(0, i, j + l), S(0, i, j - l + 1))), dvxdz);
                    dvzdx = fadd(fmul(al, fsub(S(1, i + l - 1, j), S(1, i - l, j))), dvzdx);
                }
                const float lv = __ldg(P.lam + c), mv = __ldg(P.mu_txx + c), mxz = __ldg(P.mu_txz + c);
                const float l2m = fadd(lv, fmul(2.f, mv));
                const float ex = fmul(dvxdx, P.dtx), ez = fmul(dvzdz, P.dtz);
                txx = fadd(txx, fadd(fmul(l2m, ex), fmul(lv, ez)));
                tzz = fadd(tzz, fadd(fmul(lv, ex), fmul(l2m, ez)));
                txz = fadd(txz, fmul(mxz, fadd(fmul(dvxdz, P.dtz), fmul(dvzdx, P.dtx))));
            }
            spre[idx] = txx;
            spre[W * H + idx] = tzz;
            spre[2 * W * H + idx] = txz;
        }
    }
}

// Reads field f of a value region in shared memory.
struct SmemPre {
    const float* spre;
    int xa, za, W, H, f;
    __device__ float operator()(int i, int j) const { return spre[(f * H + (j - za)) * W + (i - xa)]; }
};

// ---------------------------------------------------------------- edge tiles
template <int M, bool VEL>
__device__ void edge_tile(const StepParams& P, const TiledArgs& T, int x0, int z0, int x_end, float* smem,
                          float src_w) {
    using G = Geo<M>;
    const int xa = x0 - kEdgeX, za = z0 - kEdgeZ;
    float* sin = smem;
    float* spre = smem + (VEL ? 3 : 2) * (G::RW + 2 * M) * (G::RH + 2 * M);
    load_region_inputs<M, VEL>(P, xa, za, G::RW, G::RH, sin, src_w);
    __syncthreads();
    compute_region_pre<M, VEL>(P, T, xa, za, G::RW, G::RH, sin, spre, src_w);
    __syncthreads();
    for (int idx = threadIdx.x; idx < kTX * kTZ; idx += blockDim.x) {
        const int i = x0 + (idx % kTX), j = z0 + (idx / kTX);
        if (i >= P.nx || i >= x_end || !row_stored(P, j)) continue;
        const bool band = (i <= P.nbc) || (i >= P.nx - P.nbc - 1) || (!P.fs && j <= P.nbc);
        if (VEL) {
            float vx = SmemPre{spre, xa, za, G::RW, G::RH, 0}(i, j);
            float vz = SmemPre{spre, xa, za, G::RW, G::RH, 1}(i, j);
            if (band) {
                vx = HabcPoint<SmemPre>{P, SmemPre{spre, xa, za, G::RW, G::RH, 0}, P.in[VX], P.w_tab[0]}.final_value(i, j);
                vz = HabcPoint<SmemPre>{P, SmemPre{spre, xa, za, G::RW, G::RH, 1}, P.in[VZ], P.w_tab[1]}.final_value(i, j);
            }
            *store_at(P, T, P.out[VX], kBandVelPlane, i, j) = vx;
            *store_at(P, T, P.out[VZ], kBandVelPlane + 1, i, j) = vz;
        } else {
            float v[3];
#pragma unroll
            for (int f = 0; f < 3; ++f) {
                const SmemPre pre{spre, xa, za, G::RW, G::RH, f};
                v[f] = band ? HabcPoint<SmemPre>{P, pre, P.in[TXX + f], P.w_tab[2]}.final_value(i, j) : pre(i, j);
            }
            if (in_free_surface_rows(P, j)) v[1] = v[2] = 0.f;
            *store_at(P, T, P.out[TXX], 0, i, j) = v[0];
            *store_at(P, T, P.out[TZZ], 1, i, j) = v[1];
            *store_at(P, T, P.out[TXZ], 2, i, j) = v[2];
        }
    }
}

// ---------------------------------------------------------------- fast tiles
// x-derivative windows: NQ float4s starting HX cells left of the thread's
// first column.  win[k] is the value at column x - HX + k.
template <int M>
__device__ __forceinline__ void load_xwin(const float* row, float (&win)[4 * Geo<M>::NQ]) {
#pragma unroll
    for (int q = 0; q < Geo<M>::NQ; ++q) {
        const float4 v = lds4(row + 4 * q);
        win[4 * q] = v.x;
        win[4 * q + 1] = v.y;
        win[4 * q + 2] = v.z;
        win[4 * q + 3] = v.w;
    }
}

// d[c] = sum_l a_l (win[HX+c+l-1+s] - win[HX+c-l+s]) for the thread's 4
// columns: s = 0 for the "forward" staggering (f[i+l-1] - f[i-l]), s = 1 for
// the "backward" one (f[i+l] - f[i-l+1]).
template <int M, int S>
__device__ __forceinline__ void xderiv(const StepParams& P, const float (&w)[4 * Geo<M>::NQ], float (&d)[4]) {
    constexpr int HX = Geo<M>::HX;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float acc = 0.f;
#pragma unroll
        for (int l = 1; l <= M; ++l) acc = fadd(fmul(P.a[l - 1], fsub(w[HX + c + l - 1 + S], w[HX + c - l + S])), acc);
        d[c] = acc;
    }
}

// z-derivatives of two rows from a (2M+1)-row window wz[0..2M] starting at
// the window row of (row 0) - M + S: d[rr] = sum_l a_l (wz[rr+M+l-1] - wz[rr+M-l]),
// evaluated as column pairs.
template <int M>
__device__ __forceinline__ void zderiv(const StepParams& P, const float4 (&wz)[2 * M + 1], float2 (&lo)[2],
                                       float2 (&hi)[2]) {
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
        float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
#pragma unroll
        for (int l = 1; l <= M; ++l) {
            const float2 al = make_float2(P.a[l - 1], P.a[l - 1]);
            a = add2(mul2(al, sub2(lo2(wz[rr + M + l - 1]), lo2(wz[rr + M - l]))), a);
            b = add2(mul2(al, sub2(hi2(wz[rr + M + l - 1]), hi2(wz[rr + M - l]))), b);
        }
        lo[rr] = a;
        hi[rr] = b;
    }
}

// Stencil values of one tile cell, read back from shared memory by the HABC
// rules of band tiles.
struct TilePre {
    const float* spre;
    int x0, z0, f;
    __device__ float operator()(int i, int j) const { return spre[(f * kTZ + (j - z0)) * kTX + (i - x0)]; }
};

// L2 prefetch of the boxes of tile `tile` when it is a fast tile of this
// launch (defined after classify).  The single-shot fast tiles pass
// pf_tile = their block + T.prefetch_ahead, so that tile's DRAM reads start
// while this one is computed; the batched launches pass -1 (no prefetch).
template <int M>
__device__ void prefetch_vel(const StepParams& P, const TiledArgs& T, const VelMapRefs& mp, int tile);
template <int M>
__device__ void prefetch_str(const StepParams& P, const TiledArgs& T, const StrMapRefs& mp, int tile);

// A call thread 0 makes right after starting a tile's copies (the batched
// launches' L2 prefetch of a later block); none by default.
struct NoHook {
    __device__ void operator()() const {}
};

// live == false (a batched shot outside its step range, known only after the
// copies were started): the block waits for its boxes and stores nothing.
template <int M, class Hook = NoHook>
__device__ __forceinline__ void fast_vel(const StepParams& P, const TiledArgs& T, const VelMapRefs& mp, int x0, int z0,
                                         int x_end, bool band, bool rim, float* smem, float src_w, int pf_tile = -1,
                                         bool live = true, const Hook& hook = Hook()) {
    using G = Geo<M>;
    constexpr int BOX = G::BOXS;
    float* s_xx = smem;
    float* s_zz = smem + BOX;
    float* s_xz = smem + 2 * BOX;
    float* p_vx = smem + 3 * BOX;
    float* p_vz = p_vx + kPBox;
    float* p_b0 = p_vz + kPBox;
    float* p_b2 = p_b0 + kPBox;
    float* p_b1 = T.iso ? p_b0 : p_b2 + kPBox;
    float* p_b3 = T.iso ? p_b2 : p_b2 + 2 * kPBox;
    // bar[0]: the halo boxes (the derivatives start once they land), bar[1]:
    // the tile boxes (read by the update after the derivatives)
    uint64_t* bar = reinterpret_cast<uint64_t*>(p_b2 + (T.iso ? 1 : 3) * kPBox);
    // thread 0 starts the copies before the block barrier that lets the
    // other threads see the initialised mbarriers
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        fence_barrier_init();
        mbar_expect_tx(bar, 3 * G::BOXW * G::BOXH * 4);
        tma_load_2d(s_xx, mp.xx, x0 - G::HX, z0 - M, bar);
        tma_load_2d(s_zz, mp.zz, x0 - G::HX, z0 - M, bar);
        tma_load_2d(s_xz, mp.xz, x0 - G::HX, z0 - M, bar);
        mbar_expect_tx(bar + 1, (T.iso ? 4 : 6) * kPBox * 4);
        tma_load_2d(p_vx, mp.vx, x0, z0, bar + 1);
        tma_load_2d(p_vz, mp.vz, x0, z0, bar + 1);
        tma_load_2d(p_b0, mp.b0, x0, z0, bar + 1);
        tma_load_2d(p_b2, mp.b2, x0, z0, bar + 1);
        if (!T.iso) {
            tma_load_2d(p_b1, mp.b1, x0, z0, bar + 1);
            tma_load_2d(p_b3, mp.b3, x0, z0, bar + 1);
        }
        if (pf_tile >= 0) prefetch_vel<M>(P, T, mp, pf_tile);
        hook();
    }
    __syncthreads();
    if (!wait_tma(bar, T)) return;
    if (!live) {  // every copy of the block lands before it leaves
        wait_tma(bar + 1, T);
        return;
    }
    // The source, added to the stresses read: only the block whose halo box
    // holds it needs a block barrier (the condition is block-uniform; every
    // other thread sees the boxes through its own wait on bar[0]).
    const int si = P.src_i - (x0 - G::HX), sj = P.src_j - (z0 - M);
    if (si >= 0 && si < G::BOXW && sj >= 0 && sj < G::BOXH) {
        if (threadIdx.x == 0) {
            s_xx[sj * G::BOXW + si] = fadd(s_xx[sj * G::BOXW + si], src_w);
            s_zz[sj * G::BOXW + si] = fadd(s_zz[sj * G::BOXW + si], src_w);
        }
        __syncthreads();
    }

    const int cg = threadIdx.x % kCG, rp = threadIdx.x / kCG;
    const int x = x0 + 4 * cg, zt = z0 + 2 * rp;
    const int xr = 4 * cg;  // box column of win[0] = column x - HX
    float d1[2][4], d3[2][4];
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
        const int br = 2 * rp + rr + M;
        float w[4 * G::NQ];
        load_xwin<M>(s_xx + br * G::BOXW + xr, w);
        xderiv<M, 0>(P, w, d1[rr]);  // dtxx/dx: txx[i+l-1] - txx[i-l]
        load_xwin<M>(s_xz + br * G::BOXW + xr, w);
        xderiv<M, 1>(P, w, d3[rr]);  // dtxz/dx: txz[i+l] - txz[i-l+1]
    }
    float2 d2lo[2], d2hi[2], d4lo[2], d4hi[2];
    {
        float4 wz[2 * M + 1];
#pragma unroll
        for (int k = 0; k <= 2 * M; ++k) wz[k] = lds4(s_xz + (2 * rp + k) * G::BOXW + xr + G::HX);
        zderiv<M>(P, wz, d2lo, d2hi);  // dtxz/dz: txz[j+l-1] - txz[j-l]
#pragma unroll
        for (int k = 0; k <= 2 * M; ++k) wz[k] = lds4(s_zz + (2 * rp + 1 + k) * G::BOXW + xr + G::HX);
        zderiv<M>(P, wz, d4lo, d4hi);  // dtzz/dz: tzz[j+l] - tzz[j-l+1]
    }
    if (!wait_tma(bar + 1, T)) return;
    float4 ox[2], oz[2];
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
        const int po = (2 * rp + rr) * kTX + xr;
        const float4 vx = lds4(p_vx + po), vz = lds4(p_vz + po);
        const float4 b0 = lds4(p_b0 + po), b1 = lds4(p_b1 + po), b2 = lds4(p_b2 + po), b3 = lds4(p_b3 + po);
        const float2 xl = add2(lo2(vx), add2(mul2(lo2(b0), make_float2(d1[rr][0], d1[rr][1])), mul2(lo2(b1), d2lo[rr])));
        const float2 xh = add2(hi2(vx), add2(mul2(hi2(b0), make_float2(d1[rr][2], d1[rr][3])), mul2(hi2(b1), d2hi[rr])));
        const float2 zl = add2(lo2(vz), add2(mul2(lo2(b2), make_float2(d3[rr][0], d3[rr][1])), mul2(lo2(b3), d4lo[rr])));
        const float2 zh = add2(hi2(vz), add2(mul2(hi2(b2), make_float2(d3[rr][2], d3[rr][3])), mul2(hi2(b3), d4hi[rr])));
        ox[rr] = make_float4(xl.x, xl.y, xh.x, xh.y);
        oz[rr] = make_float4(zl.x, zl.y, zh.x, zh.y);
        if (rim) {  // cells outside the stencil domain keep their value
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (!in_stencil(P, x + c, zt + rr)) {
                    set_comp(ox[rr], c, comp(vx, c));
                    set_comp(oz[rr], c, comp(vz, c));
                }
        }
    }
    if (band) {
        __syncthreads();  // every thread is done with the boxes
        float* spre = smem;  // [2][kTZ][kTX]
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
            const int po = (2 * rp + rr) * kTX + xr;
            *reinterpret_cast<float4*>(spre + po) = ox[rr];
            *reinterpret_cast<float4*>(spre + kPBox + po) = oz[rr];
        }
        __syncthreads();
        const HabcPoint<TilePre> hx{P, TilePre{spre, x0, z0, 0}, P.in[VX], P.w_tab[0]};
        const HabcPoint<TilePre> hz{P, TilePre{spre, x0, z0, 1}, P.in[VZ], P.w_tab[1]};
#pragma unroll
        for (int rr = 0; rr < 2; ++rr)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (x + c < x_end && row_stored(P, zt + rr) && lr_band_cell(P, x + c, zt + rr)) {
                    set_comp(ox[rr], c, hx.final_value(x + c, zt + rr));
                    set_comp(oz[rr], c, hz.final_value(x + c, zt + rr));
                }
    }
    if (x < x_end) {
#pragma unroll
        for (int rr = 0; rr < 2; ++rr)
            if (row_stored(P, zt + rr)) {
                stg4(store_at(P, T, P.out[VX], kBandVelPlane, x, zt + rr), ox[rr]);
                stg4(store_at(P, T, P.out[VZ], kBandVelPlane + 1, x, zt + rr), oz[rr]);
            }
    }
}

template <int M, class Hook = NoHook>
__device__ __forceinline__ void fast_str(const StepParams& P, const TiledArgs& T, const StrMapRefs& mp, int x0, int z0,
                                         int x_end, bool band, bool rim, float* smem, float src_w, int pf_tile = -1,
                                         bool live = true, const Hook& hook = Hook()) {
    using G = Geo<M>;
    constexpr int BOX = G::BOXS;
    float* s_vx = smem;
    float* s_vz = smem + BOX;
    float* p_xx = smem + 2 * BOX;
    float* p_zz = p_xx + kPBox;
    float* p_xz = p_zz + kPBox;
    float* p_lam = p_xz + kPBox;
    float* p_mu = p_lam + kPBox;
    float* p_mxz = p_mu + kPBox;
    // bar[0]: the halo boxes, bar[1]: the tile boxes (as in fast_vel)
    uint64_t* bar = reinterpret_cast<uint64_t*>(p_mxz + kPBox);
    if (threadIdx.x == 0) {  // copies started before the block barrier, as in fast_vel
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        fence_barrier_init();
        mbar_expect_tx(bar, 2 * G::BOXW * G::BOXH * 4);
        tma_load_2d(s_vx, mp.vx, x0 - G::HX, z0 - M, bar);
        tma_load_2d(s_vz, mp.vz, x0 - G::HX, z0 - M, bar);
        mbar_expect_tx(bar + 1, 6 * kPBox * 4);
        tma_load_2d(p_xx, mp.txx, x0, z0, bar + 1);
        tma_load_2d(p_zz, mp.tzz, x0, z0, bar + 1);
        tma_load_2d(p_xz, mp.txz, x0, z0, bar + 1);
        tma_load_2d(p_lam, mp.lam, x0, z0, bar + 1);
        tma_load_2d(p_mu, mp.mu, x0, z0, bar + 1);
        tma_load_2d(p_mxz, mp.mxz, x0, z0, bar + 1);
        if (pf_tile >= 0) prefetch_str<M>(P, T, mp, pf_tile);
        hook();
    }
    __syncthreads();
    if (!wait_tma(bar, T)) return;
    if (!live) {  // every copy of the block lands before it leaves
        wait_tma(bar + 1, T);
        return;
    }

    const int cg = threadIdx.x % kCG, rp = threadIdx.x / kCG;
    const int x = x0 + 4 * cg, zt = z0 + 2 * rp;
    const int xr = 4 * cg;
    float dxx[2][4], dzx[2][4];  // dvx/dx, dvz/dx
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
        const int br = 2 * rp + rr + M;
        float w[4 * G::NQ];
        load_xwin<M>(s_vx + br * G::BOXW + xr, w);
        xderiv<M, 1>(P, w, dxx[rr]);  // vx[i+l] - vx[i-l+1]
        load_xwin<M>(s_vz + br * G::BOXW + xr, w);
        xderiv<M, 0>(P, w, dzx[rr]);  // vz[i+l-1] - vz[i-l]
    }
    float2 dzzlo[2], dzzhi[2], dxzlo[2], dxzhi[2];  // dvz/dz, dvx/dz
    {
        float4 wz[2 * M + 1];
#pragma unroll
        for (int k = 0; k <= 2 * M; ++k) wz[k] = lds4(s_vz + (2 * rp + k) * G::BOXW + xr + G::HX);
        zderiv<M>(P, wz, dzzlo, dzzhi);  // vz[j+l-1] - vz[j-l]
#pragma unroll
        for (int k = 0; k <= 2 * M; ++k) wz[k] = lds4(s_vx + (2 * rp + 1 + k) * G::BOXW + xr + G::HX);
        zderiv<M>(P, wz, dxzlo, dxzhi);  // vx[j+l] - vx[j-l+1]
    }
    if (!wait_tma(bar + 1, T)) return;
    float4 oxx[2], ozz[2], oxz[2];
    const float2 dtx2 = make_float2(P.dtx, P.dtx), dtz2 = make_float2(P.dtz, P.dtz), two = make_float2(2.f, 2.f);
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
        const int po = (2 * rp + rr) * kTX + xr;
        float4 txx = lds4(p_xx + po), tzz = lds4(p_zz + po);
        const float4 txz = lds4(p_xz + po), lam = lds4(p_lam + po), mu = lds4(p_mu + po), mxz = lds4(p_mxz + po);
        const int dc = P.src_i - x;
        if (zt + rr == P.src_j && dc >= 0 && dc < 4) {
            set_comp(txx, dc, fadd(comp(txx, dc), src_w));
            set_comp(tzz, dc, fadd(comp(tzz, dc), src_w));
        }
        float2 r_xx[2], r_zz[2], r_xz[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float2 lv = h ? hi2(lam) : lo2(lam), mv = h ? hi2(mu) : lo2(mu);
            const float2 l2m = add2(lv, mul2(two, mv));
            const float2 ex = mul2(make_float2(dxx[rr][2 * h], dxx[rr][2 * h + 1]), dtx2);
            const float2 ez = mul2(h ? dzzhi[rr] : dzzlo[rr], dtz2);
            r_xx[h] = add2(h ? hi2(txx) : lo2(txx), add2(mul2(l2m, ex), mul2(lv, ez)));
            r_zz[h] = add2(h ? hi2(tzz) : lo2(tzz), add2(mul2(lv, ex), mul2(l2m, ez)));
            const float2 sh = add2(mul2(h ? dxzhi[rr] : dxzlo[rr], dtz2),
                                   mul2(make_float2(dzx[rr][2 * h], dzx[rr][2 * h + 1]), dtx2));
            r_xz[h] = add2(h ? hi2(txz) : lo2(txz), mul2(h ? hi2(mxz) : lo2(mxz), sh));
        }
        oxx[rr] = make_float4(r_xx[0].x, r_xx[0].y, r_xx[1].x, r_xx[1].y);
        ozz[rr] = make_float4(r_zz[0].x, r_zz[0].y, r_zz[1].x, r_zz[1].y);
        oxz[rr] = make_float4(r_xz[0].x, r_xz[0].y, r_xz[1].x, r_xz[1].y);
        if (rim) {
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (!in_stencil(P, x + c, zt + rr)) {
                    set_comp(oxx[rr], c, comp(txx, c));
                    set_comp(ozz[rr], c, comp(tzz, c));
                    set_comp(oxz[rr], c, comp(txz, c));
                }
        }
    }
    if (band) {
        __syncthreads();
        float* spre = smem;  // [3][kTZ][kTX]
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
            const int po = (2 * rp + rr) * kTX + xr;
            *reinterpret_cast<float4*>(spre + po) = oxx[rr];
            *reinterpret_cast<float4*>(spre + kPBox + po) = ozz[rr];
            *reinterpret_cast<float4*>(spre + 2 * kPBox + po) = oxz[rr];
        }
        __syncthreads();
        const HabcPoint<TilePre> h0{P, TilePre{spre, x0, z0, 0}, P.in[TXX], P.w_tab[2]};
        const HabcPoint<TilePre> h1{P, TilePre{spre, x0, z0, 1}, P.in[TZZ], P.w_tab[2]};
        const HabcPoint<TilePre> h2{P, TilePre{spre, x0, z0, 2}, P.in[TXZ], P.w_tab[2]};
#pragma unroll
        for (int rr = 0; rr < 2; ++rr)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (x + c < x_end && row_stored(P, zt + rr) && lr_band_cell(P, x + c, zt + rr)) {
                    set_comp(oxx[rr], c, h0.final_value(x + c, zt + rr));
                    set_comp(ozz[rr], c, h1.final_value(x + c, zt + rr));
                    set_comp(oxz[rr], c, h2.final_value(x + c, zt + rr));
                }
    }
    if (x < x_end) {
#pragma unroll
        for (int rr = 0; rr < 2; ++rr)
            if (row_stored(P, zt + rr)) {
                if (in_free_surface_rows(P, zt + rr)) {
                    ozz[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
                    oxz[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                stg4(store_at(P, T, P.out[TXX], 0, x, zt + rr), oxx[rr]);
                stg4(store_at(P, T, P.out[TZZ], 1, x, zt + rr), ozz[rr]);
                stg4(store_at(P, T, P.out[TXZ], 2, x, zt + rr), oxz[rr]);
            }
    }
}

// Block-uniform classification of a tile.
struct TileKind {
    bool generic, band, rim;
    int x0, z0, x_end;
};

__device__ __forceinline__ TileKind classify(const StepParams& P, const TiledArgs& T, int tile) {
    TileKind k;
    const int tx = tile % T.tiles_x, tz = tile / T.tiles_x;
    k.x0 = tile_x0(T, tx);
    k.z0 = tz * kTZ;
    // Stores stop at the previous column of the last tile, and never pass
    // round_up(nx, 4) <= row pitch (grids narrower than one tile).
    k.x_end = min((tx < T.tiles_x - 1) ? min(k.x0 + kTX, T.x_last) : k.x0 + kTX, (P.nx + 3) / 4 * 4);
    const int b = P.nbc;
    const bool band_cols = (k.x0 <= b) || (k.x0 + kTX - 1 >= P.nx - b - 1);
    const int js0 = P.fs ? b : 1;
    const bool lr_rows = (k.z0 + kTZ - 1 >= js0) && (k.z0 <= P.nz - b - 2);
    k.band = band_cols && lr_rows;
    const bool top = !P.fs && k.z0 <= b;
    k.generic = top || (k.band && b + 6 > kTX);
    k.rim = k.x0 < P.M || k.x0 + kTX > P.nx - P.M || k.z0 < P.M || k.z0 + kTZ > P.nz - P.M;
    return k;
}

// A tile whose input rows (halo and edge margin included, one row to spare)
// reach the bottom band rows nz-nbc-1 .. nz-2, which the band pass of the
// previous half step writes.  Only these tiles wait for that pass.
__device__ __forceinline__ bool reads_band_rows(const StepParams& P, int z0) {
    return z0 + kTZ + kEdgeZ + P.M >= P.nz - P.nbc - 1;
}

// How far ahead a tile prefetches (TiledArgs::prefetch_ahead): two tile
// blocks per SM of the device (prefetch_distance).  Measured on the
// 4552 x 3927 grid on 148 SMs, the velocity launch was fastest 260-370 blocks
// ahead (113.8 us at one wave, 740; 140.9 us at 1480) and the stress launch
// 185-370 ahead (148.8 us at 92, 150 us at 740).
__host__ inline int prefetch_distance(int sm_count) { return 2 * sm_count; }

template <int M>
__device__ void prefetch_vel(const StepParams& P, const TiledArgs& T, const VelMapRefs& mp, int tile) {
    if (tile >= T.n_tile_blocks) return;
    const TileKind k = classify(P, T, tile);
    if (k.generic) return;
    using G = Geo<M>;
    tma_prefetch_2d(mp.xx, k.x0 - G::HX, k.z0 - M);
    tma_prefetch_2d(mp.zz, k.x0 - G::HX, k.z0 - M);
    tma_prefetch_2d(mp.xz, k.x0 - G::HX, k.z0 - M);
    tma_prefetch_2d(mp.vx, k.x0, k.z0);
    tma_prefetch_2d(mp.vz, k.x0, k.z0);
    tma_prefetch_2d(mp.b0, k.x0, k.z0);
    tma_prefetch_2d(mp.b2, k.x0, k.z0);
    if (!T.iso) {
        tma_prefetch_2d(mp.b1, k.x0, k.z0);
        tma_prefetch_2d(mp.b3, k.x0, k.z0);
    }
}

template <int M>
__device__ void prefetch_str(const StepParams& P, const TiledArgs& T, const StrMapRefs& mp, int tile) {
    if (tile >= T.n_tile_blocks) return;
    const TileKind k = classify(P, T, tile);
    if (k.generic) return;
    using G = Geo<M>;
    tma_prefetch_2d(mp.vx, k.x0 - G::HX, k.z0 - M);
    tma_prefetch_2d(mp.vz, k.x0 - G::HX, k.z0 - M);
    tma_prefetch_2d(mp.txx, k.x0, k.z0);
    tma_prefetch_2d(mp.tzz, k.x0, k.z0);
    tma_prefetch_2d(mp.txz, k.x0, k.z0);
    tma_prefetch_2d(mp.lam, k.x0, k.z0);
    tma_prefetch_2d(mp.mu, k.x0, k.z0);
    tma_prefetch_2d(mp.mxz, k.x0, k.z0);
}

// ---------------------------------------------------------------- receivers
// rec_k: 1-based step recorded from P.in (P.rec_k on the single-shot path).
__device__ inline void record_block(const StepParams& P, int rblock, int rec_k) {
    const int r = rblock * blockDim.x + threadIdx.x;
    if (r >= P.n_rec || rec_k < 1) return;
    const int c = P.rec_cell[r];
    float v;
    if (P.rec_kind == 0) v = P.in[VZ][c];
    else if (P.rec_kind == 1) v = P.in[VX][c];
    else v = fmul(fadd(P.in[TXX][c], P.in[TZZ][c]), 0.5f);
    P.gather[(size_t)(rec_k - 1) + (size_t)r * P.nt] = v;
}

// ---------------------------------------------------------------- kernels
template <int M>
__global__ void __launch_bounds__(kThreads, kTileBlocks<M>) velocity_kernel(const __grid_constant__ StepParams P, const __grid_constant__ TiledArgs T,
                                                            const __grid_constant__ VelMaps maps) {
    extern __shared__ __align__(128) float smem[];
    const int bid = blockIdx.x;
    if (bid < T.n_tile_blocks) {
        const TileKind k = classify(P, T, bid);
        if (reads_band_rows(P, k.z0)) grid_dep_wait();
        if (k.generic) edge_tile<M, true>(P, T, k.x0, k.z0, k.x_end, smem, P.src_w);
        else fast_vel<M>(P, T, refs_of(maps), k.x0, k.z0, k.x_end, k.band, k.rim, smem, P.src_w,
                         T.prefetch_ahead > 0 ? bid + T.prefetch_ahead : -1);
        return;
    }
    grid_dep_wait();  // receivers may sit in the band rows
    record_block(P, bid - T.n_tile_blocks, P.rec_k);
}

// Tile of stress block b.  The velocity launch before it ran top to bottom,
// so the last rows it read and wrote are the ones still in L2; the stress
// launch takes the tile rows that do not wait for the band pass in reverse
// raster order (bottom-right first), then the rows that read the band rows
// (they wait for the band pass) in raster order.  Blocks b >= the tile count
// map to themselves.
__device__ __forceinline__ int stress_tile(const StepParams& P, const TiledArgs& T, int b) {
    const int lim = P.nz - P.nbc - 1 - kTZ - kEdgeZ - P.M;  // a tile with z0 >= lim reads band rows
    const int tz_wait = lim <= 0 ? 0 : (lim + kTZ - 1) / kTZ;
    const int n_early = min(tz_wait * T.tiles_x, T.n_tile_blocks);
    return b < n_early ? n_early - 1 - b : b;
}

template <int M>
__global__ void __launch_bounds__(kThreads, kTileBlocks<M>) stress_kernel(const __grid_constant__ StepParams P, const __grid_constant__ TiledArgs T,
                                                          const __grid_constant__ StrMaps maps) {
    extern __shared__ __align__(128) float smem[];
    const int bid = blockIdx.x;
    if (bid < T.n_tile_blocks) {
        const TileKind k = classify(P, T, stress_tile(P, T, bid));
        if (reads_band_rows(P, k.z0)) grid_dep_wait();
        if (k.generic) edge_tile<M, false>(P, T, k.x0, k.z0, k.x_end, smem, P.src_w);
        else fast_str<M>(P, T, refs_of(maps), k.x0, k.z0, k.x_end, k.band, k.rim, smem, P.src_w,
                         T.prefetch_ahead > 0 ? stress_tile(P, T, bid + T.prefetch_ahead) : -1);
    }
}

// Receivers of the last step (the velocity launch of step k records k-1).
static __global__ void record_kernel(const StepParams P) { record_block(P, blockIdx.x, P.rec_k); }

// ---------------------------------------------------------------- bottom band
// Rows nz-nbc-1 .. nz-2: the bottom edge and the two bottom corners, whose
// HABC rules form a recurrence along j (each row reads the final values of
// the row above, nz-nbc-2 first, which the tiles stored).  The tiles left the
// stencil values of these rows (before the HABC) in the band scratch, so all
// that runs here is the recurrence.  One warp per (strip of kStripW columns,
// output field) marches down the rows: lane l holds column xs-2+l, so lanes
// 2..29 are the strip, lanes 1 and 30 carry the recurrence of the
// neighbouring columns, and lanes 0 and 31 supply values only.  Stencil and
// step-start values arrive by cp.async, kMarchRows rows per chunk, one chunk
// ahead.  A lane's column fixes its rule for every row: rim columns keep the
// stencil value; the bottom edge reads the final value of row j-1 (z term);
// corner cells add the x term of their neighbour towards the interior
// (stencil value, phase A); the last bottom-left column (nbc) and
// bottom-right chunk starts redo it with that neighbour's final value
// (phase B).  Both rules are evaluated and selected, so a warp never
// diverges.  Lane 1's values are wrong only when its column is a
// bottom-right chunk start and lane 30's only when its column is nbc; no
// strip lane reads either then.


constexpr int kMaxBandTab = 1024;                  // nbc + 2 <= this
constexpr int kMarchStage = 2 * 2 * kMarchRows * 32;  // two chunks of (stencil, step-start) values

// Band-pass warps of one half step: strips x 3 (a velocity pass leaves the
// third field's warps idle).
__host__ __device__ constexpr int band_warp_count(int nx) { return band_block_count(nx) * 3; }

template <bool VEL>
__device__ void band_march(const StepParams& P, const TiledArgs& T, int item, float* stage, float* stab) {
    constexpr unsigned FULL = 0xffffffffu;
    const int strip = item / 3, f = item % 3;
    if (VEL && f == 2) return;  // block-uniform
    const int lane = threadIdx.x & 31;
    const int b = P.nbc, nx = P.nx, nz = P.nz, r0 = nx - b - 1, j0 = nz - b - 1;
    const float* tab = P.w_tab[VEL ? f : 2];
    for (int d = lane; d < b + 2; d += 32) stab[d] = __ldg(tab + d);
    __syncwarp();
    const int i = strip * kStripW - 2 + lane;
    const bool col_ok = i >= 0 && i < nx;
    const int q = VEL ? VX + f : TXX + f;
    const int plane = VEL ? kBandVelPlane + f : f;
    const float* oin = in_field(P, q);
    float* oout = q == VX ? P.out[VX] : q == VZ ? P.out[VZ] : q == TXX ? P.out[TXX] : q == TZZ ? P.out[TZZ] : P.out[TXZ];
    // the lane's rule
    const bool rim = i <= 0 || i >= nx - 1;
    const bool left = i >= 1 && i <= b;
    const bool corner = left || (i >= r0 && i <= nx - 2);
    const bool redo = i == b || (i > r0 - 1 && i <= nx - 2 && right_chunk_start(nx, b, i));
    const int nb = min(max(lane + (left ? 1 : -1), 0), 31);  // neighbour towards the interior
    const int dxi = max(min(i, nx - 1 - i), 0);
    const size_t pitch = P.pitch;

    auto stage_chunk = [&](int c) {
        float* buf = stage + (c & 1) * (2 * kMarchRows * 32);
        for (int r = 0; r < kMarchRows; ++r) {
            const int jb = c * kMarchRows + r;
            const bool ok = col_ok && jb < b;
            cp_async4(buf + r * 32 + lane, ok ? band_pre_at(P, T, plane, jb, i) : T.band_pre, ok);
            cp_async4(buf + (kMarchRows + r) * 32 + lane, ok ? oin + cell(P, i, j0 + jb) : oin, ok);
        }
        cp_async_commit();
    };
    float fprev = col_ok ? oout[cell(P, i, j0 - 1)] : 0.f;  // final and step-start values of the row above
    float ovp = col_ok ? __ldg(oin + cell(P, i, j0 - 1)) : 0.f;
    float* dst = oout + (col_ok ? cell(P, i, j0) : 0);
    const bool store = col_ok && lane >= 2 && lane < 2 + kStripW;
    const int n_chunks = (b + kMarchRows - 1) / kMarchRows;
    stage_chunk(0);
    for (int c = 0; c < n_chunks; ++c) {
        if (c + 1 < n_chunks) {
            stage_chunk(c + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncwarp();
        const float* buf = stage + (c & 1) * (2 * kMarchRows * 32);
        const int rows = min(kMarchRows, b - c * kMarchRows);
#pragma unroll 4
        for (int r = 0; r < rows; ++r) {
            const int j = j0 + c * kMarchRows + r;
            const float pv = buf[r * 32 + lane];
            const float ov = buf[(kMarchRows + r) * 32 + lane];
            const float w = stab[min(min(dxi, nz - 1 - j), b + 1)];
            const float pv_nb = __shfl_sync(FULL, pv, nb);
            const float ov_nb = __shfl_sync(FULL, ov, nb);
            const float sz = edge_sum(P.qz, P.qt_z, P.qxt, fprev, ov, ovp);
            const float fc = blend_corner(w, pv, edge_sum(P.qx, P.qt_x, P.qxt, pv_nb, ov, ov_nb), sz);
            const float fe = blend_edge(w, pv, sz);
            const float fa = rim ? pv : (corner ? fc : fe);
            const float fa_nb = __shfl_sync(FULL, fa, nb);
            const float fb = blend_corner(w, pv, edge_sum(P.qx, P.qt_x, P.qxt, fa_nb, ov, ov_nb), sz);
            const float fin = redo ? fb : fa;
            if (store) *dst = fin;
            dst += pitch;
            fprev = fin;
            ovp = ov;
        }
        __syncwarp();  // every lane is done with this chunk's buffer
    }
}

// The band pass of one half step: one warp per (strip, field) (P, T as for
// the half step's tile launch, which must have completed).  The next tile
// launch may start beside it: it writes neither the fields nor the scratch
// planes read here, and its tiles that read the band rows wait.
template <bool VEL>
__global__ void __launch_bounds__(32) band_kernel(const __grid_constant__ StepParams P, const __grid_constant__ TiledArgs T) {
    __shared__ __align__(16) float stage[kMarchStage];
    __shared__ float stab[kMaxBandTab];
    grid_dep_trigger();
    band_march<VEL>(P, T, blockIdx.x, stage, stab);
}

// ---------------------------------------------------------------- snapshots
// One frame of a wavefield for the on_step hook (video_recorder.jl:260-297):
// frame (i, j) (1-based, nx_d = cld(nx, ds), nz_d = cld(nz, ds)) takes cell
// (min((i-1)*ds+1, nx), min((j-1)*ds+1, nz)) of
//   kind 0  p   = (txx + tzz) * 0.5
//   kind 1  vel = sqrt(vx^2 + vz^2)
//   kind 2  vx,   kind 3  vz.
static __global__ void snapshot_kernel(const float* f0, const float* f1, int kind, int nx, int nz, int pitch, int ds,
                                int nx_d, int nz_d, float* out) {
    const size_t n = (size_t)nx_d * nz_d;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(k % nx_d), j = (int)(k / nx_d);
        const int is = min(i * ds, nx - 1), js = min(j * ds, nz - 1);
        const size_t c = (size_t)is + (size_t)js * pitch;
        float v;
        if (kind == 0) v = fmul(fadd(f0[c], f1[c]), 0.5f);
        else if (kind == 1) v = __fsqrt_rn(fadd(fmul(f0[c], f0[c]), fmul(f1[c], f1[c])));
        else v = f0[c];
        out[k] = v;
    }
}

// ---------------------------------------------------------------- medium set-up
// init_medium on the device (init.jl:68-158): the (nx_in, nz_in) vp, vs, rho
// padded by edge replication (_pad_array, init.jl:119-134: a padded cell takes
// the model cell at its coordinates clamped into the model) and the staggered
// parameters of _compute_staggered_params (init.jl:136-158), in its Float32
// operation order:
//   mu = rho * (vs * vs), lam = rho * (vp * vp) - 2 * mu, rho_vx = rho,
//   rho_vz = 0.25 * (((rho[i,j] + rho[i+1,j]) + rho[i,j+1]) + rho[i+1,j+1]),
//   mu_txz = 2 / (1 / mu[i,j] + 1 / mu[i,j+1]),
// the last row and column of rho_vz and the last row of mu_txz copied from
// their neighbours.  Outputs have row pitch `pitch`.
struct ModelView {
    const float *vp, *vs, *rho;  // (nx_in, nz_in), x fastest
    int nx_in, nz_in, pad;
    __device__ __forceinline__ size_t at(int i, int j) const {
        const int ii = min(max(i - pad, 0), nx_in - 1), jj = min(max(j - pad, 0), nz_in - 1);
        return (size_t)ii + (size_t)jj * nx_in;
    }
    __device__ __forceinline__ float mu(int i, int j) const {
        const size_t k = at(i, j);
        return fmul(__ldg(rho + k), fmul(__ldg(vs + k), __ldg(vs + k)));
    }
};

static __global__ void medium_init_kernel(const ModelView V, int nx, int nz, int pitch, float* rho_vx, float* rho_vz,
                                   float* lam, float* mu_txx, float* mu_txz) {
    const size_t n = (size_t)nx * nz;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(k % nx), j = (int)(k / nx);
        const size_t m = V.at(i, j), o = (size_t)i + (size_t)j * pitch;
        const float rho = __ldg(V.rho + m), vp = __ldg(V.vp + m);
        const float mu = V.mu(i, j);
        mu_txx[o] = mu;
        lam[o] = fsub(fmul(rho, fmul(vp, vp)), fmul(2.f, mu));
        rho_vx[o] = rho;
        const int ic = min(i, nx - 2), jc = min(j, nz - 2);
        const float r00 = __ldg(V.rho + V.at(ic, jc)), r10 = __ldg(V.rho + V.at(ic + 1, jc));
        const float r01 = __ldg(V.rho + V.at(ic, jc + 1)), r11 = __ldg(V.rho + V.at(ic + 1, jc + 1));
        rho_vz[o] = fmul(0.25f, fadd(fadd(fadd(r00, r10), r01), r11));
        mu_txz[o] = fdiv(2.f, fadd(fdiv(1.f, V.mu(i, jc)), fdiv(1.f, V.mu(i, jc + 1))));
    }
}

// Buoyancy dtx/rho_vx, dtz/rho_vx, dtx/rho_vz, dtz/rho_vz: the divisions of
// update_velocity! (velocity.jl:41-42), IEEE-rounded, once per medium and dt.
static __global__ void buoyancy_kernel(const float* rho_vx, const float* rho_vz, float dtx, float dtz, size_t n,
                                float* b0, float* b1, float* b2, float* b3) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const float rx = rho_vx[k], rz = rho_vz[k];
        b0[k] = fdiv(dtx, rx);
        b2[k] = fdiv(dtx, rz);
        if (b1 != b0) b1[k] = fdiv(dtz, rx);
        if (b3 != b2) b3[k] = fdiv(dtz, rz);
    }
}

// Shared-memory bytes of one launch (the largest block role that can occur:
// generic tiles only without a free surface or with a band wider than a tile
// allows, as classify decides).
template <int M>
__host__ size_t tiled_smem_bytes(bool vel, int nbc, bool iso, bool fs) {
    using G = Geo<M>;
    const int nin = vel ? 3 : 2, nout = vel ? 2 : 3;
    const int npoint = vel ? (iso ? 4 : 6) : 6;
    const size_t interior = ((size_t)nin * G::BOXS + (size_t)npoint * kPBox) * 4 + 16;
    const size_t edge = ((size_t)nin * (G::RW + 2 * M) * (G::RH + 2 * M) + (size_t)nout * G::RW * G::RH) * 4;
    const bool generic = !fs || nbc + 6 > kTX;
    return generic ? std::max(interior, edge) : interior;
}

}  // namespace fomo
