// step_simple.cuh -- the first sm_100a kernels of the time step: one launch
// per half step (velocity, stress), operands read straight from global
// memory through the read-only cache.  They define the data flow that the
// tiled kernels keep:
//
//   * the step reads the five fields from one copy of the wavefield and
//     writes them to the other, so the reference's *_old boundary strips
//     (boundary.jl:20-56) are simply the copy being read;
//   * every written cell is a pure function of read-only inputs, so cells,
//     the HABC and the source need no ordering inside the launch;
//   * block ranges of one launch:
//       [0, n_tile_blocks)                       cell pass (32 x 8 cells)
//       [n_tile_blocks, +n_band_blocks)          bottom-band recurrence
//       [.., +record blocks)                     receivers of step rec_k
#pragma once

#include "step_common.cuh"

namespace fomo {

constexpr int kTileX = 32, kTileZ = 8;
constexpr int kBandW = 32;  // columns per bottom-band block

struct VelPreF {
    const StepParams& P;
    int q;  // VX or VZ
    __device__ float operator()(int i, int j) const {
        float vx, vz;
        vel_pre(P, i, j, vx, vz);
        return q == VX ? vx : vz;
    }
};

struct StrPreF {
    const StepParams& P;
    int q;  // TXX, TZZ or TXZ
    __device__ float operator()(int i, int j) const {
        float a, b, c;
        str_pre(P, i, j, a, b, c);
        return q == TXX ? a : (q == TZZ ? b : c);
    }
};

// Receivers of step rec_k, read from the fields the current half step reads
// (the final state of step rec_k).  record_receivers! (source_receiver.jl:65-77).
__device__ inline void record_block(const StepParams& P, int rblock) {
    const int r = rblock * blockDim.x + threadIdx.x;
    if (r >= P.n_rec || P.rec_k < 1) return;
    const int c = P.rec_cell[r];
    float v;
    if (P.rec_kind == 0) v = P.in[VZ][c];
    else if (P.rec_kind == 1) v = P.in[VX][c];
    else v = fmul(fadd(P.in[TXX][c], P.in[TZZ][c]), 0.5f);
    P.gather[(size_t)(P.rec_k - 1) + (size_t)r * P.nt] = v;
}

// Bottom band: rows nz-nbc-1 .. nz-2, columns 1 .. nx-2 (bottom edge and the
// two bottom corners).  One block owns kBandW columns; it computes the
// stencil values of its columns (plus halo) into shared memory, then marches
// down the rows, one thread per column, running the recurrence along j.
// NF fields: 2 for the velocity half step, 3 for the stress half step.
template <int NF, class PreAll>
__device__ void band_block(const StepParams& P, int bblock, PreAll pre_all, const int* fidx,
                           const float* const* tabs) {
    extern __shared__ float smem[];
    const int b = P.nbc, nx = P.nx, nz = P.nz;
    const int R = b + 1;              // rows nz-b-2 .. nz-2
    const int C = kBandW + 6;         // cols x0-3 .. x0+kBandW+2
    const int CF = kBandW + 2;        // chain cols x0-1 .. x0+kBandW
    float* Pm = smem;                 // [NF][R][C]
    float* Fa = smem + NF * R * C;    // [NF][CF]
    float* Fb = Fa + NF * CF;
    const int x0 = bblock * kBandW;
    const int j_top = nz - b - 2;

    for (int idx = threadIdx.x; idx < R * C; idx += blockDim.x) {
        const int r = idx / C, c = idx % C;
        const int i = x0 - 3 + c, j = j_top + r;
        float v[NF];
        if (i >= 0 && i < nx) {
            pre_all(i, j, v);
        } else {
#pragma unroll
            for (int f = 0; f < NF; ++f) v[f] = 0.f;
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) Pm[(f * R + r) * C + c] = v[f];
    }
    __syncthreads();

    auto PV = [&](int f, int i, int j) -> float { return Pm[(f * R + (j - j_top)) * C + (i - x0 + 3)]; };
    auto OV = [&](int f, int i, int j) -> float { return __ldg(P.in[fidx[f]] + cell(P, i, j)); };
    auto W = [&](int f, int i, int j) -> float { return habc_w(tabs[f], b, nx, nz, i, j); };
    const int r0 = nx - b - 1;

    // Row nz-b-2: final values after the edge loops (left/right edge cells
    // hold their edge result; others their stencil value).
    for (int cc = threadIdx.x; cc < CF; cc += blockDim.x) {
        const int i = x0 - 1 + cc, j = j_top;
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            float val = 0.f;
            if (i >= 0 && i < nx) {
                val = PV(f, i, j);
                if (i >= 1 && i <= b) {
                    val = blend_edge(W(f, i, j), PV(f, i, j),
                                     edge_sum(P.qx, P.qt_x, P.qxt, PV(f, i + 1, j), OV(f, i, j), OV(f, i + 1, j)));
                } else if (i >= r0 && i <= nx - 2) {
                    auto rplain = [&](int ii) {
                        return blend_edge(W(f, ii, j), PV(f, ii, j),
                                          edge_sum(P.qx, P.qt_x, P.qxt, PV(f, ii - 1, j), OV(f, ii, j), OV(f, ii - 1, j)));
                    };
                    if (i > r0 && right_chunk_start(nx, b, i)) {
                        val = blend_edge(W(f, i, j), PV(f, i, j),
                                         edge_sum(P.qx, P.qt_x, P.qxt, rplain(i - 1), OV(f, i, j), OV(f, i - 1, j)));
                    } else {
                        val = rplain(i);
                    }
                }
            }
            Fa[f * CF + cc] = val;
        }
    }
    __syncthreads();

    float* Fprev = Fa;
    float* Fcur = Fb;
    for (int j = j_top + 1; j <= nz - 2; ++j) {
        // Phase A: every column whose reads are the stencil values of row j
        // and the finals of row j-1.
        for (int cc = threadIdx.x; cc < CF; cc += blockDim.x) {
            const int i = x0 - 1 + cc;
            if (i < 0 || i >= nx) continue;
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                float val;
                const float own = PV(f, i, j);
                if (i == 0 || i == nx - 1) {
                    val = own;
                } else if (i <= b) {  // bottom-left corner
                    if (i == b) continue;  // phase B
                    const float sx = edge_sum(P.qx, P.qt_x, P.qxt, PV(f, i + 1, j), OV(f, i, j), OV(f, i + 1, j));
                    const float sz = edge_sum(P.qz, P.qt_z, P.qxt, Fprev[f * CF + cc], OV(f, i, j), OV(f, i, j - 1));
                    val = blend_corner(W(f, i, j), own, sx, sz);
                } else if (i >= r0) {  // bottom-right corner
                    if (right_chunk_start(nx, b, i)) continue;  // phase B
                    const float sx = edge_sum(P.qx, P.qt_x, P.qxt, PV(f, i - 1, j), OV(f, i, j), OV(f, i - 1, j));
                    const float sz = edge_sum(P.qz, P.qt_z, P.qxt, Fprev[f * CF + cc], OV(f, i, j), OV(f, i, j - 1));
                    val = blend_corner(W(f, i, j), own, sx, sz);
                } else {  // bottom edge
                    val = blend_edge(W(f, i, j), own,
                                     edge_sum(P.qz, P.qt_z, P.qxt, Fprev[f * CF + cc], OV(f, i, j), OV(f, i, j - 1)));
                }
                Fcur[f * CF + cc] = val;
            }
        }
        __syncthreads();
        // Phase B: the last bottom-left column reads the bottom edge's final
        // value at i+1; bottom-right chunk starts read the final value at i-1.
        for (int cc = threadIdx.x; cc < CF; cc += blockDim.x) {
            const int i = x0 - 1 + cc;
            if (i < 1 || i > nx - 2) continue;
            const bool bl_last = (i == b);
            const bool br_start = (i >= r0 && right_chunk_start(nx, b, i));
            if (!bl_last && !br_start) continue;
            if (bl_last && cc + 1 >= CF) continue;  // halo column: value unused
            if (br_start && cc == 0) continue;      // halo column: value unused
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const float own = PV(f, i, j);
                const int ix = bl_last ? i + 1 : i - 1;
                const float fx = Fcur[f * CF + (bl_last ? cc + 1 : cc - 1)];
                const float sx = edge_sum(P.qx, P.qt_x, P.qxt, fx, OV(f, i, j), OV(f, ix, j));
                const float sz = edge_sum(P.qz, P.qt_z, P.qxt, Fprev[f * CF + cc], OV(f, i, j), OV(f, i, j - 1));
                Fcur[f * CF + cc] = blend_corner(W(f, i, j), own, sx, sz);
            }
        }
        __syncthreads();
        for (int cc = 1 + threadIdx.x; cc <= kBandW; cc += blockDim.x) {
            const int i = x0 - 1 + cc;
            if (i < 1 || i > nx - 2) continue;
#pragma unroll
            for (int f = 0; f < NF; ++f) P.out[fidx[f]][cell(P, i, j)] = Fcur[f * CF + cc];
        }
        float* t = Fprev;
        Fprev = Fcur;
        Fcur = t;
        __syncthreads();
    }
}

__device__ __forceinline__ size_t band_smem_floats(int nf, int nbc) {
    return (size_t)nf * ((size_t)(nbc + 1) * (kBandW + 6) + 2 * (kBandW + 2));
}

// ---------------------------------------------------------------------------
// Velocity half step: update_velocity! + apply_habc_velocity!, with the
// source of this step injected into the stresses read and the receivers of
// the previous step recorded.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) velocity_simple_kernel(const StepParams P) {
    const int bid = blockIdx.x;
    if (bid < P.n_tile_blocks) {
        const int tx = bid % P.tiles_x, tz = bid / P.tiles_x;
        const int i = tx * kTileX + (threadIdx.x % kTileX);
        const int j = tz * kTileZ + (threadIdx.x / kTileX);
        if (i >= P.nx || j >= P.nz || in_bottom_band(P, i, j)) return;
        HabcPoint<VelPreF> hx{P, VelPreF{P, VX}, P.in[VX], P.w_tab[0]};
        HabcPoint<VelPreF> hz{P, VelPreF{P, VZ}, P.in[VZ], P.w_tab[1]};
        float vx, vz;
        vel_pre(P, i, j, vx, vz);
        const bool band = (i <= P.nbc) || (i >= P.nx - P.nbc - 1) || (!P.fs && j <= P.nbc);
        if (band) {
            vx = hx.final_value(i, j);
            vz = hz.final_value(i, j);
        }
        P.out[VX][cell(P, i, j)] = vx;
        P.out[VZ][cell(P, i, j)] = vz;
    } else if (bid < P.n_tile_blocks + P.n_band_blocks) {
        const int fidx[2] = {VX, VZ};
        const float* tabs[2] = {P.w_tab[0], P.w_tab[1]};
        band_block<2>(P, bid - P.n_tile_blocks,
                      [&](int i, int j, float* v) { vel_pre(P, i, j, v[0], v[1]); }, fidx, tabs);
    } else {
        record_block(P, bid - P.n_tile_blocks - P.n_band_blocks);
    }
}

// ---------------------------------------------------------------------------
// Stress half step: update_stress! + apply_habc_stress! + apply_free_surface!.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) stress_simple_kernel(const StepParams P) {
    const int bid = blockIdx.x;
    if (bid < P.n_tile_blocks) {
        const int tx = bid % P.tiles_x, tz = bid / P.tiles_x;
        const int i = tx * kTileX + (threadIdx.x % kTileX);
        const int j = tz * kTileZ + (threadIdx.x / kTileX);
        if (i >= P.nx || j >= P.nz || in_bottom_band(P, i, j)) return;
        float txx, tzz, txz;
        str_pre(P, i, j, txx, tzz, txz);
        const bool band = (i <= P.nbc) || (i >= P.nx - P.nbc - 1) || (!P.fs && j <= P.nbc);
        if (band) {
            HabcPoint<StrPreF> h0{P, StrPreF{P, TXX}, P.in[TXX], P.w_tab[2]};
            HabcPoint<StrPreF> h1{P, StrPreF{P, TZZ}, P.in[TZZ], P.w_tab[2]};
            HabcPoint<StrPreF> h2{P, StrPreF{P, TXZ}, P.in[TXZ], P.w_tab[2]};
            txx = h0.final_value(i, j);
            tzz = h1.final_value(i, j);
            txz = h2.final_value(i, j);
        }
        if (in_free_surface_rows(P, j)) {
            tzz = 0.f;
            txz = 0.f;
        }
        const size_t c = cell(P, i, j);
        P.out[TXX][c] = txx;
        P.out[TZZ][c] = tzz;
        P.out[TXZ][c] = txz;
    } else if (bid < P.n_tile_blocks + P.n_band_blocks) {
        const int fidx[3] = {TXX, TZZ, TXZ};
        const float* tabs[3] = {P.w_tab[2], P.w_tab[2], P.w_tab[2]};
        band_block<3>(P, bid - P.n_tile_blocks,
                      [&](int i, int j, float* v) { str_pre(P, i, j, v[0], v[1], v[2]); }, fidx, tabs);
    }
}

// Receivers of the last step (the velocity kernel of step k records k-1).
__global__ void record_kernel(const StepParams P) { record_block(P, blockIdx.x); }

}  // namespace fomo
