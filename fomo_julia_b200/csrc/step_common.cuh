// step_common.cuh -- per-cell semantics of one Elastic2D time step on sm_100a.
//
// Shared by every kernel variant.  Everything here is a pure function of the
// step's read-only inputs, so any thread may recompute any cell's value; the
// kernels use that to apply the in-place boundary updates of the reference
// without races.
//
// Arithmetic follows the reference's Float32 CPU methods operation by
// operation (no FMA contraction: __fadd_rn/__fmul_rn/__fdiv_rn are IEEE
// round-to-nearest), so results are bit-identical to a scalar CPU evaluation
// of the same expressions:
//   velocity  src/kernels/velocity.jl:30-44
//   stress    src/kernels/stress.jl:27-45
//   HABC      src/kernels/boundary.jl:68-132
//   free surf src/kernels/boundary.jl:168-181
//   source    src/kernels/source_receiver.jl:18-30
//   receivers src/kernels/source_receiver.jl:65-77
//
// Indices are 0-based here: the reference's cell (i, j) is (i-1, j-1).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fomo {

constexpr int kMaxM = 6;
enum Field { VX = 0, VZ = 1, TXX = 2, TZZ = 3, TXZ = 4 };

// Parameters of one half step (velocity or stress), passed by value.
struct StepParams {
    int nx, nz, pitch;          // padded grid; row pitch in floats
    int M, pad, nbc, fs;        // half stencil width, padding, HABC layers, free surface
    float dtx, dtz;
    float a[kMaxM];
    float qx, qz, qt_x, qt_z, qxt;
    const float* w_tab[3];      // weight by dist (nbc+2 entries): vx, vz, tau
    const float* rho_vx;
    const float* rho_vz;
    const float* lam;
    const float* mu_txx;
    const float* mu_txz;
    const float* in[5];         // fields read by this half step
    float* out[5];              // fields written by this half step
    int src_i, src_j;           // 0-based source cell
    float src_w;                // wavelet sample injected this step (0 if none)
    int rec_k;                  // 1-based step whose receivers are recorded from `in` (0 = none)
    int nt, n_rec, rec_kind;
    const int* rec_cell;        // receiver r at linear offset i + j*pitch
    float* gather;              // [nt x n_rec] column major
    int tiles_x, tiles_z;       // tile grid of the cell pass
    int n_tile_blocks, n_band_blocks;
};

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ size_t cell(const StepParams& P, int i, int j) {
    return (size_t)i + (size_t)j * (size_t)P.pitch;
}

// P.in[q] for a q known only at run time, written as selects so the
// parameter block is not copied to local memory.
__device__ __forceinline__ const float* in_field(const StepParams& P, int q) {
    const float* p = P.in[0];
    p = q == 1 ? P.in[1] : p;
    p = q == 2 ? P.in[2] : p;
    p = q == 3 ? P.in[3] : p;
    p = q == 4 ? P.in[4] : p;
    return p;
}

// P.out[q] and P.w_tab[t] for indices known only at run time, as selects.
__device__ __forceinline__ float* out_field(const StepParams& P, int q) {
    float* p = P.out[0];
    p = q == 1 ? P.out[1] : p;
    p = q == 2 ? P.out[2] : p;
    p = q == 3 ? P.out[3] : p;
    p = q == 4 ? P.out[4] : p;
    return p;
}
__device__ __forceinline__ const float* w_table(const StepParams& P, int t) {
    const float* p = P.w_tab[0];
    p = t == 1 ? P.w_tab[1] : p;
    p = t == 2 ? P.w_tab[2] : p;
    return p;
}

// ---------------------------------------------------------------------------
// Stencils.  The explosive source (txx, tzz += w at the source cell,
// source_receiver.jl:26-27) is applied to the values read, never stored, so
// the stored fields keep the pre-injection values the HABC needs as f_old.
// ---------------------------------------------------------------------------
// src_w is the wavelet sample of this step (P.src_w on the single-shot path).
__device__ __forceinline__ float tau_in(const StepParams& P, int q, int i, int j, float src_w) {
    float v = __ldg(in_field(P, q) + cell(P, i, j));
    if (q != TXZ && i == P.src_i && j == P.src_j) v = fadd(v, src_w);
    return v;
}

__device__ __forceinline__ bool in_stencil(const StepParams& P, int i, int j) {
    return i >= P.M && i <= P.nx - 1 - P.M && j >= P.M && j <= P.nz - 1 - P.M;
}

// ---------------------------------------------------------------------------
// HABC (boundary.jl:68-132).  Region loops run in program order: left,
// right, bottom, top (no free surface), then the corners bottom-left,
// bottom-right, top-left, top-right.  Within a loop the i loop runs in
// chunks of 8 cells from its first i and reads inside a chunk see the values
// held before the chunk was stored (the 8-lane Float32 AVX2 vectorisation of
// @tturbo that produced the reference's shot_1.bin); rows j run in order.
// Consequences used below:
//   left, top edges, and reads of i+1 / j+1 in corners: pre-loop values;
//   right edge, reads of i-1 in right corners: pre-loop value, except at a
//     chunk start, which reads the final value of the previous chunk's last
//     cell;
//   bottom edge, reads of j-1 in bottom corners: final value of the row above
//     (a recurrence along j, run by the band pass).
// ---------------------------------------------------------------------------
constexpr int kChunk = 8;

__device__ __forceinline__ float habc_w(const float* tab, int nbc, int nx, int nz, int i, int j) {
    int d = min(min(i, nx - 1 - i), min(j, nz - 1 - j));
    d = min(d, nbc + 1);
    return __ldg(tab + d);
}

__device__ __forceinline__ float edge_sum(float q, float qt, float qxt, float f_nb, float old_c, float old_nb) {
    return fsub(fsub(fmul(-q, f_nb), fmul(qt, old_c)), fmul(qxt, old_nb));
}

__device__ __forceinline__ float blend_edge(float w, float f, float s) {
    return fadd(fmul(w, f), fmul(fsub(1.f, w), s));
}

__device__ __forceinline__ float blend_corner(float w, float f, float sx, float sz) {
    return fadd(fmul(w, f), fmul(fmul(fsub(1.f, w), 0.5f), fadd(sx, sz)));
}

__device__ __forceinline__ bool right_chunk_start(int nx, int nbc, int i) {
    return ((i - (nx - nbc - 1)) % kChunk) == 0;
}

// Pointwise HABC evaluation for the cells outside the bottom band.  `pre(i,j)`
// returns this field's value after the stencil update; `old` is the field at
// the start of the step.
template <class PreF>
struct HabcPoint {
    const StepParams& P;
    PreF pre;
    const float* old;
    const float* tab;

    __device__ float o(int i, int j) const { return __ldg(old + cell(P, i, j)); }
    __device__ float w(int i, int j) const { return habc_w(tab, P.nbc, P.nx, P.nz, i, j); }

    __device__ float left_final(int i, int j) const {
        return blend_edge(w(i, j), pre(i, j), edge_sum(P.qx, P.qt_x, P.qxt, pre(i + 1, j), o(i, j), o(i + 1, j)));
    }
    // Right edge cell that is not a chunk start: reads the pre value of i-1.
    __device__ float right_plain(int i, int j) const {
        return blend_edge(w(i, j), pre(i, j), edge_sum(P.qx, P.qt_x, P.qxt, pre(i - 1, j), o(i, j), o(i - 1, j)));
    }
    __device__ float right_final(int i, int j) const {
        const int r0 = P.nx - P.nbc - 1;
        if (i > r0 && right_chunk_start(P.nx, P.nbc, i)) {
            const float fn = right_plain(i - 1, j);
            return blend_edge(w(i, j), pre(i, j), edge_sum(P.qx, P.qt_x, P.qxt, fn, o(i, j), o(i - 1, j)));
        }
        return right_plain(i, j);
    }
    __device__ float top_final(int i, int j) const {
        return blend_edge(w(i, j), pre(i, j), edge_sum(P.qz, P.qt_z, P.qxt, pre(i, j + 1), o(i, j), o(i, j + 1)));
    }
    __device__ float corner(int i, int j, float own, float fx, int ix, float fz, int jz) const {
        const float sx = edge_sum(P.qx, P.qt_x, P.qxt, fx, o(i, j), o(ix, j));
        const float sz = edge_sum(P.qz, P.qt_z, P.qxt, fz, o(i, j), o(i, jz));
        return blend_corner(w(i, j), own, sx, sz);
    }
    // Top-left corner (no free surface): the left edge loop already covered
    // these cells, so their own and neighbour values are post-left-edge.
    __device__ float tl_final(int i, int j) const {
        const float fx = (i + 1 <= P.nbc) ? left_final(i + 1, j) : top_final(i + 1, j);
        return corner(i, j, left_final(i, j), fx, i + 1, left_final(i, j + 1), j + 1);
    }
    __device__ float tr_plain(int i, int j) const {  // not a chunk start
        return corner(i, j, right_final(i, j), right_final(i - 1, j), i - 1, right_final(i, j + 1), j + 1);
    }
    __device__ float tr_final(int i, int j) const {
        const int r0 = P.nx - P.nbc - 1;
        if (right_chunk_start(P.nx, P.nbc, i)) {
            const float fx = (i == r0) ? top_final(i - 1, j) : tr_plain(i - 1, j);
            return corner(i, j, right_final(i, j), fx, i - 1, right_final(i, j + 1), j + 1);
        }
        return tr_plain(i, j);
    }

    // Final value of a cell outside the bottom band.
    __device__ float final_value(int i, int j) const {
        const int b = P.nbc, nx = P.nx, nz = P.nz;
        const int js0 = P.fs ? b : 1;
        const bool inL = i >= 1 && i <= b;
        const bool inR = i >= nx - b - 1 && i <= nx - 2;
        const bool top_rows = !P.fs && j >= 1 && j <= b;
        if (top_rows) {
            if (inL) return tl_final(i, j);
            if (inR) return tr_final(i, j);
            if (i >= b + 1 && i <= nx - b - 2) return top_final(i, j);
        }
        if (j >= js0 && j <= nz - b - 2) {
            if (inL) return left_final(i, j);
            if (inR) return right_final(i, j);
        }
        return pre(i, j);
    }
};

__device__ __forceinline__ bool in_bottom_band(const StepParams& P, int i, int j) {
    return j >= P.nz - P.nbc - 1 && j <= P.nz - 2 && i >= 1 && i <= P.nx - 2;
}

__device__ __forceinline__ bool in_free_surface_rows(const StepParams& P, int j) {
    return P.fs && j >= P.pad - 5 && j <= P.pad;
}

}  // namespace fomo
