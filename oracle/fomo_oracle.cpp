// fomo_oracle.cpp -- CPU restatement of the Elastic2D time-stepping path of
// Wuheng10086/Fomo_julia.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: the tests, the
// smoke check and the CPU-baseline leg of bench.py call it as the checker.
// The product (libfomo_b200.so and the fomo_julia_b200 package) never links
// or calls it.
//
// The reference is pure Julia and cannot run in this image (no julia binary),
// so this is a restatement of its CPU methods in C++17, templated on the
// arithmetic type (float reproduces the reference's Float32 path; double is
// the Float64 accuracy reference the reference itself cannot produce).
//
// Two switches cover what the Julia source leaves open:
//   * habc_mode  2 = "simd8" (canonical): program order of the Julia loops
//                    (`for j in J, i in I`: j outer, i inner) with the i loop
//                    run in chunks of 8 cells from its first i, reads inside a
//                    chunk seeing pre-chunk values -- the 8-lane Float32 AVX2
//                    vectorisation of @tturbo.  This is the mode that
//                    reproduces the reference's shot_1.bin (max 3.2e-6 per
//                    trace, against 4.8e-5 for the two modes below);
//                0 = "jacobi":     every region loop reads the values the
//                                  region held before the loop started;
//                1 = "sequential": scalar program order.
//   * contract   0 = no FMA contraction (every * and + rounded separately);
//                1 = the FMA contraction pattern documented at each site.
//
// Indices are 1-based in the comments (as in Julia) and converted with
// IX(i, j) = (i-1) + (j-1)*nx: column-major, x fastest, exactly the Julia
// memory layout of an (nx, nz) matrix.
//
// Build: see oracle/Makefile (-O3 -fno-fast-math -ffp-contract=off -fopenmp).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Shot description shared by the float and double runners.  Pointers of type
// `const void*` point at arrays of the runner's arithmetic type T.
typedef struct {
    int32_t nx, nz;            // padded grid (nx_in + 2 pad, nz_in + 2 pad)
    int32_t M, pad, nbc;       // half stencil width, padding, HABC layers
    int32_t free_surface;      // 0/1
    const void* rho_vx;        // T[nx*nz], x fastest
    const void* rho_vz;
    const void* lam;
    const void* mu_txx;
    const void* mu_txz;
    double qx, qz, qt_x, qt_z, qxt;   // HABC coefficients (converted to T)
    const void* w_vx_table;    // T[nbc+2]: weight as a function of dist
    const void* w_vz_table;
    const void* w_tau_table;
    const void* a;             // T[M] FD coefficients
    double dt, dtx, dtz;       // converted to T
    int32_t nt;
    int32_t src_i, src_j;      // 1-based
    const void* wavelet;       // T[n_wavelet]
    int32_t n_wavelet;
    int32_t n_rec;
    const int32_t* rec_i;      // 1-based
    const int32_t* rec_j;
    int32_t rec_kind;          // 0 = vz, 1 = vx, 2 = p
    int32_t habc_mode;         // 0 jacobi, 1 sequential, 2 simd8 (canonical)
    int32_t contract;          // 0 none, 1 fma
    int32_t n_threads;         // 0 = OpenMP default
} OrcShot;

}  // extern "C"

namespace {

template <class T>
struct State {
    int nx, nz;
    std::vector<T> f[5];      // vx, vz, txx, tzz, txz
    std::vector<T> old[5];    // *_old backups
    State(int nx_, int nz_) : nx(nx_), nz(nz_) {
        for (int q = 0; q < 5; ++q) {
            f[q].assign((size_t)nx * nz, T(0));
            old[q].assign((size_t)nx * nz, T(0));
        }
    }
};

enum { VX = 0, VZ = 1, TXX = 2, TZZ = 3, TXZ = 4 };

struct Grid {
    int nx, nz;
    inline size_t operator()(int i, int j) const {  // 1-based (i, j)
        return (size_t)(i - 1) + (size_t)(j - 1) * (size_t)nx;
    }
};

template <class T>
inline T madd(bool fma_on, T a, T b, T c) {  // a*b + c
    return fma_on ? std::fma(a, b, c) : a * b + c;
}

// ---------------------------------------------------------------------------
// Stage 1: backup_boundary!  (src/kernels/boundary.jl:20-56)
// Copies f -> f_old on the vertical strips i in [1, nbc+2] U [nx-nbc-1, nx]
// (rows j_top..nz) and the horizontal strips j in [j_top, nbc+2] U
// [nz-nbc-1, nz] (columns nbc+3..nx-nbc-2); j_top = fs ? nbc+1 : 1.
// ---------------------------------------------------------------------------
template <class T>
void backup_boundary(State<T>& s, int nbc, bool fs) {
    Grid G{s.nx, s.nz};
    const int nx = s.nx, nz = s.nz;
    const int j_top = fs ? nbc + 1 : 1;
    for (int q = 0; q < 5; ++q) {
        T* dst = s.old[q].data();
        const T* src = s.f[q].data();
        for (int j = j_top; j <= nz; ++j) {
            for (int i = 1; i <= nbc + 2; ++i) dst[G(i, j)] = src[G(i, j)];
            for (int i = nx - nbc - 1; i <= nx; ++i) dst[G(i, j)] = src[G(i, j)];
        }
        for (int j = j_top; j <= nbc + 2; ++j)
            for (int i = nbc + 3; i <= nx - nbc - 2; ++i) dst[G(i, j)] = src[G(i, j)];
        for (int j = nz - nbc - 1; j <= nz; ++j)
            for (int i = nbc + 3; i <= nx - nbc - 2; ++i) dst[G(i, j)] = src[G(i, j)];
    }
}

// ---------------------------------------------------------------------------
// Stage 2: inject_source!  (src/kernels/source_receiver.jl:18-30)
// ---------------------------------------------------------------------------
template <class T>
void inject_source(State<T>& s, int si, int sj, const T* wav, int n_wav, int k) {
    if (k > n_wav) return;
    Grid G{s.nx, s.nz};
    const T w = wav[k - 1];
    s.f[TXX][G(si, sj)] += w;
    s.f[TZZ][G(si, sj)] += w;
}

// ---------------------------------------------------------------------------
// Stage 3: update_velocity!  (src/kernels/velocity.jl:21-46)
// Interior i in [M+1, nx-M], j in [M+1, nz-M].  Accumulators start at 0 and
// add l = 1..M in order.  contract=1: acc = fma(a_l, diff, acc) and
// v + fma(b_x, d_x, b_z*d_z).
// ---------------------------------------------------------------------------
template <class T>
void update_velocity(State<T>& s, const T* rho_vx, const T* rho_vz, const T* a, int M,
                     T dtx, T dtz, bool fma_on) {
    Grid G{s.nx, s.nz};
    const int nx = s.nx, nz = s.nz;
    T* vx = s.f[VX].data();
    T* vz = s.f[VZ].data();
    const T* txx = s.f[TXX].data();
    const T* tzz = s.f[TZZ].data();
    const T* txz = s.f[TXZ].data();
#pragma omp parallel for schedule(static)
    for (int j = M + 1; j <= nz - M; ++j) {
        for (int i = M + 1; i <= nx - M; ++i) {
            T dtxxdx = 0, dtxzdz = 0, dtxzdx = 0, dtzzdz = 0;
            for (int l = 1; l <= M; ++l) {
                const T al = a[l - 1];
                dtxxdx = madd(fma_on, al, T(txx[G(i + l - 1, j)] - txx[G(i - l, j)]), dtxxdx);
                dtxzdz = madd(fma_on, al, T(txz[G(i, j + l - 1)] - txz[G(i, j - l)]), dtxzdz);
                dtxzdx = madd(fma_on, al, T(txz[G(i + l, j)] - txz[G(i - l + 1, j)]), dtxzdx);
                dtzzdz = madd(fma_on, al, T(tzz[G(i, j + l)] - tzz[G(i, j - l + 1)]), dtzzdz);
            }
            const size_t c = G(i, j);
            const T bxx = dtx / rho_vx[c], bxz = dtz / rho_vx[c];
            const T bzx = dtx / rho_vz[c], bzz = dtz / rho_vz[c];
            vx[c] = vx[c] + madd(fma_on, bxx, dtxxdx, T(bxz * dtxzdz));
            vz[c] = vz[c] + madd(fma_on, bzx, dtxzdx, T(bzz * dtzzdz));
        }
    }
}

// ---------------------------------------------------------------------------
// Stage 5: update_stress!  (src/kernels/stress.jl:18-47)
// contract=1: acc = fma(a_l, diff, acc);
//   txx + fma(l2m, dvxdx*dtx, l*(dvzdz*dtz));
//   tzz + fma(l,   dvxdx*dtx, l2m*(dvzdz*dtz));
//   fma(mu_xz, fma(dvxdz, dtz, dvzdx*dtx), txz).
// ---------------------------------------------------------------------------
template <class T>
void update_stress(State<T>& s, const T* lam, const T* mu_txx, const T* mu_txz, const T* a,
                   int M, T dtx, T dtz, bool fma_on) {
    Grid G{s.nx, s.nz};
    const int nx = s.nx, nz = s.nz;
    const T* vx = s.f[VX].data();
    const T* vz = s.f[VZ].data();
    T* txx = s.f[TXX].data();
    T* tzz = s.f[TZZ].data();
    T* txz = s.f[TXZ].data();
#pragma omp parallel for schedule(static)
    for (int j = M + 1; j <= nz - M; ++j) {
        for (int i = M + 1; i <= nx - M; ++i) {
            T dvxdx = 0, dvzdz = 0, dvxdz = 0, dvzdx = 0;
            for (int l = 1; l <= M; ++l) {
                const T al = a[l - 1];
                dvxdx = madd(fma_on, al, T(vx[G(i + l, j)] - vx[G(i - l + 1, j)]), dvxdx);
                dvzdz = madd(fma_on, al, T(vz[G(i, j + l - 1)] - vz[G(i, j - l)]), dvzdz);
                dvxdz = madd(fma_on, al, T(vx[G(i, j + l)] - vx[G(i, j - l + 1)]), dvxdz);
                dvzdx = madd(fma_on, al, T(vz[G(i + l - 1, j)] - vz[G(i - l, j)]), dvzdx);
            }
            const size_t c = G(i, j);
            const T l_val = lam[c];
            const T m_val = mu_txx[c];
            const T l2m = l_val + T(2) * m_val;
            const T ex = dvxdx * dtx;
            const T ez = dvzdz * dtz;
            if (fma_on) {
                txx[c] = txx[c] + std::fma(l2m, ex, T(l_val * ez));
                tzz[c] = tzz[c] + std::fma(l_val, ex, T(l2m * ez));
                txz[c] = std::fma(mu_txz[c], std::fma(dvxdz, dtz, T(dvzdx * dtx)), txz[c]);
            } else {
                txx[c] = txx[c] + (T(l2m * ex) + T(l_val * ez));
                tzz[c] = tzz[c] + (T(l_val * ex) + T(l2m * ez));
                txz[c] = txz[c] + T(mu_txz[c] * T(T(dvxdz * dtz) + T(dvzdx * dtx)));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Stage 4/6: apply_habc!  (src/kernels/boundary.jl:68-132)
//
// Regions in program order (js = fs ? nbc+1 : 2):
//   left   j in [js, nz-nbc-1], i in [2, nbc+1]       reads f[i+1,j]
//   right  j in [js, nz-nbc-1], i in [nx-nbc, nx-1]   reads f[i-1,j]
//   bottom j in [nz-nbc, nz-1], i in [nbc+2, nx-nbc-1] reads f[i,j-1]
//   top    (!fs) j in [2, nbc+1], same i as bottom    reads f[i,j+1]
//   corners bottom-left, bottom-right, then (!fs) top-left, top-right:
//     f = w f + (1-w) 0.5 (s_x + s_z)
// Edge:  s = -q f[nb] - qt f_old[c] - qxt f_old[nb];  f = w f + (1-w) s.
// contract=1: s = fma(-qxt, old_nb, fma(-qt, old_c, (-q)*f_nb));
//             f = fma(w, f, (1-w)*s)   (corner: fma(w, f, ((1-w)*0.5)*(sx+sz))).
// The weight depends only on dist = min(i-1, nx-i, j-1, nz-j)
// (src/utils/init.jl:188-195), so it is read from a table indexed by dist.
// ---------------------------------------------------------------------------
template <class T>
struct Habc {
    T qx, qz, qt_x, qt_z, qxt;
    int nbc;
    bool fs;
    bool fma_on;
};

template <class T>
inline T wt(const T* table, int nbc, int nx, int nz, int i, int j) {
    int d = std::min(std::min(i - 1, nx - i), std::min(j - 1, nz - j));
    if (d > nbc + 1) d = nbc + 1;
    return table[d];
}

template <class T>
inline T edge_sum(const Habc<T>& h, T q, T qt, T f_nb, T old_c, T old_nb) {
    if (h.fma_on) {
        T t = (-q) * f_nb;
        t = std::fma(-qt, old_c, t);
        return std::fma(-h.qxt, old_nb, t);
    }
    return T(T(T((-q) * f_nb) - T(qt * old_c)) - T(h.qxt * old_nb));
}

template <class T>
inline T blend_edge(const Habc<T>& h, T w, T f, T s) {
    if (h.fma_on) return std::fma(w, f, T(T(T(1) - w) * s));
    return T(w * f) + T(T(T(1) - w) * s);
}

template <class T>
inline T blend_corner(const Habc<T>& h, T w, T f, T sx, T sz) {
    const T c = T(T(1) - w) * T(0.5);
    if (h.fma_on) return std::fma(w, f, T(c * T(sx + sz)));
    return T(w * f) + T(c * T(sx + sz));
}

// One cell of a region, reading the current contents of f.  (di, dj) is the
// neighbour the one-way extrapolation reads: edges use one of them, corners
// both (s_x from (i+di, j), s_z from (i, j+dj)).
template <class T>
inline T habc_cell(const T* f, const T* fo, const Habc<T>& h, const T* table, int nx, int nz,
                   int i, int j, int di, int dj, bool corner) {
    Grid G{nx, nz};
    const size_t c = G(i, j);
    const T w = wt(table, h.nbc, nx, nz, i, j);
    if (corner) {
        const size_t nxb = G(i + di, j), nzb = G(i, j + dj);
        const T sx = edge_sum(h, h.qx, h.qt_x, f[nxb], fo[c], fo[nxb]);
        const T sz = edge_sum(h, h.qz, h.qt_z, f[nzb], fo[c], fo[nzb]);
        return blend_corner(h, w, f[c], sx, sz);
    }
    const size_t n = G(i + di, j + dj);
    const T q = di != 0 ? h.qx : h.qz;
    const T qt = di != 0 ? h.qt_x : h.qt_z;
    return blend_edge(h, w, f[c], edge_sum(h, q, qt, f[n], fo[c], fo[n]));
}

// One region loop of apply_habc!.
//   chunk == 0 : jacobi -- every read sees the region as it was before the loop.
//   chunk >= 1 : program order (j outer ascending, i inner ascending) with the
//                i loop run in chunks of `chunk` cells starting at i0; reads
//                inside a chunk see the values held before the chunk was
//                stored.  chunk = 1 is plain scalar order; chunk = 8 is the
//                8-lane Float32 vectorisation of @tturbo on AVX2, the mode
//                that reproduces the reference's shot_1.bin.
template <class T>
void habc_region(T* f, const T* fo, const Habc<T>& h, const T* table, int nx, int nz, int i0,
                 int i1, int j0, int j1, int di, int dj, bool corner, int chunk,
                 std::vector<T>& tmp) {
    if (i1 < i0 || j1 < j0) return;
    Grid G{nx, nz};
    const int W = i1 - i0 + 1;
    const bool reads_ahead = !corner && (di > 0 || dj > 0);  // left / top edges
    if (chunk == 0 || reads_ahead) {
        // Jacobi.  For the left and top edges every chunked order is the same:
        // the cell they read is either in the same chunk or not yet stored.
        tmp.resize((size_t)W * (j1 - j0 + 1));
#pragma omp parallel for schedule(static)
        for (int j = j0; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i)
                tmp[(size_t)(i - i0) + (size_t)(j - j0) * W] =
                    habc_cell(f, fo, h, table, nx, nz, i, j, di, dj, corner);
#pragma omp parallel for schedule(static)
        for (int j = j0; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i) f[G(i, j)] = tmp[(size_t)(i - i0) + (size_t)(j - j0) * W];
        return;
    }
    if (!corner && dj == 0) {
        // Right edge: rows are independent; chunked recurrence along i.
#pragma omp parallel for schedule(static)
        for (int j = j0; j <= j1; ++j) {
            T buf[64];
            for (int c0 = i0; c0 <= i1; c0 += chunk) {
                const int c1 = std::min(c0 + std::min(chunk, 64) - 1, i1);
                for (int i = c0; i <= c1; ++i) buf[i - c0] = habc_cell(f, fo, h, table, nx, nz, i, j, di, dj, false);
                for (int i = c0; i <= c1; ++i) f[G(i, j)] = buf[i - c0];
            }
        }
        return;
    }
    if (!corner && di == 0) {
        // Bottom edge: columns are independent; recurrence along j.
#pragma omp parallel for schedule(static)
        for (int i = i0; i <= i1; ++i)
            for (int j = j0; j <= j1; ++j) f[G(i, j)] = habc_cell(f, fo, h, table, nx, nz, i, j, di, dj, false);
        return;
    }
    // Corners: serial program order with chunks along i.
    std::vector<T> buf((size_t)std::max(chunk, 1));
    for (int j = j0; j <= j1; ++j)
        for (int c0 = i0; c0 <= i1; c0 += chunk) {
            const int c1 = std::min(c0 + chunk - 1, i1);
            for (int i = c0; i <= c1; ++i) buf[i - c0] = habc_cell(f, fo, h, table, nx, nz, i, j, di, dj, true);
            for (int i = c0; i <= c1; ++i) f[G(i, j)] = buf[i - c0];
        }
}

template <class T>
void apply_habc(T* f, const T* fo, const Habc<T>& h, const T* table, int nx, int nz, int chunk,
                std::vector<T>& tmp) {
    const int nbc = h.nbc;
    const int js = h.fs ? nbc + 1 : 2;
    // 1. edges
    habc_region(f, fo, h, table, nx, nz, 2, nbc + 1, js, nz - nbc - 1, +1, 0, false, chunk, tmp);            // left
    habc_region(f, fo, h, table, nx, nz, nx - nbc, nx - 1, js, nz - nbc - 1, -1, 0, false, chunk, tmp);      // right
    habc_region(f, fo, h, table, nx, nz, nbc + 2, nx - nbc - 1, nz - nbc, nz - 1, 0, -1, false, chunk, tmp); // bottom
    if (!h.fs)
        habc_region(f, fo, h, table, nx, nz, nbc + 2, nx - nbc - 1, 2, nbc + 1, 0, +1, false, chunk, tmp);  // top
    // 2. corners
    habc_region(f, fo, h, table, nx, nz, 2, nbc + 1, nz - nbc, nz - 1, +1, -1, true, chunk, tmp);          // bottom-left
    habc_region(f, fo, h, table, nx, nz, nx - nbc, nx - 1, nz - nbc, nz - 1, -1, -1, true, chunk, tmp);    // bottom-right
    if (!h.fs) {
        habc_region(f, fo, h, table, nx, nz, 2, nbc + 1, 2, nbc + 1, +1, +1, true, chunk, tmp);            // top-left
        habc_region(f, fo, h, table, nx, nz, nx - nbc, nx - 1, 2, nbc + 1, -1, +1, true, chunk, tmp);      // top-right
    }
}

// ---------------------------------------------------------------------------
// Stage 7: apply_free_surface!  (src/kernels/boundary.jl:168-181)
// tzz = txz = 0 on rows j in [pad-4, pad+1] (rows below 1 are skipped).
// ---------------------------------------------------------------------------
template <class T>
void free_surface(State<T>& s, int pad) {
    Grid G{s.nx, s.nz};
    const int j_fs = pad + 1;
    for (int j = std::max(1, j_fs - 5); j <= j_fs; ++j)
        for (int i = 1; i <= s.nx; ++i) {
            s.f[TZZ][G(i, j)] = T(0);
            s.f[TXZ][G(i, j)] = T(0);
        }
}

// ---------------------------------------------------------------------------
// Stage 8: record_receivers!  (src/kernels/source_receiver.jl:65-77)
// data is [nt x n_rec] column-major: data[(k-1) + r*nt].
// ---------------------------------------------------------------------------
template <class T>
void record(const State<T>& s, const int32_t* ri, const int32_t* rj, int n_rec, int kind, int k,
            int nt, T* data) {
    Grid G{s.nx, s.nz};
    for (int r = 0; r < n_rec; ++r) {
        const size_t c = G(ri[r], rj[r]);
        T v;
        if (kind == 0) v = s.f[VZ][c];
        else if (kind == 1) v = s.f[VX][c];
        else v = T(s.f[TXX][c] + s.f[TZZ][c]) * T(0.5);
        data[(size_t)(k - 1) + (size_t)r * nt] = v;
    }
}

// ---------------------------------------------------------------------------
// time_step! (src/simulation/time_stepper.jl:39-63) and the k loop of
// run_time_loop! (time_stepper.jl:97-128) inside run_shot!
// (src/simulation/shot_manager.jl:46-68): reset, run, return the gather.
// ---------------------------------------------------------------------------
template <class T>
int run_shot(const OrcShot* p, T* gather, T* final_fields, int n_steps_limit) {
    if (!p || p->nx < 3 || p->nz < 3 || p->M < 1 || p->nt < 0) return -1;
    if (p->n_threads > 0) {
#ifdef _OPENMP
        omp_set_num_threads(p->n_threads);
#endif
    }
    State<T> s(p->nx, p->nz);
    const T* rho_vx = (const T*)p->rho_vx;
    const T* rho_vz = (const T*)p->rho_vz;
    const T* lam = (const T*)p->lam;
    const T* mu_txx = (const T*)p->mu_txx;
    const T* mu_txz = (const T*)p->mu_txz;
    const T* a = (const T*)p->a;
    const T* wav = (const T*)p->wavelet;
    const T dtx = (T)p->dtx, dtz = (T)p->dtz;
    const bool fma_on = p->contract != 0;
    const int chunk = p->habc_mode == 0 ? 0 : (p->habc_mode == 1 ? 1 : 8);
    const bool fs = p->free_surface != 0;
    Habc<T> h{(T)p->qx, (T)p->qz, (T)p->qt_x, (T)p->qt_z, (T)p->qxt, p->nbc, fs, fma_on};
    std::vector<T> tmp;
    const int nsteps = n_steps_limit >= 0 ? std::min(n_steps_limit, p->nt) : p->nt;
    if (gather) std::memset(gather, 0, sizeof(T) * (size_t)p->nt * (size_t)std::max(p->n_rec, 0));
    for (int k = 1; k <= nsteps; ++k) {
        backup_boundary(s, p->nbc, fs);
        inject_source(s, p->src_i, p->src_j, wav, p->n_wavelet, k);
        update_velocity(s, rho_vx, rho_vz, a, p->M, dtx, dtz, fma_on);
        apply_habc(s.f[VX].data(), s.old[VX].data(), h, (const T*)p->w_vx_table, s.nx, s.nz, chunk, tmp);
        apply_habc(s.f[VZ].data(), s.old[VZ].data(), h, (const T*)p->w_vz_table, s.nx, s.nz, chunk, tmp);
        update_stress(s, lam, mu_txx, mu_txz, a, p->M, dtx, dtz, fma_on);
        apply_habc(s.f[TXX].data(), s.old[TXX].data(), h, (const T*)p->w_tau_table, s.nx, s.nz, chunk, tmp);
        apply_habc(s.f[TZZ].data(), s.old[TZZ].data(), h, (const T*)p->w_tau_table, s.nx, s.nz, chunk, tmp);
        apply_habc(s.f[TXZ].data(), s.old[TXZ].data(), h, (const T*)p->w_tau_table, s.nx, s.nz, chunk, tmp);
        if (fs) free_surface(s, p->pad);
        if (gather && p->n_rec > 0) record(s, p->rec_i, p->rec_j, p->n_rec, p->rec_kind, k, p->nt, gather);
    }
    if (final_fields) {
        const size_t n = (size_t)p->nx * p->nz;
        for (int q = 0; q < 5; ++q) std::memcpy(final_fields + q * n, s.f[q].data(), n * sizeof(T));
    }
    return 0;
}

// ---------------------------------------------------------------------------
// init.jl restatements
// ---------------------------------------------------------------------------

// Staggered Taylor coefficients from the linear system
// sum_l a_l (2l-1)^(2k-1) = delta_{k1}, k = 1..M, solved in long double.
void taylor_coefficients(int M, long double* out) {
    std::vector<long double> A((size_t)M * M), b(M, 0.0L);
    for (int k = 0; k < M; ++k) {
        for (int l = 0; l < M; ++l) A[(size_t)k * M + l] = std::pow((long double)(2 * l + 1), 2 * k + 1);
        b[k] = (k == 0) ? 1.0L : 0.0L;
    }
    for (int c = 0; c < M; ++c) {  // Gaussian elimination with partial pivoting
        int piv = c;
        for (int r = c + 1; r < M; ++r)
            if (std::fabs(A[(size_t)r * M + c]) > std::fabs(A[(size_t)piv * M + c])) piv = r;
        for (int q = 0; q < M; ++q) std::swap(A[(size_t)c * M + q], A[(size_t)piv * M + q]);
        std::swap(b[c], b[piv]);
        for (int r = c + 1; r < M; ++r) {
            const long double f = A[(size_t)r * M + c] / A[(size_t)c * M + c];
            for (int q = c; q < M; ++q) A[(size_t)r * M + q] -= f * A[(size_t)c * M + q];
            b[r] -= f * b[c];
        }
    }
    for (int r = M - 1; r >= 0; --r) {
        long double s = b[r];
        for (int q = r + 1; q < M; ++q) s -= A[(size_t)r * M + q] * out[q];
        out[r] = s / A[(size_t)r * M + r];
    }
}

template <class T>
void pad_array(const float* data, int nx_in, int nz_in, int pad, T* out) {
    // _pad_array (src/utils/init.jl:119-134): copy, then replicate the edges.
    const int nx = nx_in + 2 * pad, nz = nz_in + 2 * pad;
    for (int j = 1; j <= nz; ++j) {
        const int jj = std::min(std::max(j - pad, 1), nz_in);
        for (int i = 1; i <= nx; ++i) {
            const int ii = std::min(std::max(i - pad, 1), nx_in);
            out[(size_t)(i - 1) + (size_t)(j - 1) * nx] = (T)data[(size_t)(ii - 1) + (size_t)(jj - 1) * nx_in];
        }
    }
}

template <class T>
void staggered_params(const T* vp, const T* vs, const T* rho, int nx, int nz, T* lam, T* mu,
                      T* mu_txz, T* rho_vx, T* rho_vz) {
    // _compute_staggered_params (src/utils/init.jl:136-158)
    const size_t n = (size_t)nx * nz;
    for (size_t c = 0; c < n; ++c) {
        mu[c] = rho[c] * T(vs[c] * vs[c]);
        lam[c] = T(rho[c] * T(vp[c] * vp[c])) - T(T(2) * mu[c]);
        rho_vx[c] = rho[c];
    }
    Grid G{nx, nz};
    for (int j = 1; j <= nz - 1; ++j)
        for (int i = 1; i <= nx - 1; ++i)
            rho_vz[G(i, j)] = T(0.25) * T(T(T(rho[G(i, j)] + rho[G(i + 1, j)]) + rho[G(i, j + 1)]) + rho[G(i + 1, j + 1)]);
    for (int j = 1; j <= nz; ++j) rho_vz[G(nx, j)] = rho_vz[G(nx - 1, j)];
    for (int i = 1; i <= nx; ++i) rho_vz[G(i, nz)] = rho_vz[G(i, nz - 1)];
    for (int j = 1; j <= nz - 1; ++j)
        for (int i = 1; i <= nx; ++i)
            mu_txz[G(i, j)] = T(2) / T(T(T(1) / mu[G(i, j)]) + T(T(1) / mu[G(i, j + 1)]));
    for (int i = 1; i <= nx; ++i) mu_txz[G(i, nz)] = mu_txz[G(i, nz - 1)];
}

}  // namespace

extern "C" {

// get_fd_coefficients (src/utils/init.jl:13-29).  Orders 2..10 are the
// reference's Float32 table; order 12 (beyond the reference) comes from the
// Taylor system.  Returns M, or -1 for an unsupported order.
int orc_fd_coefficients_f32(int order, float* out) {
    switch (order) {
        case 2: out[0] = 1.0f; return 1;
        case 4: out[0] = 1.125f; out[1] = -0.041666667f; return 2;
        case 6: out[0] = 1.171875f; out[1] = -0.065104167f; out[2] = 0.0046875f; return 3;
        case 8:
            out[0] = 1.1962890625f; out[1] = -0.079752604167f; out[2] = 0.0095703125f;
            out[3] = -0.000697544643f; return 4;
        case 10:
            out[0] = 1.2115478515625f; out[1] = -0.089721679687f; out[2] = 0.0138427734375f;
            out[3] = -0.00176565987723f; out[4] = 0.0001186795166f; return 5;
        case 12: {
            long double c[6];
            taylor_coefficients(6, c);
            for (int l = 0; l < 6; ++l) out[l] = (float)c[l];
            return 6;
        }
        default: return -1;
    }
}

int orc_fd_coefficients_f64(int order, double* out) {
    switch (order) {
        case 2: out[0] = 1.0; return 1;
        case 4: out[0] = 1.125; out[1] = -0.041666667; return 2;
        case 6: out[0] = 1.171875; out[1] = -0.065104167; out[2] = 0.0046875; return 3;
        case 8:
            out[0] = 1.1962890625; out[1] = -0.079752604167; out[2] = 0.0095703125;
            out[3] = -0.000697544643; return 4;
        case 10:
            out[0] = 1.2115478515625; out[1] = -0.089721679687; out[2] = 0.0138427734375;
            out[3] = -0.00176565987723; out[4] = 0.0001186795166; return 5;
        case 12: {
            long double c[6];
            taylor_coefficients(6, c);
            for (int l = 0; l < 6; ++l) out[l] = (double)c[l];
            return 6;
        }
        default: return -1;
    }
}

// ricker_wavelet (src/utils/init.jl:40-49) with the reference's promotion
// rules for Float32 f0 and dt: (i-1)*dt is a Float32 product, pi*f0 is a
// Float32 product, everything else is Float64, the result is rounded to
// Float32.
void orc_ricker_f32(float f0, float dt, int nt, float* out) {
    const double t0 = 1.0 / (double)f0;
    const float pif0 = (float)M_PI * f0;
    for (int i = 1; i <= nt; ++i) {
        const float tf = (float)(i - 1) * dt;
        const double tau = (double)tf - t0;
        const double x = (double)pif0 * tau;
        const double arg = x * x;
        out[i - 1] = (float)((1.0 - 2.0 * arg) * std::exp(-arg));
    }
}

// Float64 Ricker for the double oracle.
void orc_ricker_f64(double f0, double dt, int nt, double* out) {
    const double t0 = 1.0 / f0;
    for (int i = 1; i <= nt; ++i) {
        const double tau = (double)(i - 1) * dt - t0;
        const double x = M_PI * f0 * tau;
        const double arg = x * x;
        out[i - 1] = (1.0 - 2.0 * arg) * std::exp(-arg);
    }
}

// init_medium (src/utils/init.jl:68-99): pad vp, vs, rho (Float32, (nx_in,
// nz_in), x fastest) by `pad` cells and compute the staggered arrays.
void orc_init_medium_f32(const float* vp, const float* vs, const float* rho, int nx_in, int nz_in,
                         int pad, float* rho_vx, float* rho_vz, float* lam, float* mu_txx,
                         float* mu_txz) {
    const int nx = nx_in + 2 * pad, nz = nz_in + 2 * pad;
    const size_t n = (size_t)nx * nz;
    std::vector<float> p_vp(n), p_vs(n), p_rho(n);
    pad_array(vp, nx_in, nz_in, pad, p_vp.data());
    pad_array(vs, nx_in, nz_in, pad, p_vs.data());
    pad_array(rho, nx_in, nz_in, pad, p_rho.data());
    staggered_params(p_vp.data(), p_vs.data(), p_rho.data(), nx, nz, lam, mu_txx, mu_txz, rho_vx, rho_vz);
}

void orc_init_medium_f64(const float* vp, const float* vs, const float* rho, int nx_in, int nz_in,
                         int pad, double* rho_vx, double* rho_vz, double* lam, double* mu_txx,
                         double* mu_txz) {
    const int nx = nx_in + 2 * pad, nz = nz_in + 2 * pad;
    const size_t n = (size_t)nx * nz;
    std::vector<double> p_vp(n), p_vs(n), p_rho(n);
    pad_array(vp, nx_in, nz_in, pad, p_vp.data());
    pad_array(vs, nx_in, nz_in, pad, p_vs.data());
    pad_array(rho, nx_in, nz_in, pad, p_rho.data());
    staggered_params(p_vp.data(), p_vs.data(), p_rho.data(), nx, nz, lam, mu_txx, mu_txz, rho_vx, rho_vz);
}

// init_habc (src/utils/init.jl:171-203), Float32 arithmetic throughout.
// q = {qx, qz, qt_x, qt_z, qxt}.
void orc_habc_coefficients_f32(float v_ref, float dt, float dx, float dz, float* q) {
    const float rx = (v_ref * dt) / dx;
    const float rz = (v_ref * dt) / dz;
    const float b_p = 0.45f, beta = 1.0f;
    const float one_m_bp = 1.0f - b_p;
    q[0] = (b_p * (beta + rx) - rx) / ((beta + rx) * one_m_bp);
    q[1] = (b_p * (beta + rz) - rz) / ((beta + rz) * one_m_bp);
    q[2] = (b_p * (beta + rx) - beta) / ((beta + rx) * one_m_bp);
    q[3] = (b_p * (beta + rz) - beta) / ((beta + rz) * one_m_bp);
    q[4] = b_p / (b_p - 1.0f);
}

void orc_habc_coefficients_f64(double v_ref, double dt, double dx, double dz, double* q) {
    const double rx = (v_ref * dt) / dx;
    const double rz = (v_ref * dt) / dz;
    const double b_p = 0.45, beta = 1.0;
    q[0] = (b_p * (beta + rx) - rx) / ((beta + rx) * (1 - b_p));
    q[1] = (b_p * (beta + rz) - rz) / ((beta + rz) * (1 - b_p));
    q[2] = (b_p * (beta + rx) - beta) / ((beta + rx) * (1 - b_p));
    q[3] = (b_p * (beta + rz) - beta) / ((beta + rz) * (1 - b_p));
    q[4] = b_p / (b_p - 1.0);
}

// Weight as a function of dist: Float32(clamp((dist - off)/nbc, 0, 1)),
// computed in Float64 (init.jl:188-195).  table has nbc+2 entries.
void orc_habc_weight_table_f32(int nbc, double off, float* table) {
    for (int d = 0; d <= nbc + 1; ++d) {
        double w = ((double)d - off) / (double)nbc;
        w = std::min(std::max(w, 0.0), 1.0);
        table[d] = (float)w;
    }
}

void orc_habc_weight_table_f64(int nbc, double off, double* table) {
    for (int d = 0; d <= nbc + 1; ++d) {
        double w = ((double)d - off) / (double)nbc;
        table[d] = std::min(std::max(w, 0.0), 1.0);
    }
}

// The reference's full (nz, nx) weight matrix, w[j, i] at (j-1) + (i-1)*nz.
void orc_habc_weights_full_f32(int nx, int nz, int nbc, double off, float* w) {
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= nz; ++j) {
            const int d = std::min(std::min(i - 1, nx - i), std::min(j - 1, nz - j));
            double v = ((double)d - off) / (double)nbc;
            v = std::min(std::max(v, 0.0), 1.0);
            w[(size_t)(j - 1) + (size_t)(i - 1) * nz] = (float)v;
        }
}

// round(Int, x/dx) + pad + 1 with Float32 division and ties to even
// (setup_receivers, init.jl:220-221; _coord_to_index, shot_manager.jl:189-191).
int orc_coord_to_index(float x, float dx, int pad) {
    const float r = x / dx;
    return (int)std::nearbyint(r) + pad + 1;
}

int orc_run_shot_f32(const OrcShot* p, float* gather, float* final_fields, int n_steps) {
    return run_shot<float>(p, gather, final_fields, n_steps);
}

int orc_run_shot_f64(const OrcShot* p, double* gather, double* final_fields, int n_steps) {
    return run_shot<double>(p, gather, final_fields, n_steps);
}

// create_geometry (src/io/geometry_io.jl:85-130) for one shot: coordinates
// are the discretised positions (index - pad - 1) * dx, the Int converted to
// Float32 and multiplied once in Float32 (:90-95); indices relative to the
// physical domain are index - pad (:98-101); t_max = dt * nt, the Int
// converted to Float32 (:107); the physical grid is nx - 2 pad by nz - 2 pad
// (:109).  geo_f = [src_x, src_z, t_max], geo_i = [src_i, src_j, nx, nz].
void orc_create_geometry(int src_i, int src_j, int n_rec, const int* rec_i, const int* rec_j, int pad, float dx,
                         float dz, float dt, int nt, int nx, int nz, float* geo_f, int* geo_i, float* rec_x,
                         float* rec_z, int* rec_i_phys, int* rec_j_phys) {
    volatile float t;  // each product rounded to Float32 on its own
    t = (float)(src_i - pad - 1) * dx;
    geo_f[0] = t;
    t = (float)(src_j - pad - 1) * dz;
    geo_f[1] = t;
    t = dt * (float)nt;
    geo_f[2] = t;
    geo_i[0] = src_i - pad;
    geo_i[1] = src_j - pad;
    geo_i[2] = nx - 2 * pad;
    geo_i[3] = nz - 2 * pad;
    for (int r = 0; r < n_rec; ++r) {
        t = (float)(rec_i[r] - pad - 1) * dx;
        rec_x[r] = t;
        t = (float)(rec_j[r] - pad - 1) * dz;
        rec_z[r] = t;
        rec_i_phys[r] = rec_i[r] - pad;
        rec_j_phys[r] = rec_j[r] - pad;
    }
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
