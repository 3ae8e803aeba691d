// fomo_b200.cu -- host runtime and C ABI of libfomo_b200.so (include/fomo_b200.h).
//
// Owns every device allocation behind opaque handles, one CUDA stream per
// process, and the time loop of a shot.  See include/fomo_b200.h for the
// reference interface each entry point stands in for.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cerrno>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <utility>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/fomo_b200.h"
#include "step_tiled.cuh"
#include "march_launch.h"
#include "step_march.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(FOMO_ECUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));    \
    } while (0)

struct Object {
    virtual ~Object() = default;
};

struct Buffer : Object {
    void* ptr = nullptr;
    size_t bytes = 0;
    ~Buffer() override {
        if (ptr) cudaFree(ptr);
    }
};

// Device memory of media, wavefields and shots comes from a per-device
// stream-ordered pool (on the library stream) that keeps what is freed, so
// creating and destroying them again and again costs no driver allocation
// and no device-wide synchronisation (cudaFree has both).
cudaError_t pool_alloc(void** p, size_t bytes);
void pool_free(void* p);

// Row pitch in floats: rows start on 128-byte boundaries.
inline int pitch_of(int nx) { return (nx + 31) / 32 * 32; }

struct Medium : Object {
    int nx = 0, nz = 0, pitch = 0, M = 0, pad = 0, fs = 0;
    float dx = 0, dz = 0;
    float* base = nullptr;  // 5 arrays of pitch*nz floats
    // Buoyancy dtx/rho_vx, dtz/rho_vx, dtx/rho_vz, dtz/rho_vz for the last
    // (dtx, dtz) used; when dtx == dtz the second and fourth alias the first
    // and third.
    float* buoy = nullptr;
    float buoy_dtx = 0, buoy_dtz = 0;
    bool maps_ok = false;
    CUtensorMap mod_maps[3];   // tile boxes of lam, mu_txx, mu_txz
    CUtensorMap buoy_maps[4];  // tile boxes of the four buoyancy arrays
    std::atomic<int> users{0}; // shot-server requests holding this medium
    const float* arr(int q) const { return base + (size_t)q * pitch * nz; }
    ~Medium() override {
        pool_free(base);
        pool_free(buoy);
    }
};

struct Wavefield : Object {
    int nx = 0, nz = 0, pitch = 0;
    float* base = nullptr;  // 2 copies x 5 fields of pitch*nz floats
    int cur = 0;            // copy holding the current state
    int map_M = 0;          // M the halo maps were made for (0 = none)
    CUtensorMap maps[2][5]; // halo boxes (Geo<map_M>) of every field of both copies
    CUtensorMap pmaps[2][5];// tile boxes of every field of both copies
    float* snap = nullptr;  // frame buffer of fomo_b200_wavefield_snapshot
    size_t snap_bytes = 0;
    float* field(int copy, int q) const { return base + ((size_t)copy * 5 + q) * pitch * nz; }
    ~Wavefield() override {
        pool_free(base);
        pool_free(snap);
    }
};

struct Shot : Object {
    uint64_t medium = 0, wavefield = 0;
    int nbc = 0;
    float q[5] = {0, 0, 0, 0, 0};
    float a[fomo::kMaxM] = {0};
    int M = 0;
    float dt = 0, dtx = 0, dtz = 0;
    int nt = 0, src_i = 0, src_j = 0, n_rec = 0, rec_kind = 0;
    std::vector<float> wavelet;     // host copy: one sample per step
    float* d_tabs = nullptr;        // 3 x (nbc+2)
    float* d_band = nullptr;        // band scratch: kBandPlanes planes of nbc rows x pitch
    int* d_rec = nullptr;           // n_rec linear offsets
    float* d_gather = nullptr;      // nt x n_rec
    int k_done = 0, recorded = 0;
    double device_ms = 0;
    int64_t launches = 0, h2d = 0, d2h = 0;
    ~Shot() override {
        pool_free(d_tabs);
        pool_free(d_band);
        pool_free(d_rec);
        pool_free(d_gather);
    }
};

struct Context {
    std::mutex mu;
    bool inited = false;
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int* d_status = nullptr;   // device error word of the kernels, then the fused step's work queue (2 ints)
    cudaMemPool_t pool = nullptr;
    uint64_t next = 1;
    std::unordered_map<uint64_t, std::unique_ptr<Object>> objs;
};

Context& ctx() {
    static Context c;
    return c;
}

cudaError_t pool_alloc(void** p, size_t bytes) {
    auto& C = ctx();
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, C.pool, C.stream);
    if (e == cudaErrorMemoryAllocation) {  // give the pool's cached memory back to the device, then retry once
        (void)cudaGetLastError();
        cudaStreamSynchronize(C.stream);
        cudaMemPoolTrimTo(C.pool, 0);
        e = cudaMallocFromPoolAsync(p, bytes, C.pool, C.stream);
    }
    if (e != cudaSuccess) {
        (void)cudaGetLastError();  // not a sticky error: the caller reports it
        *p = nullptr;
    }
    return e;
}

void pool_free(void* p) {
    if (p) cudaFreeAsync(p, ctx().stream);
}

template <class T>
T* get(uint64_t h) {
    auto& C = ctx();
    auto it = C.objs.find(h);
    if (it == C.objs.end()) return nullptr;
    return dynamic_cast<T*>(it->second.get());
}

uint64_t put(std::unique_ptr<Object> o) {
    auto& C = ctx();
    const uint64_t h = C.next++;
    C.objs.emplace(h, std::move(o));
    return h;
}

int ensure_init() {
    if (!ctx().inited) return fail(FOMO_ENOINIT, "fomo_b200_init has not been called");
    return FOMO_OK;
}

// SM count of the current device (grid sizes of the grid-stride kernels and
// the tile prefetch distance scale with it); 148 if the query fails.
int sm_count() {
    static std::mutex mu;
    static std::unordered_map<int, int> by_dev;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return 148;
    }
    std::lock_guard<std::mutex> lk(mu);
    auto it = by_dev.find(dev);
    if (it != by_dev.end()) return it->second;
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
        (void)cudaGetLastError();
        n = 148;
    }
    by_dev[dev] = n;
    return n;
}

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes` and never lowers it, so a launch sized by another caller for
// a larger block stays valid.  One high-water mark per (kernel, device).
template <class K>
int raise_smem_limit(K* kernel, size_t bytes) {
    static std::mutex mu;
    static std::unordered_map<uint64_t, size_t> set;
    if (bytes <= 48 * 1024) return FOMO_OK;
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    const uint64_t key = (uint64_t)(uintptr_t)(const void*)kernel * 64 + (uint64_t)dev;
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = set[key];
    if (bytes <= cur) return FOMO_OK;
    CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
    return FOMO_OK;
}

// The HABC band must fit the grid, and the free-surface rows (pad-5..pad,
// 0-based) must lie above the bottom band and the row above it.
int check_band(int nx, int nz, int pad, int fs, int nbc) {
    if (nbc < 1 || 2 * nbc + 3 > nx || 2 * nbc + 2 > nz)
        return fail(FOMO_EINVAL, "nbc=%d does not fit the %dx%d grid", nbc, nx, nz);
    if (nbc + 2 > fomo::kMaxBandTab) return fail(FOMO_EINVAL, "nbc=%d above the supported %d", nbc, fomo::kMaxBandTab - 2);
    if (fs && pad >= nz - nbc - 2)
        return fail(FOMO_EINVAL, "free-surface rows reach the bottom HABC band (pad=%d, nbc=%d, nz=%d)", pad, nbc, nz);
    return FOMO_OK;
}

int check_medium_args(int nx, int nz, int M, int pad) {
    if (M < 1 || M > fomo::kMaxM) return fail(FOMO_EINVAL, "M=%d out of range 1..%d", M, fomo::kMaxM);
    if (nx < 2 * pad + 1 || nz < 2 * pad + 1)
        return fail(FOMO_EINVAL, "grid %dx%d smaller than 2*pad+1 (pad=%d)", nx, nz, pad);
    if (pad < M) return fail(FOMO_EINVAL, "pad=%d < M=%d", pad, M);
    return FOMO_OK;
}

// ---------------------------------------------------------------- TMA descriptors
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int get_encode() {
    if (g_encode) return FOMO_OK;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !fn) return fail(FOMO_ECUDA, "cuTensorMapEncodeTiled not available");
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return FOMO_OK;
}

// 2-D Float32 descriptor of an (nx, nz) array with row pitch `pitch` floats;
// out-of-range elements of a box read as zero.
int encode_map(CUtensorMap* map, const float* base, int nx, int nz, int pitch, int boxw, int boxh) {
    if (int rc = get_encode()) return rc;
    cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)nz};
    cuuint64_t strides[1] = {(cuuint64_t)pitch * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)boxw, (cuuint32_t)boxh};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(FOMO_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return FOMO_OK;
}

template <int M>
int make_maps(Wavefield& w) {
    using G = fomo::Geo<M>;
    for (int c = 0; c < 2; ++c)
        for (int q = 0; q < 5; ++q) {
            if (int rc = encode_map(&w.maps[c][q], w.field(c, q), w.nx, w.nz, w.pitch, G::BOXW, G::BOXH)) return rc;
            if (int rc = encode_map(&w.pmaps[c][q], w.field(c, q), w.nx, w.nz, w.pitch, fomo::kTX, fomo::kTZ))
                return rc;
        }
    w.map_M = M;
    return FOMO_OK;
}

int make_medium_maps(Medium& m) {
    if (m.maps_ok) return FOMO_OK;
    for (int q = 0; q < 3; ++q)
        if (int rc = encode_map(&m.mod_maps[q], m.arr(2 + q), m.nx, m.nz, m.pitch, fomo::kTX, fomo::kTZ)) return rc;
    m.maps_ok = true;
    return FOMO_OK;
}

// ---------------------------------------------------------------- buoyancy
int ensure_buoyancy(Medium& m, float dtx, float dtz) {
    if (m.buoy && m.buoy_dtx == dtx && m.buoy_dtz == dtz) return FOMO_OK;
    const size_t plane = (size_t)m.pitch * m.nz;
    if (!m.buoy) {
        cudaError_t e = pool_alloc((void**)&m.buoy, 4 * plane * sizeof(float));
        if (e != cudaSuccess) return fail(FOMO_ENOMEM, "buoyancy allocation failed: %s", cudaGetErrorString(e));
    }
    float* b0 = m.buoy;
    float* b1 = dtx == dtz ? b0 : m.buoy + plane;
    float* b2 = m.buoy + 2 * plane;
    float* b3 = dtx == dtz ? b2 : m.buoy + 3 * plane;
    fomo::buoyancy_kernel<<<4 * sm_count(), 256, 0, ctx().stream>>>(m.arr(0), m.arr(1), dtx, dtz, plane, b0, b1, b2, b3);
    CUDA_TRY(cudaGetLastError());
    m.buoy_dtx = dtx;
    m.buoy_dtz = dtz;
    const float* bp[4] = {b0, b1, b2, b3};
    for (int q = 0; q < 4; ++q)
        if (int rc = encode_map(&m.buoy_maps[q], bp[q], m.nx, m.nz, m.pitch, fomo::kTX, fomo::kTZ)) return rc;
    return FOMO_OK;
}

void buoyancy_ptrs(const Medium& m, const float* out[4]) {
    const size_t plane = (size_t)m.pitch * m.nz;
    out[0] = m.buoy;
    out[1] = m.buoy_dtx == m.buoy_dtz ? m.buoy : m.buoy + plane;
    out[2] = m.buoy + 2 * plane;
    out[3] = m.buoy_dtx == m.buoy_dtz ? m.buoy + 2 * plane : m.buoy + 3 * plane;
}

// ---------------------------------------------------------------- launches
struct Launch {
    int tiles_x, tiles_z, n_tile, n_band, x_last;
    size_t smem_v, smem_s;
};

template <int M>
Launch launch_shape(int nx, int nz, int nbc, bool iso, bool fs) {
    Launch L;
    L.tiles_x = (nx + fomo::kTX - 1) / fomo::kTX;
    L.tiles_z = (nz + fomo::kTZ - 1) / fomo::kTZ;
    L.x_last = std::max(0, (nx + 3) / 4 * 4 - fomo::kTX);  // last tile ends at the grid's right edge
    L.n_tile = L.tiles_x * L.tiles_z;
    L.n_band = fomo::band_warp_count(nx);
    L.smem_v = fomo::tiled_smem_bytes<M>(true, nbc, iso, fs);
    L.smem_s = fomo::tiled_smem_bytes<M>(false, nbc, iso, fs);
    return L;
}

void fill_common(fomo::StepParams& P, const Medium& m, const Shot& s) {
    std::memset(&P, 0, sizeof(P));
    P.nx = m.nx;
    P.nz = m.nz;
    P.pitch = m.pitch;
    P.M = m.M;
    P.pad = m.pad;
    P.nbc = s.nbc;
    P.fs = m.fs;
    P.dtx = s.dtx;
    P.dtz = s.dtz;
    for (int l = 0; l < fomo::kMaxM; ++l) P.a[l] = s.a[l];
    P.qx = s.q[0];
    P.qz = s.q[1];
    P.qt_x = s.q[2];
    P.qt_z = s.q[3];
    P.qxt = s.q[4];
    for (int t = 0; t < 3; ++t) P.w_tab[t] = s.d_tabs + (size_t)t * (s.nbc + 2);
    P.rho_vx = m.arr(0);
    P.rho_vz = m.arr(1);
    P.lam = m.arr(2);
    P.mu_txx = m.arr(3);
    P.mu_txz = m.arr(4);
    P.src_i = s.src_i;
    P.src_j = s.src_j;
    P.nt = s.nt;
    P.n_rec = s.n_rec;
    P.rec_kind = s.rec_kind;
    P.rec_cell = s.d_rec;
    P.gather = s.d_gather;
}

// Per-launch event pairs, filled only by fomo_b200_shot_profile.
struct Profile {
    std::vector<cudaEvent_t> ev;      // 2 per launch
    std::vector<int> kind;            // 0 velocity, 1 stress, 2 band (velocity), 3 band (stress), 4 fused step
    int add(cudaStream_t st, int k) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return -1;
        ev.push_back(a);
        ev.push_back(b);
        kind.push_back(k);
        return cudaEventRecord(a, st) == cudaSuccess ? 0 : -1;
    }
    int end(cudaStream_t st) { return cudaEventRecord(ev.back(), st) == cudaSuccess ? 0 : -1; }
    ~Profile() {
        for (auto e : ev) cudaEventDestroy(e);
    }
};

int check_status() {
    int st = 0;
    CUDA_TRY(cudaMemcpyAsync(&st, ctx().d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx().stream));
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    if (st == fomo::kErrTmaTimeout) return fail(FOMO_ETIMEOUT, "a TMA load of a time-step kernel did not complete");
    if (st) return fail(FOMO_ECUDA, "time-step kernel reported error %d", st);
    return FOMO_OK;
}

// Launches a tile kernel.  With `after_band` (the launch just before it on
// the stream is a band pass) it is a programmatic dependent launch: its
// blocks start while the band pass runs, and those that read the band rows
// wait for it (grid_dep_wait).
template <class... Exp, class... Act>
static cudaError_t launch_tiles(void (*kern)(Exp...), int blocks, size_t smem, cudaStream_t st, bool after_band,
                                Act&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(fomo::kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = after_band ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Act>(args)...);
}

// ---------------------------------------------------------------- fused step
std::atomic<int> g_step_mode{FOMO_STEP_AUTO};
std::atomic<int> g_march_segs{0};

// Strips, segments and the validity check of one fused-step layout.
struct MarchPlan {
    bool ok = false;
    char why[160] = {0};
    fomo::MarchArgs A;
};

// Fused-step layout of an (nx, nz) grid, or the reason there is none.
// Every boundary rule a strip needs must read only columns the strip
// computes: the left HABC rule of cell i reads i+1, the right rule i-1 and
// (at chunk starts) i-2, for the velocity columns the strip's stress reads
// (own columns +- M, computed over own columns +- HV) and for its own stress
// columns; the corners of the bottom band read the same neighbours.
template <int M>
MarchPlan march_plan(int nx, int nz, int nbc, bool fs, int slots, int segs_req) {
    using G = fomo::MGeo<M>;
    MarchPlan p;
    std::memset(&p.A, 0, sizeof(p.A));
#define FOMO_NO(...) (std::snprintf(p.why, sizeof(p.why), __VA_ARGS__), p)
    if (!fs) return FOMO_NO("no free surface (the fused step has no top HABC band)");
    const int W = G::W, HV = G::HV, VW = fomo::kMVW;
    const int x_last = std::max(0, (nx + 3) / 4 * 4 - W);
    const int S = x_last > 0 ? (x_last + W - 1) / W + 1 : 1;
    const int r0 = nx - nbc - 1, j0 = nz - nbc - 1;
    for (int st = 0; st < S; ++st) {
        const bool last = st == S - 1;
        const int x0 = last ? x_last : st * W;
        const int x_end = last ? std::min(x0 + W, (nx + 3) / 4 * 4) : std::min(x0 + W, x_last);
        const int xa = x0 - HV;
        for (int i = std::max(0, x0 - M); i < std::min(nx, x_end + M); ++i) {
            if (i >= 1 && i <= nbc && !(i + 1 < xa + VW))
                return FOMO_NO("left HABC column %d needs column %d beyond strip %d", i, i + 1, st);
            if (i >= r0 && i <= nx - 2 && !(i - 2 >= xa))
                return FOMO_NO("right HABC column %d needs column %d before strip %d", i, i - 2, st);
        }
        for (int i = x0; i < std::min(nx, x_end); ++i) {
            if (i >= 1 && i <= nbc && !(i + 1 < x0 + W))
                return FOMO_NO("left HABC column %d needs stress column %d beyond strip %d", i, i + 1, st);
            if (i >= r0 && i <= nx - 2 && !(i - 2 >= x0))
                return FOMO_NO("right HABC column %d needs stress column %d before strip %d", i, i - 2, st);
        }
    }
    // Row segments: the last one holds the bottom band, the row above it and
    // the M rows its velocity reads above that.
    const int last_max = j0 - M;
    if (last_max < 0) return FOMO_NO("grid too shallow for the fused step");
    if ((long)((nx + 31) / 32 * 32) * nz >= (1L << 31)) return FOMO_NO("grid too large for 32-bit cell offsets");
#undef FOMO_NO
    // One table of ns segments (at most kMMaxSegs, at least min_h rows each
    // where the grid allows) whose last one starts at or above last_max.
    auto segments = [&](int ns, int min_h, int* z) {
        ns = std::max(1, std::min({ns, fomo::kMMaxSegs, std::max(1, nz / std::max(1, min_h))}));
        for (;; --ns) {
            const int h = (nz + ns - 1) / ns;
            bool okz = true;
            for (int q = 0; q < ns; ++q) z[q] = q * h;
            z[ns] = nz;
            if (ns > 1) z[ns - 1] = std::min(z[ns - 1], last_max);
            for (int q = 0; q < ns; ++q) okz = okz && z[q + 1] > z[q];
            if (okz || ns == 1) return ns;
        }
    };
    // Persistent blocks take items from a queue, so the segments only need to
    // be short enough that every block gets several items (the last item of a
    // block bounds the tail) and long enough to amortise the rows each item
    // recomputes above it.  Edge strips apply the side HABC rules on almost
    // every cell: their items are cut four times finer.
    const int n_edge = std::min(S, 2);
    const int ns = segs_req > 0 ? segs_req : (6 * slots + S - 1) / S;
    p.A.n_segs = segments(ns, segs_req > 0 ? 1 : 48, p.A.seg_z);
    p.A.n_segs_e = segments(segs_req > 0 ? segs_req : 4 * p.A.n_segs, segs_req > 0 ? 1 : 24, p.A.seg_ze);
    p.A.n_strips = S;
    p.A.n_edge = n_edge;
    p.A.n_items = n_edge * p.A.n_segs_e + (S - n_edge) * p.A.n_segs;
    p.A.x_last = x_last;
    p.ok = true;
    return p;
}

// Fused-step blocks resident on the device at once (two per SM if the
// occupancy query fails).
template <int M>
int march_slots() {
    static int slots[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        (void)cudaGetLastError();
        return 2 * sm_count();
    }
    if (!slots[dev]) {
        int per_sm = 0;
        if (raise_smem_limit(fomo::march_kernel_fn<M>(), fomo::march_smem_bytes<M>()) != FOMO_OK ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fomo::march_kernel_fn<M>(), fomo::kMThreads,
                                                          fomo::march_smem_bytes<M>()) != cudaSuccess) {
            (void)cudaGetLastError();
            per_sm = 2;
        }
        slots[dev] = std::max(1, per_sm) * sm_count();
    }
    return slots[dev];
}

template <int M>
int run_steps_march(Shot& s, Medium& m, Wavefield& w, int n_steps, Profile* prof, const MarchPlan& plan) {
    static_assert(fomo::Geo<M>::BOXW == fomo::MGeo<M>::TW && fomo::Geo<M>::BOXH == fomo::MGeo<M>::TH,
                  "the wavefield's halo descriptors are the fused step's tau boxes");
    auto& C = ctx();
    const bool iso = s.dtx == s.dtz;
    if (int rc = raise_smem_limit(fomo::march_kernel_fn<M>(), fomo::march_smem_bytes<M>())) return rc;
    if (w.map_M != M)
        if (int rc = make_maps<M>(w)) return rc;
    if (int rc = ensure_buoyancy(m, s.dtx, s.dtz)) return rc;
    if (int rc = make_medium_maps(m)) return rc;
    fomo::MarchArgs A = plan.A;
    buoyancy_ptrs(m, A.b);
    A.iso = iso ? 1 : 0;
    A.status = C.d_status;
    A.queue = C.d_status + 2;  // zero between launches: the last block to leave resets it
    const int rec_blocks = (s.n_rec + fomo::kMThreads - 1) / fomo::kMThreads;
    const int slots = march_slots<M>();
    CUDA_TRY(cudaEventRecord(C.ev0, C.stream));
    const int k_begin = s.k_done + 1, k_end = std::min(s.nt, s.k_done + n_steps);
    nvtxRangePushA("fomo_b200 time loop (fused step)");
    for (int k = k_begin; k <= k_end; ++k) {
        const int a = w.cur, b = 1 - w.cur;
        fomo::StepParams P;
        fill_common(P, m, s);
        P.src_w = (k <= (int)s.wavelet.size()) ? s.wavelet[k - 1] : 0.f;
        for (int q = 0; q < 5; ++q) {
            P.in[q] = w.field(a, q);
            P.out[q] = w.field(b, q);
        }
        P.rec_k = (k >= 2 && s.n_rec > 0) ? k - 1 : 0;
        fomo::MarchMaps mp;
        mp.xx = w.maps[a][fomo::TXX];
        mp.zz = w.maps[a][fomo::TZZ];
        mp.xz = w.maps[a][fomo::TXZ];
        mp.vx = w.pmaps[a][fomo::VX];
        mp.vz = w.pmaps[a][fomo::VZ];
        mp.b0 = m.buoy_maps[0];
        mp.b1 = m.buoy_maps[1];
        mp.b2 = m.buoy_maps[2];
        mp.b3 = m.buoy_maps[3];
        mp.lam = m.mod_maps[0];
        mp.mu = m.mod_maps[1];
        mp.mxz = m.mod_maps[2];
        if (prof && prof->add(C.stream, 4)) return fail(FOMO_ECUDA, "profiling event failed");
        A.n_rec_items = P.rec_k ? rec_blocks : 0;
        // persistent blocks: as many as are resident at once, at most one per item
        CUDA_TRY(fomo::march_launch<M>(std::min(A.n_items + A.n_rec_items, slots), C.stream, P, A, mp));
        if (prof && prof->end(C.stream)) return fail(FOMO_ECUDA, "profiling event failed");
        s.launches += 1;
        w.cur = b;
        if (k >= 2) s.recorded = k - 1;
        s.k_done = k;
    }
    nvtxRangePop();
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(C.ev1, C.stream));
    CUDA_TRY(cudaEventSynchronize(C.ev1));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, C.ev0, C.ev1));
    s.device_ms += ms;
    return check_status();
}

// The fused step's plan for a shot, or !ok (split launches): FOMO_STEP_SPLIT,
// M > 4, or a layout march_plan rejects.
template <int M>
MarchPlan shot_march_plan(const Shot& s, const Medium& m) {
    MarchPlan p;
    if (g_step_mode.load() == FOMO_STEP_SPLIT) {
        std::snprintf(p.why, sizeof(p.why), "split launches selected");
        return p;
    }
    if constexpr (M <= 4) {
        return march_plan<M>(m.nx, m.nz, s.nbc, m.fs != 0, march_slots<M>(), g_march_segs.load());
    } else {
        std::snprintf(p.why, sizeof(p.why), "M=%d above the fused step's 4", M);
        return p;
    }
}

template <int M>
int run_steps_split(Shot& s, Medium& m, Wavefield& w, int n_steps, Profile* prof);

// FOMO_STEP_AUTO's choice per grid and HABC width, made once per process by
// timing both kernels on live steps of the first shot (they give the same
// bits, so the shot itself is unaffected): 0 = split launches, 1 = fused.
struct StepKey {
    int nx, nz, M, nbc, fs, iso;
    bool operator<(const StepKey& o) const {
        return std::tie(nx, nz, M, nbc, fs, iso) < std::tie(o.nx, o.nz, o.M, o.nbc, o.fs, o.iso);
    }
};
std::mutex g_step_choice_mu;
std::map<StepKey, int> g_step_choice;
constexpr int kStepTuneWindow = 24;  // steps timed per candidate

// The autotuners' optional cache file (environment variable
// FOMO_B200_TUNE_CACHE).  Single-shot kernel choices are lines
// "step nx nz M nbc fs iso choice", read on first use and appended to when a
// choice is made; the shot server's lines have five numbers (server.cuh).
const char* tune_cache_path() {
    const char* p = std::getenv("FOMO_B200_TUNE_CACHE");
    return (p && *p) ? p : nullptr;
}

// Call with g_step_choice_mu held.
void load_step_choices() {
    static bool loaded = false;
    if (loaded) return;
    loaded = true;
    const char* path = tune_cache_path();
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char line[256];
    StepKey k;
    int c;
    while (std::fgets(line, sizeof(line), f))
        if (std::sscanf(line, "step %d %d %d %d %d %d %d", &k.nx, &k.nz, &k.M, &k.nbc, &k.fs, &k.iso, &c) == 7)
            g_step_choice[k] = c != 0;
    std::fclose(f);
}

void save_step_choice(const StepKey& k, int c) {
    const char* path = tune_cache_path();
    if (!path) return;
    if (FILE* f = std::fopen(path, "a")) {
        std::fprintf(f, "step %d %d %d %d %d %d %d\n", k.nx, k.nz, k.M, k.nbc, k.fs, k.iso, c);
        std::fclose(f);
    }
}

template <int M>
int run_steps_M(Shot& s, Medium& m, Wavefield& w, int n_steps, Profile* prof) {
    const int mode = g_step_mode.load();
    const MarchPlan plan = shot_march_plan<M>(s, m);
    if (!plan.ok) {
        if (mode == FOMO_STEP_FUSED) return fail(FOMO_EINVAL, "the fused step does not support this shot: %s", plan.why);
        return run_steps_split<M>(s, m, w, n_steps, prof);
    }
    if constexpr (M <= 4) {
        const StepKey key{m.nx, m.nz, M, s.nbc, m.fs, s.dtx == s.dtz};
        int choice = mode == FOMO_STEP_FUSED ? 1 : -1;
        if (choice < 0) {
            std::lock_guard<std::mutex> lk(g_step_choice_mu);
            load_step_choices();
            auto it = g_step_choice.find(key);
            if (it != g_step_choice.end()) choice = it->second;
        }
        if (choice < 0) {
            const int W = kStepTuneWindow;
            if (prof || std::min(n_steps, s.nt - s.k_done) < 3 * W) {
                choice = 0;  // too few steps to time both: the split launches, nothing recorded
            } else {
                double t0 = s.device_ms;
                if (int rc = run_steps_march<M>(s, m, w, W, nullptr, plan)) return rc;
                const double t_fused = s.device_ms - t0;
                t0 = s.device_ms;
                if (int rc = run_steps_split<M>(s, m, w, W, nullptr)) return rc;
                const double t_split = s.device_ms - t0;
                choice = t_fused < t_split ? 1 : 0;
                n_steps -= 2 * W;
                std::lock_guard<std::mutex> lk(g_step_choice_mu);
                g_step_choice[key] = choice;
                save_step_choice(key, choice);
            }
        }
        if (choice == 1) return run_steps_march<M>(s, m, w, n_steps, prof, plan);
    }
    return run_steps_split<M>(s, m, w, n_steps, prof);
}

// The split launches: velocity tiles, velocity band pass, stress tiles,
// stress band pass per step.
template <int M>
int run_steps_split(Shot& s, Medium& m, Wavefield& w, int n_steps, Profile* prof) {
    auto& C = ctx();
    const bool iso = s.dtx == s.dtz;
    const Launch L = launch_shape<M>(m.nx, m.nz, s.nbc, iso, m.fs != 0);
    if (int rc = raise_smem_limit(fomo::velocity_kernel<M>, L.smem_v)) return rc;
    if (int rc = raise_smem_limit(fomo::stress_kernel<M>, L.smem_s)) return rc;
    if (w.map_M != M)
        if (int rc = make_maps<M>(w)) return rc;
    if (int rc = ensure_buoyancy(m, s.dtx, s.dtz)) return rc;
    if (int rc = make_medium_maps(m)) return rc;
    fomo::TiledArgs T;
    buoyancy_ptrs(m, T.b);
    T.iso = iso ? 1 : 0;
    T.status = C.d_status;
    T.band_pre = s.d_band;
    T.n_tile_blocks = L.n_tile;
    T.tiles_x = L.tiles_x;
    T.x_last = L.x_last;
    T.prefetch_ahead = fomo::prefetch_distance(sm_count());
    const int rec_blocks = (s.n_rec + fomo::kThreads - 1) / fomo::kThreads;
    CUDA_TRY(cudaEventRecord(C.ev0, C.stream));
    const int k_begin = s.k_done + 1, k_end = std::min(s.nt, s.k_done + n_steps);
    nvtxRangePushA("fomo_b200 time loop");
    for (int k = k_begin; k <= k_end; ++k) {
        const int a = w.cur, b = 1 - w.cur;
        fomo::StepParams P;
        fill_common(P, m, s);
        P.src_w = (k <= (int)s.wavelet.size()) ? s.wavelet[k - 1] : 0.f;
        // velocity: reads v(a), tau(a); writes v(b); records step k-1 from copy a
        for (int q = 0; q < 5; ++q) P.in[q] = w.field(a, q);
        P.out[fomo::VX] = w.field(b, fomo::VX);
        P.out[fomo::VZ] = w.field(b, fomo::VZ);
        P.rec_k = (k >= 2 && s.n_rec > 0) ? k - 1 : 0;
        const int vblocks = L.n_tile + (P.rec_k ? rec_blocks : 0);
        if (prof && prof->add(C.stream, 0)) return fail(FOMO_ECUDA, "profiling event failed");
        fomo::VelMaps vm;
        vm.xx = w.maps[a][fomo::TXX];
        vm.zz = w.maps[a][fomo::TZZ];
        vm.xz = w.maps[a][fomo::TXZ];
        vm.vx = w.pmaps[a][fomo::VX];
        vm.vz = w.pmaps[a][fomo::VZ];
        vm.b0 = m.buoy_maps[0];
        vm.b1 = m.buoy_maps[1];
        vm.b2 = m.buoy_maps[2];
        vm.b3 = m.buoy_maps[3];
        // profiled launches stay serialised (events sit between them)
        CUDA_TRY(launch_tiles(fomo::velocity_kernel<M>, vblocks, L.smem_v, C.stream, !prof && k > k_begin, P, T, vm));
        if (prof && prof->end(C.stream)) return fail(FOMO_ECUDA, "profiling event failed");
        if (prof && prof->add(C.stream, 2)) return fail(FOMO_ECUDA, "profiling event failed");
        fomo::band_kernel<true><<<L.n_band, 32, 0, C.stream>>>(P, T);
        if (prof && prof->end(C.stream)) return fail(FOMO_ECUDA, "profiling event failed");
        // stress: reads v(b) (new), tau(a); writes tau(b)
        P.in[fomo::VX] = w.field(b, fomo::VX);
        P.in[fomo::VZ] = w.field(b, fomo::VZ);
        for (int q = 2; q < 5; ++q) P.out[q] = w.field(b, q);
        P.out[fomo::VX] = P.out[fomo::VZ] = nullptr;
        P.rec_k = 0;
        if (prof && prof->add(C.stream, 1)) return fail(FOMO_ECUDA, "profiling event failed");
        fomo::StrMaps sm;
        sm.vx = w.maps[b][fomo::VX];
        sm.vz = w.maps[b][fomo::VZ];
        sm.txx = w.pmaps[a][fomo::TXX];
        sm.tzz = w.pmaps[a][fomo::TZZ];
        sm.txz = w.pmaps[a][fomo::TXZ];
        sm.lam = m.mod_maps[0];
        sm.mu = m.mod_maps[1];
        sm.mxz = m.mod_maps[2];
        CUDA_TRY(launch_tiles(fomo::stress_kernel<M>, L.n_tile, L.smem_s, C.stream, !prof, P, T, sm));
        if (prof && prof->end(C.stream)) return fail(FOMO_ECUDA, "profiling event failed");
        if (prof && prof->add(C.stream, 3)) return fail(FOMO_ECUDA, "profiling event failed");
        fomo::band_kernel<false><<<L.n_band, 32, 0, C.stream>>>(P, T);
        if (prof && prof->end(C.stream)) return fail(FOMO_ECUDA, "profiling event failed");
        s.launches += 4;
        w.cur = b;
        if (k >= 2) s.recorded = k - 1;
        s.k_done = k;
    }
    nvtxRangePop();
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(C.ev1, C.stream));
    CUDA_TRY(cudaEventSynchronize(C.ev1));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, C.ev0, C.ev1));
    s.device_ms += ms;
    return check_status();
}

int run_steps(Shot& s, int n_steps, Profile* prof = nullptr) {
    Medium* m = get<Medium>(s.medium);
    Wavefield* w = get<Wavefield>(s.wavefield);
    if (!m || !w) return fail(FOMO_EINVAL, "shot refers to a destroyed medium or wavefield");
    switch (m->M) {
        case 1: return run_steps_M<1>(s, *m, *w, n_steps, prof);
        case 2: return run_steps_M<2>(s, *m, *w, n_steps, prof);
        case 3: return run_steps_M<3>(s, *m, *w, n_steps, prof);
        case 4: return run_steps_M<4>(s, *m, *w, n_steps, prof);
        case 5: return run_steps_M<5>(s, *m, *w, n_steps, prof);
        case 6: return run_steps_M<6>(s, *m, *w, n_steps, prof);
    }
    return fail(FOMO_EINVAL, "M=%d not supported", m->M);
}

// Records the receivers of the last step done (the next velocity launch would).
void shutdown_servers();  // server.cuh

int record_last(Shot& s) {
    auto& C = ctx();
    if (s.n_rec == 0 || s.k_done < 1 || s.recorded >= s.k_done) return FOMO_OK;
    Medium* m = get<Medium>(s.medium);
    Wavefield* w = get<Wavefield>(s.wavefield);
    if (!m || !w) return fail(FOMO_EINVAL, "shot refers to a destroyed medium or wavefield");
    fomo::StepParams P;
    fill_common(P, *m, s);
    for (int q = 0; q < 5; ++q) P.in[q] = w->field(w->cur, q);
    P.rec_k = s.k_done;
    fomo::record_kernel<<<(s.n_rec + fomo::kThreads - 1) / fomo::kThreads, fomo::kThreads, 0, C.stream>>>(P);
    CUDA_TRY(cudaGetLastError());
    s.launches += 1;
    s.recorded = s.k_done;
    return FOMO_OK;
}

}  // namespace

extern "C" {

int fomo_b200_version(void) { return 100; }

const char* fomo_b200_last_error(void) { return g_err.c_str(); }

int fomo_b200_init(int device) {
    auto& C = ctx();
    std::lock_guard<std::mutex> lk(C.mu);
    if (C.inited) {
        if (C.device == device) return FOMO_OK;
        return fail(FOMO_EINVAL, "already initialised on device %d", C.device);
    }
    int n = 0;
    CUDA_TRY(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(FOMO_EINVAL, "device %d not present (%d devices)", device, n);
    CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(FOMO_ECUDA, "device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
    CUDA_TRY(cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreate(&C.ev0));
    CUDA_TRY(cudaEventCreate(&C.ev1));
    CUDA_TRY(cudaMalloc(&C.d_status, 4 * sizeof(int)));
    CUDA_TRY(cudaMemset(C.d_status, 0, 4 * sizeof(int)));
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    CUDA_TRY(cudaMemPoolCreate(&C.pool, &props));
    uint64_t keep = UINT64_MAX;
    CUDA_TRY(cudaMemPoolSetAttribute(C.pool, cudaMemPoolAttrReleaseThreshold, &keep));
    C.device = device;
    C.inited = true;
    return FOMO_OK;
}

int fomo_b200_shutdown(void) {
    shutdown_servers();
    auto& C = ctx();
    std::lock_guard<std::mutex> lk(C.mu);
    if (!C.inited) return FOMO_OK;
    cudaStreamSynchronize(C.stream);
    C.objs.clear();
    cudaStreamSynchronize(C.stream);
    cudaMemPoolDestroy(C.pool);
    C.pool = nullptr;
    cudaEventDestroy(C.ev0);
    cudaEventDestroy(C.ev1);
    cudaFree(C.d_status);
    C.d_status = nullptr;
    cudaStreamDestroy(C.stream);
    C.stream = nullptr;
    C.inited = false;
    C.device = -1;
    return FOMO_OK;
}

int fomo_b200_synchronize(void) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    return FOMO_OK;
}

int fomo_b200_get_stream(void** stream) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    if (!stream) return fail(FOMO_EINVAL, "stream is NULL");
    *stream = (void*)ctx().stream;
    return FOMO_OK;
}

// ---------------------------------------------------------------- buffers
int fomo_b200_alloc(size_t bytes, uint64_t* handle) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    if (!handle) return fail(FOMO_EINVAL, "handle is NULL");
    auto b = std::make_unique<Buffer>();
    if (bytes) {
        cudaError_t e = cudaMalloc(&b->ptr, bytes);
        if (e != cudaSuccess) return fail(FOMO_ENOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    b->bytes = bytes;
    *handle = put(std::move(b));
    return FOMO_OK;
}

int fomo_b200_upload(uint64_t handle, const void* host, size_t bytes) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Buffer* b = get<Buffer>(handle);
    if (!b) return fail(FOMO_EINVAL, "unknown buffer handle %llu", (unsigned long long)handle);
    if (bytes > b->bytes || (bytes && !host)) return fail(FOMO_EINVAL, "upload of %zu bytes into a %zu-byte buffer", bytes, b->bytes);
    CUDA_TRY(cudaMemcpyAsync(b->ptr, host, bytes, cudaMemcpyHostToDevice, ctx().stream));
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    return FOMO_OK;
}

int fomo_b200_download(uint64_t handle, void* host, size_t bytes) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Buffer* b = get<Buffer>(handle);
    if (!b) return fail(FOMO_EINVAL, "unknown buffer handle %llu", (unsigned long long)handle);
    if (bytes > b->bytes || (bytes && !host)) return fail(FOMO_EINVAL, "download of %zu bytes from a %zu-byte buffer", bytes, b->bytes);
    CUDA_TRY(cudaMemcpyAsync(host, b->ptr, bytes, cudaMemcpyDeviceToHost, ctx().stream));
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    return FOMO_OK;
}

int fomo_b200_memset(uint64_t handle, float value) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Buffer* b = get<Buffer>(handle);
    if (!b) return fail(FOMO_EINVAL, "unknown buffer handle %llu", (unsigned long long)handle);
    if (b->bytes % 4) return fail(FOMO_EINVAL, "buffer of %zu bytes is not a Float32 array", b->bytes);
    if (value == 0.f) {
        CUDA_TRY(cudaMemsetAsync(b->ptr, 0, b->bytes, ctx().stream));
    } else {
        std::vector<float> h(b->bytes / 4, value);
        CUDA_TRY(cudaMemcpyAsync(b->ptr, h.data(), b->bytes, cudaMemcpyHostToDevice, ctx().stream));
    }
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    return FOMO_OK;
}

int fomo_b200_free(uint64_t handle) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    if (!get<Buffer>(handle)) return fail(FOMO_EINVAL, "unknown buffer handle %llu", (unsigned long long)handle);
    cudaStreamSynchronize(ctx().stream);
    ctx().objs.erase(handle);
    return FOMO_OK;
}

// ---------------------------------------------------------------- medium
int fomo_b200_medium_create(int32_t nx, int32_t nz, int32_t M, int32_t pad, int32_t free_surface,
                            float dx, float dz, const float* rho_vx, const float* rho_vz, const float* lam,
                            const float* mu_txx, const float* mu_txz, uint64_t* medium) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    if (!medium || !rho_vx || !rho_vz || !lam || !mu_txx || !mu_txz) return fail(FOMO_EINVAL, "NULL pointer argument");
    if (int rc = check_medium_args(nx, nz, M, pad)) return rc;
    if (free_surface && pad < 5) return fail(FOMO_EINVAL, "free surface needs pad >= 5 (rows pad-4..pad+1), got %d", pad);
    auto m = std::make_unique<Medium>();
    m->nx = nx;
    m->nz = nz;
    m->pitch = pitch_of(nx);
    m->M = M;
    m->pad = pad;
    m->fs = free_surface ? 1 : 0;
    m->dx = dx;
    m->dz = dz;
    const size_t plane = (size_t)m->pitch * nz;
    cudaError_t e = pool_alloc((void**)&m->base, 5 * plane * sizeof(float));
    if (e != cudaSuccess) return fail(FOMO_ENOMEM, "medium allocation failed: %s", cudaGetErrorString(e));
    const float* src[5] = {rho_vx, rho_vz, lam, mu_txx, mu_txz};
    for (int q = 0; q < 5; ++q)
        CUDA_TRY(cudaMemcpy2DAsync(m->base + q * plane, m->pitch * sizeof(float), src[q], nx * sizeof(float),
                                   nx * sizeof(float), nz, cudaMemcpyHostToDevice, ctx().stream));
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    *medium = put(std::move(m));
    return FOMO_OK;
}

int fomo_b200_medium_create_from_model(int32_t nx_in, int32_t nz_in, const float* vp, const float* vs,
                                       const float* rho, float dx, float dz, int32_t nbc, int32_t M,
                                       int32_t free_surface, uint64_t* medium) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    if (!medium || !vp || !vs || !rho) return fail(FOMO_EINVAL, "NULL pointer argument");
    if (nx_in < 2 || nz_in < 2 || nbc < 1) return fail(FOMO_EINVAL, "bad model size %dx%d or nbc %d", nx_in, nz_in, nbc);
    const int pad = nbc + M;
    const int nx = nx_in + 2 * pad, nz = nz_in + 2 * pad;
    if (int rc = check_medium_args(nx, nz, M, pad)) return rc;
    if (free_surface && pad < 5) return fail(FOMO_EINVAL, "free surface needs pad >= 5 (rows pad-4..pad+1), got %d", pad);
    auto m = std::make_unique<Medium>();
    m->nx = nx;
    m->nz = nz;
    m->pitch = pitch_of(nx);
    m->M = M;
    m->pad = pad;
    m->fs = free_surface ? 1 : 0;
    m->dx = dx;
    m->dz = dz;
    const size_t plane = (size_t)m->pitch * nz;
    const size_t model = (size_t)nx_in * nz_in;
    float* d_model = nullptr;
    cudaError_t e = pool_alloc((void**)&m->base, 5 * plane * sizeof(float));
    if (e == cudaSuccess) e = pool_alloc((void**)&d_model, 3 * model * sizeof(float));
    if (e != cudaSuccess) return fail(FOMO_ENOMEM, "medium allocation failed: %s", cudaGetErrorString(e));
    cudaStream_t st = ctx().stream;
    const float* src[3] = {vp, vs, rho};
    int rc = FOMO_OK;
    for (int q = 0; q < 3 && rc == FOMO_OK; ++q)
        if (cudaMemcpyAsync(d_model + q * model, src[q], model * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess)
            rc = fail(FOMO_ECUDA, "model upload failed");
    if (rc == FOMO_OK) {
        fomo::ModelView V{d_model, d_model + model, d_model + 2 * model, nx_in, nz_in, pad};
        fomo::medium_init_kernel<<<8 * sm_count(), 256, 0, st>>>(V, nx, nz, m->pitch, m->base, m->base + plane,
                                                          m->base + 2 * plane, m->base + 3 * plane, m->base + 4 * plane);
        if (cudaGetLastError() != cudaSuccess) rc = fail(FOMO_ECUDA, "medium set-up kernel launch failed");
    }
    pool_free(d_model);
    cudaStreamSynchronize(st);
    if (rc) return rc;
    *medium = put(std::move(m));
    return FOMO_OK;
}

int fomo_b200_medium_download(uint64_t medium, int32_t q, float* host) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Medium* m = get<Medium>(medium);
    if (!m) return fail(FOMO_EINVAL, "unknown medium handle %llu", (unsigned long long)medium);
    if (q < 0 || q > 4 || !host) return fail(FOMO_EINVAL, "bad array %d or NULL host pointer", q);
    CUDA_TRY(cudaMemcpy2DAsync(host, m->nx * sizeof(float), m->arr(q), m->pitch * sizeof(float),
                               m->nx * sizeof(float), m->nz, cudaMemcpyDeviceToHost, ctx().stream));
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    return FOMO_OK;
}

int fomo_b200_medium_destroy(uint64_t medium) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Medium* m = get<Medium>(medium);
    if (!m) return fail(FOMO_EINVAL, "unknown medium handle %llu", (unsigned long long)medium);
    if (int n = m->users.load())
        return fail(FOMO_EINVAL, "medium %llu is in use by %d shot-server request(s)", (unsigned long long)medium, n);
    cudaStreamSynchronize(ctx().stream);
    ctx().objs.erase(medium);
    return FOMO_OK;
}

// ---------------------------------------------------------------- wavefield
int fomo_b200_wavefield_create(int32_t nx, int32_t nz, uint64_t* wavefield) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    if (!wavefield || nx < 3 || nz < 3) return fail(FOMO_EINVAL, "bad wavefield size %dx%d", nx, nz);
    auto w = std::make_unique<Wavefield>();
    w->nx = nx;
    w->nz = nz;
    w->pitch = pitch_of(nx);
    const size_t bytes = 10 * (size_t)w->pitch * nz * sizeof(float);
    cudaError_t e = pool_alloc((void**)&w->base, bytes);
    if (e != cudaSuccess) return fail(FOMO_ENOMEM, "wavefield allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    CUDA_TRY(cudaMemsetAsync(w->base, 0, bytes, ctx().stream));
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    *wavefield = put(std::move(w));
    return FOMO_OK;
}

int fomo_b200_wavefield_destroy(uint64_t wavefield) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    if (!get<Wavefield>(wavefield)) return fail(FOMO_EINVAL, "unknown wavefield handle %llu", (unsigned long long)wavefield);
    cudaStreamSynchronize(ctx().stream);
    ctx().objs.erase(wavefield);
    return FOMO_OK;
}

static int wavefield_reset_locked(Wavefield* w) {
    CUDA_TRY(cudaMemsetAsync(w->base, 0, 10 * (size_t)w->pitch * w->nz * sizeof(float), ctx().stream));
    w->cur = 0;
    return FOMO_OK;
}

int fomo_b200_wavefield_reset(uint64_t wavefield) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Wavefield* w = get<Wavefield>(wavefield);
    if (!w) return fail(FOMO_EINVAL, "unknown wavefield handle %llu", (unsigned long long)wavefield);
    if (int rc = wavefield_reset_locked(w)) return rc;
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    return FOMO_OK;
}

int fomo_b200_wavefield_download(uint64_t wavefield, int32_t field, float* host) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Wavefield* w = get<Wavefield>(wavefield);
    if (!w) return fail(FOMO_EINVAL, "unknown wavefield handle %llu", (unsigned long long)wavefield);
    if (field < 0 || field > 4 || !host) return fail(FOMO_EINVAL, "bad field %d or NULL host pointer", field);
    CUDA_TRY(cudaMemcpy2DAsync(host, w->nx * sizeof(float), w->field(w->cur, field), w->pitch * sizeof(float),
                               w->nx * sizeof(float), w->nz, cudaMemcpyDeviceToHost, ctx().stream));
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    return FOMO_OK;
}

int fomo_b200_wavefield_upload(uint64_t wavefield, int32_t field, const float* host) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Wavefield* w = get<Wavefield>(wavefield);
    if (!w) return fail(FOMO_EINVAL, "unknown wavefield handle %llu", (unsigned long long)wavefield);
    if (field < 0 || field > 4 || !host) return fail(FOMO_EINVAL, "bad field %d or NULL host pointer", field);
    CUDA_TRY(cudaMemcpy2DAsync(w->field(w->cur, field), w->pitch * sizeof(float), host, w->nx * sizeof(float),
                               w->nx * sizeof(float), w->nz, cudaMemcpyHostToDevice, ctx().stream));
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    return FOMO_OK;
}

int fomo_b200_wavefield_snapshot(uint64_t wavefield, int32_t kind, int32_t downsample, float* host) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Wavefield* w = get<Wavefield>(wavefield);
    if (!w) return fail(FOMO_EINVAL, "unknown wavefield handle %llu", (unsigned long long)wavefield);
    if (kind < 0 || kind > 3 || downsample < 1 || !host) return fail(FOMO_EINVAL, "bad snapshot arguments");
    const int nx_d = (w->nx + downsample - 1) / downsample, nz_d = (w->nz + downsample - 1) / downsample;
    const size_t bytes = (size_t)nx_d * nz_d * sizeof(float);
    if (bytes > w->snap_bytes) {
        pool_free(w->snap);
        w->snap = nullptr;
        w->snap_bytes = 0;
        cudaError_t e = pool_alloc((void**)&w->snap, bytes);
        if (e != cudaSuccess) return fail(FOMO_ENOMEM, "snapshot buffer of %zu bytes failed", bytes);
        w->snap_bytes = bytes;
    }
    const int c = w->cur;
    const float* f0 = kind == 0 ? w->field(c, fomo::TXX) : kind == 3 ? w->field(c, fomo::VZ) : w->field(c, fomo::VX);
    const float* f1 = kind == 0 ? w->field(c, fomo::TZZ) : w->field(c, fomo::VZ);
    fomo::snapshot_kernel<<<4 * sm_count(), 256, 0, ctx().stream>>>(f0, f1, kind, w->nx, w->nz, w->pitch, downsample, nx_d,
                                                             nz_d, w->snap);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(host, w->snap, bytes, cudaMemcpyDeviceToHost, ctx().stream));
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    return FOMO_OK;
}

// ---------------------------------------------------------------- shots
int fomo_b200_shot_begin(uint64_t medium, uint64_t wavefield, const FomoHabc* habc, const FomoShot* shot,
                         uint64_t* shot_handle) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Medium* m = get<Medium>(medium);
    Wavefield* w = get<Wavefield>(wavefield);
    if (!m) return fail(FOMO_EINVAL, "unknown medium handle %llu", (unsigned long long)medium);
    if (!w) return fail(FOMO_EINVAL, "unknown wavefield handle %llu", (unsigned long long)wavefield);
    if (!habc || !shot || !shot_handle) return fail(FOMO_EINVAL, "NULL argument");
    if (w->nx != m->nx || w->nz != m->nz)
        return fail(FOMO_EINVAL, "wavefield %dx%d does not match medium %dx%d", w->nx, w->nz, m->nx, m->nz);
    if (shot->M != m->M) return fail(FOMO_EINVAL, "shot M=%d differs from medium M=%d", shot->M, m->M);
    if (!shot->a) return fail(FOMO_EINVAL, "FD coefficients are NULL");
    if (shot->nt < 0) return fail(FOMO_EINVAL, "nt=%d < 0", shot->nt);
    const int nbc = habc->nbc;
    if (int rc = check_band(m->nx, m->nz, m->pad, m->fs, nbc)) return rc;
    if (!habc->w_vx || !habc->w_vz || !habc->w_tau) return fail(FOMO_EINVAL, "HABC weight tables are NULL");
    if (shot->src_i < 1 || shot->src_i > m->nx || shot->src_j < 1 || shot->src_j > m->nz)
        return fail(FOMO_EINVAL, "source (%d, %d) outside the %dx%d grid", shot->src_i, shot->src_j, m->nx, m->nz);
    if (shot->n_wavelet < 0 || (shot->n_wavelet > 0 && !shot->wavelet)) return fail(FOMO_EINVAL, "bad wavelet");
    if (shot->n_rec < 0 || (shot->n_rec > 0 && (!shot->rec_i || !shot->rec_j)))
        return fail(FOMO_EINVAL, "bad receiver arrays");
    if (shot->rec_kind < 0 || shot->rec_kind > 2) return fail(FOMO_EINVAL, "bad receiver kind %d", shot->rec_kind);
    std::vector<int> cells(shot->n_rec);
    for (int r = 0; r < shot->n_rec; ++r) {
        const int i = shot->rec_i[r], j = shot->rec_j[r];
        if (i < 1 || i > m->nx || j < 1 || j > m->nz)
            return fail(FOMO_EINVAL, "receiver %d at (%d, %d) outside the %dx%d grid", r + 1, i, j, m->nx, m->nz);
        cells[r] = (i - 1) + (j - 1) * m->pitch;
    }
    auto s = std::make_unique<Shot>();
    s->medium = medium;
    s->wavefield = wavefield;
    s->nbc = nbc;
    s->q[0] = habc->qx;
    s->q[1] = habc->qz;
    s->q[2] = habc->qt_x;
    s->q[3] = habc->qt_z;
    s->q[4] = habc->qxt;
    s->M = shot->M;
    for (int l = 0; l < shot->M; ++l) s->a[l] = shot->a[l];
    s->dt = shot->dt;
    s->dtx = shot->dtx;
    s->dtz = shot->dtz;
    s->nt = shot->nt;
    s->src_i = shot->src_i - 1;
    s->src_j = shot->src_j - 1;
    s->wavelet.assign(shot->wavelet, shot->wavelet + shot->n_wavelet);
    s->n_rec = shot->n_rec;
    s->rec_kind = shot->rec_kind;
    const size_t tab_n = (size_t)nbc + 2;
    cudaError_t e = pool_alloc((void**)&s->d_tabs, 3 * tab_n * sizeof(float));
    if (e == cudaSuccess) e = pool_alloc((void**)&s->d_band, fomo::kBandPlanes * (size_t)nbc * m->pitch * sizeof(float));
    if (e == cudaSuccess && s->n_rec) e = pool_alloc((void**)&s->d_rec, s->n_rec * sizeof(int));
    if (e == cudaSuccess && s->n_rec && s->nt)
        e = pool_alloc((void**)&s->d_gather, (size_t)s->nt * s->n_rec * sizeof(float));
    if (e != cudaSuccess) return fail(FOMO_ENOMEM, "shot allocation failed: %s", cudaGetErrorString(e));
    cudaStream_t st = ctx().stream;
    CUDA_TRY(cudaMemcpyAsync(s->d_tabs, habc->w_vx, tab_n * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(s->d_tabs + tab_n, habc->w_vz, tab_n * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(s->d_tabs + 2 * tab_n, habc->w_tau, tab_n * 4, cudaMemcpyHostToDevice, st));
    s->h2d += 3 * tab_n * 4;
    if (s->n_rec) {
        CUDA_TRY(cudaMemcpyAsync(s->d_rec, cells.data(), s->n_rec * sizeof(int), cudaMemcpyHostToDevice, st));
        s->h2d += s->n_rec * 8;
        if (s->nt) CUDA_TRY(cudaMemsetAsync(s->d_gather, 0, (size_t)s->nt * s->n_rec * sizeof(float), st));
    }
    s->h2d += (int64_t)s->wavelet.size() * 4;
    if (int rc = wavefield_reset_locked(w)) return rc;
    CUDA_TRY(cudaMemsetAsync(ctx().d_status, 0, sizeof(int), st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *shot_handle = put(std::move(s));
    return FOMO_OK;
}

int fomo_b200_shot_advance(uint64_t shot_handle, int32_t n_steps, int32_t* k_done) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Shot* s = get<Shot>(shot_handle);
    if (!s) return fail(FOMO_EINVAL, "unknown shot handle %llu", (unsigned long long)shot_handle);
    if (n_steps < 0) return fail(FOMO_EINVAL, "n_steps=%d < 0", n_steps);
    if (int rc = run_steps(*s, n_steps)) return rc;
    if (k_done) *k_done = s->k_done;
    return FOMO_OK;
}

int fomo_b200_shot_save_gather(uint64_t shot_handle, const char* path) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Shot* s = get<Shot>(shot_handle);
    if (!s) return fail(FOMO_EINVAL, "unknown shot handle %llu", (unsigned long long)shot_handle);
    if (!path) return fail(FOMO_EINVAL, "path is NULL");
    if (int rc = record_last(*s)) return rc;
    std::vector<float> host((size_t)s->nt * s->n_rec);
    if (!host.empty()) {
        CUDA_TRY(cudaMemcpyAsync(host.data(), s->d_gather, host.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                 ctx().stream));
        s->d2h += host.size() * sizeof(float);
    }
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(FOMO_EINVAL, "cannot open %s for writing: %s", path, std::strerror(errno));
    const size_t n = host.empty() ? 0 : std::fwrite(host.data(), sizeof(float), host.size(), f);
    const int closed = std::fclose(f);
    if (n != host.size() || closed != 0) return fail(FOMO_EINVAL, "writing %s failed", path);
    return FOMO_OK;
}

int fomo_b200_shot_finish(uint64_t shot_handle, float* gather_out, FomoRunStats* stats) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Shot* s = get<Shot>(shot_handle);
    if (!s) return fail(FOMO_EINVAL, "unknown shot handle %llu", (unsigned long long)shot_handle);
    if (int rc = record_last(*s)) return rc;
    if (gather_out && s->n_rec && s->nt) {
        const size_t bytes = (size_t)s->nt * s->n_rec * sizeof(float);
        CUDA_TRY(cudaMemcpyAsync(gather_out, s->d_gather, bytes, cudaMemcpyDeviceToHost, ctx().stream));
        s->d2h += bytes;
    }
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    if (stats) {
        stats->device_ms = s->device_ms;
        stats->steps = s->k_done;
        stats->kernel_launches = s->launches;
        stats->h2d_bytes = s->h2d;
        stats->d2h_bytes = s->d2h;
    }
    ctx().objs.erase(shot_handle);
    return FOMO_OK;
}

int fomo_b200_shot_profile(uint64_t shot_handle, int32_t n_steps, FomoKernelTime* out, int32_t max_kinds,
                           int32_t* n_kinds) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    Shot* s = get<Shot>(shot_handle);
    if (!s) return fail(FOMO_EINVAL, "unknown shot handle %llu", (unsigned long long)shot_handle);
    if (n_steps < 0 || n_steps > 100000 || !out || !n_kinds || max_kinds < 4)
        return fail(FOMO_EINVAL, "bad profile arguments (max_kinds must be >= 4)");
    const int nk = max_kinds >= 5 ? 5 : 4;
    Medium* m = get<Medium>(s->medium);
    if (!m) return fail(FOMO_EINVAL, "shot refers to a destroyed medium");
    Profile prof;
    if (int rc = run_steps(*s, n_steps, &prof)) return rc;
    CUDA_TRY(cudaStreamSynchronize(ctx().stream));
    // Algorithmic bytes of one launch.  Tile launches, over the nx*nz cells:
    // velocity reads vx, vz, txx, tzz, txz, rho_vx, rho_vz and writes vx, vz
    // (36 B/cell); stress reads vx, vz, txx, tzz, txz, lam, mu_txx, mu_txz
    // and writes txx, tzz, txz (44 B/cell).  Band passes, over the nbc*nx
    // band cells: read the stencil value and the step-start value of each
    // output field and write its final value (24 B/cell velocity, 36 stress).
    // The fused step reads the five fields, two buoyancy arrays (four when
    // dx != dz) and lam, mu_txx, mu_txz, and writes the five fields
    // (60 B/cell, 68 B with four buoyancy arrays).
    const double cells = (double)m->nx * m->nz, band = (double)s->nbc * m->nx;
    const char* names[5] = {"velocity", "stress", "band_velocity", "band_stress", "step"};
    const double bytes[5] = {36.0 * cells, 44.0 * cells, 24.0 * band, 36.0 * band,
                             (s->dtx == s->dtz ? 60.0 : 68.0) * cells};
    for (size_t i = 0; i < prof.kind.size(); ++i)
        if (prof.kind[i] >= nk) return fail(FOMO_EINVAL, "the fused step ran: max_kinds must be >= 5");
    for (int k = 0; k < nk; ++k) {
        std::memset(&out[k], 0, sizeof(FomoKernelTime));
        std::snprintf(out[k].name, sizeof(out[k].name), "%s", names[k]);
        out[k].bytes_per_launch = bytes[k];
    }
    for (size_t i = 0; i < prof.kind.size(); ++i) {
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, prof.ev[2 * i], prof.ev[2 * i + 1]));
        out[prof.kind[i]].launches += 1;
        out[prof.kind[i]].total_ms += ms;
    }
    *n_kinds = nk;
    return FOMO_OK;
}

int fomo_b200_set_step_kernel(int32_t mode, int32_t n_segs) {
    if (mode != FOMO_STEP_AUTO && mode != FOMO_STEP_SPLIT && mode != FOMO_STEP_FUSED)
        return fail(FOMO_EINVAL, "unknown step kernel mode %d", mode);
    if (n_segs < 0 || n_segs > fomo::kMMaxSegs)
        return fail(FOMO_EINVAL, "n_segs=%d out of range 0..%d", n_segs, fomo::kMMaxSegs);
    g_step_mode.store(mode);
    g_march_segs.store(n_segs);
    return FOMO_OK;
}

int fomo_b200_selftest_wait(int32_t polls, int32_t* status) {
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (int rc = ensure_init()) return rc;
    if (polls < 1 || polls > (1 << 20) || !status) return fail(FOMO_EINVAL, "polls must be 1..2^20");
    cudaStream_t st = ctx().stream;
    CUDA_TRY(cudaMemsetAsync(ctx().d_status, 0, sizeof(int), st));
    fomo::wait_selftest_kernel<<<1, 32, 0, st>>>(ctx().d_status, polls);
    CUDA_TRY(cudaGetLastError());
    const int rc = check_status();
    *status = rc;
    CUDA_TRY(cudaMemsetAsync(ctx().d_status, 0, sizeof(int), st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return FOMO_OK;
}

int fomo_b200_run_shot(uint64_t medium, uint64_t wavefield, const FomoHabc* habc, const FomoShot* shot,
                       float* gather_out, FomoRunStats* stats) {
    uint64_t h = 0;
    if (int rc = fomo_b200_shot_begin(medium, wavefield, habc, shot, &h)) return rc;
    int32_t k = 0;
    if (int rc = fomo_b200_shot_advance(h, shot->nt, &k)) {
        std::string msg = g_err;
        fomo_b200_shot_finish(h, nullptr, nullptr);
        g_err = msg;
        return rc;
    }
    return fomo_b200_shot_finish(h, gather_out, stats);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free shot: fomo_b200_run_shot_noalloc.
//
// Some callers cannot call cudaMalloc while they run a shot: a serving loop
// whose memory is carved once from a fixed pool at start-up and must not run
// out later, or a host framework that forbids device allocation (and the
// device-wide synchronisation cudaFree implies) on its latency path.  For them
// this entry point runs the same time-step kernels with every scratch buffer
// taken from one static device array: the two wavefield copies, the buoyancy
// arrays, the HABC weight tables, the receiver offsets and the kernels' status
// word.  The caller passes the inputs (medium, on the device) and the output
// (gather, on the device); nothing is allocated or freed.
//
// The array (kNoAllocScratchBytes) is part of the library's device image, so
// every GPU that loads the library holds it until the process exits.  All
// calls share it and it keeps the last call's contents: each call clears the
// wavefield and the status word before its first step.  Calls that overlap on
// the GPU (two streams, two threads, two devices' worth of work aimed at one
// device) race on the array; callers must serialise them.  The first call on
// a device resolves the array's address there (noalloc_scratch); it should
// come before any stream capture on that device.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocScratchBytes = 48ull << 20;  // 48 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kMaxDevices] = {nullptr};

inline size_t align256(size_t n) { return (n + 255) / 256 * 256; }

// Device address of the scratch array for the current device.  The first call
// on a device resolves it (cudaGetSymbolAddress, with that device current).
int noalloc_scratch(unsigned char** out) {
    int dev = -1;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(FOMO_EINVAL, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return FOMO_OK;
}

template <int M>
int noalloc_loop(const fomo::StepParams& P0, fomo::TiledArgs T, float* fields, int pitch, int nx, int nz,
                 const float* const* med, const float* const* buoy, const float* wavelet, int n_wavelet,
                 int nt, int n_rec, cudaStream_t st) {
    using G = fomo::Geo<M>;
    const bool iso = T.iso != 0;
    const size_t plane = (size_t)pitch * nz;
    auto field = [&](int copy, int q) { return fields + ((size_t)copy * 5 + q) * plane; };
    CUtensorMap halo[2][5], tile[2][5], mod[3], bm[4];
    for (int c = 0; c < 2; ++c)
        for (int q = 0; q < 5; ++q) {
            if (int rc = encode_map(&halo[c][q], field(c, q), nx, nz, pitch, G::BOXW, G::BOXH)) return rc;
            if (int rc = encode_map(&tile[c][q], field(c, q), nx, nz, pitch, fomo::kTX, fomo::kTZ)) return rc;
        }
    for (int q = 0; q < 3; ++q)
        if (int rc = encode_map(&mod[q], med[2 + q], nx, nz, pitch, fomo::kTX, fomo::kTZ)) return rc;
    for (int q = 0; q < 4; ++q)
        if (int rc = encode_map(&bm[q], buoy[q], nx, nz, pitch, fomo::kTX, fomo::kTZ)) return rc;
    const Launch L = launch_shape<M>(nx, nz, P0.nbc, iso, P0.fs != 0);
    if (int rc = raise_smem_limit(fomo::velocity_kernel<M>, L.smem_v)) return rc;
    if (int rc = raise_smem_limit(fomo::stress_kernel<M>, L.smem_s)) return rc;
    T.n_tile_blocks = L.n_tile;
    T.tiles_x = L.tiles_x;
    T.x_last = L.x_last;
    T.prefetch_ahead = fomo::prefetch_distance(sm_count());
    const int rec_blocks = (n_rec + fomo::kThreads - 1) / fomo::kThreads;
    int cur = 0;
    for (int k = 1; k <= nt; ++k) {
        const int a = cur, b = 1 - cur;
        fomo::StepParams P = P0;
        P.src_w = (k <= n_wavelet) ? wavelet[k - 1] : 0.f;
        for (int q = 0; q < 5; ++q) P.in[q] = field(a, q);
        P.out[fomo::VX] = field(b, fomo::VX);
        P.out[fomo::VZ] = field(b, fomo::VZ);
        P.rec_k = (k >= 2 && n_rec > 0) ? k - 1 : 0;
        fomo::VelMaps vm;
        vm.xx = halo[a][fomo::TXX];
        vm.zz = halo[a][fomo::TZZ];
        vm.xz = halo[a][fomo::TXZ];
        vm.vx = tile[a][fomo::VX];
        vm.vz = tile[a][fomo::VZ];
        vm.b0 = bm[0];
        vm.b1 = bm[1];
        vm.b2 = bm[2];
        vm.b3 = bm[3];
        fomo::velocity_kernel<M><<<L.n_tile + (P.rec_k ? rec_blocks : 0), fomo::kThreads, L.smem_v, st>>>(P, T, vm);
        fomo::band_kernel<true><<<L.n_band, 32, 0, st>>>(P, T);
        P.in[fomo::VX] = field(b, fomo::VX);
        P.in[fomo::VZ] = field(b, fomo::VZ);
        for (int q = 2; q < 5; ++q) P.out[q] = field(b, q);
        P.out[fomo::VX] = P.out[fomo::VZ] = nullptr;
        P.rec_k = 0;
        fomo::StrMaps sm;
        sm.vx = halo[b][fomo::VX];
        sm.vz = halo[b][fomo::VZ];
        sm.txx = tile[a][fomo::TXX];
        sm.tzz = tile[a][fomo::TZZ];
        sm.txz = tile[a][fomo::TXZ];
        sm.lam = mod[0];
        sm.mu = mod[1];
        sm.mxz = mod[2];
        fomo::stress_kernel<M><<<L.n_tile, fomo::kThreads, L.smem_s, st>>>(P, T, sm);
        fomo::band_kernel<false><<<L.n_band, 32, 0, st>>>(P, T);
        cur = b;
    }
    if (n_rec > 0 && nt > 0) {  // receivers of the last step
        fomo::StepParams P = P0;
        for (int q = 0; q < 5; ++q) P.in[q] = field(cur, q);
        P.rec_k = nt;
        fomo::record_kernel<<<rec_blocks, fomo::kThreads, 0, st>>>(P);
    }
    CUDA_TRY(cudaGetLastError());
    return FOMO_OK;
}

}  // namespace

extern "C" int fomo_b200_run_shot_noalloc(int32_t nx, int32_t nz, int32_t M, int32_t pad, int32_t free_surface,
                                          const float* rho_vx, const float* rho_vz, const float* lam,
                                          const float* mu_txx, const float* mu_txz, int32_t pitch,
                                          const FomoHabc* habc, const FomoShot* shot, float* gather_out,
                                          void* stream) {
    if (!rho_vx || !rho_vz || !lam || !mu_txx || !mu_txz || !habc || !shot)
        return fail(FOMO_EINVAL, "NULL argument");
    if (int rc = check_medium_args(nx, nz, M, pad)) return rc;
    if (free_surface && pad < 5) return fail(FOMO_EINVAL, "free surface needs pad >= 5 (rows pad-4..pad+1), got %d", pad);
    if (pitch < (nx + 3) / 4 * 4 || pitch % 4)
        return fail(FOMO_EINVAL, "row pitch %d must be a multiple of 4 floats and >= round_up(nx, 4) = %d", pitch,
                    (nx + 3) / 4 * 4);
    const float* med[5] = {rho_vx, rho_vz, lam, mu_txx, mu_txz};
    for (int q = 0; q < 5; ++q)
        if ((uintptr_t)med[q] % 16) return fail(FOMO_EINVAL, "medium array %d is not 16-byte aligned", q);
    if (shot->M != M || !shot->a) return fail(FOMO_EINVAL, "shot M=%d differs from medium M=%d or no coefficients", shot->M, M);
    if (shot->nt < 0 || shot->n_wavelet < 0 || (shot->n_wavelet > 0 && !shot->wavelet)) return fail(FOMO_EINVAL, "bad nt or wavelet");
    const int nbc = habc->nbc;
    if (int rc = check_band(nx, nz, pad, free_surface ? 1 : 0, nbc)) return rc;
    if (!habc->w_vx || !habc->w_vz || !habc->w_tau) return fail(FOMO_EINVAL, "HABC weight tables are NULL");
    if (shot->src_i < 1 || shot->src_i > nx || shot->src_j < 1 || shot->src_j > nz)
        return fail(FOMO_EINVAL, "source (%d, %d) outside the %dx%d grid", shot->src_i, shot->src_j, nx, nz);
    if (shot->rec_kind < 0 || shot->rec_kind > 2) return fail(FOMO_EINVAL, "bad receiver kind %d", shot->rec_kind);
    if (shot->n_rec < 0 || (shot->n_rec > 0 && (!shot->rec_i || !shot->rec_j || !gather_out)))
        return fail(FOMO_EINVAL, "bad receiver arrays or gather pointer");
    std::vector<int> cells(shot->n_rec);
    for (int r = 0; r < shot->n_rec; ++r) {
        const int i = shot->rec_i[r], j = shot->rec_j[r];
        if (i < 1 || i > nx || j < 1 || j > nz)
            return fail(FOMO_EINVAL, "receiver %d at (%d, %d) outside the %dx%d grid", r + 1, i, j, nx, nz);
        cells[r] = (i - 1) + (j - 1) * pitch;
    }
    // Carve the scratch: status | tables | receiver offsets | buoyancy | band | wavefield.
    const bool iso = shot->dtx == shot->dtz;
    const size_t plane = (size_t)pitch * nz * sizeof(float);
    const size_t off_tab = 256;
    const size_t off_rec = off_tab + align256(3 * (size_t)(nbc + 2) * sizeof(float));
    const size_t off_buo = off_rec + align256((size_t)shot->n_rec * sizeof(int));
    const size_t off_band = off_buo + align256((iso ? 2 : 4) * plane);
    const size_t off_wf = off_band + align256(fomo::kBandPlanes * (size_t)nbc * pitch * sizeof(float));
    const size_t need = off_wf + 10 * plane;
    if (need > kNoAllocScratchBytes)
        return fail(FOMO_EINVAL, "shot needs %zu bytes of scratch, more than the %zu-byte static array of "
                    "fomo_b200_run_shot_noalloc (grid %dx%d, pitch %d, %d receivers)", need, kNoAllocScratchBytes,
                    nx, nz, pitch, shot->n_rec);
    unsigned char* base = nullptr;
    if (int rc = noalloc_scratch(&base)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    int* d_status = reinterpret_cast<int*>(base);
    float* d_tabs = reinterpret_cast<float*>(base + off_tab);
    int* d_rec = reinterpret_cast<int*>(base + off_rec);
    float* d_buo = reinterpret_cast<float*>(base + off_buo);
    float* d_fields = reinterpret_cast<float*>(base + off_wf);
    float* d_band = reinterpret_cast<float*>(base + off_band);
    const size_t tab_n = (size_t)nbc + 2;
    CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    CUDA_TRY(cudaMemsetAsync(d_fields, 0, 10 * plane, st));
    CUDA_TRY(cudaMemcpyAsync(d_tabs, habc->w_vx, tab_n * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(d_tabs + tab_n, habc->w_vz, tab_n * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(d_tabs + 2 * tab_n, habc->w_tau, tab_n * 4, cudaMemcpyHostToDevice, st));
    if (shot->n_rec) CUDA_TRY(cudaMemcpyAsync(d_rec, cells.data(), cells.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    const size_t pf = (size_t)pitch * nz;
    float* b0 = d_buo;
    float* b2 = d_buo + pf;
    float* b1 = iso ? b0 : d_buo + 2 * pf;
    float* b3 = iso ? b2 : d_buo + 3 * pf;
    fomo::buoyancy_kernel<<<4 * sm_count(), 256, 0, st>>>(rho_vx, rho_vz, shot->dtx, shot->dtz, pf, b0, b1, b2, b3);
    CUDA_TRY(cudaGetLastError());

    fomo::StepParams P;
    std::memset(&P, 0, sizeof(P));
    P.nx = nx;
    P.nz = nz;
    P.pitch = pitch;
    P.M = M;
    P.pad = pad;
    P.nbc = nbc;
    P.fs = free_surface ? 1 : 0;
    P.dtx = shot->dtx;
    P.dtz = shot->dtz;
    for (int l = 0; l < M; ++l) P.a[l] = shot->a[l];
    P.qx = habc->qx;
    P.qz = habc->qz;
    P.qt_x = habc->qt_x;
    P.qt_z = habc->qt_z;
    P.qxt = habc->qxt;
    for (int t = 0; t < 3; ++t) P.w_tab[t] = d_tabs + t * tab_n;
    P.rho_vx = rho_vx;
    P.rho_vz = rho_vz;
    P.lam = lam;
    P.mu_txx = mu_txx;
    P.mu_txz = mu_txz;
    P.src_i = shot->src_i - 1;
    P.src_j = shot->src_j - 1;
    P.nt = shot->nt;
    P.n_rec = shot->n_rec;
    P.rec_kind = shot->rec_kind;
    P.rec_cell = d_rec;
    P.gather = gather_out;
    fomo::TiledArgs T;
    std::memset(&T, 0, sizeof(T));
    T.b[0] = b0;
    T.b[1] = b1;
    T.b[2] = b2;
    T.b[3] = b3;
    T.iso = iso ? 1 : 0;
    T.status = d_status;
    T.band_pre = d_band;
    const float* bp[4] = {b0, b1, b2, b3};
    int rc = FOMO_EINVAL;
    switch (M) {
        case 1: rc = noalloc_loop<1>(P, T, d_fields, pitch, nx, nz, med, bp, shot->wavelet, shot->n_wavelet, shot->nt, shot->n_rec, st); break;
        case 2: rc = noalloc_loop<2>(P, T, d_fields, pitch, nx, nz, med, bp, shot->wavelet, shot->n_wavelet, shot->nt, shot->n_rec, st); break;
        case 3: rc = noalloc_loop<3>(P, T, d_fields, pitch, nx, nz, med, bp, shot->wavelet, shot->n_wavelet, shot->nt, shot->n_rec, st); break;
        case 4: rc = noalloc_loop<4>(P, T, d_fields, pitch, nx, nz, med, bp, shot->wavelet, shot->n_wavelet, shot->nt, shot->n_rec, st); break;
        case 5: rc = noalloc_loop<5>(P, T, d_fields, pitch, nx, nz, med, bp, shot->wavelet, shot->n_wavelet, shot->nt, shot->n_rec, st); break;
        case 6: rc = noalloc_loop<6>(P, T, d_fields, pitch, nx, nz, med, bp, shot->wavelet, shot->n_wavelet, shot->nt, shot->n_rec, st); break;
    }
    if (rc) return rc;
    int status = 0;
    CUDA_TRY(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (status == fomo::kErrTmaTimeout) return fail(FOMO_ETIMEOUT, "a TMA load of a time-step kernel did not complete");
    if (status) return fail(FOMO_ECUDA, "time-step kernel reported error %d", status);
    return FOMO_OK;
}

#include "server.cuh"
