/*
 * fomo_b200.h -- C ABI of libfomo_b200.so, the B200 (sm_100a) engine for the
 * time-stepping path of Wuheng10086/Fomo_julia's Elastic2D module.
 *
 * This is the boundary a `backend(:b200)` for the reference binds through
 * `ccall`: plain pointers, sizes and opaque 64-bit handles, no C++ or torch
 * types.  Each declaration names the reference interface it stands in for
 * (paths inside Wuheng10086/Fomo_julia).
 *
 * Conventions
 *   - Every function returns an int status: FOMO_OK (0) or a negative
 *     FOMO_E* code; fomo_b200_last_error() then holds a message for the
 *     calling thread.
 *   - Grids are the reference's padded (nx, nz) Float32 matrices, column
 *     major with x fastest: element (i, j) (1-based) at (i-1) + (j-1)*nx.
 *   - Grid indices passed in (source, receivers) are 1-based, as Julia
 *     passes them.
 *   - Host pointers are borrowed for the duration of the call only.  The
 *     library owns all device memory it allocates.  Media, wavefields and
 *     shots come from a per-device stream-ordered memory pool that keeps
 *     freed memory for reuse (destroying them returns memory to the pool,
 *     not to the device; fomo_b200_shutdown releases it).  When an
 *     allocation fails, the pool gives its cached memory back to the device
 *     and the allocation is tried once more before FOMO_ENOMEM.
 *   - Gathers are [nt x n_rec] column major: sample k (1-based) of receiver r
 *     (1-based) at (k-1) + (r-1)*nt, exactly the reference's Receivers.data.
 */
#ifndef FOMO_B200_H
#define FOMO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FOMO_OK          0
#define FOMO_EINVAL     -1   /* invalid argument, size or handle            */
#define FOMO_ENOMEM     -2   /* device allocation failed / over HBM budget  */
#define FOMO_ECUDA      -3   /* a CUDA runtime or driver call failed        */
#define FOMO_ETIMEOUT   -4   /* a bounded device-side wait gave up          */
#define FOMO_ECANCELLED -5   /* a queued request was cancelled              */
#define FOMO_ENOTREADY  -6   /* request not finished yet (poll)             */
#define FOMO_ENOINIT    -7   /* fomo_b200_init has not been called          */

/* Receiver components: Receivers.type (src/core/Structures.jl:127-132). */
#define FOMO_REC_VZ 0
#define FOMO_REC_VX 1
#define FOMO_REC_P  2        /* (txx + tzz) * 0.5, as the CPU method does   */

/* Wavefield components, in the order of Wavefield's fields. */
#define FOMO_FIELD_VX  0
#define FOMO_FIELD_VZ  1
#define FOMO_FIELD_TXX 2
#define FOMO_FIELD_TZZ 3
#define FOMO_FIELD_TXZ 4

/* ---------------------------------------------------------------------- */
/* Library lifetime                                                        */
/* ---------------------------------------------------------------------- */

/* Selects the CUDA device and creates the library's stream.  Stands in for
 * the CUDA probe of src/Elastic2D.jl:24-34 and backend(:cuda) in
 * src/backends/backend.jl:39-53. */
int fomo_b200_init(int device);

/* Frees every handle and the stream. */
int fomo_b200_shutdown(void);

/* Message for the last failing call on this thread ("" if none); stands in
 * for the reference's error(...) strings (src/backends/backend.jl:49). */
const char* fomo_b200_last_error(void);

/* Version as major*10000 + minor*100 + patch. */
int fomo_b200_version(void);

/* ---------------------------------------------------------------------- */
/* Raw device buffers (backing store of a B200Matrix / B200Vector)         */
/* ---------------------------------------------------------------------- */

/* to_device(data, backend) (src/backends/backend.jl:68-71) = alloc + upload;
 * Array(x) = download; fill!(x, v) = memset. */
int fomo_b200_alloc(size_t bytes, uint64_t* handle);
int fomo_b200_upload(uint64_t handle, const void* host, size_t bytes);
int fomo_b200_download(uint64_t handle, void* host, size_t bytes);
int fomo_b200_memset(uint64_t handle, float value);
int fomo_b200_free(uint64_t handle);

/* synchronize(::CUDABackend) (src/backends/backend.jl:78-79). */
int fomo_b200_synchronize(void);

/* The library's CUDA stream (a cudaStream_t), so a caller can order its own
 * work or timing events against the library's kernels.  No reference
 * counterpart: CUDA.jl's task-local stream plays this role there. */
int fomo_b200_get_stream(void** stream);

/* ---------------------------------------------------------------------- */
/* Medium: Medium{T} (src/core/Structures.jl:66-83) as built by           */
/* init_medium (src/utils/init.jl:68-99).                                  */
/* ---------------------------------------------------------------------- */

/* Uploads the five staggered material arrays of a padded (nx, nz) grid.
 * M = fd_order/2 (1..6), pad = nbc + M, free_surface 0/1. */
int fomo_b200_medium_create(int32_t nx, int32_t nz, int32_t M, int32_t pad,
                            int32_t free_surface, float dx, float dz,
                            const float* rho_vx, const float* rho_vz,
                            const float* lam, const float* mu_txx,
                            const float* mu_txz, uint64_t* medium);
int fomo_b200_medium_destroy(uint64_t medium);

/* init_medium (src/utils/init.jl:68-99) on the device: uploads the unpadded
 * (nx_in, nz_in) vp, vs, rho (host, column major) and computes the padding
 * (_pad_array, init.jl:119-134; pad = nbc + M) and the staggered parameters
 * (_compute_staggered_params, init.jl:136-158) in the GPU, with the same
 * Float32 operations in the same order: the medium is bit-identical to
 * fomo_b200_medium_create of the host-computed arrays, and three unpadded
 * arrays cross PCIe instead of five padded ones. */
int fomo_b200_medium_create_from_model(int32_t nx_in, int32_t nz_in, const float* vp,
                                       const float* vs, const float* rho, float dx, float dz,
                                       int32_t nbc, int32_t M, int32_t free_surface,
                                       uint64_t* medium);
/* Array(M.rho_vx) etc.: copies staggered array q (0 rho_vx, 1 rho_vz, 2 lam,
 * 3 mu_txx, 4 mu_txz) into host[nx*nz]. */
int fomo_b200_medium_download(uint64_t medium, int32_t q, float* host);

/* ---------------------------------------------------------------------- */
/* HABC: HABCConfig{T} (src/core/Structures.jl:94-105) as built by         */
/* init_habc (src/utils/init.jl:171-203).                                  */
/* ---------------------------------------------------------------------- */

/* The reference stores each weight as a full (nz, nx) matrix, but every
 * entry is a function of dist = min(i-1, nx-i, j-1, nz-j) alone
 * (init.jl:188-195); the three tables give that function for
 * dist = 0..nbc+1 (larger distances use entry nbc+1). */
typedef struct {
    int32_t nbc;
    float qx, qz, qt_x, qt_z, qxt;
    const float* w_vx;    /* host, nbc+2 entries */
    const float* w_vz;
    const float* w_tau;
} FomoHabc;

/* ---------------------------------------------------------------------- */
/* Wavefield{T} (src/core/Structures.jl:18-55)                             */
/* ---------------------------------------------------------------------- */

/* Wavefield(nx, nz, backend): device state of one shot.  The B200 engine
 * keeps two copies of the five fields (the step reads one, writes the
 * other); the reference's five *_old boundary strips are the copy being
 * read, so no separate backup pass exists. */
int fomo_b200_wavefield_create(int32_t nx, int32_t nz, uint64_t* wavefield);
int fomo_b200_wavefield_destroy(uint64_t wavefield);
/* reset!(backend, W) (src/kernels/source_receiver.jl:115-133). */
int fomo_b200_wavefield_reset(uint64_t wavefield);
/* Array(W.vx) etc.: copies the current value of one field (FOMO_FIELD_*)
 * into host[nx*nz]. */
int fomo_b200_wavefield_download(uint64_t wavefield, int32_t field, float* host);
/* to_device into W.vx etc.: overwrites the current value of one field. */
int fomo_b200_wavefield_upload(uint64_t wavefield, int32_t field, const float* host);

/* Snapshot frames for an on_step hook: the frame extraction of the
 * reference's video recorder (src/visualization/video_recorder.jl:260-297)
 * done on the device.  kind: FOMO_SNAP_P ((txx+tzz)*0.5), FOMO_SNAP_VEL
 * (sqrt(vx^2+vz^2)), FOMO_SNAP_VX, FOMO_SNAP_VZ; frame (i, j) (1-based) is
 * cell (min((i-1)*ds+1, nx), min((j-1)*ds+1, nz)) of the current state;
 * host receives cld(nx,ds) * cld(nz,ds) floats, column major.  No rendering:
 * the frames go to the caller's buffer. */
#define FOMO_SNAP_P   0
#define FOMO_SNAP_VEL 1
#define FOMO_SNAP_VX  2
#define FOMO_SNAP_VZ  3
int fomo_b200_wavefield_snapshot(uint64_t wavefield, int32_t kind, int32_t downsample, float* host);

/* ---------------------------------------------------------------------- */
/* One shot: Source (Structures.jl:116-120), Receivers (:127-132),         */
/* SimParams (:143-155) and the FD coefficients (init.jl:13-29).           */
/* ---------------------------------------------------------------------- */

typedef struct {
    const float* a;        /* host, M FD coefficients                        */
    int32_t M;             /* must equal the medium's M                      */
    float dt, dtx, dtz;    /* SimParams: dtx = Float32(dt/dx) etc.           */
    int32_t nt;            /* time steps                                     */
    int32_t src_i, src_j;  /* 1-based source cell (explosive: txx and tzz)   */
    const float* wavelet;  /* host, n_wavelet samples; step k > n_wavelet    */
    int32_t n_wavelet;     /*   injects nothing (source_receiver.jl:19-21)   */
    int32_t n_rec;         /* receivers (0 allowed)                          */
    const int32_t* rec_i;  /* host, 1-based                                  */
    const int32_t* rec_j;
    int32_t rec_kind;      /* FOMO_REC_*                                     */
} FomoShot;

typedef struct {
    double device_ms;      /* device time of the time loop (CUDA events)     */
    int64_t steps;         /* time steps run                                 */
    int64_t kernel_launches;/* kernels launched by the library for the loop  */
    int64_t h2d_bytes;     /* host->device bytes moved by the call           */
    int64_t d2h_bytes;     /* device->host bytes moved by the call           */
} FomoRunStats;

/* run_shot! (src/simulation/shot_manager.jl:46-68) with run_time_loop!
 * (src/simulation/time_stepper.jl:97-128) and time_step! (:39-63):
 * resets the wavefield, runs nt steps and writes the gather to
 * gather_out[nt*n_rec] (host).  The call blocks until the gather is on the
 * host.  stats may be NULL. */
int fomo_b200_run_shot(uint64_t medium, uint64_t wavefield, const FomoHabc* habc,
                       const FomoShot* shot, float* gather_out, FomoRunStats* stats);

/* The same loop in chunks, for an on_step callback (time_stepper.jl:112-119):
 * begin resets the wavefield and uploads the shot; advance runs up to
 * n_steps more steps (returns the number of steps done so far in *k_done);
 * the wavefield can be downloaded between advances; finish copies the
 * gather (the first k_done rows are valid) and releases the shot.  A shot
 * stopped early is finished like a complete one. */
int fomo_b200_shot_begin(uint64_t medium, uint64_t wavefield, const FomoHabc* habc,
                         const FomoShot* shot, uint64_t* shot_handle);
int fomo_b200_shot_advance(uint64_t shot_handle, int32_t n_steps, int32_t* k_done);
int fomo_b200_shot_finish(uint64_t shot_handle, float* gather_out, FomoRunStats* stats);

/* save_gather(result, path; format=:bin) (src/io/output.jl:18-33, _save_bin
 * :28-33) written straight from the shot's device seismogram: raw Float32,
 * column-major [nt x n_rec] (host byte order, little-endian on the supported
 * hosts), no header.  Call between begin and finish; the receivers of the last
 * step done are recorded first, rows after it are zero. */
int fomo_b200_shot_save_gather(uint64_t shot_handle, const char* path);

/* Per-kernel timing of a shot's loop (no reference counterpart; used by
 * bench.py for the roofline).  Runs up to n_steps more steps of the shot
 * with CUDA events around every launch and reports, per kernel kind
 * (velocity, stress, band_velocity, band_stress: max_kinds >= 4; and step,
 * the fused step, when max_kinds >= 5), the
 * launches, their summed device time and the algorithmic DRAM bytes of one
 * launch (the bytes a launch must move at minimum: each array it reads
 * once and each array it writes once, over the cells it updates). */
typedef struct {
    char name[32];
    int64_t launches;
    double total_ms;
    double bytes_per_launch;
} FomoKernelTime;

int fomo_b200_shot_profile(uint64_t shot_handle, int32_t n_steps, FomoKernelTime* out,
                           int32_t max_kinds, int32_t* n_kinds);

/* Time-step kernel selection (no reference counterpart; a tuning control).
 * Two forms of the time step give the same bits: the split launches
 * (velocity tiles, velocity band pass, stress tiles, stress band pass) and
 * the fused step -- one launch per time step that computes velocity and
 * stress together in column strips, so every field and medium array crosses
 * HBM once (free surface, M <= 4, HABC bands that fit its first and last
 * strips).  FOMO_STEP_AUTO times both on 24 live steps each of the first
 * shot of a (grid, order, HABC width) with enough steps left, keeps the
 * faster for the process (and in the FOMO_B200_TUNE_CACHE file when that is
 * set), and runs the split launches where the fused step does not apply or
 * the shot is too short to time.  FOMO_STEP_SPLIT always runs the split
 * launches; FOMO_STEP_FUSED fails a single shot that the fused step does not
 * support with FOMO_EINVAL.  n_segs > 0 fixes the fused step's row segments
 * per column strip (1..64; 0 = chosen from the grid and the SM count).
 * Process-wide.  The batched and served paths run the fused step under
 * FOMO_STEP_FUSED and the split launches otherwise;
 * fomo_b200_run_shot_noalloc runs the split launches. */
#define FOMO_STEP_AUTO 0
#define FOMO_STEP_SPLIT 1
#define FOMO_STEP_FUSED 2
int fomo_b200_set_step_kernel(int32_t mode, int32_t n_segs);

/* Self-test of the kernels' bounded device waits (no reference
 * counterpart).  Every wait of a time-step kernel on its TMA loads polls at
 * most a fixed number of times, then records an error that the call reports
 * as FOMO_ETIMEOUT instead of hanging the GPU.  This runs the same wait on a
 * barrier that nothing completes, for `polls` polls (1..2^20), and stores
 * the resulting status in *status (FOMO_ETIMEOUT when the mechanism works);
 * nothing is left outstanding on the device. */
int fomo_b200_selftest_wait(int32_t polls, int32_t* status);

/* Allocation-free shot.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory while a shot runs -- a serving
 * loop that carves all of its memory from a fixed pool at start-up and must
 * not fail for lack of memory later, or a host framework that forbids
 * cudaMalloc/cudaFree (and the device-wide synchronisation cudaFree implies)
 * on its latency path.
 *
 * Runs the same kernels as fomo_b200_run_shot and calls no cudaMalloc,
 * cudaFree or allocating library routine.  Every scratch buffer (both
 * wavefield copies, the buoyancy arrays, HABC tables, receiver offsets, the
 * kernels' status word) comes from one static device array of 48 MiB that
 * every GPU loading the library holds until the process exits; grids whose
 * scratch does not fit are rejected with FOMO_EINVAL and a message giving
 * the bytes needed.  The scratch is 10 fields (+2 buoyancy arrays when
 * dtx == dtz, +4 otherwise) of pitch*nz floats, 5*nbc rows of pitch floats
 * for the bottom band, plus a few KB, so for example a 1000 x 1000 padded
 * grid with dtx == dtz and nbc = 50 fits.
 *
 * Inputs: the five medium arrays on the device (each pitch*nz floats, row
 * pitch `pitch` floats: a multiple of 4 and >= round_up(nx, 4); 16-byte
 * aligned), the HABC and shot descriptions as for fomo_b200_run_shot (host
 * structs).  Output: gather_out, a device array of nt*n_rec floats
 * ([nt x n_rec] column major).  Work is queued on `stream` (a cudaStream_t,
 * NULL for the legacy default stream): the HABC tables and receiver offsets
 * are copied from host memory with cudaMemcpyAsync, and the call waits for
 * the stream and reads the kernels' status word back before it returns.
 * fomo_b200_init is not required; the current CUDA device is used.
 *
 * The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress, with that device current) and keeps it; make that
 * first call before any stream capture on the device.  All calls share the
 * array and it keeps the last call's contents; each call clears what must
 * start at zero (the wavefield and the status word).  Calls that overlap on
 * the GPU race on the array: serialise them. */
int fomo_b200_run_shot_noalloc(int32_t nx, int32_t nz, int32_t M, int32_t pad,
                               int32_t free_surface, const float* rho_vx,
                               const float* rho_vz, const float* lam,
                               const float* mu_txx, const float* mu_txz,
                               int32_t pitch, const FomoHabc* habc,
                               const FomoShot* shot, float* gather_out,
                               void* stream);

/* ---------------------------------------------------------------------- */
/* Batched shots and the shot server                                       */
/* ---------------------------------------------------------------------- */

/* run_shots! (src/simulation/shot_manager.jl:145-180) with the shots run
 * side by side instead of one after another: every time-step launch covers
 * all shots in flight, shots of one medium share its tiles in L2, and the
 * time loop runs as CUDA graphs of K steps.  Each shot's gather is the same
 * as fomo_b200_run_shot's for that shot, bit for bit.  The shots share the
 * medium and HABC; their sources, receivers, wavelets and nt may differ
 * (M, dtx, dtz and the coefficients a as for fomo_b200_run_shot; dtx and dtz
 * equal across the shots).  gathers_out[s] is shot s's host gather
 * (nt_s * n_rec_s floats).  Shots are admitted while their wavefields fit in
 * 90% of free device memory, so any number of shots may be passed.  The call
 * blocks until every gather is on the host.  stats (may be NULL) covers the
 * whole batch: summed steps, device time, launches and bytes moved. */
int fomo_b200_run_batch(uint64_t medium, const FomoHabc* habc, const FomoShot* shots,
                        int32_t n_shots, float* const* gathers_out, FomoRunStats* stats);

/* The shot server: a request loop (no reference counterpart; it serves
 * run_shot! requests as they arrive).  A worker thread admits queued shots
 * in arrival order while their device memory (two wavefield copies, HABC
 * tables, receivers, wavelet, gather, and the buoyancy of a medium not yet
 * resident) fits the HBM budget and the shot limit, and runs every admitted
 * shot in the same launches, K steps at a time.  A shot joins the running
 * batch at the next K-step boundary and leaves it when its nt steps are
 * done; then its gather is copied back and its memory freed.  Shots overlap
 * on the device whatever their media, orders and nt, and each result equals
 * fomo_b200_run_shot's bit for bit. */
typedef struct {
    uint64_t hbm_budget_bytes;  /* device bytes for shots; 0 = 90% of free memory   */
    int32_t max_shots;          /* shots on the device at once; 0 = budget only      */
    int32_t steps_per_launch;   /* K; 0 = autotuned per (grid, order, batch size),   */
                                /* 1 = one launch per kernel per step, no graphs     */
} FomoServerConfig;

typedef struct {
    double queue_ms;            /* submit -> admitted                                */
    double run_ms;              /* admitted -> gather on the host                    */
    double latency_ms;          /* submit -> gather on the host                      */
    int32_t steps;              /* time steps run (nt)                               */
    int32_t batch_peak;         /* most shots on the device while this one ran       */
} FomoRequestStats;

typedef struct {
    int64_t submitted, completed, failed, cancelled;
    int64_t batch_steps;        /* time steps of the batch loop                      */
    int64_t kernel_launches;    /* kernels run (graph replays count their kernels)   */
    int64_t graph_replays;
    int64_t h2d_bytes, d2h_bytes;
    int32_t peak_shots;         /* most shots on the device at once                  */
    int32_t steps_per_launch;   /* K of the last chunk                               */
    uint64_t peak_bytes;        /* most budgeted device bytes held at once           */
} FomoServerStats;

int fomo_b200_server_create(const FomoServerConfig* config, uint64_t* server);
/* Queues one shot (thread-safe, any host thread).  medium must stay alive
 * until the request completes (fomo_b200_medium_destroy refuses a medium in
 * use).  gather_out (host, nt*n_rec floats) is written by the server and
 * must stay valid until wait reports the request done.  A shot that cannot
 * fit the budget even alone fails here with FOMO_ENOMEM. */
int fomo_b200_server_submit(uint64_t server, uint64_t medium, const FomoHabc* habc,
                            const FomoShot* shot, float* gather_out, uint64_t* ticket);
/* *done = 1 once the request has finished (then the return value is its
 * status), 0 while it is queued or running. */
int fomo_b200_server_poll(uint64_t server, uint64_t ticket, int32_t* done);
/* Waits up to timeout_s seconds (< 0: no limit).  Returns the request's
 * status and releases the ticket, or FOMO_ENOTREADY on timeout (the ticket
 * stays valid).  stats may be NULL. */
int fomo_b200_server_wait(uint64_t server, uint64_t ticket, double timeout_s,
                          FomoRequestStats* stats);
/* Cancels a request that is still queued (its wait returns FOMO_ECANCELLED);
 * a running request is not interrupted and FOMO_EINVAL is returned. */
int fomo_b200_server_cancel(uint64_t server, uint64_t ticket);
int fomo_b200_server_stats(uint64_t server, FomoServerStats* stats);
/* Cancels queued requests, lets running ones finish, stops the worker. */
int fomo_b200_server_destroy(uint64_t server);

#ifdef __cplusplus
}
#endif

#endif /* FOMO_B200_H */
