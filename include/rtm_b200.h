/*
 * rtm_b200.h -- C ABI of librtm_b200.so, the B200 (sm_100a) 2D acoustic RTM
 * engine.  This is the drop-in boundary: plain C types, caller-owned host
 * buffers, an opaque handle, int status codes, no C++ exceptions crossing it.
 *
 * Each entry point replaces one member of the reference's engine interface
 * (Marouane-Djabri/RTM-Acceleration, include/rtm_engine.hpp and
 * include/rtm_factory.hpp); the citation is given beside each declaration.  The
 * C++ class rtm_b200::B200RTM (include/rtm_b200_engine.hpp of this repository) wraps these
 * calls into the reference's RTMEngine interface and throws std::runtime_error
 * on a non-zero status, like the reference.
 *
 * Conventions (same as the reference, include/rtm_types.hpp:10-57):
 *   - grids are zfast: v[ix*nz + iz], image[ix*nz + iz];
 *   - traces are trace-major: traces[ir*nt + it];
 *   - positions are in metres in the velocity model's frame.
 * One handle is used by one host thread at a time.  All work runs on one GPU.
 */
#ifndef RTM_B200_H
#define RTM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RTM_B200_ABI_VERSION 1

#if defined(__GNUC__)
#define RTM_B200_API __attribute__((visibility("default")))
#else
#define RTM_B200_API
#endif

/* ---- status codes ------------------------------------------------------ */
#define RTM_B200_OK            0
#define RTM_B200_EINVAL       -1   /* bad argument / parameter validation     */
#define RTM_B200_ENOMEM       -2   /* device or host allocation failed        */
#define RTM_B200_ECUDA        -3   /* CUDA runtime/driver error               */
#define RTM_B200_ESTATE       -4   /* call out of order (e.g. migrate before set_model) */
#define RTM_B200_ETIMEOUT     -5   /* a bounded device-side wait gave up      */
#define RTM_B200_EUNSUPPORTED -6   /* valid request the engine cannot run     */
#define RTM_B200_EREJECTED    -7   /* serving: request rejected at admission  */
#define RTM_B200_ENOTFOUND    -8   /* serving: unknown ticket                 */

/* ---- engine modes (the engine names of make_engine) --------------------- */
#define RTM_B200_MODE_PLAIN 0  /* "b200":       one shot at a time            */
#define RTM_B200_MODE_BATCH 1  /* "b200-batch": many shots per launch          */
#define RTM_B200_MODE_SERVE 2  /* "b200-serve": continuous-batching server      */

/* ---- snapshot storage --------------------------------------------------- */
#define RTM_B200_SNAP_F32  0
#define RTM_B200_SNAP_BF16 1   /* power-of-two scale per 128-cell segment     */
#define RTM_B200_SNAP_F16  2
#define RTM_B200_SNAP_RECON 3  /* no snapshots (batch/serve, FP32): the forward
                                  pass stores the band of order/2 cells around
                                  the interior at every step, the backward pass
                                  rebuilds the source field in reverse time
                                  inside the interior (snapshot-free source
                                  reconstruction); about 2*order*(nx+nz)*nt*4
                                  bytes per shot instead of nt/si*nx*nz*s */

/* ---- arithmetic --------------------------------------------------------- */
#define RTM_B200_ARITH_IEEE 0  /* FP32, unfused, reference operation order:
                                  bit-identical to the reference CPU engine   */
#define RTM_B200_ARITH_FMA  1  /* FP32 with fused multiply-adds               */
#define RTM_B200_ARITH_FP64 2  /* FP64 propagation/imaging: the FP64 run      */
#define RTM_B200_ARITH_AUTO 3  /* IEEE for the plain engine (bit-identical to
                                  the reference), FMA for batch and serve
                                  (their sums are compensated, not bitwise)  */

/* ---- accumulation of the per-shot image (batch/serve modes) ------------- */
#define RTM_B200_ACC_PLAIN        0  /* running FP32 image, reference order    */
#define RTM_B200_ACC_COMPENSATED  1  /* Kahan FP32 per shot (BF16 compensation
                                        words) + FP64 stack                   */

typedef struct rtm_b200_engine rtm_b200_engine;

/* Engine configuration.  Zero-initialise, set struct_size = sizeof, then the
 * fields you need; rtm_b200_config_init() fills the reference defaults. */
typedef struct {
    int   struct_size;
    int   mode;             /* RTM_B200_MODE_*                                 */
    int   device;           /* CUDA device ordinal                             */
    /* RTMParams (reference include/rtm_types.hpp:33-40)                        */
    int   nb;               /* sponge width, default 60                        */
    int   order;            /* FD order 2..12, default 8                       */
    float sponge_alpha;     /* default 0.0053                                  */
    int   store_interval;   /* default 1                                       */
    float f0;               /* Ricker peak frequency, default 12               */
    int   verbose;
    /* B200 engine choices                                                      */
    int   snap_precision;   /* RTM_B200_SNAP_*                                 */
    int   arithmetic;       /* RTM_B200_ARITH_*                                */
    int   accumulation;     /* RTM_B200_ACC_* (plain mode always ACC_PLAIN)    */
    int   max_shots_in_flight; /* batch/serve: 0 = 32 (batch: fewer if short) */
    long long device_mem_budget; /* bytes the engine may hold; 0 = 90% of free */
    int   tile_cols;        /* 0 = autotune; else 16 or 32 columns per tile    */
    int   chunk_steps;      /* time steps per captured CUDA graph, 0 = auto    */
    int   serve_max_nx;     /* serve: largest interior grid a request may use;  */
    int   serve_max_nz;     /*        0 = size the pool from the first requests */
} rtm_b200_config;

/* One shot gather (reference ShotRecord, include/rtm_types.hpp:49-57). */
typedef struct {
    float        sx, sz;      /* source position, metres                       */
    int          nrec;
    int          nt;          /* samples per trace (stride of traces)          */
    float        dt;          /* seconds                                       */
    const float* rx;          /* nrec                                          */
    const float* rz;          /* nrec                                          */
    const float* traces;      /* nrec*nt trace-major, or NULL for modelling    */
    /* Aperture window: migrate this shot on model columns [window_x0,
     * window_x0 + window_nx) only, exactly as the reference would migrate it on
     * the cropped model (edge-replicated padding of the window), and add its
     * image into those columns of the full image.  0,0 = whole model. */
    int          window_x0;
    int          window_nx;
} rtm_b200_shot;

/* Timings of the last call(s), seconds (reference StageTimes,
 * include/rtm_engine.hpp:8-13).  kernel = device time measured with CUDA
 * events around the propagation. */
typedef struct {
    double io, forward, backward, imaging, total, h2d, kernel, d2h;
    double cell_updates;      /* 2*nt*N_ext per migrated shot, summed          */
    double algorithmic_bytes; /* bytes the roofline counts, summed             */
    double h2d_bytes;         /* host->device bytes the engine copied          */
    double d2h_bytes;         /* device->host bytes the engine copied          */
    int    kernel_launches;   /* launches of this library's kernels            */
    int    shots;
} rtm_b200_times;

/* Serving request: its own model, parameters and shots. */
typedef struct {
    const float*         vel;      /* nx*nz zfast                              */
    int                  nx, nz;
    float                dx, dz, ox, oz;
    int                  order;
    float                f0;
    int                  nt;       /* time samples to propagate                */
    float                dt;
    int                  store_interval;
    int                  nshots;
    const rtm_b200_shot* shots;    /* borrowed until the request completes     */
    double               arrival_time; /* caller's clock, seconds (for stats)  */
} rtm_b200_request;

typedef struct {
    int    state;              /* 0 queued, 1 running, 2 done, -1 failed        */
    int    shots_done;
    double submit_time, start_time, finish_time;   /* engine clock, seconds     */
    double snapshot_bytes;     /* device snapshot footprint per shot            */
} rtm_b200_request_status;

/* Fill the reference defaults (nb 60, order 8, alpha 0.0053, store 1, f0 12)
 * and arithmetic RTM_B200_ARITH_AUTO. */
RTM_B200_API void rtm_b200_config_init(rtm_b200_config* cfg);

/* Create an engine (reference make_engine, include/rtm_factory.hpp:19-20 and
 * src/rtm/factory.cpp:17-38).  Selects the CUDA device; fails with ECUDA when
 * no usable sm_100 device is present -- there is no CPU fallback. */
RTM_B200_API int rtm_b200_create(const rtm_b200_config* cfg, rtm_b200_engine** out);

/* Release every device and host resource (reference ~CUDARTM,
 * src/cuda/rtm_cuda.cu:124-138). */
RTM_B200_API int rtm_b200_destroy(rtm_b200_engine* h);

/* Build the device tables for one model and time axis (reference
 * RTMEngine::setup, include/rtm_engine.hpp:27-29; tables as in
 * src/rtm/rtm_cpu.cpp:9-88).  Validates nb >= order/2+1, store_interval >= 1,
 * sizes, and the velocity range (0, 20000] of the reference reader. */
RTM_B200_API int rtm_b200_setup(rtm_b200_engine* h, const float* vel, int nx, int nz, float dx, float dz,
                   float ox, float oz, int nt, float dt);

/* Full migration (reference RTMEngine::migrate, include/rtm_engine.hpp:50-54,
 * src/rtm/rtm.cpp:83-103): image and illum (nx*nz, caller-owned) are
 * OVERWRITTEN with the zero-lag image and source illumination of all shots.
 * Shot traces and the image/illum buffers may be host memory (pageable or
 * page-locked) or device memory of the engine's GPU: device-resident inputs are
 * read in place, page-locked ones are DMA'd without a staging copy. */
RTM_B200_API int rtm_b200_migrate(rtm_b200_engine* h, const rtm_b200_shot* shots, int nshots, float* image,
                     float* illum);

/* As rtm_b200_migrate, returning the FP64 cross-shot stack itself. */
RTM_B200_API int rtm_b200_migrate_f64(rtm_b200_engine* h, const rtm_b200_shot* shots, int nshots, double* image,
                         double* illum);

/* Forward modelling (reference RTMEngine::model_shot, src/rtm/rtm.cpp:105-111):
 * writes nrec*nt trace-major samples of every shot into traces_out, shot after
 * shot (sum of nrec_i*nt floats). */
RTM_B200_API int rtm_b200_model_shots(rtm_b200_engine* h, const rtm_b200_shot* shots, int nshots,
                         float* traces_out);

/* Post-processing of the stack the last rtm_b200_migrate / _migrate_f64 left on
 * the device, computed on the device: the reference's
 * illumination_compensation (I / (S + eps_relative * max S + 1e-30)) and
 * laplacian_filter (second differences over dx^2 and dz^2 on the interior,
 * zero on the outermost rows and columns), src/rtm/imaging.cpp:48-75, as its
 * CLI applies them at src/main.cpp:211-223.  illum_out (nx*nz, may be NULL)
 * receives the compensated image (the `_illum` output); filtered_out (may be
 * NULL) receives the filtered image (the `_filtered` output), filtered after
 * compensation when compensate_filtered is non-zero.  The plain engine works on
 * its FP32 image with the reference's float operations (bit-identical to the
 * reference's outputs); batch and serve work on the FP64 stack and round once at
 * the end.  Buffers may be host or device memory of the engine's GPU.  ESTATE
 * before any migration. */
RTM_B200_API int rtm_b200_postprocess(rtm_b200_engine* h, float eps_relative, int compensate_filtered,
                                      float* illum_out, float* filtered_out);

/* Source propagation of one shot (reference forward_propagation,
 * include/rtm_engine.hpp:31-37).  snapshots (num_snapshots*nx*nz floats) and
 * recorded (nrec*nt) may each be NULL. */
RTM_B200_API int rtm_b200_forward(rtm_b200_engine* h, const rtm_b200_shot* shot, float* snapshots,
                     float* recorded);

/* Receiver propagation with imaging of one shot (reference
 * backward_propagation, include/rtm_engine.hpp:39-43).  If snapshots is NULL the
 * device-resident snapshots of the last rtm_b200_forward are used.  image and
 * illum (nx*nz) are ACCUMULATED into (+=), like the reference. */
RTM_B200_API int rtm_b200_backward(rtm_b200_engine* h, const rtm_b200_shot* shot, const float* snapshots,
                      float* image, float* illum);

/* Zero-lag imaging of one time step (reference RTMEngine::imaging,
 * include/rtm_engine.hpp:45-48, src/rtm/imaging.cpp:25-40): fwd_snapshot is
 * nx*nz, bwd_extended is (nx+2nb)*(nz+2nb); image/illum accumulate. */
RTM_B200_API int rtm_b200_imaging(rtm_b200_engine* h, const float* fwd_snapshot, const float* bwd_extended,
                     float* image, float* illum);

/* Grid and snapshot accounting (reference RTMEngine accessors,
 * include/rtm_engine.hpp:60-66). */
RTM_B200_API int rtm_b200_num_snapshots(const rtm_b200_engine* h);
RTM_B200_API long long rtm_b200_snapshot_bytes(const rtm_b200_engine* h);

/* Stage timings accumulated since the last reset (reference
 * RTMEngine::times, include/rtm_engine.hpp:75). */
RTM_B200_API int rtm_b200_get_times(const rtm_b200_engine* h, rtm_b200_times* out);
RTM_B200_API int rtm_b200_reset_times(rtm_b200_engine* h);

/* Device identity (reference device_name(), include/rtm_engine.hpp:70-73). */
RTM_B200_API int rtm_b200_device_name(const rtm_b200_engine* h, char* buf, size_t len);

/* What the autotuner measured and chose, as JSON text: one record per job mix
 * (stencil half-orders, tile rows, shots in flight), with the time per step of
 * every candidate (columns per consumer warp, pipeline stages) and the pick.
 * The reference has no autotuner; this reports the engine's own choices. */
RTM_B200_API int rtm_b200_autotune_report(const rtm_b200_engine* h, char* buf, size_t len);

/* Text of the last error on this handle (or of the last failed create when h
 * is NULL). */
RTM_B200_API int rtm_b200_last_error(const rtm_b200_engine* h, char* buf, size_t len);

/* ---- host-side numerics (no GPU needed) --------------------------------- */

/* Taylor second-derivative weights c[0..order/2] (reference
 * stencil_coefficients, include/rtm_types.hpp:60, src/rtm/rtm.cpp:14-36).
 * Returns order/2, or EINVAL for an unsupported order. */
RTM_B200_API int rtm_b200_stencil_coefficients(int order, float* c);

/* CFL limit (reference max_stable_dt, include/rtm_types.hpp:64,
 * src/rtm/rtm.cpp:59-62). */
RTM_B200_API float rtm_b200_max_stable_dt(float vmax, float dx, float dz, int order);

/* Ricker sample (reference ricker, include/rtm_types.hpp:63, rtm.cpp:52-55). */
RTM_B200_API float rtm_b200_ricker(float t, float f0);

/* Points per shortest wavelength (reference points_per_wavelength,
 * include/rtm_types.hpp:65, rtm.cpp:66-70). */
RTM_B200_API float rtm_b200_points_per_wavelength(float vmin, float f0, float dx, float dz);

/* Direct-arrival mute of one shot's traces in place (reference
 * mute_direct_wave, include/rtm_io.hpp:9, src/io/seismic_io.cpp:18-35).
 * shot->traces is ignored; `traces` (nrec*nt) is modified. */
RTM_B200_API void rtm_b200_mute_direct_wave(const rtm_b200_shot* shot, float* traces, float v_surface,
                                            float t_pad, float t_taper);

/* Copy-bandwidth probe on the engine's GPU (reference bandwidth probe,
 * src/tools/bandwidth_probe_cuda.cu): copies bytes/2 to bytes/2, `iters` times,
 * and reports read+write bytes per second.  A buffer well under the 126 MB L2
 * measures L2 bandwidth, one of several GB measures HBM. */
RTM_B200_API int rtm_b200_memory_probe(rtm_b200_engine* h, size_t bytes, int iters, double* gbps);

/* L2 read bandwidth on the engine's GPU: a buffer of `bytes` (small enough to
 * stay in the 126 MB L2, e.g. 24 MB) read `reps` times per launch through L2,
 * bypassing L1.  The roofline peak for work whose fields stay in L2.  The
 * reference has no L2 probe; its rtm_bandwidth_probe measures DRAM. */
RTM_B200_API int rtm_b200_l2_probe(rtm_b200_engine* h, size_t bytes, int reps, double* gbps);

/* ---- modelling without any GPU allocation ------------------------------- */

/* One shot's model, parameters and device for rtm_b200_model_shot_static. */
typedef struct {
    const float* vel;           /* nx*nz zfast, host memory                      */
    int          nx, nz;
    float        dx, dz, ox, oz;
    int          nb, order;
    float        sponge_alpha, f0;
    int          nt;
    float        dt;
    int          device;        /* CUDA device ordinal                          */
} rtm_b200_static_problem;

/* Forward modelling of one shot (the same kernel and results as
 * rtm_b200_model_shots) that allocates no GPU memory at all.  This entry point
 * has no counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc: plugins whose host application owns every byte of device memory
 * through its own pool and forbids allocations behind its back, and loops that
 * cannot afford the device-wide synchronisation that cudaMalloc/cudaFree imply.
 * The call is synchronous: it copies its tables in, runs, and waits for its own
 * work before it returns.  Its scratch (wavefields, tables, receiver lists)
 * lives in a fixed 32 MiB array inside the library's device image, which every
 * GPU that loads the library holds until the process exits; problems whose
 * scratch exceeds it (roughly more than 2.6 million extended cells) are
 * rejected with EINVAL and a message in `err`.  traces_out (nrec*nt,
 * trace-major) may be host memory or device memory of `problem->device`;
 * device memory of another GPU is rejected with EINVAL.  The first call on a
 * device looks up the array's device address, so make that first call before
 * any stream capture.  Calls share the array and find the previous call's
 * contents in it; calls that overlapped on the GPU would race on it, so this
 * function takes a per-device lock and returns only after its work is done,
 * and calls from one process never overlap.  Returns a status code; err (may be
 * NULL) receives a message. */
RTM_B200_API int rtm_b200_model_shot_static(const rtm_b200_static_problem* problem, const rtm_b200_shot* shot,
                                            float* traces_out, char* err, size_t err_len);

/* ---- serving (no reference counterpart: the continuous-batching loop) ---- */

/* Queue a request; returns a ticket.  Rejected (EREJECTED) when it can never
 * fit the device budget or fails validation (CFL, sizes, order). */
RTM_B200_API int rtm_b200_submit(rtm_b200_engine* h, const rtm_b200_request* req, long long* ticket);

/* Advance the serving loop: admit queued requests as slots and memory free up,
 * run up to max_steps time steps of every shot in flight, retire finished
 * shots.  Returns the number of requests still queued or running. */
RTM_B200_API int rtm_b200_serve_step(rtm_b200_engine* h, int max_steps, int* pending);

/* Status of a request; when done, copies its image and illumination (nx*nz)
 * into the caller's buffers (either may be NULL). */
RTM_B200_API int rtm_b200_poll(rtm_b200_engine* h, long long ticket, rtm_b200_request_status* st, float* image,
                  float* illum);

/* Run the serving loop until every submitted request is done. */
RTM_B200_API int rtm_b200_drain(rtm_b200_engine* h);

/* Engine clock (seconds since create), the clock of rtm_b200_request_status. */
RTM_B200_API double rtm_b200_clock(const rtm_b200_engine* h);

#ifdef __cplusplus
}
#endif
#endif /* RTM_B200_H */
