/* fslbm.h -- C ABI of the B200 fractional-step lattice Boltzmann (FSLBM) pipe solver.
 *
 * The reference (alparmat/FlowContrast) has no library API: its drop-in surface is the
 * executable PipeDemoStandalone/FSLBM.cu plus the files it reads and writes in the working
 * directory. Each entry point below names the reference code it replaces (file:line in
 * PipeDemoStandalone/FSLBM.cu or pipe.m). The drop-in executable `fslbm_pipe` and the Python
 * package are both built on this ABI.
 *
 * Conventions
 *  - Every function returns 0 (FSLBM_OK) or a negative FSLBM_ERR_* code; the message of the last
 *    error on the calling thread is read with fslbm_last_error().
 *  - Axes follow the reference: x and y span the pipe cross-section (x fastest in memory), z is
 *    streamwise (slowest). Host arrays are dense lx*ly*lz, index x + lx*(y + ly*z).
 *  - p is the density deviation (rho - 1) of the incompressible He-Luo equilibrium; u, v, w are
 *    the stored velocity components, which are the NEGATED physical velocity (FSLBM.cu:137-173
 *    pulls f at x+c and accumulates +c). Dumps keep this sign, as the reference's viewers expect.
 *  - Threading: a context and its solves may be used from one host thread at a time. The
 *    server (fslbm_server_*) runs its own worker thread and its calls are thread-safe.
 */
#ifndef FSLBM_H
#define FSLBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FSLBM_OK 0
#define FSLBM_ERR_ARG (-1)      /* invalid argument, size or geometry */
#define FSLBM_ERR_CUDA (-2)     /* a CUDA call failed */
#define FSLBM_ERR_STATE (-3)    /* call out of order (e.g. no fields set) */
#define FSLBM_ERR_IO (-4)       /* file missing, truncated or malformed */
#define FSLBM_ERR_DIVERGED (-5) /* non-finite values found by the divergence check */
#define FSLBM_ERR_TIMEOUT (-6)  /* a bounded device-side wait gave up */
#define FSLBM_ERR_BUDGET (-7)   /* request larger than the server's memory budget */
#define FSLBM_ERR_NOTFOUND (-8) /* unknown request id */

typedef enum {
  FSLBM_F64 = 0, /* FP64 storage and arithmetic */
  FSLBM_F32 = 1, /* FP32 storage and arithmetic (the reference's precision) */
  FSLBM_F16 = 2  /* mixed: FP16 storage of scaled deviations, FP32 arithmetic */
} fslbm_dtype;

typedef struct fslbm_ctx fslbm_ctx;
typedef struct fslbm_solve fslbm_solve;
typedef struct fslbm_batch fslbm_batch;
typedef struct fslbm_server fslbm_server;

/* Periodic pipe domain. Replaces the hard-coded dims of FSLBM.cu:512-514 and the mask read of
 * FSLBM.cu:478-485. The streamwise direction is periodic with a pressure jump `pin` across the
 * seam, which is what the reference's buffer planes and bcond copies implement
 * (FSLBM.cu:291-301); lz counts the fluid planes only (the reference's lz - 2*d2). */
typedef struct {
  int lx, ly;            /* cross-section size in cells */
  int lz;                /* streamwise period in cells */
  const uint8_t* mask;   /* lx*ly cross-section: 0 fluid, 125 wall; NULL selects the circle */
  double radius;         /* circle radius; also the r of the friction factor and Re (FSLBM.cu:650,660) */
  double cx, cy;         /* circle centre: fluid iff (x-cx)^2 + (y-cy)^2 <= radius^2 */
  int buffer_depth;      /* d2 of the reference layout used by plane dumps and statistics */
  int mask_planes;       /* 0 or 1: `mask` is one cross-section extruded along z; lz: `mask`
                            holds lx*ly*lz values, one cross-section per plane (geometry that
                            varies along the pipe, such as wall roughness; run on the one-column
                            kernel, FP32/FP64). The monitor's l1, the reference's buffer-cell
                            count over 2*d2 planes (FSLBM.cu:589-591), is then the mean fluid
                            count of the buffer_depth planes at each end of the core. */
  int periodic_xy;       /* addition: G > 0 makes the cross-section periodic in x and y with
                            period (lx - 2G, ly - 2G): a G-wide band at the box rim holds the
                            periodic images of the interior (mask value 2; refilled after every
                            step, never stepped, not counted by monitors). G >= K*d1, one
                            cross-section only. A given mask's band values are replaced; without
                            a mask the interior is all fluid (e.g. a Taylor-Green vortex). */
} fslbm_domain;

/* Run parameters: the six lines of param.txt (FSLBM.cu:502-507) plus additions. */
typedef struct {
  double tblend;        /* time-step blend b (FSLBM.cu:269) */
  double pin;           /* pressure jump across the periodic seam (FSLBM.cu:296,300) */
  double nu;            /* target viscosity; dtddy = nu - 0.16666666 (FSLBM.cu:599) */
  int d1;               /* coarse corrective stride (FSLBM.cu:243-253); 1..3 */
  int delta;            /* statistics reset policy (FSLBM.cu:683-690) */
  double blend;         /* corrector order blend, 0: order 2, 1: order 4 (FSLBM.cu:231) */
  int monitor_every;    /* monitor + pressure gauge period; 50 in the reference (FSLBM.cu:630) */
  double force[3];      /* addition: body force per step on (u,v,w), stored-velocity sign */
  int fd_order;         /* corrector order (FSLBM.cu:177-232): 0 or 4 = the reference's active
                           4<->2 blend; 6 = 6<->4 and 8 = 8<->6 blends (blend weights the higher
                           order; the paper's pipes used 6 with blend 0.4); 10, 12, 14 = fixed
                           sets (blend unused). Orders above 4 reach K*d1 cells (K = 3, 4, 5, 6,
                           8) and run on the one-column kernel: FP32 with K*d1 <= 8, FP64 with
                           K*d1 <= 4; FP16 storage supports orders 0/4 only. Not in param.txt. */
} fslbm_params;

/* One monitor record (FSLBM.cu:632-666): means over the first fluid plane (q1, p1) and over the
 * first outlet buffer plane (q2, p2) per fluid cell, friction factor f, the w sample at the box
 * centre and Re = 2 r q1 / nu. Reductions are FP64. */
typedef struct {
  int64_t step;
  double q1, q2, p1, p2, f, sample, re;
} fslbm_monitor;

typedef struct {
  int64_t cells;         /* lx*ly*lz */
  int64_t fluid_cells;   /* non-wall cells */
  int64_t bytes_device;  /* device memory held by the solve */
  int64_t steps;         /* steps advanced so far */
  int lx_pitch;          /* padded row length in device memory */
  int dtype;
  double last_step_ms;   /* device time of the last fslbm_solve_step call */
  int64_t kernel_launches; /* kernels this solve has launched (steps, monitors, statistics) */
} fslbm_info;

/* ---- errors and version ---- */
const char* fslbm_version(void);
/* Copies the calling thread's last error message into buf; returns its code. */
int fslbm_last_error(char* buf, size_t n);

/* ---- context: one device, one stream (replaces cudaSetDevice(0), FSLBM.cu:490) ---- */
int fslbm_ctx_create(int device, fslbm_ctx** out);
/* Drops the creator's reference. Each solve and batch holds its own, so the stream and memory
   pool are released when the last of the context, its solves and its batches is destroyed
   (any order is safe). */
int fslbm_ctx_destroy(fslbm_ctx* ctx);
/* Self-test of the device-side bounded waits the kernels use (no reference counterpart): a
   gpu-scope counter wait and an mbarrier phase wait, each on a condition nothing satisfies, with
   a limit of limit_ms (0 < limit_ms <= 10000). Both give up and return; *gave_up gets one bit
   per wait (3 = both) and the call returns FSLBM_ERR_TIMEOUT, the code a kernel's gave-up wait
   produces. The context stays usable. */
int fslbm_selftest_waits(fslbm_ctx* ctx, double limit_ms, unsigned* gave_up);

/* ---- solve (replaces main's set-up and time loop, FSLBM.cu:489-905) ---- */
int fslbm_solve_create(fslbm_ctx* ctx, const fslbm_domain* dom, const fslbm_params* prm,
                       fslbm_dtype dtype, fslbm_solve** out);
int fslbm_solve_destroy(fslbm_solve* s);
/* Live parameter update, as the reference's re-read of param.txt every 500 steps
 * (FSLBM.cu:669-677). d1 may change only to another supported stride. */
int fslbm_solve_set_params(fslbm_solve* s, const fslbm_params* prm);
/* Host fields in, lx*ly*lz each, FP64 (host_dtype FSLBM_F64) or FP32 (FSLBM_F32). Wall cells
 * are set to zero, the invariant the reference's bcond restores every step (FSLBM.cu:290).
 * Replaces the restart loader initphys1 (FSLBM.cu:386-418). */
int fslbm_solve_set_fields(fslbm_solve* s, fslbm_dtype host_dtype, const void* p, const void* u,
                           const void* v, const void* w);
int fslbm_solve_get_fields(fslbm_solve* s, fslbm_dtype host_dtype, void* p, void* u, void* v,
                           void* w);
/* Advances nsteps time steps, asynchronously on the context's stream. Each step is one fused
 * kernel (predictor, corrector, periodic pressure-jump and wall boundaries, gauge). Every
 * monitor_every steps a monitor record is produced on the device and its p2 gauges the next
 * step (FSLBM.cu:628, 637-647). Replaces FSLBM.cu:620-628 (about 350 launches per step). */
int fslbm_solve_step(fslbm_solve* s, int64_t nsteps);
int fslbm_solve_sync(fslbm_solve* s);
/* Latest monitor record (synchronises). Returns FSLBM_ERR_STATE if none exists yet. */
int fslbm_solve_monitor(fslbm_solve* s, fslbm_monitor* out);
/* Drains up to `max` monitor records produced since the last drain, oldest first. */
int fslbm_solve_monitor_log(fslbm_solve* s, fslbm_monitor* out, int max, int* n_out);
/* Non-finite scan of the current fields (FP64 reduction); FSLBM_ERR_DIVERGED if any. */
int fslbm_solve_check(fslbm_solve* s, double* max_abs_u);
int fslbm_solve_info(fslbm_solve* s, fslbm_info* out);
/* Per-launch device timing of the step kernel: with enable != 0 every step launch is
 * bracketed by CUDA events on the launching stream. fslbm_solve_kernel_time synchronises and
 * returns the summed step-kernel time and launch count since the previous call. */
int fslbm_solve_set_timing(fslbm_solve* s, int enable);
int fslbm_solve_kernel_time(fslbm_solve* s, double* ms_total, int64_t* launches);
/* Device pointers of the current state (p, u, v, w in the solve's storage type, row pitch
 * info.lx_pitch). Valid until the next step, set_fields or destroy. */
int fslbm_solve_device_fields(fslbm_solve* s, void** p, void** u, void** v, void** w);
/* The seeded start of fslbm_init_poiseuille generated on the device into the solve's state
 * (no host arrays, no copies); asynchronous on the context's stream. modes <= 16. */
int fslbm_solve_init_poiseuille(fslbm_solve* s, double umax, double noise, int modes,
                                double mode_amp, uint64_t seed);
/* Corrector coefficients c0..c8 of an order and blend as the solve of `dtype` uses them (FP32
 * forms for FP32 and FP16 storage); *taps = K. FSLBM_ERR_ARG for an unknown order. */
int fslbm_fd_coefficients(int order, double blend, fslbm_dtype dtype, double* c, int* taps);
/* Device bytes fslbm_solve_create allocates for a domain and dtype (an upper bound). Copying
 * host-layout fields in or out later adds a staging buffer of 4 fields in the host type when the
 * storage type differs from the host type or lx is not a multiple of 8. */
int fslbm_solve_footprint(const fslbm_domain* dom, fslbm_dtype dtype, int64_t* bytes);

/* ---- reference-layout fields: the core plus d2 buffer planes at each streamwise end,
 *      reconstructed as the bcond copies with the +-pin jump (FSLBM.cu:291-301) ---- */
/* Host arrays lx*ly*(lz+2*d2) FP32, the reference's restart layout (p3Dii etc., FSLBM.cu:830-856). */
int fslbm_solve_get_fields_ref(fslbm_solve* s, float* p, float* u, float* v, float* w);
/* Loads reference-layout fields, keeping planes d2..d2+lz-1 (FSLBM.cu:386-418). */
int fslbm_solve_set_fields_ref(fslbm_solve* s, const float* p, const float* u, const float* v,
                               const float* w);
/* One plane of the reference layout. kind 0: YZ plane x=lx/2, values y + ly*z_ref
 * (FSLBM.cu:315-324, 784-798); kind 1: XY plane z_ref = lz_ref/2, values x + lx*y
 * (FSLBM.cu:327-336, 800-814). comp 0..3 = p,u,v,w. */
int fslbm_solve_get_plane(fslbm_solve* s, int kind, int comp, float* out);

/* ---- statistics ---- */
/* Reference plane statistics (FSLBM.cu:683-768) on the YZ plane x=lx/2 of the reference layout,
 * accumulated on the device in FP64 with compensated (Neumaier) sums, so long runs of samples
 * lose no precision to rounding. fslbm_stats_sample applies the `delta` reset policy of the
 * current parameters, then adds one sample (cnt and cnt2 are incremented first, as in the
 * reference). The "RMS" sums are of |deviation|, as the reference's abs() of a double. Outputs are 11 arrays of ly*(lz+2*d2) doubles in the order
 * _p,_ux,_uy,_uz (sums / cnt), _p2,_ux2,_uy2,_uz2,_uxy2,_uxz2,_uyz2 (sums / cnt2). */
int fslbm_stats_sample(fslbm_solve* s);
int fslbm_stats_get(fslbm_solve* s, double* out, int* cnt, int* cnt2);
/* Restores averaged statistics (the `_*ii.txt` / `_avii.txt` restart, FSLBM.cu:429-468):
 * the means are multiplied back by their counts. */
int fslbm_stats_set(fslbm_solve* s, const double* means, int cnt, int cnt2);
/* Full-volume profile statistics (addition): per cross-section cell, FP64 sums over z and over
 * samples of p,u,v,w,uu,vv,ww,uv,uw,vw (10 arrays of lx*ly); samples are added with
 * compensated sums in a fixed order, so the result does not depend on scheduling. */
int fslbm_profile_sample(fslbm_solve* s);
int fslbm_profile_get(fslbm_solve* s, double* sums, int64_t* nsamples);
int fslbm_profile_reset(fslbm_solve* s);

/* ---- batched ensemble: many solves advanced together by persistent launches ---- */
int fslbm_batch_create(fslbm_ctx* ctx, fslbm_solve* const* solves, int n, fslbm_batch** out);
int fslbm_batch_destroy(fslbm_batch* b);
/* Advances every member nsteps steps, asynchronously. When every member is FP32 or FP16 storage
 * with d1 = 2, up to 16 time steps of the whole ensemble (FSLBM_BATCH_CHAIN) run in one
 * persistent launch over all members' (tile, chunk) work items, each member's next step
 * starting as soon as its previous step is complete (step counters, monitors and gauges are
 * kept inside the launch); with use_graph each such launch is replayed from a captured CUDA
 * graph. Other members step one after another. */
int fslbm_batch_step(fslbm_batch* b, int64_t nsteps, int use_graph);
int fslbm_batch_sync(fslbm_batch* b);
/* Device time of the last fslbm_batch_step call (valid after fslbm_batch_sync). */
int fslbm_batch_elapsed(fslbm_batch* b, double* ms);
/* Member `member` (index in the create call) is not stepped once its step count reaches
 * stop_step (absolute; -1 = no stop), so members with different step budgets share launches;
 * the others keep stepping. */
int fslbm_batch_set_stop(fslbm_batch* b, int member, int64_t stop_step);
/* Batch tiling (no reference counterpart). A member's work items span `chunk` streamwise planes
 * (each chunk re-reads 2*2*d1 halo planes) and use warps of 32 x 2 cells (warp_shape = 0),
 * 16 x 4 cells (1) or 8 x 8 cells (2); warps whose cells are all wall skip the arithmetic, so
 * the smaller shapes suit small cross-sections. Members fall in size classes (32-wide tiles
 * across x and y, length rounded up to a power of two); a batch takes its classes' tiling from
 * the table named by the FSLBM_BATCH_TUNING environment variable, else from batch_tiling.json
 * next to the library, else 128 planes and 16 x 4 warps. The batch marches its own 32 x 16
 * column tiles (two CTAs per SM; FSLBM_BATCH_TILE_Y=32 selects 32 x 32 tiles), independent of
 * the tiling each member uses when stepped alone. */
int fslbm_batch_set_tiling(fslbm_batch* b, int member, int chunk, int warp_shape);
int fslbm_batch_load_tiling(fslbm_batch* b, const char* path);
/* Autotuner: times each size class's candidate tilings (chunks 16..256, the three warp shapes) on the
 * batch itself, trial_steps steps per candidate, keeps the fastest per class, restores every
 * member's fields, step count, monitor log and gauge, and writes the table to `path` (JSON) if
 * not NULL. Needs members on the batched kernel (FP32 or FP16 storage, d1 = 2). If a member's
 * state cannot be restored (a CUDA error), the call fails and that member refuses to step
 * (FSLBM_ERR_STATE) until its fields are set again. */
int fslbm_batch_autotune(fslbm_batch* b, int trial_steps, const char* path);

/* ---- served solves: a request loop with continuous batching (no reference counterpart) ----
 * The server owns a context on `device` and a worker thread. Requests are admitted in arrival
 * order while their device footprint fits the HBM budget (and the resident count its limit);
 * their state stays on the device until they finish. Every round the worker advances the
 * round's solves together (batched launches per storage type) for min(quantum, most steps left
 * among them) steps, each stopping at its own step count; requests that arrive meanwhile join
 * at the next round, finished ones leave and free their memory. Which resident solves a round
 * advances is the policy: all of them (FSLBM_SERVE_ALL, the default), or those with the least
 * work left (box cells x steps left) up to round_cells box cells (FSLBM_SERVE_LEAST_WORK: short
 * requests overtake long ones, which lowers the median latency for the same total work). A
 * solve's result does not depend on what else shares its rounds (the step is bitwise
 * independent of the batch it runs in). */
enum { FSLBM_SERVE_ALL = 0, FSLBM_SERVE_LEAST_WORK = 1 };
typedef struct {
  int64_t hbm_budget;  /* bytes of solve state the server may hold; 0 = 150e9 */
  int max_resident;    /* 0 = no limit */
  int quantum;         /* steps per round; 0 = 50 */
  int policy;          /* FSLBM_SERVE_*; 0 = FSLBM_SERVE_ALL */
  int64_t round_cells; /* FSLBM_SERVE_LEAST_WORK: box cells per round (at least one request);
                          0 = 48 Mi */
} fslbm_server_config;

typedef struct {
  double umax, noise;  /* see fslbm_init_poiseuille */
  int modes;
  double mode_amp;
  uint64_t seed;
} fslbm_init_spec;

typedef struct {
  fslbm_domain domain;     /* the mask, if any, is copied at submit */
  fslbm_params params;
  int dtype;               /* fslbm_dtype */
  int64_t nsteps;
  const float* init[4];    /* host FP32 initial p,u,v,w (lx*ly*lz, copied at submit), or all NULL */
  fslbm_init_spec init_spec; /* the device-generated start used when init[0] is NULL */
  float* out[4];           /* host FP32 buffers for the final fields, or all NULL; must stay
                              valid until the request is done */
} fslbm_request;

enum { FSLBM_REQ_QUEUED = 0, FSLBM_REQ_RUNNING = 1, FSLBM_REQ_DONE = 2, FSLBM_REQ_FAILED = 3 };

typedef struct {
  int status;              /* FSLBM_REQ_* */
  int error;               /* FSLBM_ERR_* of a failed request */
  int64_t steps_done;
  double t_submit, t_admit, t_done;  /* seconds since the server started (host clock) */
  int64_t bytes_device;    /* footprint charged against the budget */
  int64_t cells;           /* lx*ly*lz */
  fslbm_monitor last;      /* latest monitor record (step 0 if none) */
} fslbm_result;

typedef struct {
  int64_t submitted, completed, failed, queued, resident;
  int64_t bytes_resident, bytes_peak;
  int64_t rounds;
  double cell_steps;       /* box cells x steps of the completed requests */
  double busy_seconds;     /* wall time from each round's launch to its completion */
  /* worker time by activity (seconds): creating admitted solves, rebuilding the batches,
   * launching rounds, waiting for rounds, handing back finished requests */
  double t_admit, t_regroup, t_launch, t_wait, t_retire;
} fslbm_server_stats;

int fslbm_server_create(int device, const fslbm_server_config* cfg, fslbm_server** out);
/* Stops the worker after the current round; unfinished requests are dropped. */
int fslbm_server_destroy(fslbm_server* srv);
/* Queues a request. FSLBM_ERR_BUDGET if it could never fit the budget, FSLBM_ERR_ARG for a
 * domain or parameter set that fslbm_solve_create would reject. */
int fslbm_server_submit(fslbm_server* srv, const fslbm_request* req, int64_t* id);
int fslbm_server_poll(fslbm_server* srv, int64_t id, fslbm_result* out);
/* Waits until the request is done or failed, at most timeout_s seconds (FSLBM_ERR_TIMEOUT). */
int fslbm_server_wait(fslbm_server* srv, int64_t id, double timeout_s, fslbm_result* out);
/* Waits until every submitted request is done or failed. */
int fslbm_server_drain(fslbm_server* srv, double timeout_s);
/* Forgets a finished request (its result can no longer be polled). */
int fslbm_server_release(fslbm_server* srv, int64_t id);
int fslbm_server_stats_get(fslbm_server* srv, fslbm_server_stats* out);

/* ---- allocation-free step ---- */
/* No counterpart in the reference. Advances a caller-owned FP32 state by one step (the same
 * fused kernel as fslbm_solve_step, d1 = 2) without allocating device memory, for callers that
 * cannot let a library call cudaMalloc: applications that give all device memory to their own
 * pool, or that step inside a loop where an allocation (which may synchronise the device and
 * fail under memory pressure) is not allowed.
 *  - state_in, state_out: device arrays of 4 fields (p,u,v,w), each lz*ly*lx_pitch floats, x
 *    fastest, field stride lz*ly*lx_pitch; 16-byte aligned; lx_pitch a multiple of 8, >= lx.
 *    They must not overlap (the step is not in place: FSLBM_ERR_ARG). Wall cells and the
 *    padding columns x >= lx must hold zero in state_in; state_out gets zero there.
 *  - mask: device array of ly*lx_pitch bytes, 0 fluid / 125 wall, with wall on the rim of the
 *    lx x ly cross-section and in the padding columns. The mask is checked on the device during
 *    the call; a mask that breaks these rules gives FSLBM_ERR_ARG, and state_out then holds no
 *    valid step.
 *  - gauge: p2 subtracted from p this step (0 outside the step after a monitor).
 *  - stream: the caller's cudaStream_t (NULL for the default stream). The call returns after
 *    the step has finished on that stream.
 * Limit: lx_pitch*ly <= 65536 cells; larger cross-sections return FSLBM_ERR_ARG. The work
 * tables live in a preallocated device array of about 1 MiB that every GPU loading the library
 * holds until exit; every call reuses it and overwrites its contents, so calls that overlap on
 * the GPU (on unordered streams) race. The first call on a device sets up that device (it looks
 * up the array's address and the kernel's attributes); make that first call before any stream
 * capture on the device. */
int fslbm_step_f32_noalloc(const float* state_in, float* state_out, const uint8_t* mask, int lx,
                           int ly, int lz, int lx_pitch, const fslbm_params* prm, double gauge,
                           void* stream);

/* ---- host-side formats and generators ---- */
/* pipe.txt: one integer per line, x fastest (pipe.m:62). Reads exactly lx*ly*lz values; extra
 * or missing values are an FSLBM_ERR_IO (the reference's feof loop writes one byte past its
 * buffer, FSLBM.cu:481-484). */
int fslbm_read_pipe_txt(const char* path, int lx, int ly, int lz, uint8_t* out);
int fslbm_write_pipe_txt(const char* path, int lx, int ly, int lz, const uint8_t* mask);
/* param.txt (FSLBM.cu:502-507): tblend, pin, nu as %e floats, d1 and delta as %d, blend as %e.
 * Values are rounded to FP32 as the reference reads them. Fields not in the file keep prm's. */
int fslbm_read_param_txt(const char* path, fslbm_params* prm);
int fslbm_write_param_txt(const char* path, const fslbm_params* prm);
/* pipe.m:36-60: circle of diameter lx0 in a (lx0+2d)^2 cross-section, l0 fluid planes between
 * d buffer planes (value 1) at each end; out holds (lx0+2d)^2 * (l0+2d) bytes. */
int fslbm_pipe_m_mask(int lx0, int l0, int d, uint8_t* out);
/* Splits a reference-layout mask (buffer planes included) into the periodic core's
 * cross-section. Rejects masks the periodic core cannot represent: values other than 0/1/125,
 * fluid on the box rim or inside the buffers, planes that differ, or buffer planes that are
 * not the wrapped copies of their source planes. */
int fslbm_ref_mask_to_core(const uint8_t* mask3d, int lx, int ly, int lz_ref, int d2,
                           uint8_t* mask2d_out);
/* The same for geometry that varies along the pipe: core_out holds lx*ly*(lz_ref - 2*d2) values
 * (one cross-section per core plane, for fslbm_domain.mask_planes = lz). Buffer planes must be
 * the wrapped core planes, as the reference's bcond copies them (FSLBM.cu:291-301). */
int fslbm_ref_mask_to_core3d(const uint8_t* mask3d, int lx, int ly, int lz_ref, int d2,
                             uint8_t* core_out);
/* Seeded initial fields (addition): Poiseuille w = -umax (1 - r^2/R^2) on the circle plus
 * uniform noise of amplitude noise*umax on u,v,w (splitmix64 of seed and cell index), and
 * `modes` random-phase sinusoidal streamwise/azimuthal perturbations of amplitude mode_amp*umax
 * (0 disables). p = 0. Host arrays of lx*ly*lz doubles. */
int fslbm_init_poiseuille(const fslbm_domain* dom, double umax, double noise, int modes,
                          double mode_amp, uint64_t seed, double* p, double* u, double* v,
                          double* w);

#ifdef __cplusplus
}
#endif
#endif /* FSLBM_H */
