// Internal declarations shared by the host runtime and the kernel launchers.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>
#include "../../include/fslbm.h"
#include "common.h"
#include "noise.h"
#include <nvtx3/nvToolsExt.h>

namespace fslbm {
// NVTX range over a host-side scope (step enqueues, batch launches, statistics, server rounds),
// so a timeline tool shows which API call issued which kernels. NVTX v3 is header-only and does
// nothing unless a tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
}  // namespace fslbm

namespace fslbm {

struct StepGeom;

// Device-side counters of a solve: steps done and monitor records written.
struct DevCounters {
  long long steps;
  long long records;
};

struct StepLaunch {
  int dtype;                 // fslbm_dtype of the storage
  int d1;
  const CUtensorMap* map;    // input state tensor map (host copy; passed by value)
  int lxp, ly, L;
  int ntiles, chunk, nchunks;
  const int2* tiles;
  const uint8_t* mask;
  const void* colcoef;
  void* out;
  const double* gauge;
  unsigned* err;
  DevCounters* counters;     // steps incremented by the launch
  long long step_no;         // the time step this launch computes (1-based; rounding seed)
  int K;                     // corrector taps (2: the reference's order 2<->4 blend)
  int mask_planes;           // 0/1: extruded cross-section; L: a mask (and CellCoef) per plane
  const float* wb;           // FP16 storage: per-column base of w and its step share, else null
  const float* wgt;
  // constants in double; converted to the compute type by the launcher
  double tb, cc, pin, dtddy, m, c0, c1, c2, fx, fy, fz;
  double ch[6];              // corrector coefficients c3..c8
};

// One-column kernel for (storage type, d1, corrector taps K).
size_t step_smem_bytes(int dtype, int d1, int K);
bool step_supported(int dtype, int d1, int K);
cudaError_t step_prepare(int dtype, int d1, int K);   // sets the dynamic shared memory attribute
cudaError_t launch_step(const StepLaunch& a, cudaStream_t st);

// Column-pair kernel (FP32 / FP16 storage, d1 = 2) and FP64 column kernel (d1 = 2, 32 x 16
// tiles): two tensor maps per input state (p box with a one-cell halo, u,v,w box with the
// corrector halo).
struct Step2Launch {
  int d1, ty;                // corrective stride, tile height (16 or 32)
  int packed;                // FP32x2 packed arithmetic (1) or scalar pairs (0)
  const CUtensorMap* map_p;
  const CUtensorMap* map_uvw;
  int grid;
};
bool step2_supported(int dtype, int d1);
bool step2_box(int dtype, int d1, int ty, int* sw, int* ph, int* uh, int* hx, int* hy);
int step2_occupancy(int dtype, int d1, int ty);   // CTAs per SM the kernel is built for
cudaError_t step2_prepare(int dtype, int d1, int ty);
cudaError_t launch_step2(const StepLaunch& a, const Step2Launch& b, cudaStream_t st);

struct MonitorLaunch {
  int dtype;
  const void* state;
  const uint8_t* mask;
  int lxp, lx, ly, L;
  double pin, nu, radius, l1;
  int sx, sy, sz;             // sample cell
  fslbm_monitor* log;
  int log_cap;
  double* gauge_out;
  DevCounters* counters;
  const float* wb = nullptr;  // FP16 storage: per-column base of w (stored w is w - wb)
};
cudaError_t launch_monitor(const MonitorLaunch& a, cudaStream_t st);
// The bounded waits against conditions nothing satisfies (counter stays 0): err bit 0 = the
// counter wait gave up, bit 1 = the mbarrier wait gave up.
cudaError_t launch_wait_selftest(const unsigned* counter, unsigned long long limit_ns, unsigned* err,
                                 cudaStream_t st);

// ---- batched ensemble (column-pair kernel, d1 = 2, tile height 16 or 32 for the whole batch)
struct BatchMon {
  MonitorLaunch mon;           // state is chosen per launch from `state`
  const void* state[2];
  long long stop_at;           // no step (and no bookkeeping) once the counter reaches this
  int monitor_every;
  int cur0;
};
cudaError_t batch_prepare(int dtype, int ty);
size_t batch_member_bytes();
// Writes one member descriptor (layout private to the kernels) into host memory at dst.
cudaError_t fill_batch_member(void* dst, const CUtensorMap* map_p, const CUtensorMap* map_u,
                              const StepLaunch& a, void* state0, void* state1,
                              const double* gauge_slot, const long long* steps, long long stop_at,
                              int monitor_every, int cur0, int nchunks, int shape);
// Advances every member `nsteps` steps (fewer for members that reach their stop) in one
// persistent launch, preceded by a reset of the launch's counters. items: nitems (member, item
// of the member) pairs, longest first; mons: per-member bookkeeping (step counter, monitor);
// sync: batch_sync_words(nmembers) counters; err: the batch's error flag. Step s of the launch
// reads buffer cur0 ^ (s & 1) of each member.
size_t batch_sync_words(int nmembers);
cudaError_t launch_batch_steps(int dtype, int ty, const void* members, const BatchMon* mons,
                               const int2* items, int nitems, int nsteps, int grid, int packed,
                               unsigned* sync, int nmembers, unsigned* err, cudaStream_t st);

// Seeded Poiseuille start written into a pitched state (walls and pad columns zero).
cudaError_t launch_init_poiseuille(int dtype, void* state, const uint8_t* mask, int planes, int lxp,
                                   const PoiseuilleInit& q, cudaStream_t st,
                                   const float* wb = nullptr);
// Periodic cross-section: pairs (ghost cell, interior image) as cross-section indices.
cudaError_t launch_fill_ghosts(int dtype, void* state, const int2* pairs, int n, int lxp, int ly,
                               int L, cudaStream_t st);
// masks: `planes` cross-sections of lxp*ly bytes (1: extruded along z)
cudaError_t launch_zero_walls(int dtype, void* state, const uint8_t* mask, int planes, int lxp,
                              int ly, int L, cudaStream_t st);
cudaError_t launch_plane_stats(int dtype, const void* state, const uint8_t* mask, int planes, int lxp, int ly,
                               int L, int d2, int xs, double pin, int cnt, int do_mean,
                               int do_fluct, double* acc, cudaStream_t st, const float* wb = nullptr);
cudaError_t launch_profile(int dtype, const void* state, int lxp, int ly, int L, double* acc,
                           cudaStream_t st, const float* wb = nullptr);
cudaError_t launch_check(int dtype, const void* state, size_t n_per_field, double* out,
                         cudaStream_t st, int lxp = 0, int ly = 0, const float* wb = nullptr);
// Converts between the storage type and FP32/FP64 staging buffers (dense per field, pitched).
// src/dst: dense [4][L][ly][lx] staging arrays; state: pitched [4][L][ly][lxp].
cudaError_t launch_convert_in(int dtype, void* state, const void* src, int src_is_f64, int lx,
                              int lxp, int ly, int L, cudaStream_t st, const float* wb = nullptr);
cudaError_t launch_convert_out(int dtype, const void* state, void* dst, int dst_is_f64, int lx,
                               int lxp, int ly, int L, cudaStream_t st, const float* wb = nullptr);
// FP16 storage keeps w as a deviation from a per-column FP32 base wb (lxp*ly): the streamwise
// mean of the given fields' w (set_fields) or the analytic Poiseuille profile (init_poiseuille),
// zero on wall and padding columns; ghost columns of a periodic cross-section take their
// images' base. wgt holds the base's share of the step of the stored w (corrector taps of the
// base and the body force, per column), recomputed when the parameters change.
cudaError_t launch_wbase_dense(const void* src, int src_is_f64, const uint8_t* mask, int lx, int lxp,
                               int ly, int L, const int2* ghosts, int nghost, float* wb,
                               cudaStream_t st);
cudaError_t launch_wbase_poiseuille(const uint8_t* mask, int lxp, const PoiseuilleInit& q,
                                    const int2* ghosts, int nghost, float* wb, cudaStream_t st);
cudaError_t launch_wgt(const float* wb, int lxp, int ly, float K0, float K1, float K2, float tfz,
                       float* wgt, cudaStream_t st);

}  // namespace fslbm

namespace fslbm {
// TMA box of the step kernel for (dtype, d1): slot row length, rows, halos.
bool step_box(int dtype, int d1, int K, int* sw, int* sh, int* hx, int* hy);
// Corrector coefficients c0..c8 of an order (0/4: the reference's 4<->2 blend, 6: 6<->4,
// 8: 8<->6, 10/12/14: fixed), formed in FP32 (fp32 != 0) or FP64 as the reference forms its
// active set. Returns the tap count K, 0 for an unknown order.
int fd_coefficients(int order, double blend, int fp32, double* c);
// Gathers the YZ plane x = idx (kind 0, out [4][L][ly]) or the XY plane z = idx
// (kind 1, out [4][ly][lx]) of the four fields as FP32 into device memory.
cudaError_t launch_gather_plane(int dtype, const void* state, int lx, int lxp, int ly, int L,
                                int kind, int idx, float* out, cudaStream_t st,
                                const float* wb = nullptr);
}  // namespace fslbm
