// Kernel launchers and the small auxiliary kernels of the solve runtime (monitor reduction,
// statistics accumulation, field conversion, divergence check).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include "internal.h"
#include "step_kernel.cuh"
#include "step2_kernel.cuh"
#include "stepcol_kernel.cuh"

namespace fslbm {

// Arithmetic type of the auxiliary kernels for a storage type (FP16 storage is read as FP32).
template <class T> struct ArithOf { using type = T; };
template <> struct ArithOf<__half> { using type = float; };
__device__ __forceinline__ double to_d(float x) { return double(x); }
__device__ __forceinline__ double to_d(double x) { return x; }
__device__ __forceinline__ double to_d(__half x) { return double(__half2float(x)); }
// A stored value as its field's value: FP16 storage keeps w as a deviation from the per-column
// base wb (w = stored + base in FP32, as the step forms it); other types and fields are as stored.
template <class TS> __device__ __forceinline__ double wval(TS v, const float*, size_t) {
  return to_d(v);
}
template <> __device__ __forceinline__ double wval<__half>(__half v, const float* wb, size_t col) {
  return wb ? double(__fadd_rn(__half2float(v), wb[col])) : to_d(v);
}

// ------------------------------------------------------------------------------------------
// step dispatch
// ------------------------------------------------------------------------------------------
template <class TS, int D1, int K>
static cudaError_t launch_step_t(const StepLaunch& a, cudaStream_t st) {
  using TC = typename Compute<TS>::type;
  using Tl = StepTile<TS, D1, K>;
  StepGeom g;
  g.lxp = a.lxp; g.ly = a.ly; g.L = a.L;
  g.ntiles = a.ntiles; g.chunk = a.chunk;
  g.tiles = a.tiles; g.mask = a.mask; g.colcoef = a.colcoef; g.out = a.out;
  g.gauge = a.gauge; g.err = a.err;
  g.step_counter = a.counters ? &a.counters->steps : nullptr;
  g.mask_planes = a.mask_planes;
  StepConst<TC> k;
  k.tb = TC(a.tb); k.cc = TC(a.cc); k.pin = TC(a.pin); k.dtddy = TC(a.dtddy); k.m = TC(a.m);
  k.c0 = TC(a.c0); k.c1 = TC(a.c1); k.c2 = TC(a.c2);
  for (int j = 0; j < 6; ++j) k.ch[j] = TC(a.ch[j]);
  k.fx = TC(a.fx); k.fy = TC(a.fy); k.fz = TC(a.fz);
  const int grid = a.ntiles * a.nchunks;
  if (a.mask_planes > 1) fslbm_step_kernel<TS, D1, K, true><<<grid, kThreads, Tl::SMEM_BYTES, st>>>(*a.map, g, k);
  else fslbm_step_kernel<TS, D1, K, false><<<grid, kThreads, Tl::SMEM_BYTES, st>>>(*a.map, g, k);
  return cudaGetLastError();
}

// (storage type, d1, corrector taps K) built for the one-column kernel: shared memory holds
// R + 3 planes of the tile with an R = K*d1 halo, which bounds R at 8 for FP32 and 4 for FP64.
#define FSLBM_STEP_COMBOS(X)                                                                    \
  X(FSLBM_F32, float, 1, 2) X(FSLBM_F32, float, 2, 2) X(FSLBM_F32, float, 3, 2)                \
  X(FSLBM_F32, float, 1, 3) X(FSLBM_F32, float, 1, 4) X(FSLBM_F32, float, 1, 5)                \
  X(FSLBM_F32, float, 1, 6) X(FSLBM_F32, float, 1, 8) X(FSLBM_F32, float, 2, 3)                \
  X(FSLBM_F32, float, 2, 4) X(FSLBM_F64, double, 1, 2) X(FSLBM_F64, double, 2, 2)              \
  X(FSLBM_F64, double, 1, 3) X(FSLBM_F64, double, 1, 4)

bool step_supported(int dtype, int d1, int K) {
#define X(DT, TS, D, KK) if (dtype == DT && d1 == D && K == KK) return true;
  FSLBM_STEP_COMBOS(X)
#undef X
  if (dtype == FSLBM_F16) return d1 == 2 && K == 2;   // column-pair kernel only
  return false;
}

size_t step_smem_bytes(int dtype, int d1, int K) {
#define X(DT, TS, D, KK) if (dtype == DT && d1 == D && K == KK) return StepTile<TS, D, KK>::SMEM_BYTES;
  FSLBM_STEP_COMBOS(X)
#undef X
  return 0;
}

cudaError_t step_prepare(int dtype, int d1, int K) {
#define X(DT, TS, D, KK)                                                                        \
  if (dtype == DT && d1 == D && K == KK) {                                                      \
    cudaError_t e = cudaFuncSetAttribute(fslbm_step_kernel<TS, D, KK, false>,                   \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,           \
                                         int(StepTile<TS, D, KK>::SMEM_BYTES));                 \
    if (e) return e;                                                                            \
    return cudaFuncSetAttribute(fslbm_step_kernel<TS, D, KK, true>,                             \
                                cudaFuncAttributeMaxDynamicSharedMemorySize,                    \
                                int(StepTile<TS, D, KK>::SMEM_BYTES));                          \
  }
  FSLBM_STEP_COMBOS(X)
#undef X
  return cudaErrorInvalidValue;
}

cudaError_t launch_step(const StepLaunch& a, cudaStream_t st) {
#define X(DT, TS, D, KK) if (a.dtype == DT && a.d1 == D && a.K == KK) return launch_step_t<TS, D, KK>(a, st);
  FSLBM_STEP_COMBOS(X)
#undef X
  return cudaErrorInvalidValue;
}

// ------------------------------------------------------------------------------------------
// column-pair kernel (FP32 / FP16 storage) and FP64 column kernel dispatch
// ------------------------------------------------------------------------------------------
bool step2_supported(int dtype, int d1) {
  return (dtype == FSLBM_F32 || dtype == FSLBM_F16 || dtype == FSLBM_F64) && d1 == 2;
}

template <int TY, class TE> static void box2(int* sw, int* ph, int* uh, int* hx, int* hy) {
  using Tl = Step2Tile<2, TY, TE>;
  *sw = Tl::SW; *ph = Tl::PH; *uh = Tl::UH; *hx = Tl::HX; *hy = Tl::HY;
}

bool step2_box(int dtype, int d1, int ty, int* sw, int* ph, int* uh, int* hx, int* hy) {
  if (d1 != 2 || (ty != 32 && ty != 16)) return false;
  if (dtype == FSLBM_F64) {          // the FP64 column kernel: 32 x 16 tiles only
    using Tl = ColTile<2, 16>;
    if (ty != 16) return false;
    *sw = Tl::SW; *ph = Tl::PH; *uh = Tl::UH; *hx = Tl::HX; *hy = Tl::HY;
    return true;
  }
  if (dtype == FSLBM_F32) {
    if (ty == 32) box2<32, float>(sw, ph, uh, hx, hy);
    else box2<16, float>(sw, ph, uh, hx, hy);
    return true;
  }
  if (dtype == FSLBM_F16) {
    if (ty == 32) box2<32, __half>(sw, ph, uh, hx, hy);
    else box2<16, __half>(sw, ph, uh, hx, hy);
    return true;
  }
  return false;
}

int step2_occupancy(int dtype, int, int ty) { return dtype != FSLBM_F64 && ty == 16 ? 2 : 1; }

template <int TY, bool PK, class TE> static cudaError_t prep2() {
  return cudaFuncSetAttribute(fslbm_step2_kernel<2, TY, PK, TE>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              int(Step2Tile<2, TY, TE>::SMEM_BYTES));
}

template <class TE> static cudaError_t prep2_all(int ty) {
  cudaError_t e;
  if (ty == 32) {
    if ((e = prep2<32, true, TE>())) return e;
    return prep2<32, false, TE>();
  }
  if (ty == 16) {
    if ((e = prep2<16, true, TE>())) return e;
    return prep2<16, false, TE>();
  }
  return cudaErrorInvalidValue;
}

cudaError_t step2_prepare(int dtype, int d1, int ty) {
  if (d1 != 2) return cudaErrorInvalidValue;
  if (dtype == FSLBM_F64)
    return ty != 16 ? cudaErrorInvalidValue
                    : cudaFuncSetAttribute(fslbm_col_kernel<2, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(ColTile<2, 16>::SMEM_BYTES));
  if (dtype == FSLBM_F32) return prep2_all<float>(ty);
  if (dtype == FSLBM_F16) return prep2_all<__half>(ty);
  return cudaErrorInvalidValue;
}

template <class TE>
static cudaError_t launch_step2_t(const Step2Launch& b, const Step2Geom& g,
                                  const StepConst<float>& k, cudaStream_t st) {
#define FSLBM_L2(TY, PK)                                                                  \
  fslbm_step2_kernel<2, TY, PK, TE><<<b.grid, Step2Tile<2, TY, TE>::THREADS,              \
                                      Step2Tile<2, TY, TE>::SMEM_BYTES, st>>>(*b.map_p,  \
                                                                          *b.map_uvw, g, k)
  if (b.ty == 32 && b.packed) FSLBM_L2(32, true);
  else if (b.ty == 32) FSLBM_L2(32, false);
  else if (b.ty == 16 && b.packed) FSLBM_L2(16, true);
  else if (b.ty == 16) FSLBM_L2(16, false);
  else return cudaErrorInvalidValue;
#undef FSLBM_L2
  return cudaGetLastError();
}

cudaError_t launch_step2(const StepLaunch& a, const Step2Launch& b, cudaStream_t st) {
  Step2Geom g;
  g.lxp = a.lxp; g.ly = a.ly; g.L = a.L; g.ntiles = a.ntiles; g.nchunks = b.grid / a.ntiles;
  g.tiles = a.tiles; g.mask = a.mask; g.colcoef = a.colcoef; g.out = a.out;
  g.gauge = a.gauge; g.err = a.err;
  g.wb = a.wb; g.wgt = a.wgt;
  g.step_counter = a.counters ? &a.counters->steps : nullptr;
  g.step_no = unsigned(a.step_no);
  StepConst<float> k;
  k.tb = float(a.tb); k.cc = float(a.cc); k.pin = float(a.pin); k.dtddy = float(a.dtddy);
  k.m = float(a.m); k.c0 = float(a.c0); k.c1 = float(a.c1); k.c2 = float(a.c2);
  k.fx = float(a.fx); k.fy = float(a.fy); k.fz = float(a.fz);
  if (b.d1 != 2) return cudaErrorInvalidValue;
  if (a.dtype == FSLBM_F64) {
    if (b.ty != 16) return cudaErrorInvalidValue;
    StepConst<double> kd;
    kd.tb = a.tb; kd.cc = a.cc; kd.pin = a.pin; kd.dtddy = a.dtddy; kd.m = a.m;
    kd.c0 = a.c0; kd.c1 = a.c1; kd.c2 = a.c2; kd.fx = a.fx; kd.fy = a.fy; kd.fz = a.fz;
    for (int j = 0; j < 6; ++j) kd.ch[j] = a.ch[j];
    fslbm_col_kernel<2, 16><<<b.grid, ColTile<2, 16>::THREADS, ColTile<2, 16>::SMEM_BYTES, st>>>(
        *b.map_p, *b.map_uvw, g, kd);
    return cudaGetLastError();
  }
  if (a.dtype == FSLBM_F32) return launch_step2_t<float>(b, g, k, st);
  if (a.dtype == FSLBM_F16) return launch_step2_t<__half>(b, g, k, st);
  return cudaErrorInvalidValue;
}

// ------------------------------------------------------------------------------------------
// block reduction helper (FP64)
// ------------------------------------------------------------------------------------------
template <int NV>
__device__ void block_sum(double (&v)[NV], double* sh /* NV * 32 */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[k * 32 + warp] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = lane < nw ? sh[k * 32 + lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      v[k] = s;
    }
  }
}

// ------------------------------------------------------------------------------------------
// monitor (FSLBM.cu:632-666), FP64 sums, one block
// ------------------------------------------------------------------------------------------
// The state is read through L2 (ld.global.cg): in a chained batched launch other CTAs of the
// same grid wrote it, and this SM's L1 may hold lines of an earlier read of the same buffer.
// The sums are formed in the order of a 512-thread block whatever the block size NT (512, or 256
// in the batched kernel's 32 x 16 tile form, where each thread takes two of the 512 strands and
// the warp partials of both), so every form books the same monitor record bit for bit.
template <class TS, int NT = 512>
__device__ void monitor_body(const MonitorLaunch& a, double* sh) {
  using TA = typename ArithOf<TS>::type;
  static_assert(NT == 512 || NT == 256, "block of 256 or 512 threads");
  const TS* st = reinterpret_cast<const TS*>(a.state);
  const size_t FS = size_t(a.lxp) * a.ly * a.L;
  const TA pin = TA(a.pin);
  double v[3] = {0, 0, 0};   // sum w, sum p, sum (p - pin) over non-wall cells of plane z=0
  auto strand = [&](int j0, double (&acc)[3]) {
    for (int j = j0; j < a.lxp * a.ly; j += 512) {
      if (a.mask[j] != 0) continue;         // walls hold zero; periodic images are not counted
      const TA p = TA(__ldcg(st + j));
      acc[0] += wval(__ldcg(st + 3 * FS + j), a.wb, size_t(j));
      acc[1] += double(p);
      acc[2] += double(TA(p - pin));        // the outlet buffer copy's p
    }
  };
  if constexpr (NT == 512) {
    for (int j = threadIdx.x; j < a.lxp * a.ly; j += blockDim.x) {
      if (a.mask[j] != 0) continue;         // walls hold zero; periodic images are not counted
      const TA p = TA(__ldcg(st + j));
      v[0] += wval(__ldcg(st + 3 * FS + j), a.wb, size_t(j));
      v[1] += double(p);
      v[2] += double(TA(p - pin));          // the outlet buffer copy's p
    }
    block_sum<3>(v, sh);
  } else {
    // strands t and t + 256, each reduced over its warp as the 512-thread block's warps w and
    // w + 8 reduce, then the 16 warp partials as block_sum's second stage adds them
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double u[3] = {0, 0, 0};
    strand(threadIdx.x, v);
    strand(threadIdx.x + 256, u);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      for (int o = 16; o > 0; o >>= 1) {
        v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        u[k] += __shfl_down_sync(0xffffffffu, u[k], o);
      }
      if (lane == 0) { sh[k * 32 + warp] = v[k]; sh[k * 32 + warp + 8] = u[k]; }
    }
    __syncthreads();
    if (warp == 0)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        double s = lane < 16 ? sh[k * 32 + lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        v[k] = s;
      }
  }
  if (threadIdx.x == 0) {
    const double q1 = v[0] / a.l1, p1 = v[1] / a.l1, p2 = v[2] / a.l1;
    fslbm_monitor r;
    r.step = a.counters->steps;
    r.q1 = q1; r.q2 = q1; r.p1 = p1; r.p2 = p2;
    r.f = (p1 - p2) / q1 / q1 / 3.0 * 4.0 * a.radius / double(a.L);
    r.sample = wval(__ldcg(st + 3 * FS + (size_t(a.sz) * a.ly + a.sy) * a.lxp + a.sx), a.wb,
                    size_t(a.sy) * a.lxp + a.sx);
    r.re = 2.0 * a.radius * q1 / a.nu;
    const long long idx = a.counters->records;
    a.log[idx % a.log_cap] = r;
    a.counters->records = idx + 1;
    *a.gauge_out = p2;
  }
}

template <class TS>
__global__ void monitor_kernel(MonitorLaunch a) {
  __shared__ double sh[3 * 32];
  monitor_body<TS>(a, sh);
}

// ------------------------------------------------------------------------------------------
// batched ensemble: chained steps in one persistent launch
// ------------------------------------------------------------------------------------------
// One member of a batched ensemble: its tensor maps for both state buffers, its step geometry
// and constants, and where its step count stops.
struct alignas(64) BatchMember {
  CUtensorMap map_p[2], map_u[2];
  Step2Geom g;                 // g.out is replaced by the buffer the step writes
  StepConst<float> k;
  void* state[2];
  const double* gauge_slot;    // the member's monitor p2, applied on the step after a monitor
  const long long* steps;      // the member's device step counter
  long long stop_at;           // the member is not stepped once its counter reaches this
  int shape;                   // warp shape of the member's items: 32 x 2, 16 x 4 or 8 x 8 (0, 1, 2)
  int monitor_every;
  int cur0;                    // input buffer at the launch's first step
};

// Bookkeeping of one member after one of its steps, by all threads of the CTA that completed
// the step's last item: the step counter advances (unless the member had reached its stop) and,
// when due, the monitor record and the gauge of the member's next step are written. Inlined: any
// call in the batched kernel makes its march spill registers (the call ABI).
template <int NT>
__device__ __forceinline__ void batch_book(const BatchMon& b, int parity_after, double* sh, int* due) {
  if (threadIdx.x == 0) {
    const long long s0 = __ldcg(&b.mon.counters->steps);
    *due = 0;
    if (s0 < b.stop_at) {
      const long long s = s0 + 1;
      b.mon.counters->steps = s;
      *due = b.monitor_every > 0 && s % b.monitor_every == 0;
    }
  }
  __syncthreads();
  if (*due) {
    MonitorLaunch a = b.mon;
    a.state = b.state[b.cur0 ^ parity_after];
    if (a.dtype == FSLBM_F16) monitor_body<__half, NT>(a, sh);
    else monitor_body<float, NT>(a, sh);
  }
}

// Thread 0, before an item of the member's step `step`: waits until the member's previous step
// is complete and booked, then stages the item's geometry and constants in shared memory.
// False when the wait gave up (error flag set). Inlined for the same reason as batch_book.
__device__ __forceinline__ bool batch_item_begin(const BatchMember& mb, int member, int step,
                                              const unsigned* sync, unsigned* err, Step2Geom* s_g,
                                              StepConst<float>* s_k, long long* s_done) {
  if (step > 0 && !wait_geq_gpu(sync + 5 + 2 * member, unsigned(step), kWaitLimitNs)) {
    atomicOr(err, 1u);
    return false;
  }
  // the member's previous step was written by other CTAs through the generic proxy; this
  // thread's TMA loads of it follow
  fence_proxy_async_global();
  const long long done = __ldcg(mb.steps);
  *s_done = done;
  const int cur = mb.cur0 ^ (step & 1);
  Step2Geom g = mb.g;
  g.out = mb.state[1 - cur];
  g.step_counter = nullptr;
  g.step_no = unsigned(done + 1);
  g.gauge = (mb.monitor_every > 0 && done > 0 && done % mb.monitor_every == 0) ? mb.gauge_slot : nullptr;
  *s_g = g;
  *s_k = mb.k;
  return true;
}

// Many pipes, `nsteps` steps each, in one persistent launch (nitems * nsteps < 2^32). Ticket t
// is step t / nitems of item items[t % nitems] = (member, item of the member); within a step the
// items are ordered longest first. Steps are chained per member instead of separated by
// launches: before it marches an item of step s > 0, a CTA waits until the member's step s - 1
// is complete and booked, so the members that finish a step early start the next one while the
// last items of the step still run, and the SMs stay busy across step boundaries. A CTA waits
// only on items that resident CTAs have already claimed (every ticket of step s precedes every
// ticket of step s + 1), so the waits end. Counters (zeroed before the launch): sync[0] = next
// ticket; per member m, sync[4 + 2m] = its items completed in this launch and sync[5 + 2m] =
// its steps released.
// A CTA counts its previous item when it claims the next one: after the claim's barrier every
// thread's stores of that item precede thread 0's fence and its acq_rel count (cumulative over
// the barrier). The CTA whose count completes a member's step books it (step counter, monitor)
// and releases it before marching on. Counting there rather than right after the march keeps
// the march free of register spills.
template <int D1, int TY, bool PK, class TE>
__global__ void __launch_bounds__(Step2Tile<D1, TY, TE>::THREADS, TY == 16 ? 2 : 1)
    fslbm_step2_batch_kernel(const BatchMember* __restrict__ members,
                             const BatchMon* __restrict__ mons, const int2* __restrict__ items,
                             int nitems, int nsteps, unsigned* sync, unsigned* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned s_ticket;
  __shared__ long long s_done;
  __shared__ int s_go, s_book, s_due;
  __shared__ double s_sh[3 * 32];
  // the item's geometry and constants, read by the march from shared memory (the single-pipe
  // kernel reads them from the parameter bank); kept in registers through the march they spill
  __shared__ StepConst<float> s_k;
  __shared__ Step2Geom s_g;
  bool first = true;
  unsigned prev = ~0u;             // the CTA's previous ticket, counted at the next claim
  for (;;) {
    if (threadIdx.x == 0) s_ticket = atomicAdd(&sync[0], 1u);
    __syncthreads();               // every thread has finished the previous item
    const unsigned t = s_ticket;
    if (threadIdx.x == 0) {
      s_book = -1;
      if (prev != ~0u) {
        __threadfence();
        const int pm = items[prev % unsigned(nitems)].x;
        const int ps = int(prev / unsigned(nitems));
        const BatchMember& pb = members[pm];
        const unsigned per_step = unsigned(pb.g.ntiles * pb.g.nchunks);
        const unsigned c = atom_add_acq_rel_gpu(sync + 4 + 2 * pm, 1u) + 1u;
        if (c == per_step * unsigned(ps + 1)) s_book = int(prev);
      }
    }
    __syncthreads();               // every thread has read the ticket before the next claim
    if (s_book >= 0) {             // the previous item completed its member's step: book, release
      const unsigned pt = unsigned(s_book);
      const int pm = items[pt % unsigned(nitems)].x;
      const int ps = int(pt / unsigned(nitems));
      batch_book<Step2Tile<D1, TY, TE>::THREADS>(mons[pm], (ps & 1) ^ 1, s_sh, &s_due);
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) st_release_gpu(sync + 5 + 2 * pm, unsigned(ps + 1));
    }
    if (t >= unsigned(nitems) * unsigned(nsteps)) return;
    const int step = int(t / unsigned(nitems));
    const int2 it = items[t % unsigned(nitems)];
    const BatchMember& mb = members[it.x];
    if (threadIdx.x == 0)          // every thread has left the previous item (ticket barriers)
      s_go = batch_item_begin(mb, it.x, step, sync, err, &s_g, &s_k, &s_done);
    __syncthreads();
    if (!s_go) return;
    prev = t;
    if (s_done < mb.stop_at) {
      const int cur = mb.cur0 ^ (step & 1);
      const int ntiles = mb.g.ntiles;
      const bool ok = step2_march<D1, TY, PK, TE>(&mb.map_p[cur], &mb.map_u[cur], s_g, s_k,
                                                  it.y % ntiles, it.y / ntiles, smem, !first,
                                                  mb.shape);
      if (!ok) return;
      first = false;
    }
  }
}

template <int TY, bool PK, class TE> static cudaError_t batch_prep() {
  return cudaFuncSetAttribute(fslbm_step2_batch_kernel<2, TY, PK, TE>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              int(Step2Tile<2, TY, TE>::SMEM_BYTES));
}

template <int TY, class TE> static cudaError_t batch_prep_all() {
  cudaError_t e;
  if ((e = batch_prep<TY, true, TE>())) return e;
  return batch_prep<TY, false, TE>();
}

cudaError_t batch_prepare(int dtype, int ty) {
  if (ty != 16 && ty != 32) return cudaErrorInvalidValue;
  if (dtype == FSLBM_F32) return ty == 16 ? batch_prep_all<16, float>() : batch_prep_all<32, float>();
  if (dtype == FSLBM_F16) return ty == 16 ? batch_prep_all<16, __half>() : batch_prep_all<32, __half>();
  return cudaErrorInvalidValue;
}

size_t batch_member_bytes() { return sizeof(BatchMember); }

cudaError_t fill_batch_member(void* dst, const CUtensorMap* mp, const CUtensorMap* mu,
                              const StepLaunch& a, void* state0, void* state1,
                              const double* gauge_slot, const long long* steps, long long stop_at,
                              int monitor_every, int cur0, int nchunks, int shape) {
  BatchMember m;
  std::memset(&m, 0, sizeof m);
  m.map_p[0] = mp[0]; m.map_p[1] = mp[1];
  m.map_u[0] = mu[0]; m.map_u[1] = mu[1];
  m.g.lxp = a.lxp; m.g.ly = a.ly; m.g.L = a.L; m.g.ntiles = a.ntiles; m.g.nchunks = nchunks;
  m.g.tiles = a.tiles; m.g.mask = a.mask; m.g.colcoef = a.colcoef; m.g.out = nullptr;
  m.g.gauge = nullptr; m.g.err = a.err; m.g.step_counter = nullptr; m.g.step_no = 0;
  m.g.wb = a.wb; m.g.wgt = a.wgt;
  m.k.tb = float(a.tb); m.k.cc = float(a.cc); m.k.pin = float(a.pin); m.k.dtddy = float(a.dtddy);
  m.k.m = float(a.m); m.k.c0 = float(a.c0); m.k.c1 = float(a.c1); m.k.c2 = float(a.c2);
  m.k.fx = float(a.fx); m.k.fy = float(a.fy); m.k.fz = float(a.fz);
  m.state[0] = state0; m.state[1] = state1;
  m.gauge_slot = gauge_slot; m.steps = steps; m.stop_at = stop_at; m.shape = shape;
  m.monitor_every = monitor_every; m.cur0 = cur0;
  std::memcpy(dst, &m, sizeof m);
  return cudaSuccess;
}

template <int TY, class TE>
static void launch_batch_t(const BatchMember* mb, const BatchMon* mons, const int2* items,
                           int nitems, int nsteps, int grid, int packed, unsigned* sync,
                           unsigned* err, cudaStream_t st) {
  using Tl = Step2Tile<2, TY, TE>;
  if (packed)
    fslbm_step2_batch_kernel<2, TY, true, TE><<<grid, Tl::THREADS, Tl::SMEM_BYTES, st>>>(
        mb, mons, items, nitems, nsteps, sync, err);
  else
    fslbm_step2_batch_kernel<2, TY, false, TE><<<grid, Tl::THREADS, Tl::SMEM_BYTES, st>>>(
        mb, mons, items, nitems, nsteps, sync, err);
}

size_t batch_sync_words(int nmembers) { return 4 + 2 * size_t(nmembers); }

cudaError_t launch_batch_steps(int dtype, int ty, const void* members, const BatchMon* mons,
                               const int2* items, int nitems, int nsteps, int grid, int packed,
                               unsigned* sync, int nmembers, unsigned* err, cudaStream_t st) {
  if (nsteps < 1) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(sync, 0, batch_sync_words(nmembers) * sizeof(unsigned), st);
  if (e) return e;
  const BatchMember* mb = reinterpret_cast<const BatchMember*>(members);
  if (ty == 32 && dtype == FSLBM_F32) launch_batch_t<32, float>(mb, mons, items, nitems, nsteps, grid, packed, sync, err, st);
  else if (ty == 32 && dtype == FSLBM_F16) launch_batch_t<32, __half>(mb, mons, items, nitems, nsteps, grid, packed, sync, err, st);
  else if (ty == 16 && dtype == FSLBM_F32) launch_batch_t<16, float>(mb, mons, items, nitems, nsteps, grid, packed, sync, err, st);
  else if (ty == 16 && dtype == FSLBM_F16) launch_batch_t<16, __half>(mb, mons, items, nitems, nsteps, grid, packed, sync, err, st);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_monitor(const MonitorLaunch& a, cudaStream_t st) {
  if (a.dtype == FSLBM_F32) monitor_kernel<float><<<1, 512, 0, st>>>(a);
  else if (a.dtype == FSLBM_F64) monitor_kernel<double><<<1, 512, 0, st>>>(a);
  else if (a.dtype == FSLBM_F16) monitor_kernel<__half><<<1, 512, 0, st>>>(a);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// seeded initial fields generated on the device (same formula as the host generator)
// ------------------------------------------------------------------------------------------
template <class TS>
__global__ void init_poiseuille_kernel(TS* s, const uint8_t* mask, int planes, int lxp,
                                       PoiseuilleInit q, const float* wb) {
  const size_t FS = size_t(lxp) * q.ly * q.L;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < FS;
       i += size_t(gridDim.x) * blockDim.x) {
    const int x = int(i % lxp);
    const size_t r = i / lxp;
    const int y = int(r % q.ly), z = int(r / q.ly);
    double c[4] = {0.0, 0.0, 0.0, 0.0};
    if (x < q.lx && mask[(planes > 1 ? size_t(z) * q.ly : 0) * lxp + size_t(y) * lxp + x] != kWall)
      poiseuille_cell(q, x, y, z, c);
    s[i] = TS(c[0]); s[FS + i] = TS(c[1]); s[2 * FS + i] = TS(c[2]);
    if (wb) s[3 * FS + i] = TS(__fsub_rn(float(c[3]), wb[size_t(y) * lxp + x]));
    else s[3 * FS + i] = TS(c[3]);
  }
}

cudaError_t launch_init_poiseuille(int dtype, void* state, const uint8_t* mask, int planes, int lxp,
                                   const PoiseuilleInit& q, cudaStream_t st, const float* wb) {
  const int grid = 1184;
  if (dtype == FSLBM_F32)
    init_poiseuille_kernel<float><<<grid, 256, 0, st>>>((float*)state, mask, planes, lxp, q, nullptr);
  else if (dtype == FSLBM_F64)
    init_poiseuille_kernel<double><<<grid, 256, 0, st>>>((double*)state, mask, planes, lxp, q, nullptr);
  else if (dtype == FSLBM_F16)
    init_poiseuille_kernel<__half><<<grid, 256, 0, st>>>((__half*)state, mask, planes, lxp, q, wb);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// periodic cross-section: ghost cells take their interior images (every plane, four fields)
// ------------------------------------------------------------------------------------------
template <class TS>
__global__ void fill_ghosts_kernel(TS* s, const int2* pairs, int n, size_t plane, int L) {
  const size_t FS = plane * L;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < size_t(n) * L;
       i += size_t(gridDim.x) * blockDim.x) {
    const int2 pr = pairs[i % n];
    const size_t z = (i / n) * plane, d = z + pr.x, sidx = z + pr.y;
    s[d] = s[sidx]; s[FS + d] = s[FS + sidx]; s[2 * FS + d] = s[2 * FS + sidx];
    s[3 * FS + d] = s[3 * FS + sidx];
  }
}

cudaError_t launch_fill_ghosts(int dtype, void* state, const int2* pairs, int n, int lxp, int ly,
                               int L, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const size_t plane = size_t(lxp) * ly;
  const int grid = int(std::min<size_t>(1184, (size_t(n) * L + 255) / 256));
  if (dtype == FSLBM_F32)
    fill_ghosts_kernel<float><<<grid, 256, 0, st>>>((float*)state, pairs, n, plane, L);
  else if (dtype == FSLBM_F64)
    fill_ghosts_kernel<double><<<grid, 256, 0, st>>>((double*)state, pairs, n, plane, L);
  else if (dtype == FSLBM_F16)
    fill_ghosts_kernel<__half><<<grid, 256, 0, st>>>((__half*)state, pairs, n, plane, L);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// wall zeroing, conversion, check
// ------------------------------------------------------------------------------------------
template <class TS>
__global__ void zero_walls_kernel(TS* s, const uint8_t* mask, int planes, int lxp, int ly, int L) {
  const size_t FS = size_t(lxp) * ly * L, plane = size_t(lxp) * ly;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < FS;
       i += size_t(gridDim.x) * blockDim.x) {
    if (mask[planes > 1 ? i : i % plane] == kWall) {
      s[i] = TS(0); s[FS + i] = TS(0); s[2 * FS + i] = TS(0); s[3 * FS + i] = TS(0);
    }
  }
}

cudaError_t launch_zero_walls(int dtype, void* state, const uint8_t* mask, int planes, int lxp,
                              int ly, int L, cudaStream_t st) {
  const int grid = 592;
  if (dtype == FSLBM_F32)
    zero_walls_kernel<float><<<grid, 256, 0, st>>>(reinterpret_cast<float*>(state), mask, planes, lxp, ly, L);
  else if (dtype == FSLBM_F64)
    zero_walls_kernel<double><<<grid, 256, 0, st>>>(reinterpret_cast<double*>(state), mask, planes, lxp, ly, L);
  else if (dtype == FSLBM_F16)
    zero_walls_kernel<__half><<<grid, 256, 0, st>>>(reinterpret_cast<__half*>(state), mask, planes, lxp, ly, L);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// Dense host-layout fields (4 x L x ly x lx) <-> the pitched state (4 x L x ly x lxp), with a type
// conversion. A warp copies one row at a time (one division per row, coalesced along x).
template <class TS, class TH>
__global__ void convert_in_kernel(TS* s, const TH* src, int lx, int lxp, int ly, int L,
                                  const float* wb) {
  const long long rows = (long long)ly * L, FS = (long long)lxp * rows;
  const int lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long rr = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; rr < 4 * rows;
       rr += nwarps) {
    const long long f = rr / rows, yz = rr - f * rows;
    const TH* in = src + rr * lx;
    TS* out = s + f * FS + yz * lxp;
    if (wb && f == 3) {                 // FP16 storage: w as the deviation from its base
      const float* b = wb + (yz % ly) * lxp;
      for (int x = lane; x < lx; x += 32) out[x] = TS(__fsub_rn(float(in[x]), b[x]));
    } else {
      for (int x = lane; x < lx; x += 32) out[x] = TS(in[x]);
    }
  }
}
template <class TS, class TH>
__global__ void convert_out_kernel(const TS* s, TH* dst, int lx, int lxp, int ly, int L,
                                   const float* wb) {
  const long long rows = (long long)ly * L, FS = (long long)lxp * rows;
  const int lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long rr = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; rr < 4 * rows;
       rr += nwarps) {
    const long long f = rr / rows, yz = rr - f * rows;
    const TS* in = s + f * FS + yz * lxp;
    TH* out = dst + rr * lx;
    if (wb && f == 3) {
      const size_t row = size_t(yz % ly) * lxp;
      for (int x = lane; x < lx; x += 32) out[x] = TH(wval(in[x], wb, row + x));
    } else {
      for (int x = lane; x < lx; x += 32) out[x] = TH(in[x]);
    }
  }
}

cudaError_t launch_convert_in(int dtype, void* state, const void* src, int src_is_f64, int lx,
                              int lxp, int ly, int L, cudaStream_t st, const float* wb) {
  const int grid = 1184;
  if (dtype == FSLBM_F32) {
    if (src_is_f64) convert_in_kernel<float, double><<<grid, 256, 0, st>>>((float*)state, (const double*)src, lx, lxp, ly, L, nullptr);
    else convert_in_kernel<float, float><<<grid, 256, 0, st>>>((float*)state, (const float*)src, lx, lxp, ly, L, nullptr);
  } else if (dtype == FSLBM_F64) {
    if (src_is_f64) convert_in_kernel<double, double><<<grid, 256, 0, st>>>((double*)state, (const double*)src, lx, lxp, ly, L, nullptr);
    else convert_in_kernel<double, float><<<grid, 256, 0, st>>>((double*)state, (const float*)src, lx, lxp, ly, L, nullptr);
  } else if (dtype == FSLBM_F16) {
    if (src_is_f64) convert_in_kernel<__half, double><<<grid, 256, 0, st>>>((__half*)state, (const double*)src, lx, lxp, ly, L, wb);
    else convert_in_kernel<__half, float><<<grid, 256, 0, st>>>((__half*)state, (const float*)src, lx, lxp, ly, L, wb);
  } else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_convert_out(int dtype, const void* state, void* dst, int dst_is_f64, int lx,
                               int lxp, int ly, int L, cudaStream_t st, const float* wb) {
  const int grid = 1184;
  if (dtype == FSLBM_F32) {
    if (dst_is_f64) convert_out_kernel<float, double><<<grid, 256, 0, st>>>((const float*)state, (double*)dst, lx, lxp, ly, L, nullptr);
    else convert_out_kernel<float, float><<<grid, 256, 0, st>>>((const float*)state, (float*)dst, lx, lxp, ly, L, nullptr);
  } else if (dtype == FSLBM_F64) {
    if (dst_is_f64) convert_out_kernel<double, double><<<grid, 256, 0, st>>>((const double*)state, (double*)dst, lx, lxp, ly, L, nullptr);
    else convert_out_kernel<double, float><<<grid, 256, 0, st>>>((const double*)state, (float*)dst, lx, lxp, ly, L, nullptr);
  } else if (dtype == FSLBM_F16) {
    if (dst_is_f64) convert_out_kernel<__half, double><<<grid, 256, 0, st>>>((const __half*)state, (double*)dst, lx, lxp, ly, L, wb);
    else convert_out_kernel<__half, float><<<grid, 256, 0, st>>>((const __half*)state, (float*)dst, lx, lxp, ly, L, wb);
  } else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// out[0] = number of non-finite values, out[1] = max |u|,|v|,|w| (FP64)
template <class TS>
__global__ void check_kernel(const TS* s, size_t n, double* out, size_t plane, const float* wb) {
  __shared__ double sh[2 * 32];
  double v[2] = {0, 0};
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < 4 * n;
       i += size_t(gridDim.x) * blockDim.x) {
    const double a = (wb && i >= 3 * n) ? wval(s[i], wb, (i - 3 * n) % plane) : to_d(s[i]);
    if (!isfinite(a)) v[0] += 1.0;
    else if (i >= n) v[1] = fmax(v[1], fabs(a));
  }
  // max via a separate warp pass: reuse block_sum for the count, max by shuffles
  double m = v[1];
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  double c[1] = {v[0]};
  block_sum<1>(c, sh);
  __shared__ double shm[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) shm[warp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = 0;
    for (int k = 0; k < int((blockDim.x + 31) >> 5); ++k) mm = fmax(mm, shm[k]);
    atomicAdd(&out[0], c[0]);
    unsigned long long* mp = reinterpret_cast<unsigned long long*>(&out[1]);
    unsigned long long old = *mp;
    while (__longlong_as_double(old) < mm) {
      const unsigned long long prev = atomicCAS(mp, old, __double_as_longlong(mm));
      if (prev == old) break;
      old = prev;
    }
  }
}

cudaError_t launch_check(int dtype, const void* state, size_t n_per_field, double* out,
                         cudaStream_t st, int lxp, int ly, const float* wb) {
  cudaError_t e = cudaMemsetAsync(out, 0, 2 * sizeof(double), st);
  if (e) return e;
  const size_t plane = size_t(lxp) * ly;
  if (dtype == FSLBM_F32) check_kernel<float><<<296, 256, 0, st>>>((const float*)state, n_per_field, out, plane, nullptr);
  else if (dtype == FSLBM_F64) check_kernel<double><<<296, 256, 0, st>>>((const double*)state, n_per_field, out, plane, nullptr);
  else if (dtype == FSLBM_F16) check_kernel<__half><<<296, 256, 0, st>>>((const __half*)state, n_per_field, out, plane, plane ? wb : nullptr);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// Compensated FP64 accumulation (Neumaier's variant of Kahan summation): *s holds the running
// sum, *c the rounding error the additions lost; the accumulated value is *s + *c. Long runs add
// thousands of samples into one accumulator, where plain FP64 sums lose about one rounding per
// addition relative to the total.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void comp_add(double* s, double* c, double x) {
  const double a = *s, t = a + x;
  *c += fabs(a) >= fabs(x) ? (a - t) + x : (x - t) + a;
  *s = t;
}

// ------------------------------------------------------------------------------------------
// reference plane statistics (FSLBM.cu:715-748) on the YZ plane x = xs of the reference
// layout: rows y, columns z_ref in [0, L+2*d2); buffer planes are the wrapped core planes with
// p +- pin on non-wall cells, in the storage type's arithmetic as the reference's bcond does.
// acc: 11 arrays of ly*(L+2*d2) running sums, then 11 arrays of their compensations; cnt is
// the mean count including this sample. The deviation is taken from the compensated mean.
// ------------------------------------------------------------------------------------------
template <class TS>
__global__ void plane_stats_kernel(const TS* s, const uint8_t* mask, int planes, int lxp, int ly,
                                   int L, int d2, int xs, double pin_d, int cnt, double* acc,
                                   const float* wb) {
  const int Lr = L + 2 * d2;
  const size_t n = size_t(ly) * Lr, FS = size_t(lxp) * ly * L;
  using TA = typename ArithOf<TS>::type;
  const TA pin = TA(pin_d);
  double* cmp = acc + 11 * n;
  for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n;
       k += size_t(gridDim.x) * blockDim.x) {
    const int y = int(k % ly), zr = int(k / ly);
    int zc = zr - d2, jump = 0;
    if (zc < 0) { zc += L; jump = 1; } else if (zc >= L) { zc -= L; jump = -1; }
    const size_t o = (size_t(zc) * ly + y) * lxp + xs;
    TA p = TA(s[o]);
    if (mask[(planes > 1 ? size_t(zc) * ly : 0) * lxp + size_t(y) * lxp + xs] != kWall) {
      if (jump == 1) p = TA(p + pin);
      else if (jump == -1) p = TA(p - pin);
    }
    const double q[4] = {double(p), to_d(s[FS + o]), to_d(s[2 * FS + o]),
                         wval(s[3 * FS + o], wb, size_t(y) * lxp + xs)};
    const double c = double(cnt);
    double dd[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {           // running mean including this sample, deviation
      comp_add(&acc[f * n + k], &cmp[f * n + k], q[f]);
      dd[f] = (acc[f * n + k] + cmp[f * n + k]) / c - q[f];
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) comp_add(&acc[(4 + f) * n + k], &cmp[(4 + f) * n + k], fabs(dd[f]));
    comp_add(&acc[8 * n + k], &cmp[8 * n + k], dd[1] * dd[2]);
    comp_add(&acc[9 * n + k], &cmp[9 * n + k], dd[1] * dd[3]);
    comp_add(&acc[10 * n + k], &cmp[10 * n + k], dd[3] * dd[2]);
  }
}

cudaError_t launch_plane_stats(int dtype, const void* state, const uint8_t* mask, int planes, int lxp, int ly,
                               int L, int d2, int xs, double pin, int cnt, int, int, double* acc,
                               cudaStream_t st, const float* wb) {
  const int grid = 148;
  if (dtype == FSLBM_F32)
    plane_stats_kernel<float><<<grid, 256, 0, st>>>((const float*)state, mask, planes, lxp, ly, L, d2, xs, pin, cnt, acc, nullptr);
  else if (dtype == FSLBM_F64)
    plane_stats_kernel<double><<<grid, 256, 0, st>>>((const double*)state, mask, planes, lxp, ly, L, d2, xs, pin, cnt, acc, nullptr);
  else if (dtype == FSLBM_F16)
    plane_stats_kernel<__half><<<grid, 256, 0, st>>>((const __half*)state, mask, planes, lxp, ly, L, d2, xs, pin, cnt, acc, wb);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// full-volume profile statistics: per column (x,y), sums over z of p,u,v,w,uu,vv,ww,uv,uw,vw
// (FP64), added to the accumulators with compensation. Block = 32 columns x 8 z-lanes over
// every plane; the lanes' partial sums are combined in a fixed order, so a sample's sums and
// hence the accumulated profile do not depend on scheduling. acc: 10 arrays of lxp*ly sums,
// then 10 arrays of their compensations.
// ------------------------------------------------------------------------------------------
template <class TS>
__global__ void profile_kernel(const TS* s, int lxp, int ly, int L, double* acc, const float* wb) {
  __shared__ double sh[10][8][33];
  const int tx = threadIdx.x & 31, tz = threadIdx.x >> 5;
  const int x = blockIdx.x * 32 + tx, y = blockIdx.y;
  const size_t FS = size_t(lxp) * ly * L, cs = size_t(lxp) * ly;
  double v[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (x < lxp) {
    for (int z = tz; z < L; z += 8) {
      const size_t o = (size_t(z) * ly + y) * lxp + x;
      const double p = to_d(s[o]), u = to_d(s[FS + o]), vv = to_d(s[2 * FS + o]),
                   w = wval(s[3 * FS + o], wb, size_t(y) * lxp + x);
      v[0] += p; v[1] += u; v[2] += vv; v[3] += w;
      v[4] += u * u; v[5] += vv * vv; v[6] += w * w; v[7] += u * vv; v[8] += u * w; v[9] += vv * w;
    }
  }
#pragma unroll
  for (int k = 0; k < 10; ++k) sh[k][tz][tx] = v[k];
  __syncthreads();
  if (tz == 0 && x < lxp) {
    const size_t i = size_t(y) * lxp + x;
#pragma unroll
    for (int k = 0; k < 10; ++k) {
      double t = 0;
      for (int j = 0; j < 8; ++j) t += sh[k][j][tx];
      comp_add(&acc[k * cs + i], &acc[(10 + k) * cs + i], t);
    }
  }
}

cudaError_t launch_profile(int dtype, const void* state, int lxp, int ly, int L, double* acc,
                           cudaStream_t st, const float* wb) {
  dim3 grid((lxp + 31) / 32, ly, 1);
  if (dtype == FSLBM_F32) profile_kernel<float><<<grid, 256, 0, st>>>((const float*)state, lxp, ly, L, acc, nullptr);
  else if (dtype == FSLBM_F64) profile_kernel<double><<<grid, 256, 0, st>>>((const double*)state, lxp, ly, L, acc, nullptr);
  else if (dtype == FSLBM_F16) profile_kernel<__half><<<grid, 256, 0, st>>>((const __half*)state, lxp, ly, L, acc, wb);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

}  // namespace fslbm

namespace fslbm {

bool step_box(int dtype, int d1, int K, int* sw, int* sh, int* hx, int* hy) {
#define X(DT, TS, D, KK)                                                                        \
  if (dtype == DT && d1 == D && K == KK) {                                                      \
    using Tl = StepTile<TS, D, KK>;                                                             \
    *sw = Tl::SW; *sh = Tl::SH; *hx = Tl::HX; *hy = Tl::HY;                                     \
    return true;                                                                                \
  }
  FSLBM_STEP_COMBOS(X)
#undef X
  return false;
}

template <class TS>
__global__ void gather_plane_kernel(const TS* s, int lx, int lxp, int ly, int L, int kind, int idx,
                                    float* out, const float* wb) {
  const size_t FS = size_t(lxp) * ly * L;
  const size_t n = kind == 0 ? size_t(L) * ly : size_t(ly) * lx;
  for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < 4 * n;
       k += size_t(gridDim.x) * blockDim.x) {
    const size_t f = k / n, r = k % n;
    size_t o;
    if (kind == 0) o = (r / ly * ly + r % ly) * lxp + idx;          // r = y + ly*z
    else o = (size_t(idx) * ly + r / lx) * lxp + r % lx;            // r = x + lx*y
    out[k] = float(f == 3 ? wval(s[f * FS + o], wb, o % (size_t(lxp) * ly)) : to_d(s[f * FS + o]));
  }
}

cudaError_t launch_gather_plane(int dtype, const void* state, int lx, int lxp, int ly, int L,
                                int kind, int idx, float* out, cudaStream_t st, const float* wb) {
  if (dtype == FSLBM_F32)
    gather_plane_kernel<float><<<148, 256, 0, st>>>((const float*)state, lx, lxp, ly, L, kind, idx, out, nullptr);
  else if (dtype == FSLBM_F64)
    gather_plane_kernel<double><<<148, 256, 0, st>>>((const double*)state, lx, lxp, ly, L, kind, idx, out, nullptr);
  else if (dtype == FSLBM_F16)
    gather_plane_kernel<__half><<<148, 256, 0, st>>>((const __half*)state, lx, lxp, ly, L, kind, idx, out, wb);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// self-test of the bounded device waits
// ------------------------------------------------------------------------------------------
// Runs the two bounded waits the kernels rely on against conditions nothing will satisfy: the
// gpu-scope counter wait of the chained batched launch (on a counter that stays 0) and the
// mbarrier phase wait of the march (on a barrier nobody arrives at; no copy is issued, so
// nothing is in flight when it gives up). err bit 0 / bit 1 record that each gave up.
__global__ void wait_selftest_kernel(const unsigned* counter, unsigned long long limit_ns,
                                     unsigned* err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  if (!wait_geq_gpu(counter, 1u, limit_ns)) atomicOr(err, 1u);
  mbar_init(&bar, 1);
  mbar_init_fence();
  if (!mbar_wait_bounded(&bar, 0u, limit_ns)) atomicOr(err, 2u);
  mbar_inval(&bar);
}

cudaError_t launch_wait_selftest(const unsigned* counter, unsigned long long limit_ns, unsigned* err,
                                 cudaStream_t st) {
  wait_selftest_kernel<<<1, 32, 0, st>>>(counter, limit_ns, err);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// FP16 storage: the per-column base of w and its share of the step
// ------------------------------------------------------------------------------------------
// Base from dense host-layout fields (4 x L x ly x lx): the streamwise mean of w per non-wall
// column x < lx (FP64 sum in z order), zero elsewhere.
template <class TH>
__global__ void wbase_dense_kernel(const TH* src, const uint8_t* mask, int lx, int lxp, int ly,
                                   int L, float* wb) {
  const size_t n = size_t(lx) * ly * L;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < lxp * ly; i += gridDim.x * blockDim.x) {
    const int x = i % lxp, y = i / lxp;
    float b = 0.0f;
    if (x < lx && mask[i] != kWall) {
      double sum = 0.0;
      for (int z = 0; z < L; ++z) sum += double(src[3 * n + (size_t(z) * ly + y) * lx + x]);
      b = float(sum / double(L));
    }
    wb[i] = b;
  }
}
// The analytic Poiseuille profile of a seeded start: -umax (1 - r^2/R^2) on non-wall columns.
__global__ void wbase_poiseuille_kernel(const uint8_t* mask, int lxp, PoiseuilleInit q, float* wb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < lxp * q.ly; i += gridDim.x * blockDim.x) {
    const int x = i % lxp, y = i / lxp;
    float b = 0.0f;
    if (x < q.lx && mask[i] != kWall) {
      const double dx = x - q.cx, dy = y - q.cy, s2 = (dx * dx + dy * dy) / (q.R * q.R);
      b = float(-q.umax * fmax(0.0, 1.0 - s2));
    }
    wb[i] = b;
  }
}
// Ghost columns of a periodic cross-section take their images' base.
__global__ void wbase_ghosts_kernel(const int2* pairs, int n, float* wb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    wb[pairs[i].x] = wb[pairs[i].y];
}
// The base's share of one step of the stored deviation s = w - wb (w's update is linear in the
// corrector taps): wgt = tb Fz + K1 T1 + K2 T2 + (K0 - 1) wb, with T1 and T2 the base summed over
// the six taps at distance 2 and 4 (the streamwise ones are the column's own base; outside the
// cross-section the base is zero).
__global__ void wgt_kernel(const float* wb, int lxp, int ly, float K0m1, float K1, float K2,
                           float tfz, float* wgt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < lxp * ly; i += gridDim.x * blockDim.x) {
    const int x = i % lxp, y = i / lxp;
    auto b = [&](int xx, int yy) {
      return (xx < 0 || yy < 0 || xx >= lxp || yy >= ly) ? 0.0f : wb[yy * lxp + xx];
    };
    const float c = wb[i];
    const float t1 = __fadd_rn(__fadd_rn(__fadd_rn(b(x - 2, y), b(x + 2, y)), __fadd_rn(b(x, y - 2), b(x, y + 2))),
                               __fadd_rn(c, c));
    const float t2 = __fadd_rn(__fadd_rn(__fadd_rn(b(x - 4, y), b(x + 4, y)), __fadd_rn(b(x, y - 4), b(x, y + 4))),
                               __fadd_rn(c, c));
    wgt[i] = __fmaf_rn(K1, t1, __fmaf_rn(K2, t2, __fmaf_rn(K0m1, c, tfz)));
  }
}

cudaError_t launch_wbase_dense(const void* src, int src_is_f64, const uint8_t* mask, int lx, int lxp,
                               int ly, int L, const int2* ghosts, int nghost, float* wb,
                               cudaStream_t st) {
  const int grid = std::max(1, std::min(592, (lxp * ly + 255) / 256));
  if (src_is_f64) wbase_dense_kernel<double><<<grid, 256, 0, st>>>((const double*)src, mask, lx, lxp, ly, L, wb);
  else wbase_dense_kernel<float><<<grid, 256, 0, st>>>((const float*)src, mask, lx, lxp, ly, L, wb);
  if (nghost > 0) wbase_ghosts_kernel<<<std::min(592, (nghost + 255) / 256), 256, 0, st>>>(ghosts, nghost, wb);
  return cudaGetLastError();
}

cudaError_t launch_wbase_poiseuille(const uint8_t* mask, int lxp, const PoiseuilleInit& q,
                                    const int2* ghosts, int nghost, float* wb, cudaStream_t st) {
  const int grid = std::max(1, std::min(592, (lxp * q.ly + 255) / 256));
  wbase_poiseuille_kernel<<<grid, 256, 0, st>>>(mask, lxp, q, wb);
  if (nghost > 0) wbase_ghosts_kernel<<<std::min(592, (nghost + 255) / 256), 256, 0, st>>>(ghosts, nghost, wb);
  return cudaGetLastError();
}

cudaError_t launch_wgt(const float* wb, int lxp, int ly, float K0, float K1, float K2, float tfz,
                       float* wgt, cudaStream_t st) {
  const int grid = std::max(1, std::min(592, (lxp * ly + 255) / 256));
  wgt_kernel<<<grid, 256, 0, st>>>(wb, lxp, ly, K0 - 1.0f, K1, K2, tfz, wgt);
  return cudaGetLastError();
}

}  // namespace fslbm
