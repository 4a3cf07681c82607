// Host runtime behind the C ABI (include/fslbm.h): contexts, solves, statistics, the batched
// ensemble and the device-side monitor log. The reference keeps all of this in main()
// (FSLBM.cu:489-905); here it is a library with explicit error codes.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <dlfcn.h>

#include "internal.h"

using namespace fslbm;

// ------------------------------------------------------------------------------------------
// errors
// ------------------------------------------------------------------------------------------
static thread_local std::string g_err;
static thread_local int g_err_code = 0;

int fslbm_set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  g_err_code = code;
  return code;
}

#define CUDA_TRY(expr)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (expr);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fslbm_set_error(FSLBM_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)

extern "C" const char* fslbm_version(void) { return "fslbm-b200 0.1"; }

extern "C" int fslbm_last_error(char* buf, size_t n) {
  if (buf && n) {
    std::strncpy(buf, g_err.c_str(), n - 1);
    buf[n - 1] = 0;
  }
  return g_err_code;
}

// ------------------------------------------------------------------------------------------
// context
// ------------------------------------------------------------------------------------------
// Device memory of a context's solves and batches comes from the context's own stream-ordered
// pool, which keeps freed blocks (release threshold: never), so creating and destroying solves
// in a serving loop neither maps nor unmaps device memory nor synchronises the device. All
// set-up copies run on the context's stream, behind the allocations.
// A context is reference-counted: the creator holds one reference and every live solve and
// batch one more, so destroying the context before its solves (an error path, or objects
// finalised in any order at interpreter exit) defers the teardown to the last of them.
struct fslbm_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  int sm_count = 0;
  std::atomic<int> refs{1};
};

static void ctx_retain(fslbm_ctx* c) { c->refs.fetch_add(1); }

static void ctx_release(fslbm_ctx* c) {
  if (c->refs.fetch_sub(1) != 1) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaMemPoolDestroy(c->pool);
  cudaStreamDestroy(c->stream);
  delete c;
}

static cudaError_t ctx_alloc(fslbm_ctx* c, void** p, size_t bytes) {
  return cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 1), c->pool, c->stream);
}

static void ctx_free(fslbm_ctx* c, void* p) {
  if (p) cudaFreeAsync(p, c->stream);
}

extern "C" int fslbm_ctx_create(int device, fslbm_ctx** out) {
  if (!out) return fslbm_set_error(FSLBM_ERR_ARG, "ctx_create: null output");
  int n = 0;
  CUDA_TRY(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n)
    return fslbm_set_error(FSLBM_ERR_ARG, "ctx_create: device %d of %d", device, n);
  CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return fslbm_set_error(FSLBM_ERR_ARG, "ctx_create: device %d is sm_%d%d; the library is compiled for sm_100a",
                           device, prop.major, prop.minor);
  auto* c = new fslbm_ctx;
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (!e) {
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = device;
    e = cudaMemPoolCreate(&c->pool, &pp);
  }
  if (!e) {
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (e) {
    if (c->pool) cudaMemPoolDestroy(c->pool);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return fslbm_set_error(FSLBM_ERR_CUDA, "ctx_create: %s", cudaGetErrorString(e));
  }
  *out = c;
  return FSLBM_OK;
}

extern "C" int fslbm_ctx_destroy(fslbm_ctx* c) {
  if (c) ctx_release(c);
  return FSLBM_OK;
}

// Self-test of the device-side bounded waits (no reference counterpart): both give up after
// limit_ms, the kernel returns, and the error is reported like any other gave-up wait.
extern "C" int fslbm_selftest_waits(fslbm_ctx* c, double limit_ms, unsigned* gave_up) {
  if (!c || !gave_up || !(limit_ms > 0.0) || limit_ms > 10000.0)
    return fslbm_set_error(FSLBM_ERR_ARG, "selftest_waits: bad argument");
  CUDA_TRY(cudaSetDevice(c->device));
  unsigned* d = nullptr;                      // [0] the counter nobody sets, [1] error bits
  CUDA_TRY(ctx_alloc(c, reinterpret_cast<void**>(&d), 2 * sizeof(unsigned)));
  cudaError_t e = cudaMemsetAsync(d, 0, 2 * sizeof(unsigned), c->stream);
  if (!e) e = launch_wait_selftest(d, static_cast<unsigned long long>(limit_ms * 1e6), d + 1, c->stream);
  unsigned err = 0;
  if (!e) e = cudaMemcpyAsync(&err, d + 1, sizeof err, cudaMemcpyDeviceToHost, c->stream);
  ctx_free(c, d);
  if (!e) e = cudaStreamSynchronize(c->stream);
  if (e) return fslbm_set_error(FSLBM_ERR_CUDA, "selftest_waits: %s", cudaGetErrorString(e));
  *gave_up = err;
  if (err) return fslbm_set_error(FSLBM_ERR_TIMEOUT, "selftest_waits: bounded device waits gave up (bits %u)", err);
  return FSLBM_OK;
}

// ------------------------------------------------------------------------------------------
// tensor-map encoding through the driver entry point (no link-time libcuda dependency)
// ------------------------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// ------------------------------------------------------------------------------------------
// solve
// ------------------------------------------------------------------------------------------
struct fslbm_solve {
  fslbm_ctx* ctx = nullptr;
  int lx = 0, ly = 0, L = 0, lxp = 0, d2 = 10;
  double radius = 0, cx = 0, cy = 0;
  bool from_mask = false;          // geometry given as a mask (else the analytic circle)
  int K = 2;                       // corrector taps of prm.fd_order
  int dtype = FSLBM_F32;
  size_t es = 4;
  fslbm_params prm{};
  std::vector<uint8_t> mask;   // lxp*ly, padded columns are wall
  int64_t fluid2d = 0;             // fluid cells of the (first) cross-section
  double l1 = 0;                   // the monitor's l1 (FSLBM.cu:589-591)
  int64_t fluid_total = 0;         // fluid cells of the core
  int planes = 1;                  // mask cross-sections: 1 (extruded) or L (one per plane)
  int ghost = 0;                   // periodic cross-section: ghost band width (0: walls)
  int2* d_ghosts = nullptr;        // (ghost cell, interior image) per ghost cell of a cross-section
  int nghost = 0;
  int sx = 0, sy = 0, sz = 0;  // monitor sample cell
  // device
  void* state[2] = {nullptr, nullptr};
  int cur = 0;
  uint8_t* d_mask = nullptr;
  void* d_colcoef = nullptr;
  int2* d_tiles = nullptr;
  int ntiles = 0, chunk = 0, nchunks = 0;
  CUtensorMap maps[2];
  // FP32 column-pair kernel (even d1): tile height, persistent grid, two maps per buffer
  bool use2 = false;
  int ty2 = 32, grid2 = 0, packed2 = 1;
  std::vector<int> tile_warps[3];  // per column-pair tile: warps holding fluid, [shape] 32 x 2, 16 x 4, 8 x 8
  CUtensorMap maps2p[2], maps2u[2];
  DevCounters* d_counters = nullptr;
  fslbm_monitor* d_log = nullptr;
  int log_cap = 4096;
  int64_t drained = 0;
  double* d_gauge = nullptr;
  unsigned* d_err = nullptr;
  double* d_scratch = nullptr;     // small reductions
  // FP16 storage: stored w is the deviation from the per-column base d_wbase (lxp*ly FP32);
  // d_wgt is the base's share of a step of the stored w (see launch_wgt)
  float* d_wbase = nullptr;
  float* d_wgt = nullptr;
  double* d_stats = nullptr;       // 11 * ly * (L + 2 d2) sums, then their 11 compensations
  int cnt = 0, cnt2 = 0;
  double* d_prof = nullptr;        // 10 * lxp * ly sums, then their 10 compensations
  int64_t prof_n = 0;
  void* d_stage = nullptr;         // conversion staging (dense 4 fields)
  size_t stage_bytes = 0;
  float* d_plane = nullptr;        // plane gather buffer
  int64_t steps = 0;
  bool fields_set = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0;
  int64_t bytes_device = 0;
  int64_t launches = 0;            // kernels launched by this solve
  bool timing = false;             // bracket every step launch with events
  std::vector<cudaEvent_t> tev;    // event pairs of the launches since the last read
  size_t tev_used = 0;
};

static size_t field_stride(const fslbm_solve* s) { return size_t(s->lxp) * s->ly * s->L; }

// Mask byte of cell (x, y) in core plane z (one cross-section, or one per plane).
static uint8_t mask_at(const fslbm_solve* s, int x, int y, int z) {
  return s->mask[((s->planes > 1 ? size_t(z) : 0) * s->ly + y) * s->lxp + x];
}

// Milliseconds between two events, if both were recorded. A failed query (events never
// recorded) is cleared from the runtime's last-error slot, where a later launch check would
// otherwise report it.
static void elapsed_if_recorded(cudaEvent_t a, cudaEvent_t b, double* out) {
  float ms = 0;
  if (cudaEventElapsedTime(&ms, a, b) == cudaSuccess) *out = ms;
  else (void)cudaGetLastError();
}

static int validate_params(const fslbm_params* p, int dtype) {
  if (!p) return fslbm_set_error(FSLBM_ERR_ARG, "params: null");
  double c[9];
  const int K = fd_coefficients(p->fd_order, p->blend, dtype != FSLBM_F64, c);
  if (K == 0) return fslbm_set_error(FSLBM_ERR_ARG, "params: unknown corrector order %d", p->fd_order);
  if (!step_supported(dtype, p->d1, K))
    return fslbm_set_error(FSLBM_ERR_ARG, "params: d1=%d with corrector order %d is not supported for dtype %d",
                           p->d1, p->fd_order, dtype);
  if (!std::isfinite(p->tblend) || !std::isfinite(p->pin) || !std::isfinite(p->nu) ||
      !std::isfinite(p->blend))
    return fslbm_set_error(FSLBM_ERR_ARG, "params: non-finite value");
  if (p->monitor_every < 0) return fslbm_set_error(FSLBM_ERR_ARG, "params: monitor_every < 0");
  if (p->delta < 0 || p->delta > 2) return fslbm_set_error(FSLBM_ERR_ARG, "params: delta must be 0, 1 or 2");
  return FSLBM_OK;
}

// Tensor maps of the column-pair kernel with tile height ty over the solve's two state buffers:
// the p box (one-cell halo) and the u,v,w box (the corrector's halo).
static int encode_pair_maps(const fslbm_solve* s, int ty, CUtensorMap mp[2], CUtensorMap mu[2]) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return fslbm_set_error(FSLBM_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  const CUtensorMapDataType dt = s->dtype == FSLBM_F64   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                 : s->dtype == FSLBM_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                         : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  int sw2, ph, uh, hx2, hy2;
  if (!step2_box(s->dtype, s->prm.d1, ty, &sw2, &ph, &uh, &hx2, &hy2))
    return fslbm_set_error(FSLBM_ERR_ARG, "no column-pair kernel for d1 %d, tile height %d", s->prm.d1, ty);
  cuuint64_t dims[4] = {cuuint64_t(s->lxp), cuuint64_t(s->ly), cuuint64_t(s->L), 4};
  cuuint64_t strides[3] = {cuuint64_t(s->lxp) * s->es, cuuint64_t(s->lxp) * s->ly * s->es,
                           cuuint64_t(field_stride(s)) * s->es};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  cuuint32_t boxp[4] = {cuuint32_t(sw2), cuuint32_t(ph), 1, 1};
  cuuint32_t boxu[4] = {cuuint32_t(sw2), cuuint32_t(uh), 1, 3};
  for (int b = 0; b < 2; ++b) {
    CUresult r = enc(&mp[b], dt, 4, s->state[b], dims, strides, boxp, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r == CUDA_SUCCESS)
      r = enc(&mu[b], dt, 4, s->state[b], dims, strides, boxu, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
      return fslbm_set_error(FSLBM_ERR_CUDA, "cuTensorMapEncodeTiled (pair kernel) failed (%d)", int(r));
  }
  return FSLBM_OK;
}

static int build_tensor_maps(fslbm_solve* s) {
  if (s->use2) return encode_pair_maps(s, s->ty2, s->maps2p, s->maps2u);
  EncodeTiledFn enc = encode_fn();
  if (!enc) return fslbm_set_error(FSLBM_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  const CUtensorMapDataType dt = s->dtype == FSLBM_F64   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                 : s->dtype == FSLBM_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                         : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  int sw, sh, hx, hy;
  if (!step_box(s->dtype, s->prm.d1, s->K, &sw, &sh, &hx, &hy))
    return fslbm_set_error(FSLBM_ERR_ARG, "no step kernel for dtype %d d1 %d", s->dtype, s->prm.d1);
  cuuint64_t dims[4] = {cuuint64_t(s->lxp), cuuint64_t(s->ly), cuuint64_t(s->L), 4};
  cuuint64_t strides[3] = {cuuint64_t(s->lxp) * s->es, cuuint64_t(s->lxp) * s->ly * s->es,
                           cuuint64_t(field_stride(s)) * s->es};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  cuuint32_t box[4] = {cuuint32_t(sw), cuuint32_t(sh), 1, 4};
  for (int b = 0; b < 2; ++b) {
    const CUresult r = enc(&s->maps[b], dt, 4, s->state[b], dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
      return fslbm_set_error(FSLBM_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", int(r));
  }
  return FSLBM_OK;
}

// Tile list (tiles holding fluid) for a tile of kTX x th cells.
static std::vector<int2> fluid_tiles(const fslbm_solve* s, int th) {
  std::vector<int2> tiles;
  for (int y0 = 0; y0 < s->ly; y0 += th)
    for (int x0 = 0; x0 < s->lxp; x0 += kTX) {
      bool any = false;
      for (int z = 0; z < s->planes && !any; ++z)
        for (int y = y0; y < std::min(y0 + th, s->ly) && !any; ++y)
          for (int x = x0; x < std::min(x0 + kTX, s->lxp); ++x)
            if (s->mask[(size_t(z) * s->ly + y) * s->lxp + x] == 0) { any = true; break; }
      if (any) tiles.push_back(make_int2(x0, y0));
    }
  return tiles;
}

// Warps of each column-pair tile (32 x ty cells) that hold fluid, for the three warp shapes:
// warps[0] 32 x 2 cells, warps[1] 16 x 4 cells, warps[2] 8 x 8 cells (the kernel's lane maps).
static void tile_warp_counts(const fslbm_solve* s, const std::vector<int2>& tiles, int ty,
                             std::vector<int> (&warps)[3]) {
  static const int kWx[3] = {32, 16, 8}, kWy[3] = {2, 4, 8};
  for (const int2 org : tiles)
    for (int shape = 0; shape < 3; ++shape) {
      const int wx = kWx[shape], wy = kWy[shape], across = 32 / wx;
      int n = 0;
      for (int w = 0; w < ty / 2; ++w) {
        const int x0 = org.x + wx * (w % across), y0 = org.y + wy * (w / across);
        bool any = false;
        for (int y = y0; y < std::min(y0 + wy, s->ly) && !any; ++y)
          for (int x = x0; x < std::min(x0 + wx, s->lxp) && !any; ++x)
            any = s->mask[size_t(y) * s->lxp + x] == 0;
        n += any;
      }
      warps[shape].push_back(n);
    }
}

static void choose_chunks(fslbm_solve* s);

// Selects the step kernel for the current dtype and d1, uploads its tile list, builds its
// tensor maps and sizes its grid. FSLBM_STEP_KERNEL=1 forces the one-column kernel and
// FSLBM_PACKED=0 uses scalar pair arithmetic and FSLBM_TILE_Y=16|32 picks the column-pair kernel's tile height (for comparisons).
static int configure_kernel(fslbm_solve* s) {
  const char* ek = std::getenv("FSLBM_STEP_KERNEL");
  const char* et = std::getenv("FSLBM_TILE_Y");
  double cf[9];
  s->K = fd_coefficients(s->prm.fd_order, s->prm.blend, s->dtype != FSLBM_F64, cf);
  // FP16 storage exists only in the column-pair kernel, which has the 2-tap corrector
  s->use2 = step2_supported(s->dtype, s->prm.d1) && s->K == 2 && s->planes == 1 &&
            (s->dtype == FSLBM_F16 || !(ek && std::atoi(ek) == 1));
  // FP64 runs the column kernel on 32 x 16 tiles
  s->ty2 = (s->dtype == FSLBM_F64 || (et && std::atoi(et) == 16)) ? 16 : 32;
  const char* ep = std::getenv("FSLBM_PACKED");
  s->packed2 = (ep && std::atoi(ep) == 0) ? 0 : 1;
  const std::vector<int2> tiles = fluid_tiles(s, s->use2 ? s->ty2 : kTY);
  for (auto& v : s->tile_warps) v.clear();
  if (s->use2) tile_warp_counts(s, tiles, s->ty2, s->tile_warps);
  if (s->d_tiles) {
    ctx_free(s->ctx, s->d_tiles);
    s->bytes_device -= int64_t(s->ntiles) * sizeof(int2);
    s->d_tiles = nullptr;
  }
  s->ntiles = int(tiles.size());
  CUDA_TRY(ctx_alloc(s->ctx, reinterpret_cast<void**>(&s->d_tiles), tiles.size() * sizeof(int2)));
  s->bytes_device += int64_t(tiles.size() * sizeof(int2));
  CUDA_TRY(cudaMemcpyAsync(s->d_tiles, tiles.data(), tiles.size() * sizeof(int2),
                           cudaMemcpyHostToDevice, s->ctx->stream));
  if (s->use2) {
    CUDA_TRY(step2_prepare(s->dtype, s->prm.d1, s->ty2));
    // tiles x streamwise chunks, at most one CTA per SM slot and chunks of at least 2R planes
    // (chunk counts weighted by each tile's fluid warps measured no faster: a tile with wall in
    // it is not proportionally faster per plane)
    const int slots = s->ctx->sm_count * step2_occupancy(s->dtype, s->prm.d1, s->ty2);
    int nch = std::max(1, slots / s->ntiles);
    nch = std::min(nch, std::max(1, s->L / (4 * s->prm.d1)));
    s->grid2 = s->ntiles * nch;
  } else {
    CUDA_TRY(step_prepare(s->dtype, s->prm.d1, s->K));
    choose_chunks(s);
  }
  return build_tensor_maps(s);
}

// Static wall sums per column (see step_kernel.cuh): sums of w(cx)w(cy) cx^a cy^b over the
// wall cells of the 3x3 cross-section neighbourhood; outside the box counts as wall.
template <class TC>
static std::vector<ColCoef<TC>> column_coefs(const fslbm_solve* s) {
  std::vector<ColCoef<TC>> cc(size_t(s->lxp) * s->ly);
  const double wv[3] = {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0};
  for (int y = 0; y < s->ly; ++y)
    for (int x = 0; x < s->lxp; ++x) {
      double a = 0, bx = 0, by = 0;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int gx = x + dx, gy = y + dy;
          const bool wall = gx < 0 || gy < 0 || gx >= s->lxp || gy >= s->ly ||
                            s->mask[size_t(gy) * s->lxp + gx] == kWall;
          if (!wall) continue;
          const double w = wv[dx + 1] * wv[dy + 1];
          a += w; bx += dx * w; by += dy * w;
        }
      ColCoef<TC>& c = cc[size_t(y) * s->lxp + x];
      c.ws0 = TC(a); c.wsx = TC(bx); c.wsy = TC(by);
      c.fluid = TC(s->mask[size_t(y) * s->lxp + x] == 0 ? 1 : 0);
    }
  return cc;
}

// Wall sums per cell for masks that vary along z: sums of w(cx)w(cy)w(cz) c^k over the wall
// cells of the 3x3x3 neighbourhood (periodic in z, outside the cross-section counts as wall).
template <class TC>
static std::vector<CellCoef<TC>> cell_coefs(const fslbm_solve* s) {
  const size_t plane = size_t(s->lxp) * s->ly;
  std::vector<CellCoef<TC>> cc(plane * s->L);
  const double wv[3] = {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0};
  for (int z = 0; z < s->L; ++z)
    for (int y = 0; y < s->ly; ++y)
      for (int x = 0; x < s->lxp; ++x) {
        double a = 0, bx = 0, by = 0, bz = 0;
        for (int dz = -1; dz <= 1; ++dz) {
          const int gz = (z + dz + s->L) % s->L;
          for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
              const int gx = x + dx, gy = y + dy;
              const bool wall = gx < 0 || gy < 0 || gx >= s->lxp || gy >= s->ly ||
                                s->mask[gz * plane + size_t(gy) * s->lxp + gx] == kWall;
              if (!wall) continue;
              const double w = wv[dx + 1] * wv[dy + 1] * wv[dz + 1];
              a += w; bx += dx * w; by += dy * w; bz += dz * w;
            }
        }
        CellCoef<TC>& c = cc[z * plane + size_t(y) * s->lxp + x];
        c.ws0 = TC(a); c.wsx = TC(bx); c.wsy = TC(by); c.wsz = TC(bz);
      }
  return cc;
}

// Picks the streamwise chunking: minimises waves * (chunk + 2R) over chunk counts.
static void choose_chunks(fslbm_solve* s) {
  int occ = 1;
  const size_t smem = step_smem_bytes(s->dtype, s->prm.d1, s->K);
  occ = s->dtype == FSLBM_F64 ? 1 : 2;
  if (smem * occ > 227 * 1024) occ = 1;
  const int slots = std::max(1, s->ctx->sm_count * occ);
  const int R = s->K * s->prm.d1;
  double best = 1e300;
  int best_n = 1;
  for (int n = 1; n <= s->L; ++n) {
    const int chunk = (s->L + n - 1) / n;
    if (n > 1 && chunk < 2 * R) break;
    const int ctas = s->ntiles * n;
    const int waves = (ctas + slots - 1) / slots;
    const double t = double(waves) * double(chunk + 2 * R);
    if (t < best - 1e-9) { best = t; best_n = n; }
  }
  s->nchunks = best_n;
  s->chunk = (s->L + best_n - 1) / best_n;
  s->nchunks = (s->L + s->chunk - 1) / s->chunk;
}

static void free_solve(fslbm_solve* s) {
  if (!s) return;
  cudaSetDevice(s->ctx->device);
  void* ptrs[] = {s->state[0], s->state[1], s->d_mask, s->d_colcoef, s->d_tiles, s->d_ghosts, s->d_counters,
                  s->d_log, s->d_gauge, s->d_err, s->d_scratch, s->d_stats, s->d_prof,
                  s->d_stage, s->d_plane, s->d_wbase, s->d_wgt};
  for (void* p : ptrs) ctx_free(s->ctx, p);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  for (cudaEvent_t e : s->tev) cudaEventDestroy(e);
  fslbm_ctx* c = s->ctx;
  delete s;
  ctx_release(c);
}

template <class T>
static cudaError_t dalloc(fslbm_solve* s, T** p, size_t bytes) {
  cudaError_t e = ctx_alloc(s->ctx, reinterpret_cast<void**>(p), bytes);
  if (!e) s->bytes_device += int64_t(bytes);
  return e;
}

extern "C" int fslbm_solve_create(fslbm_ctx* ctx, const fslbm_domain* dom, const fslbm_params* prm,
                                  fslbm_dtype dtype, fslbm_solve** out) {
  if (!ctx || !dom || !out) return fslbm_set_error(FSLBM_ERR_ARG, "solve_create: null argument");
  if (dtype != FSLBM_F32 && dtype != FSLBM_F64 && dtype != FSLBM_F16)
    return fslbm_set_error(FSLBM_ERR_ARG, "solve_create: dtype %d is not available", int(dtype));
  int rc = validate_params(prm, dtype);
  if (rc) return rc;
  if (dom->lx < 3 || dom->ly < 3 || dom->lz < 1)
    return fslbm_set_error(FSLBM_ERR_ARG, "solve_create: box %dx%dx%d too small", dom->lx, dom->ly, dom->lz);
  double cf[9];
  const int R = fd_coefficients(prm->fd_order, prm->blend, dtype != FSLBM_F64, cf) * prm->d1;
  if (dom->lz < std::max(R, 1) + 1)
    return fslbm_set_error(FSLBM_ERR_ARG, "solve_create: streamwise period %d shorter than the stencil reach %d",
                           dom->lz, R + 1);
  if (dom->buffer_depth < 0 || (dom->buffer_depth > 0 && dom->buffer_depth > dom->lz))
    return fslbm_set_error(FSLBM_ERR_ARG, "solve_create: buffer_depth %d out of range", dom->buffer_depth);
  CUDA_TRY(cudaSetDevice(ctx->device));

  auto* s = new fslbm_solve;
  s->ctx = ctx;
  ctx_retain(ctx);
  s->lx = dom->lx; s->ly = dom->ly; s->L = dom->lz;
  s->lxp = (dom->lx + 7) / 8 * 8;
  s->d2 = dom->buffer_depth;
  s->dtype = dtype;
  s->es = dtype == FSLBM_F64 ? 8 : (dtype == FSLBM_F16 ? 2 : 4);
  s->prm = *prm;
  if (dom->mask_planes > 1 && (dom->mask_planes != dom->lz || !dom->mask)) {
    free_solve(s);
    return fslbm_set_error(FSLBM_ERR_ARG, "solve_create: mask_planes must be 0, 1 or lz (%d) with a mask", dom->lz);
  }
  s->planes = dom->mask_planes > 1 ? dom->lz : 1;
  // periodic cross-section: the band G cells wide at the rim takes the periodic images of the
  // interior (2 where the image is fluid, 125 where it is wall)
  std::vector<uint8_t> pmask;
  if (dom->periodic_xy > 0) {
    const int G = dom->periodic_xy, nx = dom->lx - 2 * G, ny = dom->ly - 2 * G;
    double cf[9];
    const int reach = fd_coefficients(prm->fd_order, prm->blend, dtype != FSLBM_F64, cf) * prm->d1;
    if (s->planes > 1 || nx < 1 || ny < 1 || G < std::max(1, reach)) {
      free_solve(s);
      return fslbm_set_error(FSLBM_ERR_ARG,
                             "solve_create: periodic_xy %d needs one cross-section, an interior of at "
                             "least one cell and a band at least the corrector reach %d wide", G, reach);
    }
    s->ghost = G;
    pmask.assign(size_t(dom->lx) * dom->ly, 0);
    for (int y = 0; y < dom->ly; ++y)
      for (int x = 0; x < dom->lx; ++x) {
        const int sx = G + ((x - G) % nx + nx) % nx, sy = G + ((y - G) % ny + ny) % ny;
        const uint8_t src = dom->mask ? dom->mask[size_t(sy) * dom->lx + sx] : uint8_t(0);
        if (src != 0 && src != kWall) {
          free_solve(s);
          return fslbm_set_error(FSLBM_ERR_ARG, "solve_create: mask value %d at (%d,%d); expected 0 or 125",
                                 int(src), sx, sy);
        }
        const bool band = sx != x || sy != y;
        pmask[size_t(y) * dom->lx + x] = band ? (src == kWall ? kWall : kGhost) : src;
      }
  }
  const size_t plane = size_t(s->lxp) * s->ly;
  s->mask.assign(plane * s->planes, kWall);
  std::vector<int64_t> per_plane(s->planes, 0);
  double sxs = 0, sys = 0;
  for (int z = 0; z < s->planes; ++z)
    for (int y = 0; y < s->ly; ++y)
      for (int x = 0; x < s->lx; ++x) {
        uint8_t v;
        if (!pmask.empty()) {
          v = pmask[size_t(y) * s->lx + x];
          if (v != 0 && v != kWall && v != kGhost) {
            free_solve(s);
            return fslbm_set_error(FSLBM_ERR_ARG, "solve_create: mask value %d at (%d,%d); expected 0 or 125", v, x, y);
          }
        } else if (dom->mask) {
          v = dom->mask[(size_t(z) * s->ly + y) * s->lx + x];
          if (v != 0 && v != kWall) {
            free_solve(s);
            return fslbm_set_error(FSLBM_ERR_ARG, "solve_create: mask value %d at (%d,%d,%d); expected 0 or 125",
                                   v, x, y, z);
          }
        } else {
          const double dx = x - dom->cx, dy = y - dom->cy;
          v = (dx * dx + dy * dy <= dom->radius * dom->radius) ? 0 : kWall;
        }
        if (v == 0 && (x == 0 || y == 0 || x == s->lx - 1 || y == s->ly - 1)) {
          free_solve(s);
          return fslbm_set_error(FSLBM_ERR_ARG,
                                 "solve_create: fluid cell (%d,%d,%d) on the box rim; the cross-section must "
                                 "be enclosed by wall", x, y, z);
        }
        s->mask[z * plane + size_t(y) * s->lxp + x] = v;
        if (v == 0) { ++per_plane[z]; sxs += x; sys += y; }
      }
  for (int64_t c : per_plane) s->fluid_total += c;
  if (s->planes == 1) s->fluid_total *= s->L;
  if (s->fluid_total == 0) {
    free_solve(s);
    return fslbm_set_error(FSLBM_ERR_ARG, "solve_create: no fluid cells");
  }
  // l1 of the monitor: the reference counts its buffer cells over 2*d2 planes (FSLBM.cu:589-591),
  // i.e. the mean fluid count of the core planes the buffers copy
  {
    const int d2 = std::max(1, std::min(s->d2 > 0 ? s->d2 : 1, s->L));
    int64_t c = 0;
    for (int j = 0; j < d2; ++j) c += per_plane[s->planes == 1 ? 0 : j] + per_plane[s->planes == 1 ? 0 : s->L - 1 - j];
    s->l1 = double(c) / double(2 * d2);
    if (s->l1 <= 0) s->l1 = 1.0;
    s->fluid2d = per_plane[0];
  }
  const double nfl = s->planes == 1 ? double(per_plane[0]) : double(s->fluid_total);
  s->from_mask = dom->mask != nullptr;
  s->radius = dom->radius > 0 ? dom->radius : std::sqrt(double(s->fluid_total) / s->L / M_PI);
  s->cx = dom->mask ? sxs / nfl : dom->cx;
  s->cy = dom->mask ? sys / nfl : dom->cy;
  // monitor sample: linear index (ly*lx)/2 + lx/2 of the plane z = lz_ref/2 (FSLBM.cu:653,665)
  {
    const long idx = (long(s->ly) * s->lx) / 2 + s->lx / 2;
    s->sx = int(idx % s->lx);
    s->sy = int(idx / s->lx);
    if (s->sy >= s->ly) s->sy = s->ly - 1;
    s->sz = s->L / 2;
  }

  const size_t fs = field_stride(s);
  cudaError_t e = cudaSuccess;
  auto fail = [&](const char* what) {
    const int r = fslbm_set_error(FSLBM_ERR_CUDA, "solve_create: %s: %s", what, cudaGetErrorString(e));
    free_solve(s);
    return r;
  };
  // set-up on the context's stream (pageable host sources are staged before each call returns)
  cudaStream_t st = ctx->stream;
  for (int b = 0; b < 2; ++b) {
    if ((e = dalloc(s, &s->state[b], 4 * fs * s->es))) return fail("state");
    if ((e = cudaMemsetAsync(s->state[b], 0, 4 * fs * s->es, st))) return fail("memset");
  }
  if ((e = dalloc(s, &s->d_mask, s->mask.size()))) return fail("mask");
  if ((e = cudaMemcpyAsync(s->d_mask, s->mask.data(), s->mask.size(), cudaMemcpyHostToDevice, st)))
    return fail("mask copy");
  if (s->planes > 1 && dtype == FSLBM_F16) {
    e = cudaErrorInvalidValue;
    const int r = fslbm_set_error(FSLBM_ERR_ARG, "solve_create: masks varying along z need FP32 or FP64 storage");
    free_solve(s);
    return r;
  }
  if (s->planes > 1 && dtype == FSLBM_F64) {
    auto cc = cell_coefs<double>(s);
    if ((e = dalloc(s, &s->d_colcoef, cc.size() * sizeof(cc[0])))) return fail("colcoef");
    e = cudaMemcpyAsync(s->d_colcoef, cc.data(), cc.size() * sizeof(cc[0]), cudaMemcpyHostToDevice, st);
    if (!e) e = cudaStreamSynchronize(st);       // the table is a local vector
  } else if (s->planes > 1) {
    auto cc = cell_coefs<float>(s);
    if ((e = dalloc(s, &s->d_colcoef, cc.size() * sizeof(cc[0])))) return fail("colcoef");
    e = cudaMemcpyAsync(s->d_colcoef, cc.data(), cc.size() * sizeof(cc[0]), cudaMemcpyHostToDevice, st);
    if (!e) e = cudaStreamSynchronize(st);
  } else if (dtype == FSLBM_F64) {
    auto cc = column_coefs<double>(s);
    if ((e = dalloc(s, &s->d_colcoef, cc.size() * sizeof(cc[0])))) return fail("colcoef");
    e = cudaMemcpyAsync(s->d_colcoef, cc.data(), cc.size() * sizeof(cc[0]), cudaMemcpyHostToDevice, st);
  } else {
    auto cc = column_coefs<float>(s);
    if ((e = dalloc(s, &s->d_colcoef, cc.size() * sizeof(cc[0])))) return fail("colcoef");
    e = cudaMemcpyAsync(s->d_colcoef, cc.data(), cc.size() * sizeof(cc[0]), cudaMemcpyHostToDevice, st);
  }
  if (e) return fail("colcoef copy");
  if ((e = dalloc(s, &s->d_counters, sizeof(DevCounters)))) return fail("counters");
  if ((e = cudaMemsetAsync(s->d_counters, 0, sizeof(DevCounters), st))) return fail("memset");
  if ((e = dalloc(s, &s->d_log, sizeof(fslbm_monitor) * s->log_cap))) return fail("log");
  if ((e = dalloc(s, &s->d_gauge, sizeof(double)))) return fail("gauge");
  if ((e = cudaMemsetAsync(s->d_gauge, 0, sizeof(double), st))) return fail("memset");
  if ((e = dalloc(s, &s->d_err, sizeof(unsigned)))) return fail("err");
  if ((e = cudaMemsetAsync(s->d_err, 0, sizeof(unsigned), st))) return fail("memset");
  if ((e = dalloc(s, &s->d_scratch, 8 * sizeof(double)))) return fail("scratch");
  if (dtype == FSLBM_F16) {
    const size_t cs = size_t(s->lxp) * s->ly * sizeof(float);
    if ((e = dalloc(s, &s->d_wbase, cs)) || (e = dalloc(s, &s->d_wgt, cs))) return fail("w base");
    if ((e = cudaMemsetAsync(s->d_wbase, 0, cs, st)) || (e = cudaMemsetAsync(s->d_wgt, 0, cs, st)))
      return fail("memset");
  }
  if (s->ghost > 0) {
    const int G = s->ghost, nx = s->lx - 2 * G, ny = s->ly - 2 * G;
    std::vector<int2> pairs;
    for (int y = 0; y < s->ly; ++y)
      for (int x = 0; x < s->lx; ++x) {
        if (s->mask[size_t(y) * s->lxp + x] != kGhost) continue;
        const int sx = G + ((x - G) % nx + nx) % nx, sy = G + ((y - G) % ny + ny) % ny;
        pairs.push_back(make_int2(y * s->lxp + x, sy * s->lxp + sx));
      }
    s->nghost = int(pairs.size());
    if ((e = dalloc(s, &s->d_ghosts, pairs.size() * sizeof(int2)))) return fail("ghosts");
    if ((e = cudaMemcpyAsync(s->d_ghosts, pairs.data(), pairs.size() * sizeof(int2),
                             cudaMemcpyHostToDevice, st)))
      return fail("ghosts copy");
    if ((e = cudaStreamSynchronize(st))) return fail("ghosts copy");   // pairs is a local vector
  }
  if ((e = cudaEventCreate(&s->ev0)) || (e = cudaEventCreate(&s->ev1))) return fail("events");
  if (int r = configure_kernel(s)) { free_solve(s); return r; }
  *out = s;
  return FSLBM_OK;
}

extern "C" int fslbm_solve_destroy(fslbm_solve* s) {
  free_solve(s);
  return FSLBM_OK;
}

static void fill_constants(const fslbm_solve* s, StepLaunch& a);

// FP16 storage: the base's share of a step of the stored w, from the current parameters.
static int update_wgt(fslbm_solve* s) {
  if (!s->d_wgt) return FSLBM_OK;
  StepLaunch a{};
  fill_constants(s, a);
  // the step kernel's folded constants, formed the same way (FP32, K0 with one fused rounding)
  const float tb = float(a.tb), am = (tb * float(a.dtddy)) * float(a.m);
  const float K0 = std::fmaf(am, float(a.c0), float(a.cc)), K1 = am * float(a.c1), K2 = am * float(a.c2);
  CUDA_TRY(launch_wgt(s->d_wbase, s->lxp, s->ly, K0, K1, K2, tb * float(a.fz), s->d_wgt,
                      s->ctx->stream));
  return FSLBM_OK;
}

extern "C" int fslbm_solve_set_params(fslbm_solve* s, const fslbm_params* prm) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "set_params: null solve");
  int rc = validate_params(prm, s->dtype);
  if (rc) return rc;
  const bool d1_changed = prm->d1 != s->prm.d1 || prm->fd_order != s->prm.fd_order;
  s->prm = *prm;
  if (d1_changed) {
    CUDA_TRY(cudaSetDevice(s->ctx->device));
    CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
    if (int r = configure_kernel(s)) return r;
  }
  if (s->d_wgt) {
    CUDA_TRY(cudaSetDevice(s->ctx->device));
    if (int r = update_wgt(s)) return r;
  }
  return FSLBM_OK;
}

static int ensure_stage(fslbm_solve* s, size_t bytes) {
  if (s->stage_bytes >= bytes) return FSLBM_OK;
  if (s->d_stage) {
    ctx_free(s->ctx, s->d_stage);
    s->bytes_device -= int64_t(s->stage_bytes);
    s->d_stage = nullptr;
    s->stage_bytes = 0;
  }
  CUDA_TRY(dalloc(s, &s->d_stage, bytes));
  s->stage_bytes = bytes;
  return FSLBM_OK;
}

extern "C" int fslbm_solve_set_fields(fslbm_solve* s, fslbm_dtype hd, const void* p, const void* u,
                                      const void* v, const void* w) {
  if (!s || !p || !u || !v || !w) return fslbm_set_error(FSLBM_ERR_ARG, "set_fields: null argument");
  if (hd != FSLBM_F64 && hd != FSLBM_F32)
    return fslbm_set_error(FSLBM_ERR_ARG, "set_fields: host dtype must be F64 or F32");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  const size_t n = size_t(s->lx) * s->ly * s->L, hes = hd == FSLBM_F64 ? 8 : 4;
  cudaStream_t st = s->ctx->stream;
  void* dst = s->state[s->cur];
  if (int(hd) == s->dtype && s->lx == s->lxp) {
    // same type and no pitch padding: one contiguous copy per field straight into the state
    // (narrow pitched rows would make slow DMA; those go through the staging buffer)
    const void* src[4] = {p, u, v, w};
    for (int f = 0; f < 4; ++f)
      CUDA_TRY(cudaMemcpy2DAsync(static_cast<char*>(dst) + f * field_stride(s) * s->es,
                                 size_t(s->lxp) * s->es, src[f], size_t(s->lx) * hes,
                                 size_t(s->lx) * hes, size_t(s->ly) * s->L,
                                 cudaMemcpyHostToDevice, st));
  } else {
    if (int r = ensure_stage(s, 4 * n * hes)) return r;
    const void* src[4] = {p, u, v, w};
    for (int f = 0; f < 4; ++f)
      CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(s->d_stage) + f * n * hes, src[f], n * hes,
                               cudaMemcpyHostToDevice, st));
    if (s->d_wbase)                 // FP16: w is stored as the deviation from its column mean
      CUDA_TRY(launch_wbase_dense(s->d_stage, hd == FSLBM_F64, s->d_mask, s->lx, s->lxp, s->ly, s->L,
                                  s->d_ghosts, s->nghost, s->d_wbase, st));
    CUDA_TRY(launch_convert_in(s->dtype, dst, s->d_stage, hd == FSLBM_F64, s->lx, s->lxp, s->ly,
                               s->L, st, s->d_wbase));
  }
  CUDA_TRY(launch_zero_walls(s->dtype, dst, s->d_mask, s->planes, s->lxp, s->ly, s->L, st));
  CUDA_TRY(launch_fill_ghosts(s->dtype, dst, s->d_ghosts, s->nghost, s->lxp, s->ly, s->L, st));
  // the other buffer's walls (never written by the step) must be zero too
  CUDA_TRY(launch_zero_walls(s->dtype, s->state[1 - s->cur], s->d_mask, s->planes, s->lxp, s->ly, s->L, st));
  if (int r = update_wgt(s)) return r;
  s->fields_set = true;
  return FSLBM_OK;
}

int fslbm_poiseuille_setup(const fslbm_domain* dom, double umax, double noise, int modes,
                           double mode_amp, uint64_t seed, fslbm::PoiseuilleInit* q,
                           std::vector<uint8_t>* fluid_out);

extern "C" int fslbm_solve_init_poiseuille(fslbm_solve* s, double umax, double noise, int modes,
                                           double mode_amp, uint64_t seed) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "init_poiseuille: null solve");
  std::vector<uint8_t> dense;
  fslbm_domain dom{};
  dom.lx = s->lx; dom.ly = s->ly; dom.lz = s->L;
  dom.radius = s->radius; dom.cx = s->cx; dom.cy = s->cy; dom.buffer_depth = s->d2;
  if (s->from_mask) {
    dense.resize(size_t(s->lx) * s->ly);
    for (int y = 0; y < s->ly; ++y)
      for (int x = 0; x < s->lx; ++x) dense[size_t(y) * s->lx + x] = s->mask[size_t(y) * s->lxp + x];
    dom.mask = dense.data();
  }
  PoiseuilleInit q;
  std::vector<uint8_t> fluid;
  if (int r = fslbm_poiseuille_setup(&dom, umax, noise, modes, mode_amp, seed, &q, &fluid)) return r;
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  cudaStream_t st = s->ctx->stream;
  if (s->d_wbase)                     // FP16: w is stored as the deviation from the profile
    CUDA_TRY(launch_wbase_poiseuille(s->d_mask, s->lxp, q, s->d_ghosts, s->nghost, s->d_wbase, st));
  CUDA_TRY(launch_init_poiseuille(s->dtype, s->state[s->cur], s->d_mask, s->planes, s->lxp, q, st,
                                  s->d_wbase));
  CUDA_TRY(launch_fill_ghosts(s->dtype, s->state[s->cur], s->d_ghosts, s->nghost, s->lxp, s->ly,
                              s->L, st));
  CUDA_TRY(launch_zero_walls(s->dtype, s->state[1 - s->cur], s->d_mask, s->planes, s->lxp, s->ly, s->L, st));
  if (int r = update_wgt(s)) return r;
  s->fields_set = true;
  return FSLBM_OK;
}

// Device bytes fslbm_solve_create allocates for this domain and dtype (state ping-pong, mask,
// column sums, tile list, monitor log and small buffers). Host-layout copies in or out
// (set/get fields) of a solve whose storage type differs from the host type, or whose width is
// not a multiple of 8, add a staging buffer of 4 fields in the host type.
extern "C" int fslbm_solve_footprint(const fslbm_domain* dom, fslbm_dtype dtype, int64_t* bytes) {
  if (!dom || !bytes || dom->lx < 1 || dom->ly < 1 || dom->lz < 1)
    return fslbm_set_error(FSLBM_ERR_ARG, "solve_footprint: bad argument");
  const int64_t es = dtype == FSLBM_F64 ? 8 : (dtype == FSLBM_F16 ? 2 : 4);
  const int64_t lxp = (dom->lx + 7) / 8 * 8, cs = lxp * dom->ly, fs = cs * dom->lz;
  const int64_t cc = dtype == FSLBM_F64 ? int64_t(sizeof(ColCoef<double>)) : int64_t(sizeof(ColCoef<float>));
  const int64_t tiles = ((lxp + kTX - 1) / kTX) * ((dom->ly + kTY - 1) / kTY) * int64_t(sizeof(int2));
  const int64_t masks = dom->mask_planes > 1
                            ? cs * dom->lz * (1 + int64_t(dtype == FSLBM_F64 ? sizeof(CellCoef<double>)
                                                                                : sizeof(CellCoef<float>)))
                            : cs + cs * cc;
  const int64_t wtabs = dtype == FSLBM_F16 ? 2 * cs * int64_t(sizeof(float)) : 0;
  *bytes = 2 * 4 * fs * es + masks + tiles + wtabs + int64_t(sizeof(DevCounters)) +
           4096 * int64_t(sizeof(fslbm_monitor)) + int64_t(sizeof(double)) * 9 + int64_t(sizeof(unsigned));
  return FSLBM_OK;
}

extern "C" int fslbm_solve_get_fields(fslbm_solve* s, fslbm_dtype hd, void* p, void* u, void* v,
                                      void* w) {
  if (!s || !p || !u || !v || !w) return fslbm_set_error(FSLBM_ERR_ARG, "get_fields: null argument");
  if (hd != FSLBM_F64 && hd != FSLBM_F32)
    return fslbm_set_error(FSLBM_ERR_ARG, "get_fields: host dtype must be F64 or F32");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  const size_t n = size_t(s->lx) * s->ly * s->L, hes = hd == FSLBM_F64 ? 8 : 4;
  cudaStream_t st = s->ctx->stream;
  const void* src = s->state[s->cur];
  void* dst[4] = {p, u, v, w};
  if (int(hd) == s->dtype && s->lx == s->lxp) {
    for (int f = 0; f < 4; ++f)
      CUDA_TRY(cudaMemcpy2DAsync(dst[f], size_t(s->lx) * hes,
                                 static_cast<const char*>(src) + f * field_stride(s) * s->es,
                                 size_t(s->lxp) * s->es, size_t(s->lx) * hes,
                                 size_t(s->ly) * s->L, cudaMemcpyDeviceToHost, st));
  } else {
    if (int r = ensure_stage(s, 4 * n * hes)) return r;
    CUDA_TRY(launch_convert_out(s->dtype, src, s->d_stage, hd == FSLBM_F64, s->lx, s->lxp, s->ly,
                                s->L, st, s->d_wbase));
    for (int f = 0; f < 4; ++f)
      CUDA_TRY(cudaMemcpyAsync(dst[f], static_cast<char*>(s->d_stage) + f * n * hes, n * hes,
                               cudaMemcpyDeviceToHost, st));
  }
  CUDA_TRY(cudaStreamSynchronize(st));
  return FSLBM_OK;
}

// Per-step constants formed as the reference forms them (FSLBM.cu:231, 269, 599, 624): in FP32
// for the FP32-arithmetic forms (FP32 and FP16 storage), in FP64 otherwise.
static void fill_constants(const fslbm_solve* s, StepLaunch& a) {
  const fslbm_params& p = s->prm;
  if (s->dtype != FSLBM_F64) {
    const float tb = float(p.tblend), nu = float(p.nu), blend = float(p.blend);
    a.tb = tb;
    a.cc = float(1.0 - double(tb));
    a.pin = float(p.pin);
    a.dtddy = nu - 0.16666666f;
    a.m = float(1.0 / double(float(p.d1 * p.d1)));
    (void)blend;
    a.fx = float(p.force[0]); a.fy = float(p.force[1]); a.fz = float(p.force[2]);
  } else {
    a.tb = p.tblend;
    a.cc = 1.0 - p.tblend;
    a.pin = p.pin;
    a.dtddy = p.nu - 0.16666666;
    a.m = 1.0 / double(p.d1 * p.d1);
    a.fx = p.force[0]; a.fy = p.force[1]; a.fz = p.force[2];
  }
  // corrector coefficients of the order (FSLBM.cu:177-232), formed as the reference forms them
  double c[9];
  a.K = fd_coefficients(p.fd_order, p.blend, s->dtype != FSLBM_F64, c);
  a.c0 = c[0]; a.c1 = c[1]; a.c2 = c[2];
  for (int j = 0; j < 6; ++j) a.ch[j] = c[3 + j];
}

static int enqueue_steps(fslbm_solve* s, int64_t nsteps) {
  cudaStream_t st = s->ctx->stream;
  StepLaunch a{};
  a.dtype = s->dtype; a.d1 = s->prm.d1;
  a.lxp = s->lxp; a.ly = s->ly; a.L = s->L;
  a.ntiles = s->ntiles; a.chunk = s->chunk; a.nchunks = s->nchunks;
  a.tiles = s->d_tiles; a.mask = s->d_mask; a.colcoef = s->d_colcoef;
  a.err = s->d_err; a.counters = s->d_counters; a.mask_planes = s->planes;
  a.wb = s->d_wbase; a.wgt = s->d_wgt;
  fill_constants(s, a);
  MonitorLaunch m{};
  m.dtype = s->dtype; m.mask = s->d_mask;
  m.lxp = s->lxp; m.lx = s->lx; m.ly = s->ly; m.L = s->L;
  m.pin = s->dtype != FSLBM_F64 ? double(float(s->prm.pin)) : s->prm.pin;
  m.nu = s->prm.nu; m.radius = s->radius; m.l1 = s->l1;
  m.sx = s->sx; m.sy = s->sy; m.sz = s->sz;
  m.log = s->d_log; m.log_cap = s->log_cap; m.gauge_out = s->d_gauge; m.counters = s->d_counters;
  m.wb = s->d_wbase;
  const int me = s->prm.monitor_every;
  for (int64_t n = 0; n < nsteps; ++n) {
    const int64_t c = s->steps + 1;
    a.map = &s->maps[s->cur];
    a.out = s->state[1 - s->cur];
    a.step_no = c;
    a.gauge = (me > 0 && c > 1 && (c - 1) % me == 0) ? s->d_gauge : nullptr;
    if (s->timing) {
      while (s->tev.size() < s->tev_used + 2) {
        cudaEvent_t e;
        CUDA_TRY(cudaEventCreate(&e));
        s->tev.push_back(e);
      }
      CUDA_TRY(cudaEventRecord(s->tev[s->tev_used], st));
    }
    if (s->use2) {
      Step2Launch b2{s->prm.d1, s->ty2, s->packed2, &s->maps2p[s->cur], &s->maps2u[s->cur], s->grid2};
      CUDA_TRY(launch_step2(a, b2, st));
    } else {
      CUDA_TRY(launch_step(a, st));
    }
    if (s->timing) {
      CUDA_TRY(cudaEventRecord(s->tev[s->tev_used + 1], st));
      s->tev_used += 2;
    }
    ++s->launches;
    if (s->nghost) {                 // periodic cross-section: refresh the ghost band
      CUDA_TRY(launch_fill_ghosts(s->dtype, a.out, s->d_ghosts, s->nghost, s->lxp, s->ly, s->L, st));
      ++s->launches;
    }
    s->cur ^= 1;
    s->steps = c;
    if (me > 0 && c % me == 0) {
      m.state = s->state[s->cur];
      CUDA_TRY(launch_monitor(m, st));
      ++s->launches;
    }
  }
  return FSLBM_OK;
}

extern "C" int fslbm_solve_step(fslbm_solve* s, int64_t nsteps) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "step: null solve");
  if (nsteps < 0) return fslbm_set_error(FSLBM_ERR_ARG, "step: negative step count");
  if (!s->fields_set) return fslbm_set_error(FSLBM_ERR_STATE, "step: fields were never set");
  NvtxRange range("fslbm_solve_step");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  CUDA_TRY(cudaEventRecord(s->ev0, s->ctx->stream));
  if (int r = enqueue_steps(s, nsteps)) return r;
  CUDA_TRY(cudaEventRecord(s->ev1, s->ctx->stream));
  return FSLBM_OK;
}

extern "C" int fslbm_solve_sync(fslbm_solve* s) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "sync: null solve");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  elapsed_if_recorded(s->ev0, s->ev1, &s->last_ms);
  unsigned err = 0;
  CUDA_TRY(cudaMemcpy(&err, s->d_err, sizeof err, cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemsetAsync(s->d_err, 0, sizeof(unsigned), s->ctx->stream);
    return fslbm_set_error(FSLBM_ERR_TIMEOUT, "a bounded device wait gave up (flags 0x%x)", err);
  }
  return FSLBM_OK;
}

extern "C" int fslbm_solve_monitor_log(fslbm_solve* s, fslbm_monitor* out, int max, int* n_out) {
  if (!s || (!out && max > 0)) return fslbm_set_error(FSLBM_ERR_ARG, "monitor_log: null argument");
  if (int r = fslbm_solve_sync(s)) return r;
  DevCounters c;
  CUDA_TRY(cudaMemcpy(&c, s->d_counters, sizeof c, cudaMemcpyDeviceToHost));
  int64_t first = std::max<int64_t>(s->drained, c.records - s->log_cap);
  int n = 0;
  for (int64_t k = first; k < c.records && n < max; ++k, ++n)
    CUDA_TRY(cudaMemcpy(&out[n], s->d_log + (k % s->log_cap), sizeof(fslbm_monitor),
                        cudaMemcpyDeviceToHost));
  s->drained = first + n;
  if (n_out) *n_out = n;
  return FSLBM_OK;
}

extern "C" int fslbm_solve_monitor(fslbm_solve* s, fslbm_monitor* out) {
  if (!s || !out) return fslbm_set_error(FSLBM_ERR_ARG, "monitor: null argument");
  if (int r = fslbm_solve_sync(s)) return r;
  DevCounters c;
  CUDA_TRY(cudaMemcpy(&c, s->d_counters, sizeof c, cudaMemcpyDeviceToHost));
  if (c.records == 0) return fslbm_set_error(FSLBM_ERR_STATE, "monitor: no record yet");
  CUDA_TRY(cudaMemcpy(out, s->d_log + ((c.records - 1) % s->log_cap), sizeof(fslbm_monitor),
                      cudaMemcpyDeviceToHost));
  return FSLBM_OK;
}

extern "C" int fslbm_solve_check(fslbm_solve* s, double* max_abs_u) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "check: null solve");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  CUDA_TRY(launch_check(s->dtype, s->state[s->cur], field_stride(s), s->d_scratch, s->ctx->stream,
                        s->lxp, s->ly, s->d_wbase));
  double r[2];
  CUDA_TRY(cudaMemcpyAsync(r, s->d_scratch, sizeof r, cudaMemcpyDeviceToHost, s->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  if (max_abs_u) *max_abs_u = r[1];
  if (r[0] > 0)
    return fslbm_set_error(FSLBM_ERR_DIVERGED, "check: %.0f non-finite values in the fields", r[0]);
  return FSLBM_OK;
}

extern "C" int fslbm_solve_info(fslbm_solve* s, fslbm_info* out) {
  if (!s || !out) return fslbm_set_error(FSLBM_ERR_ARG, "info: null argument");
  out->cells = int64_t(s->lx) * s->ly * s->L;
  out->fluid_cells = s->fluid_total;
  out->bytes_device = s->bytes_device;
  out->steps = s->steps;
  out->lx_pitch = s->lxp;
  out->dtype = s->dtype;
  out->last_step_ms = s->last_ms;
  out->kernel_launches = s->launches;
  return FSLBM_OK;
}

extern "C" int fslbm_solve_set_timing(fslbm_solve* s, int enable) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "set_timing: null solve");
  s->timing = enable != 0;
  return FSLBM_OK;
}

extern "C" int fslbm_solve_kernel_time(fslbm_solve* s, double* ms_total, int64_t* launches) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "kernel_time: null solve");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  double t = 0;
  for (size_t k = 0; k + 1 < s->tev_used; k += 2) {
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, s->tev[k], s->tev[k + 1]));
    t += ms;
  }
  if (ms_total) *ms_total = t;
  if (launches) *launches = int64_t(s->tev_used / 2);
  s->tev_used = 0;
  return FSLBM_OK;
}

extern "C" int fslbm_solve_device_fields(fslbm_solve* s, void** p, void** u, void** v, void** w) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "device_fields: null solve");
  char* b = static_cast<char*>(s->state[s->cur]);
  const size_t fb = field_stride(s) * s->es;
  if (p) *p = b;
  if (u) *u = b + fb;
  if (v) *v = b + 2 * fb;
  if (w) *w = b + 3 * fb;
  return FSLBM_OK;
}

// ------------------------------------------------------------------------------------------
// reference layout (buffer planes reconstructed as bcond copies, FSLBM.cu:291-301)
// ------------------------------------------------------------------------------------------
extern "C" int fslbm_solve_get_fields_ref(fslbm_solve* s, float* p, float* u, float* v, float* w) {
  if (!s || !p || !u || !v || !w) return fslbm_set_error(FSLBM_ERR_ARG, "get_fields_ref: null argument");
  const size_t plane = size_t(s->lx) * s->ly, n = plane * s->L;
  std::vector<float> core(4 * n);
  if (int r = fslbm_solve_get_fields(s, FSLBM_F32, core.data(), core.data() + n,
                                     core.data() + 2 * n, core.data() + 3 * n))
    return r;
  const int d2 = s->d2, Lr = s->L + 2 * d2;
  const float pin = float(s->prm.pin);
  float* dst[4] = {p, u, v, w};
  for (int zr = 0; zr < Lr; ++zr) {
    int zc = zr - d2, jump = 0;
    if (zc < 0) { zc += s->L; jump = 1; } else if (zc >= s->L) { zc -= s->L; jump = -1; }
    for (int f = 0; f < 4; ++f)
      std::memcpy(dst[f] + plane * zr, core.data() + f * n + plane * zc, plane * sizeof(float));
    if (jump)
      for (size_t j = 0; j < plane; ++j) {
        const int x = int(j % s->lx), y = int(j / s->lx);
        if (mask_at(s, x, y, zc) == kWall) continue;
        float& pv = p[plane * zr + j];
        pv = jump > 0 ? pv + pin : pv - pin;
      }
  }
  return FSLBM_OK;
}

extern "C" int fslbm_solve_set_fields_ref(fslbm_solve* s, const float* p, const float* u,
                                          const float* v, const float* w) {
  if (!s || !p || !u || !v || !w) return fslbm_set_error(FSLBM_ERR_ARG, "set_fields_ref: null argument");
  const size_t off = size_t(s->lx) * s->ly * s->d2;
  return fslbm_solve_set_fields(s, FSLBM_F32, p + off, u + off, v + off, w + off);
}

extern "C" int fslbm_solve_get_plane(fslbm_solve* s, int kind, int comp, float* out) {
  if (!s || !out || comp < 0 || comp > 3 || kind < 0 || kind > 1)
    return fslbm_set_error(FSLBM_ERR_ARG, "get_plane: bad argument");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  cudaStream_t st = s->ctx->stream;
  const int Lr = s->L + 2 * s->d2;
  if (!s->d_plane) {
    const size_t need = 4 * std::max(size_t(s->L) * s->ly, size_t(s->ly) * s->lx) * sizeof(float);
    CUDA_TRY(dalloc(s, &s->d_plane, need));
  }
  std::vector<float> buf;
  if (kind == 0) {
    const int xs = s->lx / 2;
    CUDA_TRY(launch_gather_plane(s->dtype, s->state[s->cur], s->lx, s->lxp, s->ly, s->L, 0, xs,
                                 s->d_plane, st, s->d_wbase));
    buf.resize(4 * size_t(s->L) * s->ly);
    CUDA_TRY(cudaMemcpyAsync(buf.data(), s->d_plane, buf.size() * sizeof(float),
                             cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    const size_t n = size_t(s->L) * s->ly;
    const float pin = float(s->prm.pin);
    for (int zr = 0; zr < Lr; ++zr) {
      int zc = zr - s->d2, jump = 0;
      if (zc < 0) { zc += s->L; jump = 1; } else if (zc >= s->L) { zc -= s->L; jump = -1; }
      for (int y = 0; y < s->ly; ++y) {
        float val = buf[comp * n + size_t(zc) * s->ly + y];
        if (comp == 0 && jump && mask_at(s, xs, y, zc) != kWall)
          val = jump > 0 ? val + pin : val - pin;
        out[size_t(zr) * s->ly + y] = val;
      }
    }
  } else {
    int zr = Lr / 2, zc = zr - s->d2, jump = 0;
    if (zc < 0) { zc += s->L; jump = 1; } else if (zc >= s->L) { zc -= s->L; jump = -1; }
    CUDA_TRY(launch_gather_plane(s->dtype, s->state[s->cur], s->lx, s->lxp, s->ly, s->L, 1, zc,
                                 s->d_plane, st, s->d_wbase));
    const size_t n = size_t(s->ly) * s->lx;
    buf.resize(4 * n);
    CUDA_TRY(cudaMemcpyAsync(buf.data(), s->d_plane, buf.size() * sizeof(float),
                             cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    const float pin = float(s->prm.pin);
    for (size_t j = 0; j < n; ++j) {
      float val = buf[comp * n + j];
      const int x = int(j % s->lx), y = int(j / s->lx);
      if (comp == 0 && jump && mask_at(s, x, y, zc) != kWall)
        val = jump > 0 ? val + pin : val - pin;
      out[j] = val;
    }
  }
  return FSLBM_OK;
}

// ------------------------------------------------------------------------------------------
// statistics
// ------------------------------------------------------------------------------------------
static int ensure_stats(fslbm_solve* s) {
  if (s->d_stats) return FSLBM_OK;
  const size_t n = size_t(s->ly) * (s->L + 2 * s->d2);
  CUDA_TRY(dalloc(s, &s->d_stats, 22 * n * sizeof(double)));
  CUDA_TRY(cudaMemsetAsync(s->d_stats, 0, 22 * n * sizeof(double), s->ctx->stream));
  return FSLBM_OK;
}

extern "C" int fslbm_stats_sample(fslbm_solve* s) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "stats_sample: null solve");
  NvtxRange range("fslbm_stats_sample");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  if (int r = ensure_stats(s)) return r;
  const size_t n = size_t(s->ly) * (s->L + 2 * s->d2);
  cudaStream_t st = s->ctx->stream;
  // reset policy (FSLBM.cu:683-690)
  if (s->prm.delta == 0) {
    s->cnt = 0; s->cnt2 = 0;
    CUDA_TRY(cudaMemsetAsync(s->d_stats, 0, 22 * n * sizeof(double), st));
  } else if (s->prm.delta == 1) {
    s->cnt2 = 0;
    CUDA_TRY(cudaMemsetAsync(s->d_stats + 4 * n, 0, 7 * n * sizeof(double), st));
    CUDA_TRY(cudaMemsetAsync(s->d_stats + 15 * n, 0, 7 * n * sizeof(double), st));
  }
  s->cnt += 1; s->cnt2 += 1;                                   // FSLBM.cu:715
  const double pin = s->dtype != FSLBM_F64 ? double(float(s->prm.pin)) : s->prm.pin;
  CUDA_TRY(launch_plane_stats(s->dtype, s->state[s->cur], s->d_mask, s->planes, s->lxp, s->ly, s->L, s->d2,
                              s->lx / 2, pin, s->cnt, 1, 1, s->d_stats, st, s->d_wbase));
  return FSLBM_OK;
}

extern "C" int fslbm_stats_get(fslbm_solve* s, double* out, int* cnt, int* cnt2) {
  if (!s || !out) return fslbm_set_error(FSLBM_ERR_ARG, "stats_get: null argument");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  if (int r = ensure_stats(s)) return r;
  const size_t n = size_t(s->ly) * (s->L + 2 * s->d2);
  std::vector<double> acc(22 * n);
  CUDA_TRY(cudaMemcpyAsync(acc.data(), s->d_stats, 22 * n * sizeof(double), cudaMemcpyDeviceToHost,
                           s->ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  for (size_t k = 0; k < 11 * n; ++k) {
    const int c = k < 4 * n ? s->cnt : s->cnt2;
    out[k] = c ? (acc[k] + acc[11 * n + k]) / double(c) : 0.0;   // compensated sum / count
  }
  if (cnt) *cnt = s->cnt;
  if (cnt2) *cnt2 = s->cnt2;
  return FSLBM_OK;
}

extern "C" int fslbm_stats_set(fslbm_solve* s, const double* means, int cnt, int cnt2) {
  if (!s || !means || cnt < 0 || cnt2 < 0) return fslbm_set_error(FSLBM_ERR_ARG, "stats_set: bad argument");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  if (int r = ensure_stats(s)) return r;
  const size_t n = size_t(s->ly) * (s->L + 2 * s->d2);
  std::vector<double> sums(22 * n, 0.0);                                      // compensations 0
  for (size_t k = 0; k < 4 * n; ++k) sums[k] = means[k] * double(cnt);        // FSLBM.cu:453-456
  for (size_t k = 4 * n; k < 11 * n; ++k) sums[k] = means[k] * double(cnt2);  // FSLBM.cu:457-463
  CUDA_TRY(cudaMemcpyAsync(s->d_stats, sums.data(), sums.size() * sizeof(double),
                           cudaMemcpyHostToDevice, s->ctx->stream));
  s->cnt = cnt; s->cnt2 = cnt2;
  return FSLBM_OK;
}

extern "C" int fslbm_profile_sample(fslbm_solve* s) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "profile_sample: null solve");
  NvtxRange range("fslbm_profile_sample");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  const size_t n = size_t(s->lxp) * s->ly;
  if (!s->d_prof) {
    CUDA_TRY(dalloc(s, &s->d_prof, 20 * n * sizeof(double)));
    CUDA_TRY(cudaMemsetAsync(s->d_prof, 0, 20 * n * sizeof(double), s->ctx->stream));
  }
  CUDA_TRY(launch_profile(s->dtype, s->state[s->cur], s->lxp, s->ly, s->L, s->d_prof, s->ctx->stream,
                          s->d_wbase));
  s->prof_n += 1;
  return FSLBM_OK;
}

extern "C" int fslbm_profile_get(fslbm_solve* s, double* sums, int64_t* nsamples) {
  if (!s || !sums) return fslbm_set_error(FSLBM_ERR_ARG, "profile_get: null argument");
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  const size_t n = size_t(s->lxp) * s->ly;
  std::vector<double> buf(20 * n, 0.0);
  if (s->d_prof) {
    CUDA_TRY(cudaMemcpyAsync(buf.data(), s->d_prof, buf.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, s->ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  }
  for (int k = 0; k < 10; ++k)
    for (int y = 0; y < s->ly; ++y)
      for (int x = 0; x < s->lx; ++x)
        sums[(size_t(k) * s->ly + y) * s->lx + x] =
            buf[(size_t(k) * s->ly + y) * s->lxp + x] + buf[(size_t(10 + k) * s->ly + y) * s->lxp + x];
  if (nsamples) *nsamples = s->prof_n;
  return FSLBM_OK;
}

extern "C" int fslbm_profile_reset(fslbm_solve* s) {
  if (!s) return fslbm_set_error(FSLBM_ERR_ARG, "profile_reset: null solve");
  if (s->d_prof) {
    CUDA_TRY(cudaSetDevice(s->ctx->device));
    CUDA_TRY(cudaMemsetAsync(s->d_prof, 0, 20 * size_t(s->lxp) * s->ly * sizeof(double), s->ctx->stream));
  }
  s->prof_n = 0;
  return FSLBM_OK;
}

// ------------------------------------------------------------------------------------------
// batched ensemble: `chain` time steps of all members in one persistent launch (FP32 or FP16
// storage, d1 = 2), steps chained per member inside the launch (step counters, monitors and
// gauges booked there too); the launch is captured once as a CUDA graph and replayed. Members
// of other kinds step one after another.
// ------------------------------------------------------------------------------------------
struct fslbm_batch {
  fslbm_ctx* ctx = nullptr;
  std::vector<fslbm_solve*> members;
  std::vector<int64_t> stop;       // per member: step count at which it stops (-1: never)
  bool fast = false;
  void* d_members = nullptr;
  BatchMon* d_mons = nullptr;
  int2* d_items = nullptr;         // (member, item of the member), longest first
  unsigned* d_tickets = nullptr;   // [2] the batch's error flag ([0], [1], [3] unused)
  unsigned* d_sync = nullptr;      // counters of the chained launch (batch_sync_words)
  int chain = 16;                  // steps per chained launch (and per graph replay)
  std::vector<unsigned char> h_members;
  std::vector<BatchMon> h_mons;
  std::vector<int2> h_items;
  std::vector<int2> item_shape;    // per member: (tiles, chunks) the item table was built for
  int nitems = 0, grid = 0, packed = 1;
  // the batch's own column-pair tiling of every member (32 x ty tiles, one height for the whole
  // batch): tile list, fluid warps per tile for the two warp shapes, tensor maps of both buffers.
  // 32 x 16 tiles, two 256-thread CTAs per SM: on the 64-pipe ensemble (cross-sections 24..96)
  // +1.0 % against 32 x 32 tiles; the members' own single-pipe tiling is not affected
  int ty = 16;
  struct Tiling {
    int ntiles = 0;
    int2* d_tiles = nullptr;
    std::vector<int> warps[3];
    CUtensorMap mp[2], mu[2];
  };
  std::vector<Tiling> mt;
  // per member tiling: streamwise planes per work item and warp shape (0: 32 x 2, 1: 16 x 4,
  // 2: 8 x 8), from the tuning table by size class, else 128 (FSLBM_BATCH_CHUNK) and 16 x 4
  std::vector<int> m_chunk, m_shape;
  int shrink = 1;                  // chunk divisor for batches with fewer than 2 items per SM
  cudaGraphExec_t exec2 = nullptr;  // one chained launch of `chain` steps
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0;
};

static void free_batch(fslbm_batch* b) {
  if (!b) return;
  cudaSetDevice(b->ctx->device);
  if (b->exec2) cudaGraphExecDestroy(b->exec2);
  for (auto& t : b->mt) ctx_free(b->ctx, t.d_tiles);
  ctx_free(b->ctx, b->d_members);
  ctx_free(b->ctx, b->d_mons);
  ctx_free(b->ctx, b->d_items);
  ctx_free(b->ctx, b->d_tickets);
  ctx_free(b->ctx, b->d_sync);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  fslbm_ctx* c = b->ctx;
  delete b;
  ctx_release(c);
}

// Work of one (tile, chunk) item of the column-pair kernel, for ordering the items: planes
// marched (the chunk plus the 2R pipeline planes) times the tile's warps that compute plus two
// for the pipeline's fixed cost.
static int64_t item_cost(const fslbm_solve* s, const std::vector<int> (&warps)[3], int tile, int nout,
                         int shape) {
  return int64_t(nout + 4 * s->prm.d1) * (warps[shape][tile] + 2);
}

// Resident CTAs of the batched kernel: one per SM for 32 x 32 tiles, two for 32 x 16 tiles.
static int batch_slots(const fslbm_batch* b) {
  return b->ctx->sm_count * step2_occupancy(b->members[0]->dtype, 2, b->ty);
}

// Streamwise chunks of a member: about `chunk` planes each, at least 4*d1 planes.
static int member_chunks(const fslbm_solve* s, int chunk) {
  int nch = (s->L + chunk - 1) / chunk;
  return std::max(1, std::min(nch, std::max(1, s->L / (4 * s->prm.d1))));
}

// Member descriptors for the members' current buffers, step counts and stops, and the work-item
// table (rebuilt only when the membership or chunking changed: nitems == 0).
static int batch_upload(fslbm_batch* b) {
  const size_t mbytes = batch_member_bytes();
  const int n = int(b->members.size());
  cudaStream_t st = b->ctx->stream;
  b->h_members.assign(mbytes * n, 0);
  b->h_mons.resize(n);
  // the batched kernel counts a member's step complete after ntiles * nchunks items, so the
  // item table must match every member as it is now: a member reconfigured since the table was
  // built (fslbm_solve_set_params) forces a rebuild, and one that no longer fits the kernel
  // (stride, corrector order or storage type changed) is refused
  for (int i = 0; i < n; ++i) {
    const fslbm_solve* s = b->members[i];
    if (!(s->use2 && s->prm.d1 == 2 && s->dtype == b->members[0]->dtype && s->dtype != FSLBM_F64 &&
          s->nghost == 0))
      return fslbm_set_error(FSLBM_ERR_STATE, "batch_step: member %d was reconfigured and no longer "
                             "fits the batched kernel; create a new batch", i);
  }
  auto eff_chunk = [&](int i) { return std::max(4 * b->members[i]->prm.d1, b->m_chunk[i] / b->shrink); };
  if (!b->h_items.empty() && b->item_shape.size() == size_t(n))
    for (int i = 0; i < n; ++i)
      if (b->item_shape[i].x != b->mt[i].ntiles ||
          b->item_shape[i].y != member_chunks(b->members[i], eff_chunk(i))) {
        b->h_items.clear();
        break;
      }
  const bool build_items = b->h_items.empty();
  struct Item { int64_t cost; int2 it; };
  std::vector<Item> items;
  if (build_items) {
    // shorter chunks while there are fewer than two items per SM (few or small members)
    auto count = [&]() {
      int64_t c = 0;
      for (int i = 0; i < n; ++i) c += int64_t(b->mt[i].ntiles) * member_chunks(b->members[i], eff_chunk(i));
      return c;
    };
    b->shrink = 1;
    while (b->shrink < 64 && count() < 2 * batch_slots(b)) b->shrink *= 2;
  }
  for (int i = 0; i < n; ++i) {
    fslbm_solve* s = b->members[i];
    const fslbm_batch::Tiling& tl = b->mt[i];
    StepLaunch a{};
    a.dtype = s->dtype; a.d1 = s->prm.d1;
    a.lxp = s->lxp; a.ly = s->ly; a.L = s->L; a.ntiles = tl.ntiles;
    a.tiles = tl.d_tiles; a.mask = s->d_mask; a.colcoef = s->d_colcoef;
    a.err = b->d_tickets + 2;        // one flag for the whole batch
    a.wb = s->d_wbase; a.wgt = s->d_wgt;
    fill_constants(s, a);
    const int nch = member_chunks(s, eff_chunk(i));
    const long long stop_at = b->stop[i] >= 0 ? (long long)b->stop[i] : LLONG_MAX;
    CUDA_TRY(fill_batch_member(b->h_members.data() + mbytes * i, tl.mp, tl.mu, a,
                               s->state[0], s->state[1], s->d_gauge, &s->d_counters->steps,
                               stop_at, s->prm.monitor_every, s->cur, nch, b->m_shape[i]));
    if (build_items) {
      if (i == 0) b->item_shape.assign(n, make_int2(0, 0));
      b->item_shape[i] = make_int2(tl.ntiles, nch);
    }
    if (build_items)
      for (int c = 0; c < nch; ++c) {
        const int nout = int((long long)s->L * (c + 1) / nch - (long long)s->L * c / nch);
        for (int t = 0; t < tl.ntiles; ++t)
          items.push_back({item_cost(s, tl.warps, t, nout, b->m_shape[i]), make_int2(i, c * tl.ntiles + t)});
        // the chunk's tiles are ordered by the chunk's longest tile, so neighbouring tiles are
        // claimed one after another and read their shared halo planes while they are in L2
        int64_t longest = 0;
        for (size_t k = items.size() - size_t(tl.ntiles); k < items.size(); ++k)
          longest = std::max(longest, items[k].cost);
        for (size_t k = items.size() - size_t(tl.ntiles); k < items.size(); ++k) items[k].cost = longest;
      }
    BatchMon& m = b->h_mons[i];
    std::memset(&m, 0, sizeof m);
    m.mon.dtype = s->dtype; m.mon.mask = s->d_mask;
    m.mon.lxp = s->lxp; m.mon.lx = s->lx; m.mon.ly = s->ly; m.mon.L = s->L;
    m.mon.pin = double(float(s->prm.pin)); m.mon.nu = s->prm.nu; m.mon.radius = s->radius;
    m.mon.l1 = s->l1; m.mon.sx = s->sx; m.mon.sy = s->sy; m.mon.sz = s->sz;
    m.mon.log = s->d_log; m.mon.log_cap = s->log_cap; m.mon.gauge_out = s->d_gauge;
    m.mon.counters = s->d_counters;
    m.mon.wb = s->d_wbase;
    m.state[0] = s->state[0]; m.state[1] = s->state[1];
    m.stop_at = stop_at;
    m.monitor_every = s->prm.monitor_every; m.cur0 = s->cur;
  }
  if (build_items) {
    std::stable_sort(items.begin(), items.end(), [](const Item& x, const Item& y) { return x.cost > y.cost; });
    b->h_items.resize(items.size());
    for (size_t k = 0; k < items.size(); ++k) b->h_items[k] = items[k].it;
    b->nitems = int(items.size());
    b->grid = std::max(1, std::min(b->nitems, batch_slots(b)));
    ctx_free(b->ctx, b->d_items);
    b->d_items = nullptr;
    CUDA_TRY(ctx_alloc(b->ctx, reinterpret_cast<void**>(&b->d_items), b->h_items.size() * sizeof(int2)));
    CUDA_TRY(cudaMemcpyAsync(b->d_items, b->h_items.data(), b->h_items.size() * sizeof(int2),
                             cudaMemcpyHostToDevice, st));
    if (b->exec2) {                // the graph holds the old table's address and size
      cudaGraphExecDestroy(b->exec2);
      b->exec2 = nullptr;
    }
  }
  CUDA_TRY(cudaMemcpyAsync(b->d_members, b->h_members.data(), b->h_members.size(),
                           cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(b->d_mons, b->h_mons.data(), sizeof(BatchMon) * n,
                           cudaMemcpyHostToDevice, st));
  return FSLBM_OK;
}

// One chained launch of `nsteps` steps for every member (each starting at its buffer cur0).
static cudaError_t batch_enqueue(fslbm_batch* b, int nsteps, cudaStream_t st) {
  return launch_batch_steps(b->members[0]->dtype, b->ty, b->d_members, b->d_mons, b->d_items, b->nitems,
                            nsteps, b->grid, b->packed, b->d_sync, int(b->members.size()),
                            b->d_tickets + 2, st);
}

// ------------------------------------------------------------------------------------------
// batch tiling by size class: table, autotuner
// ------------------------------------------------------------------------------------------
// Size class of a member: 32-wide column tiles across x and y, and the streamwise length
// rounded up to a power of two ("TXxTY:L<log2>"); members of a class share chunk and warp shape.
static std::string class_key(const fslbm_solve* s) {
  int lb = 0;
  while ((1 << lb) < s->L) ++lb;
  char buf[64];
  std::snprintf(buf, sizeof buf, "%dx%d:L%d", (s->lxp + kTX - 1) / kTX, (s->ly + 31) / 32, lb);
  return buf;
}

struct Tiling { int chunk = 128, shape = 1; double ms = 0; };
using TilingTable = std::map<std::string, Tiling>;

static bool write_tiling(const char* path, const TilingTable& t) {
  FILE* f = std::fopen(path, "wt");
  if (!f) return false;
  std::fprintf(f, "{\n  \"format\": \"fslbm batch tiling 1\",\n  \"classes\": {");
  bool first = true;
  for (const auto& kv : t) {
    std::fprintf(f, "%s\n    \"%s\": {\"chunk\": %d, \"warp_shape\": %d, \"trial_ms\": %.4f}",
                 first ? "" : ",", kv.first.c_str(), kv.second.chunk, kv.second.shape, kv.second.ms);
    first = false;
  }
  std::fprintf(f, "\n  }\n}\n");
  return std::fclose(f) == 0;
}

// Reads the table written by write_tiling: every `"<key>": {"chunk": N, "warp_shape": M` entry
// (M = 0, 1, 2; tables of the earlier form name it "warp16x4", 0 or 1, with the same meaning).
static bool read_tiling(const char* path, TilingTable& t) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::string s;
  char buf[4096];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) s.append(buf, n);
  std::fclose(f);
  size_t pos = 0;
  while ((pos = s.find("{\"chunk\":", pos)) != std::string::npos) {
    const size_t q1 = s.rfind('"', s.rfind(':', pos));
    const size_t q0 = q1 == std::string::npos ? q1 : s.rfind('"', q1 - 1);
    Tiling v;
    if (q0 != std::string::npos &&
        (std::sscanf(s.c_str() + pos, "{\"chunk\": %d, \"warp_shape\": %d", &v.chunk, &v.shape) == 2 ||
         std::sscanf(s.c_str() + pos, "{\"chunk\": %d, \"warp16x4\": %d", &v.chunk, &v.shape) == 2) &&
        v.chunk >= 4 && v.shape >= 0 && v.shape <= 2)
      t[s.substr(q0 + 1, q1 - q0 - 1)] = v;
    pos += 9;
  }
  return true;
}

static void apply_tiling(fslbm_batch* b, const TilingTable& t) {
  for (size_t i = 0; i < b->members.size(); ++i) {
    auto it = t.find(class_key(b->members[i]));
    if (it == t.end()) continue;
    b->m_chunk[i] = it->second.chunk;
    b->m_shape[i] = it->second.shape;
  }
  b->h_items.clear();              // rebuild the work items
}

// The tuning table used when a batch is created: FSLBM_BATCH_TUNING, else batch_tiling.json next
// to this library (a table measured on a B200 ships with the package), else none.
static void default_tiling(fslbm_batch* b) {
  std::string path;
  if (const char* e = std::getenv("FSLBM_BATCH_TUNING")) {
    path = e;
  } else {
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&fslbm_version), &info) && info.dli_fname) {
      path = info.dli_fname;
      const size_t slash = path.rfind('/');
      path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/batch_tiling.json";
    }
  }
  TilingTable t;
  if (!path.empty() && read_tiling(path.c_str(), t)) apply_tiling(b, t);
}

extern "C" int fslbm_batch_create(fslbm_ctx* ctx, fslbm_solve* const* solves, int n, fslbm_batch** out) {
  if (!ctx || !out || n < 1 || !solves) return fslbm_set_error(FSLBM_ERR_ARG, "batch_create: bad argument");
  auto* b = new fslbm_batch;
  b->ctx = ctx;
  ctx_retain(ctx);
  bool fast = true;
  for (int i = 0; i < n; ++i) {
    if (!solves[i] || solves[i]->ctx != ctx) {
      free_batch(b);
      return fslbm_set_error(FSLBM_ERR_ARG, "batch_create: member %d is null or of another context", i);
    }
    b->members.push_back(solves[i]);
    b->stop.push_back(-1);
    b->m_chunk.push_back(128);
    b->m_shape.push_back(1);
    fast = fast && solves[i]->use2 && solves[i]->prm.d1 == 2 && solves[i]->dtype != FSLBM_F64 &&
           solves[i]->dtype == solves[0]->dtype && solves[i]->nghost == 0;
  }
  b->fast = fast;
  default_tiling(b);
  if (const char* ec = std::getenv("FSLBM_BATCH_CHUNK"))
    for (int& c : b->m_chunk) c = std::max(8, std::atoi(ec));
  // packed FP32x2 pair arithmetic, as the single-pipe kernel (FSLBM_BATCH_PACKED=0 selects the
  // scalar form, for comparisons; both give the same bits)
  const char* ebp = std::getenv("FSLBM_BATCH_PACKED");
  b->packed = (ebp && std::atoi(ebp) == 0) ? 0 : 1;
  cudaError_t e = cudaSetDevice(ctx->device);
  // tile height of the batch's tiles (FSLBM_BATCH_TILE_Y=16|32 overrides the default)
  if (const char* ety = std::getenv("FSLBM_BATCH_TILE_Y")) b->ty = std::atoi(ety) == 16 ? 16 : 32;
  if (!e && fast) e = batch_prepare(solves[0]->dtype, b->ty);
  if (!e && fast) {
    b->mt.resize(n);
    for (int i = 0; i < n && !e; ++i) {
      fslbm_solve* s = solves[i];
      fslbm_batch::Tiling& tl = b->mt[i];
      const std::vector<int2> tiles = fluid_tiles(s, b->ty);
      tl.ntiles = int(tiles.size());
      tile_warp_counts(s, tiles, b->ty, tl.warps);
      const int rc = encode_pair_maps(s, b->ty, tl.mp, tl.mu);
      if (rc != FSLBM_OK) {
        free_batch(b);
        return rc;
      }
      e = ctx_alloc(ctx, reinterpret_cast<void**>(&tl.d_tiles), std::max<size_t>(1, tiles.size()) * sizeof(int2));
      if (!e) e = cudaMemcpyAsync(tl.d_tiles, tiles.data(), tiles.size() * sizeof(int2),
                                  cudaMemcpyHostToDevice, ctx->stream);
    }
  }
  if (!e && fast) e = ctx_alloc(ctx, &b->d_members, batch_member_bytes() * n);
  if (!e && fast) e = ctx_alloc(ctx, reinterpret_cast<void**>(&b->d_mons), sizeof(BatchMon) * n);
  if (!e && fast) e = ctx_alloc(ctx, reinterpret_cast<void**>(&b->d_tickets), 4 * sizeof(unsigned));
  if (!e && fast) e = cudaMemsetAsync(b->d_tickets, 0, 4 * sizeof(unsigned), ctx->stream);
  if (!e && fast)
    e = ctx_alloc(ctx, reinterpret_cast<void**>(&b->d_sync), batch_sync_words(n) * sizeof(unsigned));
  if (const char* ech = std::getenv("FSLBM_BATCH_CHAIN")) b->chain = std::max(1, std::atoi(ech));
  if (!e) e = cudaEventCreate(&b->ev0);
  if (!e) e = cudaEventCreate(&b->ev1);
  if (e) {
    free_batch(b);
    return fslbm_set_error(FSLBM_ERR_CUDA, "batch_create: %s", cudaGetErrorString(e));
  }
  *out = b;
  return FSLBM_OK;
}

extern "C" int fslbm_batch_destroy(fslbm_batch* b) {
  free_batch(b);
  return FSLBM_OK;
}

extern "C" int fslbm_batch_step(fslbm_batch* b, int64_t nsteps, int use_graph) {
  if (!b) return fslbm_set_error(FSLBM_ERR_ARG, "batch_step: null batch");
  if (nsteps < 0) return fslbm_set_error(FSLBM_ERR_ARG, "batch_step: negative step count");
  for (fslbm_solve* s : b->members)
    if (!s->fields_set) return fslbm_set_error(FSLBM_ERR_STATE, "batch_step: a member has no fields");
  NvtxRange range("fslbm_batch_step");
  CUDA_TRY(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  // steps each member actually takes (a member stops at its stop step)
  std::vector<int64_t> take(b->members.size(), nsteps);
  for (size_t i = 0; i < b->members.size(); ++i)
    if (b->stop[i] >= 0) take[i] = std::max<int64_t>(0, std::min(nsteps, b->stop[i] - b->members[i]->steps));
  if (!b->fast) {
    CUDA_TRY(cudaEventRecord(b->ev0, st));
    for (size_t i = 0; i < b->members.size(); ++i)
      if (int r = enqueue_steps(b->members[i], take[i])) return r;
    CUDA_TRY(cudaEventRecord(b->ev1, st));
    return FSLBM_OK;
  }
  if (int r = batch_upload(b)) return r;
  CUDA_TRY(cudaEventRecord(b->ev0, st));
  // chained launches of `chain` steps (one graph replay each when use_graph), then the rest in
  // one more launch; every launch leaves the members on their launch-start buffer when it has an
  // even step count, so the graph replays from the same descriptors
  // steps per launch: even (the graph replays from the same buffers) and few enough that the
  // launch's 32-bit ticket count nitems * steps stays below 2^31
  const int64_t cap = std::max<int64_t>(2, (int64_t(INT_MAX) / std::max(1, b->nitems)) & ~int64_t(1));
  const int G = int(std::min<int64_t>(b->chain + (b->chain & 1), cap));
  int64_t left = nsteps, nlaunch = 0;
  if (use_graph && left >= G) {
    if (!b->exec2) {
      cudaGraph_t graph;
      CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      cudaError_t e1 = batch_enqueue(b, G, st);
      cudaError_t e2 = cudaStreamEndCapture(st, &graph);
      if (e1 || e2)
        return fslbm_set_error(FSLBM_ERR_CUDA, "batch_step: graph capture: %s",
                               cudaGetErrorString(e1 ? e1 : e2));
      cudaError_t e3 = cudaGraphInstantiate(&b->exec2, graph, 0);
      cudaGraphDestroy(graph);
      if (e3) return fslbm_set_error(FSLBM_ERR_CUDA, "batch_step: graph instantiate: %s", cudaGetErrorString(e3));
    }
    for (; left >= G; left -= G, ++nlaunch) CUDA_TRY(cudaGraphLaunch(b->exec2, st));
  }
  for (; left >= G; left -= G, ++nlaunch) CUDA_TRY(batch_enqueue(b, G, st));
  if (left > 0) {                  // left < G
    CUDA_TRY(batch_enqueue(b, int(left), st));
    ++nlaunch;
  }
  CUDA_TRY(cudaEventRecord(b->ev1, st));
  for (size_t i = 0; i < b->members.size(); ++i) {
    fslbm_solve* s = b->members[i];
    s->steps += take[i];
    s->cur ^= int(take[i] & 1);
    // counted per member: each chained launch serves all members
    s->launches += std::min<int64_t>(nlaunch, (take[i] + G - 1) / G);
  }
  return FSLBM_OK;
}

extern "C" int fslbm_batch_set_stop(fslbm_batch* b, int member, int64_t stop_step) {
  if (!b || member < 0 || member >= int(b->members.size()))
    return fslbm_set_error(FSLBM_ERR_ARG, "batch_set_stop: bad batch or member index");
  b->stop[member] = stop_step < 0 ? -1 : stop_step;
  return FSLBM_OK;
}

extern "C" int fslbm_batch_sync(fslbm_batch* b) {
  if (!b) return fslbm_set_error(FSLBM_ERR_ARG, "batch_sync: null batch");
  CUDA_TRY(cudaSetDevice(b->ctx->device));
  CUDA_TRY(cudaStreamSynchronize(b->ctx->stream));
  elapsed_if_recorded(b->ev0, b->ev1, &b->last_ms);
  std::vector<unsigned*> flags;
  if (b->fast) flags.push_back(b->d_tickets + 2);
  else
    for (fslbm_solve* s : b->members) flags.push_back(s->d_err);
  for (unsigned* f : flags) {
    unsigned err = 0;
    CUDA_TRY(cudaMemcpy(&err, f, sizeof err, cudaMemcpyDeviceToHost));
    if (err) {
      cudaMemsetAsync(f, 0, sizeof(unsigned), b->ctx->stream);
      return fslbm_set_error(FSLBM_ERR_TIMEOUT, "batch_sync: a bounded device wait gave up");
    }
  }
  return FSLBM_OK;
}

extern "C" int fslbm_batch_elapsed(fslbm_batch* b, double* ms) {
  if (!b || !ms) return fslbm_set_error(FSLBM_ERR_ARG, "batch_elapsed: null argument");
  *ms = b->last_ms;
  return FSLBM_OK;
}

extern "C" int fslbm_batch_set_tiling(fslbm_batch* b, int member, int chunk, int warp_shape) {
  if (!b || member < 0 || member >= int(b->members.size()) || chunk < 1 || warp_shape < 0 || warp_shape > 2)
    return fslbm_set_error(FSLBM_ERR_ARG, "batch_set_tiling: bad batch, member, chunk or warp shape");
  b->m_chunk[member] = chunk;
  b->m_shape[member] = warp_shape;
  b->h_items.clear();
  return FSLBM_OK;
}

extern "C" int fslbm_batch_load_tiling(fslbm_batch* b, const char* path) {
  if (!b || !path) return fslbm_set_error(FSLBM_ERR_ARG, "batch_load_tiling: null argument");
  TilingTable t;
  if (!read_tiling(path, t)) return fslbm_set_error(FSLBM_ERR_IO, "batch_load_tiling: cannot read %s", path);
  apply_tiling(b, t);
  return FSLBM_OK;
}

// Times candidate tilings on the batch itself: first one tiling for all members (chunks 64, 128,
// 256 planes, the three warp shapes), then per size class, largest first, the neighbouring chunks
// and the other warp shapes while the other classes keep theirs; a change is kept only when it is at
// least 0.3 % faster (each timing is the better of two trials). The members' fields, step
// counts, monitor logs and gauges are restored afterwards.
extern "C" int fslbm_batch_autotune(fslbm_batch* b, int trial_steps, const char* path) {
  if (!b || trial_steps < 1) return fslbm_set_error(FSLBM_ERR_ARG, "batch_autotune: bad argument");
  if (!b->fast)
    return fslbm_set_error(FSLBM_ERR_STATE, "batch_autotune: the members do not use the batched kernel");
  for (fslbm_solve* s : b->members)
    if (!s->fields_set) return fslbm_set_error(FSLBM_ERR_STATE, "batch_autotune: a member has no fields");
  CUDA_TRY(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  const int n = int(b->members.size());
  // snapshot
  struct Snap { void* state = nullptr; DevCounters c{}; double gauge = 0; int64_t steps = 0, launches = 0, drained = 0; int cur = 0; };
  std::vector<Snap> snap(n);
  CUDA_TRY(cudaStreamSynchronize(st));
  int rc = FSLBM_OK;
  for (int i = 0; i < n && !rc; ++i) {
    fslbm_solve* s = b->members[i];
    const size_t bytes = 4 * field_stride(s) * s->es;
    Snap& q = snap[i];
    q.steps = s->steps; q.cur = s->cur; q.launches = s->launches; q.drained = s->drained;
    cudaError_t e = ctx_alloc(b->ctx, &q.state, bytes);
    if (!e) e = cudaMemcpyAsync(q.state, s->state[s->cur], bytes, cudaMemcpyDeviceToDevice, st);
    if (!e) e = cudaMemcpyAsync(&q.c, s->d_counters, sizeof q.c, cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaMemcpyAsync(&q.gauge, s->d_gauge, sizeof q.gauge, cudaMemcpyDeviceToHost, st);
    if (e) rc = fslbm_set_error(FSLBM_ERR_CUDA, "batch_autotune: snapshot: %s", cudaGetErrorString(e));
  }
  if (!rc && cudaStreamSynchronize(st)) rc = fslbm_set_error(FSLBM_ERR_CUDA, "batch_autotune: snapshot sync");
  const std::vector<int64_t> stops = b->stop;
  for (int64_t& x : b->stop) x = -1;
  // classes, largest first
  std::map<std::string, std::vector<int>> cls;
  for (int i = 0; i < n; ++i) cls[class_key(b->members[i])].push_back(i);
  std::vector<std::pair<int64_t, std::string>> order;
  for (const auto& kv : cls) {
    int64_t cells = 0;
    for (int i : kv.second) cells += int64_t(b->members[i]->lx) * b->members[i]->ly * b->members[i]->L;
    order.push_back({-cells, kv.first});
  }
  std::sort(order.begin(), order.end());
  auto trial = [&](double* ms) -> int {
    double best = 1e30;
    for (int rep = 0; rep < 2; ++rep) {
      if (int r = fslbm_batch_step(b, 2, 1)) return r;       // warm: items, graph
      if (int r = fslbm_batch_sync(b)) return r;
      if (int r = fslbm_batch_step(b, trial_steps, 1)) return r;
      if (int r = fslbm_batch_sync(b)) return r;
      best = std::min(best, b->last_ms);
    }
    *ms = best;
    return FSLBM_OK;
  };
  auto set = [&](const std::vector<int>& mem, int c, int w) {
    for (int i : mem) { b->m_chunk[i] = c; b->m_shape[i] = w; }
    b->h_items.clear();
  };
  std::vector<int> all(n);
  for (int i = 0; i < n; ++i) all[i] = i;
  Tiling glob;
  glob.ms = 1e30;
  for (int w : {1, 2, 0}) {
    if (rc) break;
    for (int c : {64, 128, 256}) {
      set(all, c, w);
      double ms = 0;
      if ((rc = trial(&ms))) break;
      if (ms < glob.ms) { glob.ms = ms; glob.chunk = c; glob.shape = w; }
    }
  }
  set(all, glob.chunk, glob.shape);
  double cur_ms = glob.ms;
  TilingTable table;
  for (size_t oi = 0; oi < order.size() && !rc; ++oi) {
    const std::vector<int>& mem = cls[order[oi].second];
    int maxL = 0;
    for (int i : mem) maxL = std::max(maxL, b->members[i]->L);
    Tiling best = glob;
    best.ms = cur_ms;
    const std::pair<int, int> cands[] = {{glob.chunk / 2, glob.shape}, {glob.chunk * 2, glob.shape},
                                         {glob.chunk, (glob.shape + 1) % 3}, {glob.chunk, (glob.shape + 2) % 3}};
    for (const auto& cw : cands) {
      if (cw.first < 16 || (cw.first / 2 >= maxL && cw.first > glob.chunk)) continue;
      set(mem, cw.first, cw.second);
      double ms = 0;
      if ((rc = trial(&ms))) break;
      if (ms < best.ms * 0.997) { best.ms = ms; best.chunk = cw.first; best.shape = cw.second; }
    }
    set(mem, best.chunk, best.shape);
    cur_ms = best.ms;
    table[order[oi].second] = best;
  }
  // Restore every member and free every snapshot even when a step fails; keep the first error.
  // A member's host-side counters are put back only with its device state, counters and gauge;
  // a member whose copies could not be queued is marked as having no fields, so it refuses to
  // step (FSLBM_ERR_STATE) until its fields are set again, instead of stepping a state that
  // disagrees with its counters.
  b->stop = stops;
  cudaError_t re = cudaStreamSynchronize(st);
  int unrestored = 0;
  for (int i = 0; i < n; ++i) {
    fslbm_solve* s = b->members[i];
    Snap& q = snap[i];
    if (!q.state) continue;
    if (!re) re = cudaMemcpyAsync(s->state[q.cur], q.state, 4 * field_stride(s) * s->es,
                                  cudaMemcpyDeviceToDevice, st);
    if (!re) re = cudaMemcpyAsync(s->d_counters, &q.c, sizeof q.c, cudaMemcpyHostToDevice, st);
    if (!re) re = cudaMemcpyAsync(s->d_gauge, &q.gauge, sizeof q.gauge, cudaMemcpyHostToDevice, st);
    if (!re) {
      s->steps = q.steps; s->cur = q.cur; s->launches = q.launches; s->drained = q.drained;
    } else {
      s->fields_set = false;
      ++unrestored;
    }
    ctx_free(b->ctx, q.state);                     // stream-ordered: after the copy
  }
  if (!re) re = cudaMemsetAsync(b->d_tickets + 2, 0, sizeof(unsigned), st);
  const cudaError_t se = cudaStreamSynchronize(st);  // host snapshots stay alive until copied
  if (!re) re = se;
  b->h_items.clear();
  if (rc) return rc;
  if (re) return fslbm_set_error(FSLBM_ERR_CUDA, "batch_autotune: restoring the members: %s (%d "
                                 "members not restored: their fields must be set again)",
                                 cudaGetErrorString(re), unrestored);
  if (path && !write_tiling(path, table))
    return fslbm_set_error(FSLBM_ERR_IO, "batch_autotune: cannot write %s", path);
  return FSLBM_OK;
}
