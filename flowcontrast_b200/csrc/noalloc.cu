// Allocation-free FSLBM step: fslbm_step_f32_noalloc (declared in include/fslbm.h).
//
// Some callers cannot let a library call cudaMalloc: applications that hand every byte of
// device memory to their own pool or arena, and hosts that run the solver inside a budgeted or
// real-time loop where a device allocation (which can synchronise the device and fail under
// memory pressure) is not allowed. This entry point advances a state the caller owns by one
// FP32 step and allocates nothing. The work tables the step kernel needs (per-column wall
// sums, the tile list, the gauge value and the error flag) live in the file-scope device array
// below, which every GPU that loads the library holds until the process exits.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "internal.h"
#include "step2_kernel.cuh"

int fslbm_set_error(int code, const char* fmt, ...);

namespace {

using namespace fslbm;

constexpr int kNoallocMaxCells = 65536;   // lx_pitch * ly of the cross-section
constexpr int kNoallocMaxTiles = 2048;
constexpr int kNoallocTY = 32;            // tile height of the FP32 column-pair kernel used here
constexpr size_t kCoefBytes = size_t(kNoallocMaxCells) * sizeof(ColCoef<float>);
constexpr size_t kTileBytes = size_t(kNoallocMaxTiles) * sizeof(int2);
constexpr size_t kGaugeOffset = kCoefBytes + kTileBytes;
constexpr size_t kErrOffset = kGaugeOffset + sizeof(double);
constexpr size_t kScratchBytes = kErrOffset + 256;

// The step's work tables, shared by every call on a device. Calls that overlap on the GPU
// (different streams, no ordering between them) race on it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};
int g_sm_count[kMaxDevices] = {};

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn g_encode = nullptr;

// Error word bits: the step kernel's bounded waits set bit 0; the mask check sets bit 1.
constexpr unsigned kErrBadMask = 2u;

// Per-column wall sums (the same arithmetic, in the same order, as the solve's host-side
// table), the tile list (every tile of the padded cross-section) and the gauge, written into
// the scratch array (the host clears the error word first). The mask must hold only 0 and 125,
// with wall on the cross-section rim and in the padding columns (the conditions the solve
// checks at creation); anything else sets kErrBadMask.
__global__ void noalloc_prepare(const uint8_t* mask, int lx, int lxp, int ly, int ntx, int ntiles,
                                double gauge, unsigned char* scratch) {
  ColCoef<float>* cc = reinterpret_cast<ColCoef<float>*>(scratch);
  int2* tiles = reinterpret_cast<int2*>(scratch + kCoefBytes);
  const double wv[3] = {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0};
  const int n = lxp * ly;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int x = i % lxp, y = i / lxp;
    double a = 0, bx = 0, by = 0;
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int gx = x + dx, gy = y + dy;
        const bool wall = gx < 0 || gy < 0 || gx >= lxp || gy >= ly || mask[gy * lxp + gx] == kWall;
        if (!wall) continue;
        const double w = wv[dx + 1] * wv[dy + 1];
        a += w; bx += dx * w; by += dy * w;
      }
    ColCoef<float> c;
    c.ws0 = float(a); c.wsx = float(bx); c.wsy = float(by);
    c.fluid = mask[i] == 0 ? 1.0f : 0.0f;
    cc[i] = c;
    const uint8_t m = mask[i];
    const bool rim = x == 0 || y == 0 || x >= lx - 1 || y == ly - 1;
    if ((m != 0 && m != kWall) || (m == 0 && rim))
      atomicOr(reinterpret_cast<unsigned*>(scratch + kErrOffset), kErrBadMask);
  }
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x)
    tiles[t] = make_int2(kTX * (t % ntx), kNoallocTY * (t / ntx));
  if (blockIdx.x == 0 && threadIdx.x == 0) *reinterpret_cast<double*>(scratch + kGaugeOffset) = gauge;
}

// [a, a + na) and [b, b + nb) share a byte
bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + nb && y < x + na;
}

// Once per device, with that device current: the scratch array's device address, the
// kernel's shared-memory attribute, the SM count and the tensor-map encoder.
int setup_device(int dev) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_scratch_ptr[dev]) return FSLBM_OK;
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess)
    return fslbm_set_error(FSLBM_ERR_CUDA, "step_f32_noalloc: cudaGetSymbolAddress: %s",
                           cudaGetErrorString(e));
  if ((e = step2_prepare(FSLBM_F32, 2, kNoallocTY)) != cudaSuccess)
    return fslbm_set_error(FSLBM_ERR_CUDA, "step_f32_noalloc: kernel set-up: %s", cudaGetErrorString(e));
  int sms = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return fslbm_set_error(FSLBM_ERR_CUDA, "step_f32_noalloc: %s", cudaGetErrorString(e));
  if (!g_encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return fslbm_set_error(FSLBM_ERR_CUDA, "step_f32_noalloc: cuTensorMapEncodeTiled is unavailable");
    g_encode = reinterpret_cast<EncodeTiledFn>(fn);
  }
  g_sm_count[dev] = sms;
  g_scratch_ptr[dev] = p;
  return FSLBM_OK;
}

}  // namespace

extern "C" int fslbm_step_f32_noalloc(const float* state_in, float* state_out,
                                      const uint8_t* mask, int lx, int ly, int lz, int lx_pitch,
                                      const fslbm_params* prm, double gauge, void* stream) {
  if (!state_in || !state_out || !mask || !prm)
    return fslbm_set_error(FSLBM_ERR_ARG, "step_f32_noalloc: null argument");
  if (lx < 3 || ly < 3 || lx_pitch < lx || lx_pitch % 8 != 0)
    return fslbm_set_error(FSLBM_ERR_ARG,
                           "step_f32_noalloc: need lx, ly >= 3 and lx_pitch >= lx, a multiple of 8");
  if (long(lx_pitch) * ly > kNoallocMaxCells)
    return fslbm_set_error(FSLBM_ERR_ARG,
                           "step_f32_noalloc: cross-section %d x %d exceeds the %d cells of the "
                           "preallocated scratch", lx_pitch, ly, kNoallocMaxCells);
  if (prm->d1 != 2)
    return fslbm_set_error(FSLBM_ERR_ARG, "step_f32_noalloc: only d1 = 2 is available (got %d)", prm->d1);
  if (prm->fd_order != 0 && prm->fd_order != 4)
    return fslbm_set_error(FSLBM_ERR_ARG, "step_f32_noalloc: corrector order %d needs the one-column kernel; "
                           "this entry point runs orders 0/4 only", prm->fd_order);
  if (lz < 2 * prm->d1 + 1)
    return fslbm_set_error(FSLBM_ERR_ARG, "step_f32_noalloc: lz = %d shorter than the stencil reach", lz);
  if ((reinterpret_cast<uintptr_t>(state_in) | reinterpret_cast<uintptr_t>(state_out)) % 16)
    return fslbm_set_error(FSLBM_ERR_ARG, "step_f32_noalloc: state pointers must be 16-byte aligned");
  const int ntx = (lx_pitch + kTX - 1) / kTX, nty = (ly + kNoallocTY - 1) / kNoallocTY;
  if (ntx * nty > kNoallocMaxTiles)
    return fslbm_set_error(FSLBM_ERR_ARG, "step_f32_noalloc: too many tiles");
  // the step reads state_in by TMA while other CTAs write state_out: they must not overlap
  const size_t state_bytes = 4 * size_t(lx_pitch) * ly * lz * sizeof(float);
  if (overlaps(state_in, state_bytes, state_out, state_bytes) ||
      overlaps(mask, size_t(lx_pitch) * ly, state_out, state_bytes))
    return fslbm_set_error(FSLBM_ERR_ARG,
                           "step_f32_noalloc: state_out overlaps state_in or mask (the step is not in place)");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fslbm_set_error(FSLBM_ERR_CUDA, "step_f32_noalloc: no usable current device");
  if (int r = setup_device(dev)) return r;
  unsigned char* scratch = static_cast<unsigned char*>(g_scratch_ptr[dev]);
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  if ((e = cudaMemsetAsync(scratch + kErrOffset, 0, sizeof(unsigned), st)) != cudaSuccess)
    return fslbm_set_error(FSLBM_ERR_CUDA, "step_f32_noalloc: %s", cudaGetErrorString(e));
  noalloc_prepare<<<64, 256, 0, st>>>(mask, lx, lx_pitch, ly, ntx, ntx * nty, gauge, scratch);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return fslbm_set_error(FSLBM_ERR_CUDA, "step_f32_noalloc: prepare: %s", cudaGetErrorString(e));

  // tensor maps of the input state: p box (one-cell halo) and u,v,w box (corrector halo)
  int sw, ph, uh, hx, hy;
  step2_box(FSLBM_F32, 2, kNoallocTY, &sw, &ph, &uh, &hx, &hy);
  const cuuint64_t fs = cuuint64_t(lx_pitch) * ly * lz;
  cuuint64_t dims[4] = {cuuint64_t(lx_pitch), cuuint64_t(ly), cuuint64_t(lz), 4};
  cuuint64_t strides[3] = {cuuint64_t(lx_pitch) * 4, cuuint64_t(lx_pitch) * ly * 4, fs * 4};
  cuuint32_t boxp[4] = {cuuint32_t(sw), cuuint32_t(ph), 1, 1};
  cuuint32_t boxu[4] = {cuuint32_t(sw), cuuint32_t(uh), 1, 3};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUtensorMap mp, mu;
  CUresult r1 = g_encode(&mp, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(state_in),
                         dims, strides, boxp, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  CUresult r2 = g_encode(&mu, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(state_in),
                         dims, strides, boxu, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r1 != CUDA_SUCCESS || r2 != CUDA_SUCCESS)
    return fslbm_set_error(FSLBM_ERR_CUDA, "step_f32_noalloc: tensor map encoding failed");

  // step constants formed as the reference forms them in FP32 (FSLBM.cu:231, 269, 599, 624)
  StepLaunch a{};
  a.dtype = FSLBM_F32; a.d1 = 2;
  a.lxp = lx_pitch; a.ly = ly; a.L = lz;
  a.ntiles = ntx * nty;
  a.tiles = reinterpret_cast<const int2*>(scratch + kCoefBytes);
  a.mask = mask;
  a.colcoef = scratch;
  a.out = state_out;
  a.gauge = reinterpret_cast<const double*>(scratch + kGaugeOffset);
  a.err = reinterpret_cast<unsigned*>(scratch + kErrOffset);
  a.counters = nullptr;
  const float tb = float(prm->tblend), nu = float(prm->nu), blend = float(prm->blend);
  a.tb = tb;
  a.cc = float(1.0 - double(tb));
  a.pin = float(prm->pin);
  a.dtddy = nu - 0.16666666f;
  a.m = float(1.0 / double(float(prm->d1 * prm->d1)));
  a.c0 = -6.0f - 1.5f * blend;
  a.c1 = 1.0f + 0.3333333333f * blend;
  a.c2 = -0.0833333333f * blend;
  a.fx = float(prm->force[0]); a.fy = float(prm->force[1]); a.fz = float(prm->force[2]);
  int nch = g_sm_count[dev] / a.ntiles;
  if (nch < 1) nch = 1;
  if (nch > lz / (4 * prm->d1)) nch = lz / (4 * prm->d1) > 0 ? lz / (4 * prm->d1) : 1;
  Step2Launch b{2, kNoallocTY, 1, &mp, &mu, a.ntiles * nch};
  if ((e = launch_step2(a, b, st)) != cudaSuccess)
    return fslbm_set_error(FSLBM_ERR_CUDA, "step_f32_noalloc: step launch: %s", cudaGetErrorString(e));

  // synchronous: wait for the step, then read the kernel's bounded-wait error flag
  unsigned err = 0;
  e = cudaMemcpyFromSymbolAsync(&err, g_noalloc_scratch, sizeof(err), kErrOffset,
                                cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return fslbm_set_error(FSLBM_ERR_CUDA, "step_f32_noalloc: %s", cudaGetErrorString(e));
  if (err & kErrBadMask)
    return fslbm_set_error(FSLBM_ERR_ARG,
                           "step_f32_noalloc: mask values must be 0 or 125, with wall on the rim and "
                           "in the padding columns (state_out is not a valid step)");
  if (err)
    return fslbm_set_error(FSLBM_ERR_TIMEOUT, "step_f32_noalloc: a bounded device wait gave up");
  return FSLBM_OK;
}
