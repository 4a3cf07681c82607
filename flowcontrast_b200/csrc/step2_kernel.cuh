// FSLBM time step, FP32 column-pair kernel for sm_100a (even corrective strides).
//
// Same step as step_kernel.cuh (predictor factored by neighbour plane, coarse corrector,
// periodic +-pin seam, walls, gauge, body force), organised for throughput:
//  - every thread owns two adjacent columns (x, x+1) and computes both with packed FP32x2
//    arithmetic (__ffma2_rn / __fadd2_rn / __fmul2_rn); neighbour pairs come from 64-bit
//    shared-memory loads;
//  - a 32 x TY tile per CTA, 16 warps per SM either way (TY = 32: one 512-thread CTA per SM;
//    TY = 16: two 256-thread CTAs, which suit small cross-sections); p is staged with a one-cell
//    halo, u,v,w with the corrector's 2*d1 halo, as two TMA boxes per plane into a window of 8
//    planes for TY = 32 (output plane .. 3 planes ahead for d1 = 2), 7 for TY = 16;
//  - no block-wide barrier in the march and no producer thread: per-slot "full" mbarriers count
//    TMA completion, each warp releases the slots of a pair of planes after its last read of
//    them, and the last warp to release a pair refills both slots, so warps drift within the
//    window and none waits for a free slot;
//  - the streamwise corrector taps behind the output plane come from a 2*d1 register history
//    of the thread's own columns, the taps ahead from the window; in the FP32 single-pipe
//    kernel the output plane's own centre pairs come from the predictor's centre row of the
//    same plane, read one iteration earlier;
//  - grid = tiles x streamwise chunks in chunk-major order, so concurrent CTAs work at nearby
//    planes and halos hit L2; odd chunks march downwards, so the planes two neighbouring
//    chunks share are read by both at the same time;
//  - warps whose cells are all wall keep the pipeline protocol but skip the arithmetic.
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "common.h"
#include "ptx.cuh"
#include "step_kernel.cuh"

namespace fslbm {

// TE is the storage type of the state (float, or __half for FP16 storage); arithmetic is FP32
// either way. Halo widths and paddings keep every TMA box start and destination on 16 bytes.
template <int D1, int TY, class TE = float> struct Step2Tile {
  static_assert(D1 % 2 == 0, "pair loads of the corrector taps need an even stride");
  static constexpr int ES = int(sizeof(TE));
  static constexpr int A16 = 16 / ES;                   // elements per 16 bytes
  static constexpr int TX = 32;
  static constexpr int THREADS = TX / 2 * TY;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int R = 2 * D1;                      // farthest corrector tap
  static constexpr int HX = (R + A16 - 1) / A16 * A16;  // x halo, TMA-aligned (16 bytes)
  static constexpr int HY = R;
  static constexpr int SW = TX + 2 * HX;                // row length of both boxes
  static constexpr int PH = TY + 2;                     // p rows (halo 1)
  static constexpr int UH = TY + 2 * HY;                // u,v,w rows
  static constexpr int PPLANE = (SW * PH * ES + 127) / 128 * 128 / ES;   // 128-byte aligned
  static constexpr int UPLANE = SW * UH;
  static constexpr int SLOT = PPLANE + 3 * UPLANE;
  // window slots: 8 for 32 x 32 tiles (one 512-thread CTA per SM), 7 for 32 x 16 tiles, so that
  // two 256-thread CTAs fit an SM's shared memory
  static constexpr int S = TY == 16 ? 7 : 8;
  static constexpr int AHEAD = S - R - 1;               // planes loaded beyond the current one
  static_assert(AHEAD >= 1, "window too small for the corrector reach");
  static constexpr uint32_t TX_BYTES = uint32_t((SW * PH + 3 * UPLANE) * ES);
  static constexpr size_t RING_BYTES = size_t(S) * SLOT * ES;
  static constexpr size_t BAR_OFFSET = RING_BYTES;
  // FP16 storage: the tile's base of w (FP32) for columns org.x-2 .. org.x+TX+1 and rows
  // org.y-1 .. org.y+TY, after the barriers and counters
  static constexpr int BW = TX + 4, BH = TY + 2;
  static constexpr size_t BASE_OFFSET = (BAR_OFFSET + S * sizeof(uint64_t) + S * sizeof(uint32_t) + 15) / 16 * 16;
  static constexpr size_t BASE_BYTES = std::is_same<TE, __half>::value ? size_t(BW) * BH * sizeof(float) : 0;
  // a "full" mbarrier per slot, then a release counter per slot
  static constexpr size_t SMEM_BYTES = BASE_BYTES ? BASE_OFFSET + BASE_BYTES
                                                  : BAR_OFFSET + S * sizeof(uint64_t) + S * sizeof(uint32_t);
  static_assert((PPLANE * ES) % 128 == 0 && (UPLANE * ES) % 16 == 0 && (SLOT * ES) % 128 == 0,
                "TMA destinations must stay aligned");
  static_assert((HX * ES) % 16 == 0, "TMA box x start must be 16-byte aligned");
};

struct Step2Geom {
  int lxp, ly, L;
  int ntiles, nchunks;     // grid = ntiles * nchunks, chunk-major
  const int2* tiles;
  const uint8_t* mask;
  const void* colcoef;     // ColCoef<float>[lxp*ly]
  void* out;
  const double* gauge;
  unsigned* err;
  long long* step_counter;
  unsigned step_no;        // time step being computed (seed of the FP16 stochastic rounding)
  // FP16 storage: stored w is w - wb (per-column base, FP32); wgt is the base's share of a step
  // of the stored w. Null for other storage types.
  const float* wb;
  const float* wgt;
};

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 lds2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ float2 lds2(const __half* p) {
  return __half22float2(*reinterpret_cast<const __half2*>(p));
}

// 32-bit integer hash (the "lowbias32" finaliser of C. Wellons' hash-prospector, public domain).
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}

// FP32 -> FP16 with stochastic rounding: uniform noise below FP16's last kept bit is added to
// the magnitude, which is then truncated. The result is unbiased, so increments far below half
// an FP16 ulp (the body force and the slow relaxation of the step) survive in expectation
// instead of being rounded away. The kept bit is the 11th of the significand, 2^(e-10) for
// |x| in [2^e, 2^(e+1)), and fixed at 2^-24 below 2^-14 (FP16 subnormals, which the deviations
// of FP16 storage often reach): the noise is 13 random bits scaled to 2^(max(e,-14)-23), formed
// without a branch (measured +0.9 % on the FP16 step against branching on the subnormal range).
// In FP16's normal range the noise's lowest bit is x's FP32 resolution, so the sum is exact.
__device__ __forceinline__ __half sr_half(float x, uint32_t r) {
  const uint32_t ex = max(__float_as_uint(x) & 0x7f800000u, 0x38800000u);   // exponent of max(|x|, 2^-14)
  const float noise = float(r & 0x1fffu) * __uint_as_float(ex - (23u << 23));
  return __float2half_rz(x + copysignf(noise, x));
}

// Stores of one column pair's four fields. FP32 storage stores the values; FP16 storage rounds
// stochastically with noise from (pair index, field, time step) only, so a pipe's result does
// not depend on which other work shares the launch.
template <class TE> struct PairStore;
template <> struct PairStore<float> {
  static __device__ __forceinline__ void put(float* o, size_t fs, float2 p, float2 u, float2 v,
                                             float2 w, const float*, uint32_t) {
    *reinterpret_cast<float2*>(o) = p;
    *reinterpret_cast<float2*>(o + fs) = u;
    *reinterpret_cast<float2*>(o + 2 * fs) = v;
    *reinterpret_cast<float2*>(o + 3 * fs) = w;
  }
};
template <> struct PairStore<__half> {
  static __device__ __forceinline__ __half2 sr2(float2 a, uint32_t r) {
    return __halves2half2(sr_half(a.x, r), sr_half(a.y, r >> 16));
  }
  static __device__ __forceinline__ void put(__half* o, size_t fs, float2 p, float2 u, float2 v,
                                             float2 w, const __half* base, uint32_t seed) {
    const uint32_t key = uint32_t(o - base) << 2;
    *reinterpret_cast<__half2*>(o) = sr2(p, hash32(key ^ seed));
    *reinterpret_cast<__half2*>(o + fs) = sr2(u, hash32((key | 1u) ^ seed));
    *reinterpret_cast<__half2*>(o + 2 * fs) = sr2(v, hash32((key | 2u) ^ seed));
    *reinterpret_cast<__half2*>(o + 3 * fs) = sr2(w, hash32((key | 3u) ^ seed));
  }
};

// Column-pair arithmetic: packed FP32x2 instructions (PK = true) or two scalar ones.
template <bool PK> struct Pair;
template <> struct Pair<true> {
  static __device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
  static __device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
  static __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
};
template <> struct Pair<false> {
  static __device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
  static __device__ __forceinline__ float2 mul(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
  static __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) {
    return make_float2(__fmaf_rn(a.x, b.x, c.x), __fmaf_rn(a.y, b.y, c.y));
  }
};

// Predictor brackets of one in-plane neighbour (cx, cy), see step_kernel.cuh:
// P0 = q + a(3 + 4.5a), P1' = w(1 + 3a) (= P1/3), P2' = w^2 (= P2/4.5), a = cx u + cy v.
template <bool PK, int CX, int CY>
__device__ __forceinline__ void brackets(float2 Q, float2 U, float2 V, float2 W, float2& P0,
                                         float2& P1, float2& P2) {
  using F = Pair<PK>;
  P2 = F::mul(W, W);
  if (CX == 0 && CY == 0) {
    P0 = Q;
    P1 = W;
  } else if (CY == 0 || CX == 0) {
    // a = s*B, s = +-1: a(3 + 4.5a) = B(3s + 4.5B), 1 + 3a = 1 + 3sB
    const float2 B = CY == 0 ? U : V;
    constexpr float s = float(CX + CY);
    P0 = F::fma(B, F::fma(B, f2(4.5f), f2(3.0f * s)), Q);
    P1 = F::mul(W, F::fma(B, f2(3.0f * s), f2(1.0f)));
  } else {
    // a = CX (U + CX*CY V) = CX a': a(3 + 4.5a) = a'(3 CX + 4.5 a'), 1 + 3a = 1 + 3 CX a'
    const float2 a1 = F::fma(V, f2(float(CX * CY)), U);
    P0 = F::fma(a1, F::fma(a1, f2(4.5f), f2(3.0f * CX)), Q);
    P1 = F::mul(W, F::fma(a1, f2(3.0f * CX), f2(1.0f)));
  }
}

template <bool PK>
__device__ __forceinline__ float2 qof(float2 P, float2 U, float2 V, float2 W) {
  using F = Pair<PK>;
  return F::fma(f2(-1.5f), F::fma(U, U, F::fma(V, V, F::mul(W, W))), P);
}

// Marches one (tile, chunk) work item of one pipe: the step of every cell of the tile's columns
// in the chunk's planes. `reinit` re-arms the CTA's mbarriers when the CTA has marched an item
// before (persistent grids). Returns false when a bounded wait gave up (error flag set).
// Freed window slots are refilled by the last warp to release them (no warp waits for a free
// slot); measured +2 % on the single pipe and +1.7 % on the batched ensemble against thread 0
// waiting on per-slot "empty" mbarriers and refilling.
// The warp shape (below) is a runtime argument: it only places each thread in the tile, and a
// kernel that inlines one march for every shape (the batched kernel, whose members choose their
// shape) keeps one copy of the march instead of one per shape, which ended its register spills.
// kCarry: the output plane's centre pairs come from the predictor's centre row of the same plane
// (one iteration earlier, 8 registers held) instead of 4 shared loads per plane: +1.0 % on the
// single FP32 pipe, -9 % in the batched kernel and -3 % with FP16 storage, which therefore do
// not use it.
template <int D1, int TY, bool PK, class TE, bool kCarry = false>
__device__ __forceinline__ bool step2_march(const CUtensorMap* tmap_p, const CUtensorMap* tmap_uvw,
                                            const Step2Geom& g, const StepConst<float>& k,
                                            int tile, int chunk, unsigned char* smem, bool reinit,
                                            int shape = 0) {
  using Tl = Step2Tile<D1, TY, TE>;
  using F = Pair<PK>;
  static_assert(D1 == 2, "the march prologue below is written for d1 = 2 (R = 4)");
  constexpr int R = Tl::R, HX = Tl::HX, HY = Tl::HY, SW = Tl::SW, S = Tl::S;
  constexpr int PPL = Tl::PPLANE, UPL = Tl::UPLANE, SLOT = Tl::SLOT;

  // window slot of march plane m and the parity of its fill (m >= 0)
  auto slot_of = [](int m) { return int(unsigned(m) % unsigned(S)); };
  auto phase_of = [](int m) { return uint32_t((unsigned(m) / unsigned(S)) & 1u); };
  TE* ring = reinterpret_cast<TE*>(smem);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + Tl::BAR_OFFSET);
  // per slot: warp releases, counted to elect the refilling warp
  unsigned* released = reinterpret_cast<unsigned*>(full + S);

  // Warp shape. 0: 32 columns x 2 rows (each half-warp reads one contiguous row); 1: 16 columns
  // (8 pairs) x 4 rows; 2: 8 columns (4 pairs) x 8 rows. The smaller shapes let warps over wall
  // skip at a finer grain, which pays for small cross-sections (16 x 4: measured +6 % on the
  // mixed-size ensemble, -2 % on the 128 x 128 pipe). 16 x 4: lanes 0-15 take rows 0 and 2 of
  // the warp, lanes 16-31 rows 1 and 3; 8 x 8: lanes 4r .. 4r+3 take row r. With the 160-byte
  // FP32 row stride each half-warp's 64-bit shared loads fall on distinct banks in every shape
  // (FP16 rows of 96 bytes: conflict-free for 32 x 2 and 16 x 4, two-way for 8 x 8). The map
  // changes no thread's arithmetic.
  static_assert(Tl::TX == 32 && TY % 8 == 0, "warp shapes within a 32-wide tile");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int tp = tid % (Tl::TX / 2), ty = tid / (Tl::TX / 2);
  if (shape == 1) {
    tp = (warp & 1) * 8 + (lane & 7);
    ty = (warp >> 1) * 4 + ((lane >> 3) & 1) * 2 + (lane >> 4);
  } else if (shape == 2) {
    tp = (warp & 3) * 4 + (lane & 3);
    ty = (warp >> 2) * 8 + (lane >> 2);
  }

  // ---- work: one (tile, chunk); odd chunks march towards -z
  const int zb = int((long long)g.L * chunk / g.nchunks);
  const int ze = int((long long)g.L * (chunk + 1) / g.nchunks);
  const int dir = (chunk & 1) ? -1 : 1;
  const int nout = ze - zb, niter = nout + 2 * R;
  const int start = dir > 0 ? zb - R : ze - 1 + R;      // real plane of march index 0
  const int2 org = g.tiles[tile];
  const int xa = org.x + 2 * tp, y = org.y + ty;
  const bool inside = xa < g.lxp && y < g.ly;

  float2 ws0 = f2(0.f), wsx = f2(0.f), wsy = f2(0.f), fl = f2(0.f);
  if (inside) {
    const ColCoef<float>* cp = reinterpret_cast<const ColCoef<float>*>(g.colcoef) + size_t(y) * g.lxp + xa;
    const ColCoef<float> ca = cp[0], cb = cp[1];
    ws0 = make_float2(ca.ws0, cb.ws0); wsx = make_float2(ca.wsx, cb.wsx);
    wsy = make_float2(ca.wsy, cb.wsy); fl = make_float2(ca.fluid, cb.fluid);
  }
  const bool warp_on = __any_sync(0xffffffffu, fl.x != 0.f || fl.y != 0.f);

  __syncthreads();   // a previous item (persistent grids) is fully consumed
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      if (reinit) mbar_inval(&full[s]);
      mbar_init(&full[s], 1);
      released[s] = 0u;
    }
    mbar_init_fence();
  }
  // FP16 storage: the tile's base of w (zero outside the cross-section), read by the predictor
  constexpr bool kBase = std::is_same<TE, __half>::value;
  float* wbs = reinterpret_cast<float*>(smem + Tl::BASE_OFFSET);
  if (kBase && g.wb)
    for (int i = tid; i < Tl::BW * Tl::BH; i += Tl::THREADS) {
      const int gx = org.x - 2 + i % Tl::BW, gy = org.y - 1 + i / Tl::BW;
      wbs[i] = (gx >= 0 && gy >= 0 && gx < g.lxp && gy < g.ly) ? g.wb[size_t(gy) * g.lxp + gx] : 0.0f;
    }
  __syncthreads();

  auto issue = [&](int m) {            // load march plane m into slot m % S
    const int slot = slot_of(m);
    int zz = (start + dir * m) % g.L;
    if (zz < 0) zz += g.L;
    TE* dst = ring + slot * SLOT;
    mbar_arrive_expect_tx(&full[slot], Tl::TX_BYTES);
    tma_load_4d(dst, tmap_p, &full[slot], org.x - HX, org.y - 1, zz, 0);
    tma_load_4d(dst + PPL, tmap_uvw, &full[slot], org.x - HX, org.y - HY, zz, 1);
  };
  if (tid == 0) {                      // the whole ring up front
    prefetch_tensormap(tmap_p);
    prefetch_tensormap(tmap_uvw);
    for (int m = 0; m < S && m < niter; ++m) issue(m);
  }
  // failure path: any warp may have issued loads up to S planes ahead; let them land (bounded)
  auto drain = [&](int from) {
    if (lane == 0)
      for (int q = from; q < niter && q < from + S; ++q)
        mbar_wait_bounded(&full[slot_of(q)], phase_of(q), kWaitLimitNs / 8);
  };
  // wait for march plane m; false after flagging a failure (the caller returns)
  auto arrive_wait = [&](int m) -> bool {
    if (mbar_wait_bounded(&full[slot_of(m)], phase_of(m), kWaitLimitNs)) return true;
    if (lane == 0) atomicOr(g.err, 1u);
    drain(m + 1);
    return false;
  };
  // Plane m - R leaves the window at iteration m (its last reader is output(m - R)). Planes leave
  // in pairs: at odd p = m - R, planes p - 1 and p, whose slots take planes p - 1 + S and p + S.
  // __syncwarp orders the warp's shared loads before lane 0's acq_rel add to the pair's counter
  // (the slot of plane p); the warp whose add completes the count has acquired every warp's loads
  // and orders them before its TMA writes with a proxy fence. One add per two planes halves the
  // release cost, which is a fence-like wait (measured: plain step +1.5 %, batched ensemble +9 %).
  // Plane m fills the slot of plane m - S, so a warp waiting for plane m needs every warp to have
  // released at iteration m - AHEAD at the latest (instead of m - AHEAD - 1): an earlier
  // iteration, as AHEAD >= 1, so no wait depends on itself. A counter's next use (2S planes later
  // for odd S, S for S = 8) comes only after every warp has passed its previous use, so the count
  // is a multiple of WARPS exactly when a pair is complete.
  auto release_produce = [&](int m) -> bool {
    __syncwarp();
    if (m >= R && ((m - R) & 1) && lane == 0) {
      const int slot = slot_of(m - R);
      const unsigned seen = atom_add_acq_rel_cta(&released[slot], 1u) + 1u;
      const int mn = m - R + S - 1;
      if (seen % unsigned(Tl::WARPS) == 0u && mn < niter) {
        fence_proxy_async_smem();
        issue(mn);
        if (mn + 1 < niter) issue(mn + 1);
      }
    }
    return true;
  };

  if (!warp_on) {   // all-wall warps keep the pipeline protocol only
    for (int m = 0; m < niter; ++m)
      if (!arrive_wait(m) || !release_produce(m)) return false;
    return true;
  }

  // the gauge may have been written by another CTA of the same (chained batched) launch: read
  // it from L2, not from a possibly stale L1 line
  const float gauge = g.gauge ? float(__ldcg(g.gauge)) : 0.0f;
  const float2 wgt2 = (kBase && g.wgt && inside) ? *reinterpret_cast<const float2*>(g.wgt + size_t(y) * g.lxp + xa)
                                                 : f2(0.f);
  const size_t FS = size_t(g.lxp) * g.ly * g.L;
  const TE* obase = reinterpret_cast<const TE*>(g.out);
  const uint32_t seed = hash32(g.step_no * 0x9e3779b9u + 0x632be5abu);
  TE* outp = reinterpret_cast<TE*>(g.out) + (size_t(start + dir * R) * g.ly + y) * g.lxp + xa;
  const long long ostep = (long long)dir * g.ly * g.lxp;     // output pointer step per plane
  const int po = (ty + 1) * SW + HX + 2 * tp;                 // p box
  const int uo = PPL + (ty + HY) * SW + HX + 2 * tp;          // u box (v, w at +UPL, +2 UPL)
  // seam pressure jump: a wrapped plane adds off to p on its non-wall cells, i.e. off times the
  // non-wall weight sums (raw units, x36) to the row-factored A0, X0, Y0
  const float n0[2] = {36.f - 36.f * ws0.x, 36.f - 36.f * ws0.y};
  const float nx[2] = {-36.f * wsx.x, -36.f * wsx.y};
  const float ny[2] = {-36.f * wsy.x, -36.f * wsy.y};
  const float h6 = float(dir) / 72.0f;
  // folded update: u_new = K1 t1 + K2 t2 + K0 u + tb (u* + F), the corrector's taps t1 / t2 at
  // distance d1 / 2 d1, K0 = tb dtddy m c0 + (1 - tb), K1 = tb dtddy m c1, K2 = tb dtddy m c2
  const float kam = __fmul_rn(__fmul_rn(k.tb, k.dtddy), k.m);
  const float kK0 = __fmaf_rn(kam, k.c0, k.cc), kK1 = __fmul_rn(kam, k.c1), kK2 = __fmul_rn(kam, k.c2);
  const float ktz = __fmul_rn(float(dir), k.tb);              // the z-moment carries the sign

  float2 hu[4], hv[4], hw[4];                                 // own columns of planes jo-4..jo-1
  // Predictor terms waiting for their output plane: b2 = the march-previous plane's share of the
  // output being completed, b1 = the same for the next output, s1 = the self-plane moments of
  // the next output. Each output sums its two neighbour planes' shares first (a commutative
  // add) and then fuses its own plane's share, so the FP32 result of a cell does not depend on
  // the march direction and hence not on how the pipe is split into streamwise chunks.
  float b2[4][2], b1[4][2], s1[3][2];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    hu[j] = hv[j] = hw[j] = f2(0.f);
    b2[j][0] = b2[j][1] = b1[j][0] = b1[j][1] = 0.f;
    if (j < 3) s1[j][0] = s1[j][1] = 0.f;
  }
  float2 comp0, comp1, comp2, comp3;
  float2 cen[4] = {}, cnx[4] = {};   // kCarry: centre pairs p,u,v,w of the output plane / the predictor plane

  // predictor contribution of march plane ma (see step_kernel.cuh for the factorisation)
  auto predictor = [&](int ma) {
    const TE* ss = ring + slot_of(ma) * SLOT;
    const int sp = start + dir * ma;                          // real plane
    const float off = sp < 0 ? k.pin : (sp >= g.L ? -k.pin : 0.0f);
    // Row-factored weights w(cx)w(cy) = {4,1,1}x{4,1,1}/36, per column of the pair: per row
    // R = P(-1)+P(+1)+4P(0), D = P(+1)-P(-1); across rows A = R(-1)+R(+1)+4R(0), X likewise on
    // D, Y = R(+1)-R(-1). The four cells x-1..x+2 of a row are shared by the two columns, so q
    // and w^2 are formed once per cell.
    float A[2][3], X[2][3], Y[2][3];
#pragma unroll
    for (int cy = -1; cy <= 1; ++cy) {
      const TE* rp = ss + po + cy * SW;
      const TE* rq = ss + uo + cy * SW;
      const float2 pL = lds2(rp - 2), pC = lds2(rp), pR = lds2(rp + 2);
      if (kCarry && cy == 0) cnx[0] = pC;
      const float2 uL = lds2(rq - 2), uC = lds2(rq), uR = lds2(rq + 2);
      const float2 vL = lds2(rq + UPL - 2), vC = lds2(rq + UPL), vR = lds2(rq + UPL + 2);
      const float2 wL = lds2(rq + 2 * UPL - 2), wC = lds2(rq + 2 * UPL), wR = lds2(rq + 2 * UPL + 2);
      if (kCarry && cy == 0) { cnx[1] = uC; cnx[2] = vC; cnx[3] = wC; }
      const float pc4[4] = {pL.y, pC.x, pC.y, pR.x};
      const float uc4[4] = {uL.y, uC.x, uC.y, uR.x};
      const float vc4[4] = {vL.y, vC.x, vC.y, vR.x};
      float wc4[4] = {wL.y, wC.x, wC.y, wR.x};
      if (kBase && g.wb) {             // w = stored deviation + the column's base
        const float* br = wbs + (ty + 1 + cy) * Tl::BW + 2 * tp;
        const float2 bL = *reinterpret_cast<const float2*>(br), bC = *reinterpret_cast<const float2*>(br + 2),
                     bR = *reinterpret_cast<const float2*>(br + 4);
        wc4[0] = __fadd_rn(wc4[0], bL.y); wc4[1] = __fadd_rn(wc4[1], bC.x);
        wc4[2] = __fadd_rn(wc4[2], bC.y); wc4[3] = __fadd_rn(wc4[3], bR.x);
      }
      float q4[4], w24[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        w24[j] = wc4[j] * wc4[j];
        q4[j] = __fmaf_rn(-1.5f, __fmaf_rn(uc4[j], uc4[j], __fmaf_rn(vc4[j], vc4[j], w24[j])), pc4[j]);
      }
#pragma unroll
      for (int col = 0; col < 2; ++col) {
        float P[3][3];   // [cx+1][k]
#pragma unroll
        for (int cx = -1; cx <= 1; ++cx) {
          const int j = col + 1 + cx;
          const float u = uc4[j], v = vc4[j], w = wc4[j];
          float P0, P1;
          if (cx == 0 && cy == 0) {
            P0 = q4[j];
            P1 = w;
          } else if (cx == 0 || cy == 0) {
            const float Bv = cy == 0 ? u : v;
            const float s3 = 3.0f * float(cx + cy);
            P0 = __fmaf_rn(Bv, __fmaf_rn(Bv, 4.5f, s3), q4[j]);
            P1 = w * __fmaf_rn(Bv, s3, 1.0f);
          } else {
            const float a1 = __fmaf_rn(v, float(cx * cy), u);
            const float s3 = 3.0f * float(cx);
            P0 = __fmaf_rn(a1, __fmaf_rn(a1, 4.5f, s3), q4[j]);
            P1 = w * __fmaf_rn(a1, s3, 1.0f);
          }
          P[cx + 1][0] = P0; P[cx + 1][1] = P1; P[cx + 1][2] = w24[j];
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const float Rq = __fmaf_rn(4.0f, P[1][q], P[0][q] + P[2][q]);
          const float Dq = P[2][q] - P[0][q];
          if (cy == -1) { A[col][q] = Rq; X[col][q] = Dq; Y[col][q] = Rq; }
          else if (cy == 0) { A[col][q] = __fmaf_rn(4.0f, Rq, A[col][q]); X[col][q] = __fmaf_rn(4.0f, Dq, X[col][q]); }
          else { A[col][q] += Rq; X[col][q] += Dq; Y[col][q] = Rq - Y[col][q]; }
        }
      }
    }
    // True sums are A0'/36, dir A1'/12, A2'/8 (P1 and P2 were formed as P1/3 and P2/4.5).
    // Plane ma is the march-next neighbour of output ma-1 (completed here), itself, and the
    // march-previous neighbour of ma+1: with e = (A0 + A2)/6 and h = A1/6 the shares are
    // e + h (next), (2/3) A0 (self) and e - h (previous); for the z-moment h - e (previous),
    // none (self) and e + h (next), times dir.
    float cmp[4][2];
    if (sp < 0 || sp >= g.L) {         // seam plane (CTA-uniform): the pressure jump's share
#pragma unroll
      for (int col = 0; col < 2; ++col) {
        A[col][0] = __fmaf_rn(off, n0[col], A[col][0]);
        X[col][0] = __fmaf_rn(off, nx[col], X[col][0]);
        Y[col][0] = __fmaf_rn(off, ny[col], Y[col][0]);
      }
    }
#pragma unroll
    for (int col = 0; col < 2; ++col) {
      const float A0 = A[col][0], X0 = X[col][0], Y0 = Y[col][0];
      const float eA = __fmaf_rn(A[col][2], 1.0f / 48.0f, __fmul_rn(A0, 1.0f / 216.0f));
      const float eX = __fmaf_rn(X[col][2], 1.0f / 48.0f, __fmul_rn(X0, 1.0f / 216.0f));
      const float eY = __fmaf_rn(Y[col][2], 1.0f / 48.0f, __fmul_rn(Y0, 1.0f / 216.0f));
      // e + h and e - h with h = A1 h6, each one fused rounding
      const float sA = __fmaf_rn(A[col][1], h6, eA), dA = __fmaf_rn(A[col][1], -h6, eA);
      const float sX = __fmaf_rn(X[col][1], h6, eX), dX = __fmaf_rn(X[col][1], -h6, eX);
      const float sY = __fmaf_rn(Y[col][1], h6, eY), dY = __fmaf_rn(Y[col][1], -h6, eY);
      cmp[0][col] = __fmaf_rn(s1[0][col], 1.0f / 54.0f, __fadd_rn(b2[0][col], sA));
      cmp[1][col] = __fmaf_rn(s1[1][col], 1.0f / 54.0f, __fadd_rn(b2[1][col], sX));
      cmp[2][col] = __fmaf_rn(s1[2][col], 1.0f / 54.0f, __fadd_rn(b2[2][col], sY));
      cmp[3][col] = __fadd_rn(b2[3][col], sA);
#pragma unroll
      for (int q = 0; q < 4; ++q) b2[q][col] = b1[q][col];
      b1[0][col] = dA;
      b1[1][col] = dX;
      b1[2][col] = dY;
      b1[3][col] = -dA;
      s1[0][col] = A0;
      s1[1][col] = X0;
      s1[2][col] = Y0;
    }
    comp0 = make_float2(cmp[0][0], cmp[0][1]);
    comp1 = make_float2(cmp[1][0], cmp[1][1]);
    comp2 = make_float2(cmp[2][0], cmp[2][1]);
    comp3 = make_float2(cmp[3][0], cmp[3][1]);
  };

  // own columns of march plane jo (for the history)
  auto own = [&](int jo, float2& uc, float2& vc, float2& wc) {
    const TE* so = ring + slot_of(jo) * SLOT;
    uc = lds2(so + uo); vc = lds2(so + uo + UPL); wc = lds2(so + uo + 2 * UPL);
  };

  // corrector and update of output march plane jo; hist slot ROT holds plane jo-4 and is then
  // overwritten with plane jo
  auto output = [&](int jo, auto rot_c) {
    constexpr int ROT = decltype(rot_c)::value;
    const TE* so = ring + slot_of(jo) * SLOT;
    const TE* sa1 = ring + slot_of(jo + D1) * SLOT;   // march planes ahead
    const TE* sa2 = ring + slot_of(jo + 2 * D1) * SLOT;
    float2 pc, uc, vc, wc;
    if (kCarry) {
      pc = cen[0]; uc = cen[1]; vc = cen[2]; wc = cen[3];
#pragma unroll
      for (int q = 0; q < 4; ++q) cen[q] = cnx[q];
    } else {
      pc = lds2(so + po);
      uc = lds2(so + uo); vc = lds2(so + uo + UPL); wc = lds2(so + uo + 2 * UPL);
    }
    // u_new = K1 t1 + K2 t2 + K0 u + tb m* + tb F
    auto update = [&](int f, float2 c, float2 zb1, float2 zb2, float2 mom, float tm, float2 tf) {
      const TE* q = so + uo + f * UPL;
      const float2 za1 = lds2(sa1 + uo + f * UPL), za2 = lds2(sa2 + uo + f * UPL);
      const float2 t1 = F::add(F::add(F::add(lds2(q - D1), lds2(q + D1)),
                                      F::add(lds2(q - D1 * SW), lds2(q + D1 * SW))),
                               F::add(zb1, za1));
      const float2 t2 = F::add(F::add(F::add(lds2(q - 2 * D1), lds2(q + 2 * D1)),
                                      F::add(lds2(q - 2 * D1 * SW), lds2(q + 2 * D1 * SW))),
                               F::add(zb2, za2));
      return F::fma(f2(kK1), t1, F::fma(f2(kK2), t2, F::fma(f2(kK0), c, F::fma(f2(tm), mom, tf))));
    };
    constexpr int H2 = (ROT + 2) & 3;                         // plane jo-2
    const float2 rho = F::add(F::fma(pc, ws0, comp0), f2(-gauge));
    const float2 us = F::fma(pc, wsx, comp1), vs = F::fma(pc, wsy, comp2);
    const float2 un = update(0, uc, hu[H2], hu[ROT], us, k.tb, f2(__fmul_rn(k.tb, k.fx)));
    const float2 vn = update(1, vc, hv[H2], hv[ROT], vs, k.tb, f2(__fmul_rn(k.tb, k.fy)));
    // FP16 storage updates the stored deviation of w: the force's term becomes the column's share
    // of the step of the base (tb fz included), see launch_wgt
    const float2 wn = update(2, wc, hw[H2], hw[ROT], comp3, ktz,
                             (kBase && g.wgt) ? wgt2 : f2(__fmul_rn(k.tb, k.fz)));
    hu[ROT] = uc; hv[ROT] = vc; hw[ROT] = wc;
    if (inside) {   // wall columns get zero (fl = 0)
      if (fl.x != 0.f && fl.y != 0.f)
        PairStore<TE>::put(outp, FS, rho, un, vn, wn, obase, seed);
      else
        PairStore<TE>::put(outp, FS, F::mul(rho, fl), F::mul(un, fl), F::mul(vn, fl),
                           F::mul(wn, fl), obase, seed);
    }
    outp += ostep;
  };

  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  using I3 = std::integral_constant<int, 3>;
  // ---- prologue (R = 4): planes 0..3 arrive; 4..5 enter the history; 6..7 also start the
  // predictor sums of the first output
#pragma unroll
  for (int m = 0; m < 2 * R; ++m) {
    if (!arrive_wait(m)) return false;
    if (m >= 2 * R - 2) predictor(m - R + 1);
    if (m >= R) {
      float2 uc, vc, wc;
      own(m - R, uc, vc, wc);
      const int h = (m - R) & 3;
      if (h == 0) { hu[0] = uc; hv[0] = vc; hw[0] = wc; }
      else if (h == 1) { hu[1] = uc; hv[1] = vc; hw[1] = wc; }
      else if (h == 2) { hu[2] = uc; hv[2] = vc; hw[2] = wc; }
      else { hu[3] = uc; hv[3] = vc; hw[3] = wc; }
    }
    if (!release_produce(m)) return false;
  }
  if (kCarry)                          // the first output's centre pairs
#pragma unroll
    for (int q = 0; q < 4; ++q) cen[q] = cnx[q];
  // ---- steady state, four planes per pass (the history period)
  for (int m = 2 * R; m < niter; m += 4) {
    if (!arrive_wait(m)) return false;
    predictor(m - R + 1);
    output(m - R, I0{});
    if (!release_produce(m)) return false;
    if (m + 1 >= niter) break;
    if (!arrive_wait(m + 1)) return false;
    predictor(m - R + 2);
    output(m - R + 1, I1{});
    if (!release_produce(m + 1)) return false;
    if (m + 2 >= niter) break;
    if (!arrive_wait(m + 2)) return false;
    predictor(m - R + 3);
    output(m - R + 2, I2{});
    if (!release_produce(m + 2)) return false;
    if (m + 3 >= niter) break;
    if (!arrive_wait(m + 3)) return false;
    predictor(m - R + 4);
    output(m - R + 3, I3{});
    if (!release_produce(m + 3)) return false;
  }
  return true;
}

// One pipe, one step: CTA b marches (tile b % ntiles, chunk b / ntiles).
template <int D1, int TY, bool PK, class TE>
__global__ void __launch_bounds__(Step2Tile<D1, TY, TE>::THREADS, TY == 16 ? 2 : 1)
    fslbm_step2_kernel(const __grid_constant__ CUtensorMap tmap_p,
                       const __grid_constant__ CUtensorMap tmap_uvw, const Step2Geom g,
                       const StepConst<float> k) {
  extern __shared__ __align__(128) unsigned char smem[];
  if (threadIdx.x == 0 && blockIdx.x == 0 && g.step_counter) *g.step_counter += 1;
  // centre pairs carried for FP32 storage (FP16 storage measured 3 % slower with them)
  step2_march<D1, TY, PK, TE, std::is_same<TE, float>::value>(&tmap_p, &tmap_uvw, g, k, blockIdx.x % g.ntiles,
                                                              blockIdx.x / g.ntiles, smem, false);
}

}  // namespace fslbm
