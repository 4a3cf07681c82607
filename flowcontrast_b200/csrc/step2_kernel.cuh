// FSLBM time step, FP32 column-pair kernel for sm_100a (even corrective strides).
//
// Same step as step_kernel.cuh (predictor factored by neighbour plane, coarse corrector,
// periodic +-pin seam, walls, gauge, body force), organised for throughput:
//  - every thread owns two adjacent columns (x, x+1) and computes both with packed FP32x2
//    arithmetic (__ffma2_rn / __fadd2_rn / __fmul2_rn); neighbour pairs come from 64-bit
//    shared-memory loads;
//  - a 32 x TY tile per CTA (512 threads for TY = 32, 16 warps per SM); p is staged with a
//    one-cell halo, u,v,w with the corrector's 2*d1 halo, as two TMA boxes per plane into a
//    window of 8 planes (output plane .. 3 planes ahead for d1 = 2);
//  - no block-wide barrier in the march: per-slot "full" mbarriers (TMA completion) and
//    "empty" mbarriers (one arrival per warp after its last read of a plane) pace one producer
//    thread, so warps drift within the window;
//  - the streamwise corrector taps behind the output plane come from a 2*d1 register history
//    of the thread's own columns, the taps ahead from the window;
//  - grid = tiles x streamwise chunks in chunk-major order, so concurrent CTAs work at nearby
//    planes and halos hit L2; odd chunks march downwards, so the planes two neighbouring
//    chunks share are read by both at the same time;
//  - warps whose columns are all wall keep the pipeline protocol but skip the arithmetic.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>
#include "common.h"
#include "ptx.cuh"
#include "step_kernel.cuh"

namespace fslbm {

template <int D1, int TY> struct Step2Tile {
  static_assert(D1 % 2 == 0, "pair loads of the corrector taps need an even stride");
  static constexpr int TX = 32;
  static constexpr int THREADS = TX / 2 * TY;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int R = 2 * D1;                      // farthest corrector tap
  static constexpr int HX = (R + 3) / 4 * 4;            // x halo, TMA-aligned (16 bytes)
  static constexpr int HY = R;
  static constexpr int SW = TX + 2 * HX;                // row length of both boxes
  static constexpr int PH = TY + 2;                     // p rows (halo 1)
  static constexpr int UH = TY + 2 * HY;                // u,v,w rows
  static constexpr int PPLANE = (SW * PH + 31) / 32 * 32;   // padded for 128-byte alignment
  static constexpr int UPLANE = SW * UH;
  static constexpr int SLOT = PPLANE + 3 * UPLANE;
  static constexpr int S = 8;                           // window slots (power of two)
  static constexpr int AHEAD = S - R - 1;               // planes loaded beyond the current one
  static_assert(AHEAD >= 1, "window too small for the corrector reach");
  static constexpr uint32_t TX_BYTES = uint32_t((SW * PH + 3 * UPLANE) * 4);
  static constexpr size_t RING_BYTES = size_t(S) * SLOT * 4;
  static constexpr size_t BAR_OFFSET = RING_BYTES;
  static constexpr size_t SMEM_BYTES = BAR_OFFSET + 2 * S * sizeof(uint64_t);
  static_assert((PPLANE * 4) % 128 == 0 && (UPLANE * 4) % 16 == 0 && (SLOT * 4) % 128 == 0,
                "TMA destinations must stay aligned");
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
};

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 lds2(const float* p) { return *reinterpret_cast<const float2*>(p); }

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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

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

template <int D1, int TY, bool PK>
__global__ void __launch_bounds__(Step2Tile<D1, TY>::THREADS, 1)
    fslbm_step2_kernel(const __grid_constant__ CUtensorMap tmap_p,
                       const __grid_constant__ CUtensorMap tmap_uvw, const Step2Geom g,
                       const StepConst<float> k) {
  using Tl = Step2Tile<D1, TY>;
  using F = Pair<PK>;
  constexpr int R = Tl::R, HX = Tl::HX, HY = Tl::HY, SW = Tl::SW, S = Tl::S, AH = Tl::AHEAD;
  constexpr int PPL = Tl::PPLANE, UPL = Tl::UPLANE, SLOT = Tl::SLOT;

  extern __shared__ __align__(128) unsigned char smem[];
  float* ring = reinterpret_cast<float*>(smem);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + Tl::BAR_OFFSET);
  uint64_t* empty = full + S;

  const int tid = threadIdx.x, lane = tid & 31, tp = tid % (Tl::TX / 2), ty = tid / (Tl::TX / 2);
  if (tid == 0 && blockIdx.x == 0 && g.step_counter) *g.step_counter += 1;

  // ---- work: one (tile, chunk); odd chunks march towards -z
  const int tile = blockIdx.x % g.ntiles, chunk = blockIdx.x / g.ntiles;
  const int zb = int((long long)g.L * chunk / g.nchunks);
  const int ze = int((long long)g.L * (chunk + 1) / g.nchunks);
  const int dir = (chunk & 1) ? -1 : 1;
  const int nout = ze - zb, niter = nout + 2 * R;
  const int start = dir > 0 ? zb - R : ze - 1 + R;      // real plane of march index 0
  const int2 org = g.tiles[tile];
  const int xa = org.x + 2 * tp, y = org.y + ty;

  float2 ws0 = f2(0.f), wsx = f2(0.f), wsy = f2(0.f), fl = f2(0.f);
  if (xa < g.lxp && y < g.ly) {
    const ColCoef<float>* cp = reinterpret_cast<const ColCoef<float>*>(g.colcoef) + size_t(y) * g.lxp + xa;
    const ColCoef<float> ca = cp[0], cb = cp[1];
    ws0 = make_float2(ca.ws0, cb.ws0); wsx = make_float2(ca.wsx, cb.wsx);
    wsy = make_float2(ca.wsy, cb.wsy); fl = make_float2(ca.fluid, cb.fluid);
  }
  const bool fluid_any = fl.x != 0.f || fl.y != 0.f;
  const bool warp_on = __any_sync(0xffffffffu, fluid_any);
  // non-wall flags of the 4 x 3 neighbourhood (columns xa-1..xa+2), for the seam jump
  unsigned nwbits = 0;
  if (warp_on) {
    for (int cy = -1; cy <= 1; ++cy)
      for (int j = 0; j < 4; ++j) {
        const int gx = xa - 1 + j, gy = y + cy;
        const bool nwall = gx >= 0 && gy >= 0 && gx < g.lxp && gy < g.ly &&
                           g.mask[size_t(gy) * g.lxp + gx] != kWall;
        nwbits |= unsigned(nwall) << ((cy + 1) * 4 + j);
      }
  }

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], Tl::WARPS);
    }
    mbar_init_fence();
  }
  __syncthreads();

  auto issue = [&](int m) {            // load march plane m into slot m % S
    const int slot = m & (S - 1);
    int zz = (start + dir * m) % g.L;
    if (zz < 0) zz += g.L;
    float* dst = ring + slot * SLOT;
    mbar_arrive_expect_tx(&full[slot], Tl::TX_BYTES);
    tma_load_4d(dst, &tmap_p, &full[slot], org.x - HX, org.y - 1, zz, 0);
    tma_load_4d(dst + PPL, &tmap_uvw, &full[slot], org.x - HX, org.y - HY, zz, 1);
  };
  int issued = -1;                                            // last march plane issued (thread 0)
  if (tid == 0) {
    prefetch_tensormap(&tmap_p);
    prefetch_tensormap(&tmap_uvw);
    for (int m = 0; m <= AH && m < niter; ++m) { issue(m); issued = m; }
  }
  auto drain = [&](int from) {                                // failure path: let loads land
    if (tid == 0)
      for (int q = from; q <= issued; ++q)
        mbar_wait_bounded(&full[q & (S - 1)], uint32_t((q / S) & 1), kWaitLimitNs / 8);
  };

  const float gauge = g.gauge ? float(*g.gauge) : 0.0f;
  const size_t FS = size_t(g.lxp) * g.ly * g.L;
  float* out = reinterpret_cast<float*>(g.out);
  // true predictor sums from the row-factored ones: A0/36, dir*A1'/12, A2'/8
  const float2 s0 = f2(1.0f / 36.0f), s1 = f2(float(dir) / 12.0f), s2 = f2(1.0f / 8.0f);
  const int po = (ty + 1) * SW + HX + 2 * tp;                 // p box
  const int uo = PPL + (ty + HY) * SW + HX + 2 * tp;          // u box (v, w at +UPL, +2 UPL)

  float2 hu[R], hv[R], hw[R];                                 // own columns, march planes j-R..j-1
#pragma unroll
  for (int j = 0; j < R; ++j) { hu[j] = f2(0.f); hv[j] = f2(0.f); hw[j] = f2(0.f); }
  float2 aA[4], aB[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) { aA[j] = f2(0.f); aB[j] = f2(0.f); }

  for (int m = 0; m < niter; ++m) {
    if (!mbar_wait_bounded(&full[m & (S - 1)], uint32_t((m / S) & 1), kWaitLimitNs)) {
      if (lane == 0) atomicOr(g.err, 1u);
      drain(m + 1);
      return;
    }
    const int ma = m - R + 1;                                 // predictor plane (march index)
    const int jo = m - R;                                     // output plane (march index)
    if (warp_on) {
      float2 comp0 = f2(0.f), comp1 = f2(0.f), comp2 = f2(0.f), comp3 = f2(0.f);
      if (ma >= R - 1) {
        const float* ss = ring + (ma & (S - 1)) * SLOT;
        const int sp = start + dir * ma;                      // real plane
        const float off = sp < 0 ? k.pin : (sp >= g.L ? -k.pin : 0.0f);
        // row-factored weights w(cx)w(cy) = {4,1,1}x{4,1,1}/36: per row R = P(-1)+P(+1)+4P(0),
        // D = P(+1)-P(-1); across rows A = R(-1)+R(+1)+4R(0), X likewise on D, Y = R(+1)-R(-1)
        float2 A[3], X[3], Y[3];
#pragma unroll
        for (int cy = -1; cy <= 1; ++cy) {
          const float* rp = ss + po + cy * SW;
          const float* rq = ss + uo + cy * SW;
          const float2 pL = lds2(rp - 2), pC = lds2(rp), pR = lds2(rp + 2);
          const float2 uL = lds2(rq - 2), uC = lds2(rq), uR = lds2(rq + 2);
          const float2 vL = lds2(rq + UPL - 2), vC = lds2(rq + UPL), vR = lds2(rq + UPL + 2);
          const float2 wL = lds2(rq + 2 * UPL - 2), wC = lds2(rq + 2 * UPL), wR = lds2(rq + 2 * UPL + 2);
          float2 pm = make_float2(pL.y, pC.x), p0 = pC, pp = make_float2(pC.y, pR.x);
          if (off != 0.0f) {
            const unsigned bb = nwbits >> ((cy + 1) * 4);
            pm.x += (bb & 1u) ? off : 0.f; pm.y += (bb & 2u) ? off : 0.f;
            p0.x += (bb & 2u) ? off : 0.f; p0.y += (bb & 4u) ? off : 0.f;
            pp.x += (bb & 4u) ? off : 0.f; pp.y += (bb & 8u) ? off : 0.f;
          }
          const float2 um = make_float2(uL.y, uC.x), up = make_float2(uC.y, uR.x);
          const float2 vm = make_float2(vL.y, vC.x), vp = make_float2(vC.y, vR.x);
          const float2 wm = make_float2(wL.y, wC.x), wp = make_float2(wC.y, wR.x);
          float2 Pm[3], P0[3], Pp[3];
          if (cy == -1) {
            brackets<PK, -1, -1>(qof<PK>(pm, um, vm, wm), um, vm, wm, Pm[0], Pm[1], Pm[2]);
            brackets<PK, 0, -1>(qof<PK>(p0, uC, vC, wC), uC, vC, wC, P0[0], P0[1], P0[2]);
            brackets<PK, 1, -1>(qof<PK>(pp, up, vp, wp), up, vp, wp, Pp[0], Pp[1], Pp[2]);
          } else if (cy == 0) {
            brackets<PK, -1, 0>(qof<PK>(pm, um, vm, wm), um, vm, wm, Pm[0], Pm[1], Pm[2]);
            brackets<PK, 0, 0>(qof<PK>(p0, uC, vC, wC), uC, vC, wC, P0[0], P0[1], P0[2]);
            brackets<PK, 1, 0>(qof<PK>(pp, up, vp, wp), up, vp, wp, Pp[0], Pp[1], Pp[2]);
          } else {
            brackets<PK, -1, 1>(qof<PK>(pm, um, vm, wm), um, vm, wm, Pm[0], Pm[1], Pm[2]);
            brackets<PK, 0, 1>(qof<PK>(p0, uC, vC, wC), uC, vC, wC, P0[0], P0[1], P0[2]);
            brackets<PK, 1, 1>(qof<PK>(pp, up, vp, wp), up, vp, wp, Pp[0], Pp[1], Pp[2]);
          }
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            const float2 Rq = F::fma(f2(4.0f), P0[q], F::add(Pm[q], Pp[q]));
            const float2 Dq = F::fma(f2(-1.0f), Pm[q], Pp[q]);
            if (cy == -1) { A[q] = Rq; X[q] = Dq; Y[q] = Rq; }
            else if (cy == 0) { A[q] = F::fma(f2(4.0f), Rq, A[q]); X[q] = F::fma(f2(4.0f), Dq, X[q]); }
            else { A[q] = F::add(A[q], Rq); X[q] = F::add(X[q], Dq); Y[q] = F::fma(f2(-1.0f), Y[q], Rq); }
          }
        }
        const float2 tA0 = F::mul(A[0], s0), tA1 = F::mul(A[1], s1), tA2 = F::mul(A[2], s2);
        const float2 tX0 = F::mul(X[0], s0), tX1 = F::mul(X[1], s1), tX2 = F::mul(X[2], s2);
        const float2 tY0 = F::mul(Y[0], s0), tY1 = F::mul(Y[1], s1), tY2 = F::mul(Y[2], s2);
        // plane ma is the march-next neighbour of output ma-1 (completed here), itself, and
        // the march-previous neighbour of ma+1
        const float2 A02 = F::add(tA0, tA2), X02 = F::add(tX0, tX2), Y02 = F::add(tY0, tY2);
        const float2 sP = F::add(A02, tA1), sM = F::fma(tA1, f2(-1.f), A02);
        const float2 xP = F::add(X02, tX1), xM = F::fma(tX1, f2(-1.f), X02);
        const float2 yP = F::add(Y02, tY1), yM = F::fma(tY1, f2(-1.f), Y02);
        const float2 cw0 = f2(2.0f / 3.0f), cw1 = f2(1.0f / 6.0f);
        comp0 = F::fma(cw1, sP, aA[0]);
        comp1 = F::fma(cw1, xP, aA[1]);
        comp2 = F::fma(cw1, yP, aA[2]);
        comp3 = F::fma(cw1, sP, aA[3]);
        aA[0] = F::fma(cw0, tA0, aB[0]);
        aA[1] = F::fma(cw0, tX0, aB[1]);
        aA[2] = F::fma(cw0, tY0, aB[2]);
        aA[3] = aB[3];
        aB[0] = F::mul(cw1, sM);
        aB[1] = F::mul(cw1, xM);
        aB[2] = F::mul(cw1, yM);
        aB[3] = F::mul(f2(-1.0f / 6.0f), sM);
      }
      if (jo >= 0) {
        const float* so = ring + (jo & (S - 1)) * SLOT;
        const float2 uc = lds2(so + uo), vc = lds2(so + uo + UPL), wc = lds2(so + uo + 2 * UPL);
        if (jo >= R && fluid_any) {
          // ---- output plane: corrector and update
          const float* sa1 = ring + ((jo + D1) & (S - 1)) * SLOT;   // march planes ahead
          const float* sa2 = ring + ((jo + 2 * D1) & (S - 1)) * SLOT;
          const float2 pc = lds2(so + po);
          auto lap = [&](int f, float2 c, float2 zb1, float2 zb2) {
            const float* q = so + uo + f * UPL;
            const float2 za1 = lds2(sa1 + uo + f * UPL), za2 = lds2(sa2 + uo + f * UPL);
            const float2 t1 = F::add(F::add(F::add(lds2(q - D1), lds2(q + D1)),
                                            F::add(lds2(q - D1 * SW), lds2(q + D1 * SW))),
                                     F::add(zb1, za1));
            const float2 t2 = F::add(F::add(F::add(lds2(q - 2 * D1), lds2(q + 2 * D1)),
                                            F::add(lds2(q - 2 * D1 * SW), lds2(q + 2 * D1 * SW))),
                                     F::add(zb2, za2));
            return F::fma(f2(k.c2), t2, F::fma(f2(k.c1), t1, F::mul(f2(k.c0), c)));
          };
          const float2 Lu = lap(0, uc, hu[R - D1], hu[0]);
          const float2 Lv = lap(1, vc, hv[R - D1], hv[0]);
          const float2 Lw = lap(2, wc, hw[R - D1], hw[0]);
          const float2 rho = F::add(F::fma(pc, ws0, comp0), f2(-gauge));
          const float2 us = F::fma(pc, wsx, comp1), vs = F::fma(pc, wsy, comp2);
          const float2 wsz = F::mul(comp3, f2(float(dir)));
          const float2 dt = f2(k.dtddy), mm = f2(k.m), tb = f2(k.tb), cc = f2(k.cc);
          const float2 un = F::fma(F::add(F::fma(F::mul(dt, Lu), mm, us), f2(k.fx)), tb, F::mul(uc, cc));
          const float2 vn = F::fma(F::add(F::fma(F::mul(dt, Lv), mm, vs), f2(k.fy)), tb, F::mul(vc, cc));
          const float2 wn = F::fma(F::add(F::fma(F::mul(dt, Lw), mm, wsz), f2(k.fz)), tb, F::mul(wc, cc));
          const int zo = start + dir * jo;
          const size_t o = (size_t(zo) * g.ly + y) * g.lxp + xa;
          auto put = [&](float* dst, float2 v) {
            v.x = fl.x != 0.f ? v.x : 0.f;
            v.y = fl.y != 0.f ? v.y : 0.f;
            *reinterpret_cast<float2*>(dst) = v;
          };
          put(out + o, rho);
          put(out + FS + o, un);
          put(out + 2 * FS + o, vn);
          put(out + 3 * FS + o, wn);
        }
        // own columns of plane jo join the history of streamwise taps
#pragma unroll
        for (int j = 0; j < R - 1; ++j) { hu[j] = hu[j + 1]; hv[j] = hv[j + 1]; hw[j] = hw[j + 1]; }
        hu[R - 1] = uc; hv[R - 1] = vc; hw[R - 1] = wc;
      }
    }
    // plane jo leaves the window: release its slot, then refill it with march plane m + AH + 1
    __syncwarp();
    if (jo >= 0 && lane == 0) mbar_arrive(&empty[jo & (S - 1)]);
    if (tid == 0 && m + AH + 1 < niter) {
      const int mn = m + AH + 1;
      if (mn >= S &&
          !mbar_wait_bounded(&empty[mn & (S - 1)], uint32_t(((mn - S) / S) & 1), kWaitLimitNs)) {
        atomicOr(g.err, 1u);
        drain(m + 1);
        return;
      }
      fence_proxy_async_smem();
      issue(mn);
      issued = mn;
    }
  }
}

}  // namespace fslbm
