// FSLBM time step, FP64 column kernel for sm_100a (d1 = 2, the reference's order 2<->4 corrector).
//
// The column-pair kernel's pipeline (step2_kernel.cuh) with one FP64 column per thread:
//  - a 32 x 16 tile per CTA, 512 threads, one warp per tile row: a warp's 64-bit shared loads
//    read 32 consecutive doubles (two wavefronts, no bank conflict); 16 warps per SM;
//  - p is staged with a one-cell halo and u,v,w with the corrector's 2*d1 halo, as two TMA boxes
//    per plane (no multicast) into a window of 7 planes (201 KB);
//  - no block-wide barrier in the march and no producer thread: per-slot "full" mbarriers count
//    TMA completion, planes leave the window in pairs and the last warp to release a pair
//    refills both slots (the protocol of step2_march, same bounded waits and failure path);
//  - the predictor is row-factored per column, the streamwise corrector taps behind the output
//    plane come from a register history of the thread's own column, the taps ahead from the
//    window; the update is folded as in the FP32 kernel;
//  - grid = tiles x streamwise chunks in chunk-major order, odd chunks marching downwards, and a
//    cell's predictor adds its two neighbour planes' shares before its own plane's, so results do
//    not depend on the chunking.
// It replaces the one-column kernel of step_kernel.cuh (one block barrier per plane, a single
// 4-field box with the corrector halo on p too, 8 warps per SM) for FP64 solves with d1 = 2 and
// the 2-tap corrector; other orders, strides and per-plane masks keep that kernel.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>
#include "common.h"
#include "ptx.cuh"
#include "step_kernel.cuh"
#include "step2_kernel.cuh"

namespace fslbm {

template <int D1, int TY> struct ColTile {
  static constexpr int ES = int(sizeof(double));
  static constexpr int TX = 32;
  static constexpr int THREADS = TX * TY;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int R = 2 * D1;                      // farthest corrector tap
  static constexpr int HX = (R * ES + 15) / 16 * 16 / ES;   // x halo, TMA-aligned (16 bytes)
  static constexpr int HY = R;
  static constexpr int SW = TX + 2 * HX;                // row length of both boxes
  static constexpr int PH = TY + 2;                     // p rows (halo 1)
  static constexpr int UH = TY + 2 * HY;                // u,v,w rows
  static constexpr int PPLANE = (SW * PH * ES + 127) / 128 * 128 / ES;
  static constexpr int UPLANE = SW * UH;
  static constexpr int SLOT = PPLANE + 3 * UPLANE;
  static constexpr int S = 7;                           // window slots
  static constexpr int AHEAD = S - R - 1;
  static_assert(AHEAD >= 1, "window too small for the corrector reach");
  static constexpr uint32_t TX_BYTES = uint32_t((SW * PH + 3 * UPLANE) * ES);
  static constexpr size_t BAR_OFFSET = size_t(S) * SLOT * ES;
  static constexpr size_t SMEM_BYTES = BAR_OFFSET + S * sizeof(uint64_t) + S * sizeof(uint32_t);
  static_assert((PPLANE * ES) % 128 == 0 && (UPLANE * ES) % 16 == 0 && (SLOT * ES) % 128 == 0,
                "TMA destinations must stay aligned");
  static_assert((HX * ES) % 16 == 0, "TMA box x start must be 16-byte aligned");
  static_assert(SMEM_BYTES <= 227 * 1024, "window exceeds a CTA's shared memory");
};

// Marches one (tile, chunk) work item: the step of every cell of the tile's columns in the
// chunk's planes. Returns false when a bounded wait gave up (error flag set).
template <int D1, int TY>
__device__ __forceinline__ bool col_march(const CUtensorMap* tmap_p, const CUtensorMap* tmap_uvw,
                                          const Step2Geom& g, const StepConst<double>& k, int tile,
                                          int chunk, unsigned char* smem) {
  using Tl = ColTile<D1, TY>;
  static_assert(D1 == 2, "the march prologue below is written for d1 = 2 (R = 4)");
  constexpr int R = Tl::R, HX = Tl::HX, HY = Tl::HY, SW = Tl::SW, S = Tl::S;
  constexpr int PPL = Tl::PPLANE, UPL = Tl::UPLANE, SLOT = Tl::SLOT;

  auto slot_of = [](int m) { return int(unsigned(m) % unsigned(S)); };
  auto phase_of = [](int m) { return uint32_t((unsigned(m) / unsigned(S)) & 1u); };
  double* ring = reinterpret_cast<double*>(smem);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + Tl::BAR_OFFSET);
  unsigned* released = reinterpret_cast<unsigned*>(full + S);

  const int tid = threadIdx.x, lane = tid & 31;
  const int tx = lane, ty = tid >> 5;                  // one warp per tile row

  // ---- work: one (tile, chunk); odd chunks march towards -z
  const int zb = int((long long)g.L * chunk / g.nchunks);
  const int ze = int((long long)g.L * (chunk + 1) / g.nchunks);
  const int dir = (chunk & 1) ? -1 : 1;
  const int nout = ze - zb, niter = nout + 2 * R;
  const int start = dir > 0 ? zb - R : ze - 1 + R;      // real plane of march index 0
  const int2 org = g.tiles[tile];
  const int x = org.x + tx, y = org.y + ty;
  const bool inside = x < g.lxp && y < g.ly;

  double ws0 = 0, wsx = 0, wsy = 0, fl = 0;
  if (inside) {
    const ColCoef<double> c = reinterpret_cast<const ColCoef<double>*>(g.colcoef)[size_t(y) * g.lxp + x];
    ws0 = c.ws0; wsx = c.wsx; wsy = c.wsy; fl = c.fluid;
  }
  const bool warp_on = __any_sync(0xffffffffu, fl != 0.0);

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      released[s] = 0u;
    }
    mbar_init_fence();
  }
  __syncthreads();

  auto issue = [&](int m) {            // load march plane m into its slot
    const int slot = slot_of(m);
    int zz = (start + dir * m) % g.L;
    if (zz < 0) zz += g.L;
    double* dst = ring + slot * SLOT;
    mbar_arrive_expect_tx(&full[slot], Tl::TX_BYTES);
    tma_load_4d(dst, tmap_p, &full[slot], org.x - HX, org.y - 1, zz, 0);
    tma_load_4d(dst + PPL, tmap_uvw, &full[slot], org.x - HX, org.y - HY, zz, 1);
  };
  if (tid == 0) {                      // the whole ring up front
    prefetch_tensormap(tmap_p);
    prefetch_tensormap(tmap_uvw);
    for (int m = 0; m < S && m < niter; ++m) issue(m);
  }
  auto drain = [&](int from) {         // failure path: let this CTA's loads land (bounded)
    if (lane == 0)
      for (int q = from; q < niter && q < from + S; ++q)
        mbar_wait_bounded(&full[slot_of(q)], phase_of(q), kWaitLimitNs / 8);
  };
  auto arrive_wait = [&](int m) -> bool {
    if (mbar_wait_bounded(&full[slot_of(m)], phase_of(m), kWaitLimitNs)) return true;
    if (lane == 0) atomicOr(g.err, 1u);
    drain(m + 1);
    return false;
  };
  // planes p - 1 and p (p = m - R odd) leave the window; see step2_march for the ordering
  auto release_produce = [&](int m) {
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
  };

  if (!warp_on) {   // all-wall warps keep the pipeline protocol only
    for (int m = 0; m < niter; ++m) {
      if (!arrive_wait(m)) return false;
      release_produce(m);
    }
    return true;
  }

  const double gauge = g.gauge ? __ldcg(g.gauge) : 0.0;
  const size_t FS = size_t(g.lxp) * g.ly * g.L;
  double* outp = reinterpret_cast<double*>(g.out) + (size_t(start + dir * R) * g.ly + y) * g.lxp + x;
  const long long ostep = (long long)dir * g.ly * g.lxp;     // output pointer step per plane
  const int po = (ty + 1) * SW + HX + tx;                     // p box
  const int uo = PPL + (ty + HY) * SW + HX + tx;              // u box (v, w at +UPL, +2 UPL)
  // seam pressure jump: off times the non-wall weight sums (raw units, x36) on A0, X0, Y0
  const double n0 = 36.0 - 36.0 * ws0, nx = -36.0 * wsx, ny = -36.0 * wsy;
  const double h6 = double(dir) / 72.0;
  // folded update: u_new = K1 t1 + K2 t2 + K0 u + tb (u* + F)
  const double kam = __dmul_rn(__dmul_rn(k.tb, k.dtddy), k.m);
  const double kK0 = __fma_rn(kam, k.c0, k.cc), kK1 = __dmul_rn(kam, k.c1), kK2 = __dmul_rn(kam, k.c2);
  const double ktz = double(dir) * k.tb;

  double hu[4], hv[4], hw[4];          // own column of planes jo-4..jo-1
  // b2: the march-previous plane's share of the output being completed, b1: the same for the
  // next output, s1: the self-plane moments of the next output (see step2_march)
  double b2[4], b1[4], s1[3];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    hu[j] = hv[j] = hw[j] = 0.0;
    b2[j] = b1[j] = 0.0;
    if (j < 3) s1[j] = 0.0;
  }
  double comp0 = 0, comp1 = 0, comp2 = 0, comp3 = 0;

  // predictor contribution of march plane ma (factorisation: step_kernel.cuh, step2_march)
  auto predictor = [&](int ma) {
    const double* ss = ring + slot_of(ma) * SLOT;
    const int sp = start + dir * ma;
    double A[3], X[3], Y[3];
#pragma unroll
    for (int cy = -1; cy <= 1; ++cy) {
      const double* rp = ss + po + cy * SW;
      const double* rq = ss + uo + cy * SW;
      double q3[3], u3[3], v3[3], w3[3], w23[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const double pv = rp[j - 1];
        u3[j] = rq[j - 1];
        v3[j] = rq[UPL + j - 1];
        w3[j] = rq[2 * UPL + j - 1];
        w23[j] = __dmul_rn(w3[j], w3[j]);
        q3[j] = __fma_rn(-1.5, __fma_rn(u3[j], u3[j], __fma_rn(v3[j], v3[j], w23[j])), pv);
      }
      double P[3][3];   // [cx+1][k]
#pragma unroll
      for (int cx = -1; cx <= 1; ++cx) {
        const int j = cx + 1;
        const double u = u3[j], v = v3[j], w = w3[j];
        double P0, P1;
        if (cx == 0 && cy == 0) {
          P0 = q3[j];
          P1 = w;
        } else if (cx == 0 || cy == 0) {
          const double Bv = cy == 0 ? u : v;
          const double s3 = 3.0 * double(cx + cy);
          P0 = __fma_rn(Bv, __fma_rn(Bv, 4.5, s3), q3[j]);
          P1 = __dmul_rn(w, __fma_rn(Bv, s3, 1.0));
        } else {
          const double a1 = __fma_rn(v, double(cx * cy), u);
          const double s3 = 3.0 * double(cx);
          P0 = __fma_rn(a1, __fma_rn(a1, 4.5, s3), q3[j]);
          P1 = __dmul_rn(w, __fma_rn(a1, s3, 1.0));
        }
        P[j][0] = P0; P[j][1] = P1; P[j][2] = w23[j];
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const double Rq = __fma_rn(4.0, P[1][q], __dadd_rn(P[0][q], P[2][q]));
        const double Dq = __dsub_rn(P[2][q], P[0][q]);
        if (cy == -1) { A[q] = Rq; X[q] = Dq; Y[q] = Rq; }
        else if (cy == 0) { A[q] = __fma_rn(4.0, Rq, A[q]); X[q] = __fma_rn(4.0, Dq, X[q]); }
        else { A[q] = __dadd_rn(A[q], Rq); X[q] = __dadd_rn(X[q], Dq); Y[q] = __dsub_rn(Rq, Y[q]); }
      }
    }
    if (sp < 0 || sp >= g.L) {         // seam plane (CTA-uniform): the pressure jump's share
      const double off = sp < 0 ? k.pin : -k.pin;
      A[0] = __fma_rn(off, n0, A[0]);
      X[0] = __fma_rn(off, nx, X[0]);
      Y[0] = __fma_rn(off, ny, Y[0]);
    }
    // true sums are A0/36, dir A1/12, A2/8; shares e + h (next), (2/3) A0 (self), e - h (previous)
    const double eA = __fma_rn(A[2], 1.0 / 48.0, __dmul_rn(A[0], 1.0 / 216.0));
    const double eX = __fma_rn(X[2], 1.0 / 48.0, __dmul_rn(X[0], 1.0 / 216.0));
    const double eY = __fma_rn(Y[2], 1.0 / 48.0, __dmul_rn(Y[0], 1.0 / 216.0));
    const double sA = __fma_rn(A[1], h6, eA), dA = __fma_rn(A[1], -h6, eA);
    const double sX = __fma_rn(X[1], h6, eX), dX = __fma_rn(X[1], -h6, eX);
    const double sY = __fma_rn(Y[1], h6, eY), dY = __fma_rn(Y[1], -h6, eY);
    comp0 = __fma_rn(s1[0], 1.0 / 54.0, __dadd_rn(b2[0], sA));
    comp1 = __fma_rn(s1[1], 1.0 / 54.0, __dadd_rn(b2[1], sX));
    comp2 = __fma_rn(s1[2], 1.0 / 54.0, __dadd_rn(b2[2], sY));
    comp3 = __dadd_rn(b2[3], sA);
#pragma unroll
    for (int q = 0; q < 4; ++q) b2[q] = b1[q];
    b1[0] = dA; b1[1] = dX; b1[2] = dY; b1[3] = -dA;
    s1[0] = A[0]; s1[1] = X[0]; s1[2] = Y[0];
  };

  // corrector and update of output march plane jo; history slot ROT holds plane jo-4 and is then
  // overwritten with plane jo
  auto output = [&](int jo, auto rot_c) {
    constexpr int ROT = decltype(rot_c)::value;
    const double* so = ring + slot_of(jo) * SLOT;
    const double* sa1 = ring + slot_of(jo + D1) * SLOT;   // march planes ahead
    const double* sa2 = ring + slot_of(jo + 2 * D1) * SLOT;
    const double pc = so[po];
    const double uc = so[uo], vc = so[uo + UPL], wc = so[uo + 2 * UPL];
    auto update = [&](int f, double c, double zb1, double zb2, double mom, double tm, double tf) {
      const double* q = so + uo + f * UPL;
      const double za1 = sa1[uo + f * UPL], za2 = sa2[uo + f * UPL];
      const double t1 = __dadd_rn(__dadd_rn(__dadd_rn(q[-D1], q[D1]), __dadd_rn(q[-D1 * SW], q[D1 * SW])),
                                  __dadd_rn(zb1, za1));
      const double t2 = __dadd_rn(__dadd_rn(__dadd_rn(q[-2 * D1], q[2 * D1]),
                                            __dadd_rn(q[-2 * D1 * SW], q[2 * D1 * SW])),
                                  __dadd_rn(zb2, za2));
      return __fma_rn(kK1, t1, __fma_rn(kK2, t2, __fma_rn(kK0, c, __fma_rn(tm, mom, tf))));
    };
    constexpr int H2 = (ROT + 2) & 3;                         // plane jo-2
    const double rho = __dadd_rn(__fma_rn(pc, ws0, comp0), -gauge);
    const double us = __fma_rn(pc, wsx, comp1), vs = __fma_rn(pc, wsy, comp2);
    const double un = update(0, uc, hu[H2], hu[ROT], us, k.tb, __dmul_rn(k.tb, k.fx));
    const double vn = update(1, vc, hv[H2], hv[ROT], vs, k.tb, __dmul_rn(k.tb, k.fy));
    const double wn = update(2, wc, hw[H2], hw[ROT], comp3, ktz, __dmul_rn(k.tb, k.fz));
    hu[ROT] = uc; hv[ROT] = vc; hw[ROT] = wc;
    if (inside) {   // wall columns get zero (fl = 0)
      outp[0] = rho * fl;
      outp[FS] = un * fl;
      outp[2 * FS] = vn * fl;
      outp[3 * FS] = wn * fl;
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
      const double* so = ring + slot_of(m - R) * SLOT;
      const double uc = so[uo], vc = so[uo + UPL], wc = so[uo + 2 * UPL];
      const int h = (m - R) & 3;
      if (h == 0) { hu[0] = uc; hv[0] = vc; hw[0] = wc; }
      else if (h == 1) { hu[1] = uc; hv[1] = vc; hw[1] = wc; }
      else if (h == 2) { hu[2] = uc; hv[2] = vc; hw[2] = wc; }
      else { hu[3] = uc; hv[3] = vc; hw[3] = wc; }
    }
    release_produce(m);
  }
  // ---- steady state, four planes per pass (the history period)
  for (int m = 2 * R; m < niter; m += 4) {
    if (!arrive_wait(m)) return false;
    predictor(m - R + 1);
    output(m - R, I0{});
    release_produce(m);
    if (m + 1 >= niter) break;
    if (!arrive_wait(m + 1)) return false;
    predictor(m - R + 2);
    output(m - R + 1, I1{});
    release_produce(m + 1);
    if (m + 2 >= niter) break;
    if (!arrive_wait(m + 2)) return false;
    predictor(m - R + 3);
    output(m - R + 2, I2{});
    release_produce(m + 2);
    if (m + 3 >= niter) break;
    if (!arrive_wait(m + 3)) return false;
    predictor(m - R + 4);
    output(m - R + 3, I3{});
    release_produce(m + 3);
  }
  return true;
}

// One pipe, one step: CTA b marches (tile b % ntiles, chunk b / ntiles).
template <int D1, int TY>
__global__ void __launch_bounds__(ColTile<D1, TY>::THREADS, 1)
    fslbm_col_kernel(const __grid_constant__ CUtensorMap tmap_p,
                     const __grid_constant__ CUtensorMap tmap_uvw, const Step2Geom g,
                     const StepConst<double> k) {
  extern __shared__ __align__(128) unsigned char smem[];
  if (threadIdx.x == 0 && blockIdx.x == 0 && g.step_counter) *g.step_counter += 1;
  col_march<D1, TY>(&tmap_p, &tmap_uvw, g, k, blockIdx.x % g.ntiles, blockIdx.x / g.ntiles, smem);
}

}  // namespace fslbm
