// Fused FSLBM time step for sm_100a.
//
// One launch advances the whole periodic pipe by one step: predictor (D3Q27 equilibrium pull,
// FSLBM.cu:130-173), corrector (coarse-stride reverse diffusion, FSLBM.cu:231-273), the
// periodic seam with its +-pin pressure jump (FSLBM.cu:291-301), walls (FSLBM.cu:290), the
// gauge p -= p2 (FSLBM.cu:303) and an optional body force. It replaces the reference's 38 slab
// launches, 310 shiftback launches and one bcond per step; fields ping-pong between two
// buffers, so no shift copy exists.
//
// Work decomposition. A CTA owns a kTX x kTY tile of the cross-section (one thread per
// column) and marches along the streamwise axis z over a chunk of planes. Each plane of the
// tile, with an x/y halo of R = 2*d1 cells, is brought into a shared-memory ring by one 4-D TMA
// load (p,u,v,w in one box; out-of-box cells read as zero, which equals the reference's clamp
// addressing because the box rim is wall). Loads run P planes ahead on per-slot mbarriers.
//
// Predictor, factored by neighbour plane. With D3Q27 weights W_c = w(cx)w(cy)w(cz),
// w(0)=2/3, w(+-1)=1/6, and q = p - 1.5|u|^2, each bracket q + 3c.u + 4.5(c.u)^2 of a
// neighbour splits as P0 + cz*P1 + cz^2*P2 with a = cx*u + cy*v:
//   P0 = q + a(3 + 4.5a),  P1 = w(3 + 9a),  P2 = 4.5 w^2.
// So one pass over the 3x3 in-plane neighbours of a plane gives that plane's contribution to
// the three outputs it touches (z-1, z, z+1); partial sums ride in registers along the march.
// The wall rule "a wall neighbour contributes with the centre's p" (FSLBM.cu:138-140) is the
// static per-column sum of W_c c^k over wall neighbours times the centre p, because wall cells
// hold zero (bcond, FSLBM.cu:290); the mask is extruded along z.
//
// Corrector: in-plane taps at +-d1 .. +-K*d1 (K = 2 for the reference's order 2<->4 blend, up to
// 8 for its order-14 set) come from the ring slot of the output plane, the streamwise taps from a
// 2R+1 register ring of the thread's own column (R = K*d1).
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>
#include "common.h"
#include "ptx.cuh"

namespace fslbm {

constexpr uint64_t kWaitLimitNs = 2000000000ull;   // 2 s bound on every mbarrier wait

template <class TS> struct Compute { using type = TS; };

template <class TS, int D1, int K = 2> struct StepTile {
  static constexpr int R = K * D1;                              // farthest corrector tap
  static constexpr int AL = 16 / int(sizeof(TS));               // elements per 16 bytes
  static constexpr int HX = ((R + AL - 1) / AL) * AL;           // x halo, TMA-aligned start
  static constexpr int HY = R;
  static constexpr int SW = kTX + 2 * HX;                       // slot row length
  static constexpr int SH = kTY + 2 * HY;
  static constexpr int PLANE = SW * SH;                         // elements per field plane
  static constexpr int P = 2;                                   // planes loaded ahead of use
  static constexpr int S = R + 1 + P;                           // ring slots
  static constexpr int SLOT = 4 * PLANE;                        // p,u,v,w
  static constexpr int QW = kTX + 2, QH = kTY + 2, QN = QW * QH;
  using TC = typename Compute<TS>::type;
  static constexpr size_t RING_BYTES = size_t(S) * SLOT * sizeof(TS);
  static constexpr size_t Q_OFFSET = RING_BYTES;
  static constexpr size_t NW_OFFSET = Q_OFFSET + 2 * QN * sizeof(TC);
  static constexpr size_t BAR_OFFSET = (NW_OFFSET + QN + 15) / 16 * 16;
  static constexpr size_t SMEM_BYTES = BAR_OFFSET + S * sizeof(uint64_t);
  static_assert((SW * sizeof(TS)) % 16 == 0, "TMA box rows must be 16-byte multiples");
  static_assert((SLOT * sizeof(TS)) % 128 == 0, "ring slots must stay 128-byte aligned");
};

template <class TC> struct StepConst {
  TC tb, cc, pin, dtddy, m, c0, c1, c2, fx, fy, fz;
  TC ch[6];                // corrector coefficients c3..c8 (orders above 4)
};

struct StepGeom {
  int lxp, ly, L;          // row pitch (padded lx), rows, streamwise planes
  int ntiles, chunk;       // tiles in the list; planes per chunk
  const int2* tiles;       // tile origins
  const uint8_t* mask;     // lxp*ly per plane: 0 fluid, 125 wall (padding columns are wall)
  const void* colcoef;     // ColCoef<TC>[lxp*ly], or CellCoef<TC>[lxp*ly*L] for mask_planes > 1
  int mask_planes;         // 0 or 1: one cross-section extruded along z; L: one per plane
                           // (the kernel's MP parameter must match: MP = mask_planes > 1)
  void* out;               // output state: 4 fields, field stride lxp*ly*L
  const double* gauge;     // p2 of the previous monitor (applied this step) or null
  unsigned* err;           // bit 0: a bounded wait gave up
  long long* step_counter; // device step count, advanced by block 0
};

// MP: masks that vary along z (one cross-section and per-cell wall sums per plane). A template
// parameter rather than a runtime test: the test sat in per-element loops and cost 17 % in FP64.
template <class TS, int D1, int K = 2, bool MP = false>
__global__ void __launch_bounds__(kThreads, sizeof(TS) == 8 ? 1 : 2)
    fslbm_step_kernel(const __grid_constant__ CUtensorMap tin, const StepGeom g,
                      const StepConst<typename Compute<TS>::type> k) {
  using Tl = StepTile<TS, D1, K>;
  using TC = typename Tl::TC;
  constexpr int R = Tl::R, HX = Tl::HX, HY = Tl::HY, SW = Tl::SW, PL = Tl::PLANE;
  constexpr int S = Tl::S, P = Tl::P, QW = Tl::QW, QN = Tl::QN;

  extern __shared__ __align__(128) unsigned char smem[];
  TS* ring = reinterpret_cast<TS*>(smem);
  TC* qbuf = reinterpret_cast<TC*>(smem + Tl::Q_OFFSET);
  uint8_t* nw = smem + Tl::NW_OFFSET;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + Tl::BAR_OFFSET);

  const int tid = threadIdx.x, tx = tid % kTX, ty = tid / kTX;
  const int tile = blockIdx.x % g.ntiles, chunk = blockIdx.x / g.ntiles;
  const int2 org = g.tiles[tile];
  const int x = org.x + tx, y = org.y + ty;
  const int zb = chunk * g.chunk, ze = min(zb + g.chunk, g.L);
  const int t0 = zb - R, t1 = ze + R;

  if (tid == 0) {
    if (blockIdx.x == 0 && g.step_counter) *g.step_counter += 1;
    for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
    mbar_init_fence();
    prefetch_tensormap(&tin);
  }
  // non-wall flags of the predictor tile (columns x0-1..x0+kTX, rows y0-1..y0+kTY)
  for (int j = tid; j < QN; j += kThreads) {
    const int gx = org.x - 1 + j % QW, gy = org.y - 1 + j / QW;
    nw[j] = (gx >= 0 && gy >= 0 && gx < g.lxp && gy < g.ly && g.mask[gy * g.lxp + gx] != kWall);
  }
  bool fluid = false;
  TC ws0 = 0, wsx = 0, wsy = 0;
  if (x < g.lxp && y < g.ly && !MP) {
    const ColCoef<TC> c = reinterpret_cast<const ColCoef<TC>*>(g.colcoef)[y * g.lxp + x];
    fluid = c.fluid != TC(0);
    ws0 = c.ws0; wsx = c.wsx; wsy = c.wsy;
  }
  __syncthreads();

  int issued = t0 - 1;   // last plane whose load was issued (thread 0 only)
  auto issue = [&](int t) {
    const int s = (t - t0) % S;
    int zz = t % g.L;
    if (zz < 0) zz += g.L;
    mbar_arrive_expect_tx(&bar[s], uint32_t(Tl::SLOT * sizeof(TS)));
    tma_load_4d(ring + size_t(s) * Tl::SLOT, &tin, &bar[s], org.x - HX, org.y - HY, zz, 0);
    issued = t;
  };
  if (tid == 0)
    for (int j = 0; j < P && t0 + j < t1; ++j) issue(t0 + j);

  TC ru[2 * R + 1], rv[2 * R + 1], rw[2 * R + 1];
#pragma unroll
  for (int j = 0; j <= 2 * R; ++j) { ru[j] = 0; rv[j] = 0; rw[j] = 0; }
  TC aA[4] = {0, 0, 0, 0}, aB[4] = {0, 0, 0, 0};
  const TC gauge = g.gauge ? TC(*g.gauge) : TC(0);
  const size_t FS = size_t(g.lxp) * g.ly * g.L;
  TS* out = reinterpret_cast<TS*>(g.out);
  const int cidx = (ty + HY) * SW + tx + HX;
  constexpr TC w0 = TC(2.0 / 3.0), w1 = TC(1.0 / 6.0);

  for (int t = t0; t < t1; ++t) {
    const int i = t - t0;
    const bool ok = mbar_wait_bounded(&bar[i % S], uint32_t((i / S) & 1), kWaitLimitNs);
    const TS* pl = ring + size_t(i % S) * Tl::SLOT;
#pragma unroll
    for (int j = 0; j < 2 * R; ++j) { ru[j] = ru[j + 1]; rv[j] = rv[j + 1]; rw[j] = rw[j + 1]; }
    ru[2 * R] = TC(pl[PL + cidx]);
    rv[2 * R] = TC(pl[2 * PL + cidx]);
    rw[2 * R] = TC(pl[3 * PL + cidx]);

    // q = p (+ seam jump on non-wall cells) - 1.5|u|^2 on the predictor plane sp
    const int sp = t - R + 1;
    const bool pred = sp >= zb - 1;
    TC* q = qbuf + (i & 1) * QN;
    const TS* pp = ring + size_t(pred ? (i - R + 1) % S : 0) * Tl::SLOT;
    if (pred) {
      const TC off = sp < 0 ? k.pin : (sp >= g.L ? -k.pin : TC(0));
      // a mask per plane: the seam offset goes on the non-wall cells of the wrapped plane
      const uint8_t* mz = nullptr;
      if (MP && off != TC(0)) {
        int zz = sp % g.L;
        if (zz < 0) zz += g.L;
        mz = g.mask + size_t(zz) * g.lxp * g.ly;
      }
      for (int j = tid; j < QN; j += kThreads) {
        const int e = (j / QW - 1 + HY) * SW + (j % QW - 1 + HX);
        const TC pv = TC(pp[e]), uv = TC(pp[PL + e]), vv = TC(pp[2 * PL + e]),
                 wv = TC(pp[3 * PL + e]);
        bool nwj = nw[j];
        if (mz) {
          const int gx = org.x - 1 + j % QW, gy = org.y - 1 + j / QW;
          nwj = gx >= 0 && gy >= 0 && gx < g.lxp && gy < g.ly && mz[gy * g.lxp + gx] != kWall;
        }
        q[j] = (nwj ? pv + off : pv) - TC(1.5) * (uv * uv + vv * vv + wv * wv);
      }
    }
    if (__syncthreads_or(!ok)) {
      // A load never completed: flag it, give the loads still in flight a bounded chance to
      // land, and leave.
      if (tid == 0) {
        atomicOr(g.err, 1u);
        for (int tt = t; tt <= issued; ++tt) {
          const int ii = tt - t0;
          mbar_wait_bounded(&bar[ii % S], uint32_t((ii / S) & 1), kWaitLimitNs / 4);
        }
      }
      return;
    }
    if (tid == 0 && t + P < t1) {
      fence_proxy_async_smem();
      issue(t + P);
    }

    TC comp[4] = {0, 0, 0, 0};
    if (pred) {
      TC A0 = 0, A1 = 0, A2 = 0, X0 = 0, X1 = 0, X2 = 0, Y0 = 0, Y1 = 0, Y2 = 0;
      const TC* qc = q + (ty + 1) * QW + (tx + 1);
      const TS* pu = pp + PL + cidx;
      const TS* pv = pp + 2 * PL + cidx;
      const TS* pw = pp + 3 * PL + cidx;
#pragma unroll
      for (int cy = -1; cy <= 1; ++cy) {
#pragma unroll
        for (int cx = -1; cx <= 1; ++cx) {
          constexpr double wa0 = 2.0 / 3.0, wa1 = 1.0 / 6.0;
          const TC wgt = TC((cx == 0 ? wa0 : wa1) * (cy == 0 ? wa0 : wa1));
          const int so = cy * SW + cx;
          const TC qn = qc[cy * QW + cx];
          const TC un = TC(pu[so]), vn = TC(pv[so]), wn = TC(pw[so]);
          TC a;
          if (cx != 0 && cy != 0) a = TC(cx) * un + TC(cy) * vn;
          else if (cx != 0) a = TC(cx) * un;
          else if (cy != 0) a = TC(cy) * vn;
          else a = TC(0);
          const TC P0 = qn + a * (TC(3) + TC(4.5) * a);
          const TC P1 = wn * (TC(3) + TC(9) * a);
          const TC P2 = TC(4.5) * wn * wn;
          A0 += wgt * P0; A1 += wgt * P1; A2 += wgt * P2;
          if (cx != 0) {
            const TC wx = TC(cx) * wgt;
            X0 += wx * P0; X1 += wx * P1; X2 += wx * P2;
          }
          if (cy != 0) {
            const TC wy = TC(cy) * wgt;
            Y0 += wy * P0; Y1 += wy * P1; Y2 += wy * P2;
          }
        }
      }
      // plane sp is the cz=+1 neighbour of output sp-1, cz=0 of sp, cz=-1 of sp+1
      const TC sPlus = A0 + A1 + A2, sMinus = A0 - A1 + A2;
      comp[0] = aA[0] + w1 * sPlus;
      comp[1] = aA[1] + w1 * (X0 + X1 + X2);
      comp[2] = aA[2] + w1 * (Y0 + Y1 + Y2);
      comp[3] = aA[3] + w1 * sPlus;
      aA[0] = aB[0] + w0 * A0;
      aA[1] = aB[1] + w0 * X0;
      aA[2] = aB[2] + w0 * Y0;
      aA[3] = aB[3];
      aB[0] = w1 * sMinus;
      aB[1] = w1 * (X0 - X1 + X2);
      aB[2] = w1 * (Y0 - Y1 + Y2);
      aB[3] = -w1 * sMinus;
    }

    const int zo = t - R;   // output plane; its predictor sums completed just above
    TC wsz = 0;
    if (MP && zo >= zb && x < g.lxp && y < g.ly) {
      const size_t cell = (size_t(zo) * g.ly + y) * g.lxp + x;
      fluid = g.mask[cell] == 0;
      const CellCoef<TC> c = reinterpret_cast<const CellCoef<TC>*>(g.colcoef)[cell];
      ws0 = c.ws0; wsx = c.wsx; wsy = c.wsy; wsz = c.wsz;
    }
    if (zo >= zb && fluid) {
      const TS* po = ring + size_t((i - R) % S) * Tl::SLOT + cidx;
      const TC pc = TC(po[0]);
      const TC uc = ru[R], vc = rv[R], wc = rw[R];
      // L = c0 u + sum_k c_k (six taps at k*d1), k = 1..K
      auto lap = [&](const TS* f, const TC* rz, TC c) {
        TC acc = c * k.c0;
#pragma unroll
        for (int kk = 1; kk <= K; ++kk) {
          const int o = kk * D1;
          const TC s = TC(f[o]) + TC(f[-o]) + TC(f[o * SW]) + TC(f[-o * SW]) + rz[R + o] + rz[R - o];
          const TC ck = kk == 1 ? k.c1 : (kk == 2 ? k.c2 : k.ch[kk - 3]);
          acc += ck * s;
        }
        return acc;
      };
      const TC Lu = lap(po + PL, ru, uc), Lv = lap(po + 2 * PL, rv, vc),
               Lw = lap(po + 3 * PL, rw, wc);
      const TC rho = comp[0] + pc * ws0;
      const TC us = comp[1] + pc * wsx, vs = comp[2] + pc * wsy, wzs = comp[3] + pc * wsz;
      const size_t o = (size_t(zo) * g.ly + y) * g.lxp + x;
      out[o] = TS(rho - gauge);
      out[FS + o] = TS((us + k.dtddy * Lu * k.m + k.fx) * k.tb + uc * k.cc);
      out[2 * FS + o] = TS((vs + k.dtddy * Lv * k.m + k.fy) * k.tb + vc * k.cc);
      out[3 * FS + o] = TS((wzs + k.dtddy * Lw * k.m + k.fz) * k.tb + wc * k.cc);
    }
  }
}

}  // namespace fslbm
