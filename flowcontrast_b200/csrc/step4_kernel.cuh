// FSLBM time step, multi-column march for sm_100a (d1 = 2): the kernel that the single-pipe
// step, the batched persistent kernel and the allocation-free step run for FP32 and FP16
// storage (four columns per thread, FP32 arithmetic, 32 x 32 tiles), and the single-pipe FP64
// step (two columns per thread, FP64 arithmetic, 32 x 16 tiles).
//
// Same step and pipeline as the column-pair march of step2_kernel.cuh (predictor factored by
// neighbour plane and by row, coarse corrector, periodic +-pin seam, walls, gauge, body force;
// TMA window of S planes with per-slot full mbarriers and last-warp refill, no block barrier),
// organised to cut the shared-memory traffic and the instruction count per cell:
//  - every thread owns C adjacent columns (x .. x+C-1, x a multiple of C), read as one 16-byte
//    vector per field and row (float4, four halves widened, or double2); a CTA is 256 threads;
//  - the predictor's edge cells x-1 and x+C of a row come from the neighbouring threads of the
//    row by warp shuffles (a scalar shared load only at the tile edge: with 16-byte row strides
//    the edge cells of all rows share one bank class, so loading them directly serialises);
//  - q = p - 1.5|u|^2 and w^2 are formed once per cell for the thread's C + 2 cells of a row;
//  - the corrector's x taps (x-4 .. x+C+3) are 16-byte loads, its y and z taps one each;
//  - the update folds the step constants: u_new = K1 t1 + K2 t2 + K0 u + tb (u* + F), with
//    K0 = tb dtddy m c0 + (1 - tb), K1 = tb dtddy m c1, K2 = tb dtddy m c2;
//  - all arithmetic is written with explicit round-to-nearest intrinsics, so the compiler does
//    not contract it and every launch that marches a cell forms it the same way (batched and
//    single-pipe results are equal bit for bit, and independent of the march direction).
#pragma once
#include "step2_kernel.cuh"

namespace fslbm {

// Uncontracted arithmetic in the compute type.
template <class T> struct Ar;
template <> struct Ar<float> {
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
};
template <> struct Ar<double> {
  static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
};

// Constants of the folded update, formed on the host in the compute type.
template <class T> struct Step4Const {
  T K0, K1, K2;        // corrector weights folded with tblend, dtddy and m
  T tb;                // tblend
  T tfx, tfy, tfz;     // tblend * body force
  T pin;
};

// Per storage type: compute type, columns per thread, tile height and window depth. The window
// holds the output plane, the four planes its corrector and predictor reach ahead, and S - 5
// planes in flight; FP64 tiles are 32 x 16 so that 7 slots fit in shared memory.
template <class TE> struct MarchCfg;
template <> struct MarchCfg<float> { using T = float; static constexpr int C = 4, TY = 32, S = 8; };
template <> struct MarchCfg<__half> { using T = float; static constexpr int C = 4, TY = 32, S = 8; };
template <> struct MarchCfg<double> { using T = double; static constexpr int C = 2, TY = 16, S = 7; };

template <class TE> struct Step4Tile {
  using Cfg = MarchCfg<TE>;
  using T = typename Cfg::T;
  static constexpr int C = Cfg::C, TX = 32, TY = Cfg::TY, S = Cfg::S;
  static constexpr int THREADS = TX / C * TY;           // 256
  static constexpr int WARPS = THREADS / 32;
  // shared-memory layout: per slot a p box (one-cell halo) and a u,v,w box (corrector halo)
  static constexpr int ES = int(sizeof(TE));
  static constexpr int A16 = 16 / ES;                   // elements per 16 bytes
  static constexpr int R = 4;                           // farthest corrector tap (2 d1)
  static constexpr int HX = (R + A16 - 1) / A16 * A16;  // x halo, TMA-aligned (16 bytes)
  static constexpr int HY = R;
  static constexpr int SW = TX + 2 * HX;                // row length of both boxes
  static constexpr int PH = TY + 2;                     // p rows
  static constexpr int UH = TY + 2 * HY;                // u,v,w rows
  static constexpr int PPLANE = (SW * PH * ES + 127) / 128 * 128 / ES;   // 128-byte aligned
  static constexpr int UPLANE = SW * UH;
  static constexpr int SLOT = PPLANE + 3 * UPLANE;
  static constexpr uint32_t TX_BYTES = uint32_t((SW * PH + 3 * UPLANE) * ES);
  static constexpr size_t RING_BYTES = size_t(S) * SLOT * ES;
  static constexpr size_t BAR_OFFSET = RING_BYTES;
  // FP16 storage: the tile's base of w (FP32) for columns org.x-4 .. org.x+TX+3 and rows
  // org.y-1 .. org.y+TY, after the barriers and counters
  static constexpr bool BASE = std::is_same<TE, __half>::value;
  static constexpr int BW = TX + 8, BH = TY + 2;
  static constexpr size_t BASE_OFFSET = (BAR_OFFSET + S * sizeof(uint64_t) + S * sizeof(uint32_t) + 15) / 16 * 16;
  static constexpr size_t SMEM_BYTES = BASE ? BASE_OFFSET + size_t(BW) * BH * sizeof(float)
                                            : BAR_OFFSET + S * sizeof(uint64_t) + S * sizeof(uint32_t);
  static_assert(S >= R + 2, "window too small for the corrector reach");
  static_assert((PPLANE * ES) % 128 == 0 && (UPLANE * ES) % 16 == 0 && (SLOT * ES) % 128 == 0,
                "TMA destinations must stay aligned");
  static_assert((HX * ES) % 16 == 0 && C * ES <= 16 && 4 % C == 0, "vector loads stay aligned");
  static_assert(SMEM_BYTES <= 227 * 1024, "window exceeds shared memory");
};

// C-element vector loads (16 bytes, or 8 for four halves) widened to the compute type.
__device__ __forceinline__ void ldv(const float* p, float (&o)[4]) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
}
__device__ __forceinline__ void ldv(const __half* p, float (&o)[4]) {
  const uint2 t = *reinterpret_cast<const uint2*>(p);
  __half2 h0, h1;
  memcpy(&h0, &t.x, 4);
  memcpy(&h1, &t.y, 4);
  const float2 a = __half22float2(h0), b = __half22float2(h1);
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void ldv(const double* p, double (&o)[2]) {
  const double2 t = *reinterpret_cast<const double2*>(p);
  o[0] = t.x; o[1] = t.y;
}
__device__ __forceinline__ float ld1(const float* p) { return *p; }
__device__ __forceinline__ float ld1(const __half* p) { return __half2float(*p); }
__device__ __forceinline__ double ld1(const double* p) { return *p; }

// Stores of one thread's C columns of the four fields. FP32/FP64 storage stores the values;
// FP16 storage rounds stochastically with noise from (cell index, field, time step) only, so a
// pipe's result does not depend on which other work shares the launch.
template <class TE> struct VecStore;
template <> struct VecStore<float> {
  static __device__ __forceinline__ void put(float* o, size_t fs, const float (&f)[4][4],
                                             const float*, uint32_t) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      *reinterpret_cast<float4*>(o + k * fs) = make_float4(f[k][0], f[k][1], f[k][2], f[k][3]);
  }
};
template <> struct VecStore<double> {
  static __device__ __forceinline__ void put(double* o, size_t fs, const double (&f)[4][2],
                                             const double*, uint32_t) {
#pragma unroll
    for (int k = 0; k < 4; ++k) *reinterpret_cast<double2*>(o + k * fs) = make_double2(f[k][0], f[k][1]);
  }
};
template <> struct VecStore<__half> {
  static __device__ __forceinline__ uint32_t sr2(float a, float b, uint32_t r) {
    const __half2 h = __halves2half2(sr_half(a, r), sr_half(b, r >> 16));
    uint32_t u;
    memcpy(&u, &h, 4);
    return u;
  }
  static __device__ __forceinline__ void put(__half* o, size_t fs, const float (&f)[4][4],
                                             const __half* base, uint32_t seed) {
    const uint32_t key = uint32_t(o - base) << 2;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      uint2 v;
      v.x = sr2(f[k][0], f[k][1], hash32((key | uint32_t(k)) ^ seed));
      v.y = sr2(f[k][2], f[k][3], hash32(((key + 8u) | uint32_t(k)) ^ seed));
      *reinterpret_cast<uint2*>(o + k * fs) = v;
    }
  }
};

// Marches one (tile, chunk) work item of one pipe: the step of every cell of the tile's columns
// in the chunk's planes. `reinit` re-arms the CTA's mbarriers when the CTA has marched an item
// before (persistent grids). Returns false when a bounded wait gave up (error flag set).
// W16X8 (four columns only): warps of 16 columns x 8 rows (finer skipping of all-wall warps on
// small cross-sections) instead of 32 x 4.
template <class TE, bool W16X8 = false>
__device__ __forceinline__ bool step4_march(const CUtensorMap* tmap_p, const CUtensorMap* tmap_uvw,
                                            const Step2Geom& g,
                                            const Step4Const<typename MarchCfg<TE>::T>& k,
                                            int tile, int chunk, unsigned char* smem, bool reinit) {
  using Tl = Step4Tile<TE>;
  using T = typename Tl::T;
  using F = Ar<T>;
  constexpr int C = Tl::C, D1 = 2, R = Tl::R, HX = Tl::HX, HY = Tl::HY, SW = Tl::SW, S = Tl::S;
  constexpr int PPL = Tl::PPLANE, UPL = Tl::UPLANE, SLOT = Tl::SLOT;
  static_assert(!W16X8 || C == 4, "the 16 x 8 warp shape is for four columns per thread");

  TE* ring = reinterpret_cast<TE*>(smem);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + Tl::BAR_OFFSET);
  unsigned* released = reinterpret_cast<unsigned*>(full + S);

  // thread -> (column group tp, row ty); TPR threads of a warp share a row
  constexpr int TPR = W16X8 ? 4 : Tl::TX / C;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int qx = lane % TPR;                             // column group within the warp's row
  const int tp = W16X8 ? (warp & 1) * 4 + qx : qx;
  const int ty = W16X8 ? (warp >> 1) * 8 + (lane >> 2) : warp * (32 / TPR) + lane / TPR;
  const bool edge_l = qx == 0, edge_r = qx == TPR - 1;   // the row's outermost threads

  // ---- work: one (tile, chunk); odd chunks march towards -z
  const int zb = int((long long)g.L * chunk / g.nchunks);
  const int ze = int((long long)g.L * (chunk + 1) / g.nchunks);
  const int dir = (chunk & 1) ? -1 : 1;
  const int nout = ze - zb, niter = nout + 2 * R;
  const int start = dir > 0 ? zb - R : ze - 1 + R;      // real plane of march index 0
  const int2 org = g.tiles[tile];
  const int xa = org.x + C * tp, y = org.y + ty;
  const bool inside = xa < g.lxp && y < g.ly;           // lxp is a multiple of 8: all C columns

  T ws0[C], wsx[C], wsy[C], fl[C];
#pragma unroll
  for (int i = 0; i < C; ++i) ws0[i] = wsx[i] = wsy[i] = fl[i] = T(0);
  if (inside) {
    const ColCoef<T>* cp = reinterpret_cast<const ColCoef<T>*>(g.colcoef) + size_t(y) * g.lxp + xa;
#pragma unroll
    for (int i = 0; i < C; ++i) {
      const ColCoef<T> c = cp[i];
      ws0[i] = c.ws0; wsx[i] = c.wsx; wsy[i] = c.wsy; fl[i] = c.fluid;
    }
  }
  bool any = false, all = true;
#pragma unroll
  for (int i = 0; i < C; ++i) { any = any || fl[i] != T(0); all = all && fl[i] != T(0); }
  const bool warp_on = __any_sync(0xffffffffu, any);

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
  float* wbs = reinterpret_cast<float*>(smem + Tl::BASE_OFFSET);
  if constexpr (Tl::BASE) {
    if (g.wb)
      for (int i = tid; i < Tl::BW * Tl::BH; i += Tl::THREADS) {
        const int gx = org.x - 4 + i % Tl::BW, gy = org.y - 1 + i / Tl::BW;
        wbs[i] = (gx >= 0 && gy >= 0 && gx < g.lxp && gy < g.ly) ? g.wb[size_t(gy) * g.lxp + gx] : 0.0f;
      }
  }
  __syncthreads();

  auto slot_of = [](int m) { return unsigned(m) % unsigned(S); };
  auto phase_of = [](int m) { return uint32_t((unsigned(m) / unsigned(S)) & 1u); };
  auto issue = [&](int m) {            // load march plane m into its slot
    const unsigned slot = slot_of(m);
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
  auto arrive_wait = [&](int m) -> bool {
    if (mbar_wait_bounded(&full[slot_of(m)], phase_of(m), kWaitLimitNs)) return true;
    if (lane == 0) atomicOr(g.err, 1u);
    drain(m + 1);
    return false;
  };
  // Plane m - R leaves the window and its slot takes plane m - R + S. __syncwarp orders the
  // warp's shared loads before lane 0's acq_rel add to the slot's counter; the warp whose add
  // completes the count has acquired every warp's loads and orders them before its TMA write
  // with a proxy fence. A slot's next cycle starts only after its refill lands, which needs all
  // WARPS releases of this cycle, so the count is a multiple of WARPS exactly when a cycle is
  // complete.
  auto release_produce = [&](int m) {
    __syncwarp();
    if (m >= R && lane == 0) {
      const unsigned slot = slot_of(m - R);
      const unsigned seen = atom_add_acq_rel_cta(&released[slot], 1u) + 1u;
      const int mn = m - R + S;
      if (seen % unsigned(Tl::WARPS) == 0u && mn < niter) {
        fence_proxy_async_smem();
        issue(mn);
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

  // the gauge may have been written by another CTA of the same (chained batched) launch: read
  // it from L2, not from a possibly stale L1 line
  const T gauge = g.gauge ? T(__ldcg(g.gauge)) : T(0);
  const size_t FS = size_t(g.lxp) * g.ly * g.L;
  const TE* obase = reinterpret_cast<const TE*>(g.out);
  const uint32_t seed = hash32(g.step_no * 0x9e3779b9u + 0x632be5abu);
  TE* outp = reinterpret_cast<TE*>(g.out) + (size_t(start + dir * R) * g.ly + y) * g.lxp + xa;
  const long long ostep = (long long)dir * g.ly * g.lxp;     // output pointer step per plane
  const int po = (ty + 1) * SW + HX + C * tp;                 // p box
  const int uo = PPL + (ty + HY) * SW + HX + C * tp;          // u box (v, w at +UPL, +2 UPL)
  const T h6 = T(dir) / T(72);
  const T tbz = T(dir) * k.tb;                                // the z-moment carries the sign
  const T k48 = T(1) / T(48), k216 = T(1) / T(216), k54 = T(1) / T(54);

  T hu[4][C], hv[4][C], hw[4][C];                             // [plane jo-4..jo-1 slot][column]
  // Predictor terms waiting for their output plane: b2 = the march-previous plane's share of the
  // output being completed, b1 = the same for the next output, s1 = the self-plane moments of
  // the next output. Each output sums its two neighbour planes' shares first (a commutative
  // add) and then fuses its own plane's share, so the result of a cell does not depend on the
  // march direction and hence not on how the pipe is split into streamwise chunks.
  T b2[4][C], b1[4][C], s1[3][C];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int i = 0; i < C; ++i) {
      hu[j][i] = hv[j][i] = hw[j][i] = T(0);
      b2[j][i] = b1[j][i] = T(0);
      if (j < 3) s1[j][i] = T(0);
    }
  T comp[4][C];                                               // [moment][column]

  // one row of a plane: the thread's cells x-1 .. x+C of a field
  auto rowc = [&](const TE* p, T (&o)[C + 2]) {
    T q[C];
    ldv(p, q);
    T l = __shfl_up_sync(0xffffffffu, q[C - 1], 1);
    T r = __shfl_down_sync(0xffffffffu, q[0], 1);
    if (edge_l) l = ld1(p - 1);
    if (edge_r) r = ld1(p + C);
    o[0] = l;
#pragma unroll
    for (int i = 0; i < C; ++i) o[i + 1] = q[i];
    o[C + 1] = r;
  };

  // predictor contribution of march plane ma (see step_kernel.cuh for the factorisation)
  auto predictor = [&](int ma) {
    const TE* ss = ring + slot_of(ma) * SLOT;
    const int sp = start + dir * ma;                          // real plane
    // Row-factored weights w(cx)w(cy) = {4,1,1}x{4,1,1}/36, per column: per row
    // R = P(-1)+P(+1)+4P(0), D = P(+1)-P(-1); across rows A = R(-1)+R(+1)+4R(0), X likewise on
    // D, Y = R(+1)-R(-1). q and w^2 are formed once per cell of the row.
    T A[C][3], X[C][3], Y[C][3];
#pragma unroll
    for (int cy = -1; cy <= 1; ++cy) {
      T pr[C + 2], ur[C + 2], vr[C + 2], wr[C + 2];
      rowc(ss + po + cy * SW, pr);
      rowc(ss + uo + cy * SW, ur);
      rowc(ss + uo + UPL + cy * SW, vr);
      rowc(ss + uo + 2 * UPL + cy * SW, wr);
      if constexpr (Tl::BASE) {        // w = stored deviation + the column's base
        if (g.wb) {
          const float* br = wbs + (ty + 1 + cy) * Tl::BW + 4 + C * tp;
          float q[C];
          ldv(br, q);
          float l = __shfl_up_sync(0xffffffffu, q[C - 1], 1);
          float r = __shfl_down_sync(0xffffffffu, q[0], 1);
          if (edge_l) l = br[-1];
          if (edge_r) r = br[C];
          wr[0] = F::add(wr[0], l);
#pragma unroll
          for (int i = 0; i < C; ++i) wr[i + 1] = F::add(wr[i + 1], q[i]);
          wr[C + 1] = F::add(wr[C + 1], r);
        }
      }
      T qr[C + 2], w2r[C + 2];
#pragma unroll
      for (int j = 0; j < C + 2; ++j) {
        w2r[j] = F::mul(wr[j], wr[j]);
        qr[j] = F::fma(T(-1.5), F::fma(ur[j], ur[j], F::fma(vr[j], vr[j], w2r[j])), pr[j]);
      }
#pragma unroll
      for (int col = 0; col < C; ++col) {
        T P[3][3];   // [cx+1][k]: P0, P1' = P1/3, P2' = P2/4.5
#pragma unroll
        for (int cx = -1; cx <= 1; ++cx) {
          const int j = col + 1 + cx;
          const T u = ur[j], v = vr[j], w = wr[j];
          T P0, P1;
          if (cx == 0 && cy == 0) {
            P0 = qr[j];
            P1 = w;
          } else if (cx == 0 || cy == 0) {
            const T Bv = cy == 0 ? u : v;
            const T s3 = T(3 * (cx + cy));
            P0 = F::fma(Bv, F::fma(Bv, T(4.5), s3), qr[j]);
            P1 = F::mul(w, F::fma(Bv, s3, T(1)));
          } else {
            const T a1 = F::fma(v, T(cx * cy), u);
            const T s3 = T(3 * cx);
            P0 = F::fma(a1, F::fma(a1, T(4.5), s3), qr[j]);
            P1 = F::mul(w, F::fma(a1, s3, T(1)));
          }
          P[cx + 1][0] = P0; P[cx + 1][1] = P1; P[cx + 1][2] = w2r[j];
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const T Rq = F::fma(T(4), P[1][q], F::add(P[0][q], P[2][q]));
          const T Dq = F::sub(P[2][q], P[0][q]);
          if (cy == -1) { A[col][q] = Rq; X[col][q] = Dq; Y[col][q] = Rq; }
          else if (cy == 0) { A[col][q] = F::fma(T(4), Rq, A[col][q]); X[col][q] = F::fma(T(4), Dq, X[col][q]); }
          else { A[col][q] = F::add(A[col][q], Rq); X[col][q] = F::add(X[col][q], Dq); Y[col][q] = F::sub(Rq, Y[col][q]); }
        }
      }
    }
    // seam pressure jump: a wrapped plane adds off to p on its non-wall cells, i.e. off times
    // the non-wall weight sums (raw units, x36) to A0, X0, Y0 (a CTA-uniform branch)
    if (sp < 0 || sp >= g.L) {
      const T off = sp < 0 ? k.pin : -k.pin;
#pragma unroll
      for (int col = 0; col < C; ++col) {
        A[col][0] = F::fma(off, F::fma(T(-36), ws0[col], T(36)), A[col][0]);
        X[col][0] = F::fma(off, F::mul(T(-36), wsx[col]), X[col][0]);
        Y[col][0] = F::fma(off, F::mul(T(-36), wsy[col]), Y[col][0]);
      }
    }
    // True sums are A0'/36, dir A1'/12, A2'/8 (P1 and P2 were formed as P1/3 and P2/4.5).
    // Plane ma is the march-next neighbour of output ma-1 (completed here), itself, and the
    // march-previous neighbour of ma+1: with e = (A0 + A2)/6 and h = A1/6 the shares are
    // e + h (next), (2/3) A0 (self) and e - h (previous); for the z-moment h - e (previous),
    // none (self) and e + h (next), times dir.
#pragma unroll
    for (int col = 0; col < C; ++col) {
      const T eA = F::fma(A[col][2], k48, F::mul(A[col][0], k216));
      const T eX = F::fma(X[col][2], k48, F::mul(X[col][0], k216));
      const T eY = F::fma(Y[col][2], k48, F::mul(Y[col][0], k216));
      const T sA = F::fma(A[col][1], h6, eA), dA = F::fma(A[col][1], -h6, eA);
      const T sX = F::fma(X[col][1], h6, eX), dX = F::fma(X[col][1], -h6, eX);
      const T sY = F::fma(Y[col][1], h6, eY), dY = F::fma(Y[col][1], -h6, eY);
      comp[0][col] = F::fma(s1[0][col], k54, F::add(b2[0][col], sA));
      comp[1][col] = F::fma(s1[1][col], k54, F::add(b2[1][col], sX));
      comp[2][col] = F::fma(s1[2][col], k54, F::add(b2[2][col], sY));
      comp[3][col] = F::add(b2[3][col], sA);
#pragma unroll
      for (int q = 0; q < 4; ++q) b2[q][col] = b1[q][col];
      b1[0][col] = dA;
      b1[1][col] = dX;
      b1[2][col] = dY;
      b1[3][col] = -dA;
      s1[0][col] = A[col][0];
      s1[1][col] = X[col][0];
      s1[2][col] = Y[col][0];
    }
  };

  // own columns of march plane jo (for the history)
  auto own = [&](int jo, T (&uc)[C], T (&vc)[C], T (&wc)[C]) {
    const TE* so = ring + slot_of(jo) * SLOT;
    ldv(so + uo, uc); ldv(so + uo + UPL, vc); ldv(so + uo + 2 * UPL, wc);
  };

  // corrector and update of output march plane jo; history slot ROT holds plane jo-4 and is
  // then overwritten with plane jo
  auto output = [&](int jo, auto rot_c) {
    constexpr int ROT = decltype(rot_c)::value;
    constexpr int H2 = (ROT + 2) & 3;                         // plane jo-2
    const TE* so = ring + slot_of(jo) * SLOT;
    const TE* sa1 = ring + slot_of(jo + D1) * SLOT;           // march planes ahead
    const TE* sa2 = ring + slot_of(jo + 2 * D1) * SLOT;
    T pc[C], uc[C], vc[C], wc[C];
    ldv(so + po, pc);
    ldv(so + uo, uc); ldv(so + uo + UPL, vc); ldv(so + uo + 2 * UPL, wc);
    T res[4][C];                                              // [field][column]
    // u_new = K1 t1 + K2 t2 + K0 u + tb m* + tb F, t1 / t2 the six taps at distance d1 / 2 d1
    auto field = [&](int f, const T (&c)[C], const T (&zb1)[C], const T (&zb2)[C],
                     const T (&mom)[C], T tbm, T tf, T (&out)[C]) {
      const TE* q = so + uo + f * UPL;
      T ext[C + 8];                                           // cells x-4 .. x+C+3 of the row
#pragma unroll
      for (int v = 0; v < 4 / C; ++v) {
        T a[C], b[C];
        ldv(q - 4 + v * C, a);
        ldv(q + C + v * C, b);
#pragma unroll
        for (int i = 0; i < C; ++i) { ext[v * C + i] = a[i]; ext[4 + C + v * C + i] = b[i]; }
      }
#pragma unroll
      for (int i = 0; i < C; ++i) ext[4 + i] = c[i];
      T ym1[C], yp1[C], ym2[C], yp2[C], za1[C], za2[C];
      ldv(q - D1 * SW, ym1); ldv(q + D1 * SW, yp1);
      ldv(q - 2 * D1 * SW, ym2); ldv(q + 2 * D1 * SW, yp2);
      ldv(sa1 + uo + f * UPL, za1); ldv(sa2 + uo + f * UPL, za2);
#pragma unroll
      for (int i = 0; i < C; ++i) {
        const T t1 = F::add(F::add(F::add(ext[4 + i - D1], ext[4 + i + D1]), F::add(ym1[i], yp1[i])),
                            F::add(zb1[i], za1[i]));
        const T t2 = F::add(F::add(F::add(ext[i], ext[4 + i + 2 * D1]), F::add(ym2[i], yp2[i])),
                            F::add(zb2[i], za2[i]));
        out[i] = F::fma(k.K1, t1, F::fma(k.K2, t2, F::fma(k.K0, c[i], F::fma(tbm, mom[i], tf))));
      }
    };
    T mx[C], my[C];
#pragma unroll
    for (int i = 0; i < C; ++i) {
      res[0][i] = F::add(F::fma(pc[i], ws0[i], comp[0][i]), -gauge);
      mx[i] = F::fma(pc[i], wsx[i], comp[1][i]);
      my[i] = F::fma(pc[i], wsy[i], comp[2][i]);
    }
    field(0, uc, hu[H2], hu[ROT], mx, k.tb, k.tfx, res[1]);
    field(1, vc, hv[H2], hv[ROT], my, k.tb, k.tfy, res[2]);
    if constexpr (Tl::BASE) {          // the stored deviation of w: the column's base share
      if (g.wgt) {
        T tw[C];
        if (inside) ldv(g.wgt + size_t(y) * g.lxp + xa, tw);
        else for (int i = 0; i < C; ++i) tw[i] = T(0);
        auto fieldw = [&](T (&out)[C]) {
          const TE* q = so + uo + 2 * UPL;
          T ext[C + 8];
#pragma unroll
          for (int v = 0; v < 4 / C; ++v) {
            T a[C], b[C];
            ldv(q - 4 + v * C, a);
            ldv(q + C + v * C, b);
#pragma unroll
            for (int i = 0; i < C; ++i) { ext[v * C + i] = a[i]; ext[4 + C + v * C + i] = b[i]; }
          }
#pragma unroll
          for (int i = 0; i < C; ++i) ext[4 + i] = wc[i];
          T ym1[C], yp1[C], ym2[C], yp2[C], za1[C], za2[C];
          ldv(q - D1 * SW, ym1); ldv(q + D1 * SW, yp1);
          ldv(q - 2 * D1 * SW, ym2); ldv(q + 2 * D1 * SW, yp2);
          ldv(sa1 + uo + 2 * UPL, za1); ldv(sa2 + uo + 2 * UPL, za2);
#pragma unroll
          for (int i = 0; i < C; ++i) {
            const T t1 = F::add(F::add(F::add(ext[4 + i - D1], ext[4 + i + D1]), F::add(ym1[i], yp1[i])),
                                F::add(hw[H2][i], za1[i]));
            const T t2 = F::add(F::add(F::add(ext[i], ext[4 + i + 2 * D1]), F::add(ym2[i], yp2[i])),
                                F::add(hw[ROT][i], za2[i]));
            out[i] = F::fma(k.K1, t1, F::fma(k.K2, t2, F::fma(k.K0, wc[i], F::fma(tbz, comp[3][i], tw[i]))));
          }
        };
        fieldw(res[3]);
      } else {
        field(2, wc, hw[H2], hw[ROT], comp[3], tbz, k.tfz, res[3]);
      }
    } else {
      field(2, wc, hw[H2], hw[ROT], comp[3], tbz, k.tfz, res[3]);
    }
#pragma unroll
    for (int i = 0; i < C; ++i) { hu[ROT][i] = uc[i]; hv[ROT][i] = vc[i]; hw[ROT][i] = wc[i]; }
    if (inside) {   // wall and padding columns get zero (fl = 0)
      if (!all) {
#pragma unroll
        for (int f = 0; f < 4; ++f)
#pragma unroll
          for (int i = 0; i < C; ++i) res[f][i] = F::mul(res[f][i], fl[i]);
      }
      VecStore<TE>::put(outp, FS, res, obase, seed);
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
      const int h = (m - R) & 3;
      if (h == 0) own(m - R, hu[0], hv[0], hw[0]);
      else if (h == 1) own(m - R, hu[1], hv[1], hw[1]);
      else if (h == 2) own(m - R, hu[2], hv[2], hw[2]);
      else own(m - R, hu[3], hv[3], hw[3]);
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

// Folded update constants from the step constants, in the compute type in a fixed order.
template <class T> inline Step4Const<T> step4_const(const StepConst<T>& c) {
  Step4Const<T> k;
  const T a = c.tb * c.dtddy * c.m;
  k.K0 = a * c.c0 + c.cc;
  k.K1 = a * c.c1;
  k.K2 = a * c.c2;
  k.tb = c.tb;
  k.tfx = c.tb * c.fx; k.tfy = c.tb * c.fy; k.tfz = c.tb * c.fz;
  k.pin = c.pin;
  return k;
}

// One pipe, one step: CTA b marches (tile b % ntiles, chunk b / ntiles).
template <class TE>
__global__ void __launch_bounds__(Step4Tile<TE>::THREADS, 1)
    fslbm_step4_kernel(const __grid_constant__ CUtensorMap tmap_p,
                       const __grid_constant__ CUtensorMap tmap_uvw, const Step2Geom g,
                       const Step4Const<typename MarchCfg<TE>::T> k) {
  extern __shared__ __align__(128) unsigned char smem[];
  if (threadIdx.x == 0 && blockIdx.x == 0 && g.step_counter) *g.step_counter += 1;
  step4_march<TE>(&tmap_p, &tmap_uvw, g, k, blockIdx.x % g.ntiles, blockIdx.x / g.ntiles, smem,
                  false);
}

}  // namespace fslbm
