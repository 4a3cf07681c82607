// FSLBM oracle: CPU restatement of the reference's fractional-step lattice Boltzmann
// pipe step, for TEST USE ONLY. Nothing in the product links or calls this file; only the
// test-suite, the smoke check and the CPU-baseline leg of the benchmark load it.
//
// What it restates (file:line in PipeDemoStandalone/FSLBM.cu of alparmat/FlowContrast):
//   predictor  (D3Q27 equilibrium pull, wall rule "p_n := p_centre")   FSLBM.cu:60-63, 130-173
//   corrector  (coarse-stride FD reverse diffusion, order 2<->4 blend)   FSLBM.cu:231-257, 269-273
//              and the orders 6..14 / blends the reference keeps as alternatives  FSLBM.cu:177-229
//   constants  dtddy = nu - 0.16666666, m = 1/d1^2                       FSLBM.cu:599, 624
//   boundaries walls := 0, buffer planes := copy +-pin, gauge p -= p2   FSLBM.cu:280-303
//   step order sweep -> BC(gauge of step c-1) -> monitor every 50 steps FSLBM.cu:620-647
//   monitor    q1,q2,p1,p2 over planes z=d2 and z=lz-d2, f, Re         FSLBM.cu:630-666
//   statistics plane x=lx/2 running means, |dev| and cross products     FSLBM.cu:683-768
//   geometry   pipe.m:38-62 (circle, 10-plane buffers, 10-cell wall pad)
//
// Semantics are Jacobi: every read of a step sees the time-n field and the boundary copy
// reads the swept field before it writes. The reference's in-place "shift" sweep has
// intra-launch read-after-write races when blend != 0 (corrector taps at z+2*d1 read planes
// the same launch writes, FSLBM.cu:253,275) and in bcond when p2 != 0 (FSLBM.cu:295,303);
// those are not reproduced. p2 is 0 before the first monitor (the reference leaves it
// uninitialised, FSLBM.cu:496).
//
// Constants: the D3Q27 weights are the exact rationals 8/27, 2/27, 1/54, 1/216 (the
// reference's float literals at FSLBM.cu:60-61 are their FP32 roundings). The literal
// decimals 0.16666666 (FSLBM.cu:599), 0.3333333333 and 0.0833333333 (FSLBM.cu:231) are kept
// as written; in the float instantiation they are the reference's own float literals.
//
// Extension beyond the reference (documented, zero by default): a body force F added inside
// the tblend bracket, u_new = (u* + dtddy*m*L(u) + F)*tb + u*(1-tb). With F = 0 the added
// term is an exact +0 and the reference arithmetic is unchanged.
//
// Parity pinning: the float instantiation of oracle_step_ref is compared in the test-suite
// against golden fields produced by the reference's own kernels (FSLBMcalc, shiftback, bcond)
// run on a B200 (tests/golden/).
#include <cstdint>
#include <cstring>
#include <cmath>
#include <cstdio>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int WALL = 125;
constexpr int BUF = 1;
constexpr int GHOST = 2;   // addition: periodic image cell of a cross-section periodic in x and y

template <class T> struct Consts {
  T tb, cc, pin, dtddy, m, c0, c1, c2, gauge, fx, fy, fz;
  T c[9];   // c[0] = c0 .. c[K]: corrector coefficients
  int d1, K;
};

// Corrector coefficient sets of FSLBM.cu:177-232 (orders 14..2 and the 8<->6, 6<->4, 4<->2
// blends; only 4<->2 is active in the reference, the others are its commented alternatives),
// formed in T as the reference forms its active set. order 0 or 4: the 4<->2 blend; 6: 6<->4;
// 8: 8<->6 (blend weights the higher order); 10, 12, 14: fixed. Returns K (taps), 0 if unknown.
template <class T>
int fd_coefficients(int order, T b, T* c) {
  for (int k = 0; k < 9; ++k) c[k] = T(0);
  switch (order) {
    case 0: case 4:
      c[0] = T(-6.0) - T(1.5) * b; c[1] = T(1.0) + T(0.3333333333) * b; c[2] = T(-0.0833333333) * b;
      return 2;
    case 6:
      c[0] = T(-7.5) - T(0.66666666666) * b; c[1] = T(1.3333333) + T(0.16666666666) * b;
      c[2] = T(-0.08333333) - T(0.0666666666666) * b; c[3] = T(0.01111111) * b;
      return 3;
    case 8:
      c[0] = T(-8.166666666666666) - T(0.375) * b; c[1] = T(1.5) + T(0.1) * b;
      c[2] = T(-0.15) - T(0.05) * b; c[3] = T(0.01111111) + T(0.014285714285714) * b;
      c[4] = T(-0.001785714285714) * b;
      return 4;
    case 10:
      c[0] = T(-8.78166666666); c[1] = T(1.66666666); c[2] = T(-0.23809523809);
      c[3] = T(0.03968253968); c[4] = T(-0.00496031746); c[5] = T(0.00031746031);
      return 5;
    case 12:
      c[0] = T(-8.94833333333); c[1] = T(1.71428571429); c[2] = T(-0.26785714285);
      c[3] = T(0.05291005291); c[4] = T(-0.00892857142); c[5] = T(0.00103896103);
      c[6] = T(-0.00006012506);
      return 6;
    case 14:
      c[0] = T(-9.16453231293); c[1] = T(1.77777777778); c[2] = T(-0.31111111111);
      c[3] = T(0.07542087542); c[4] = T(-0.01767676767); c[5] = T(3.48096348e-3);
      c[6] = T(-5.1800052e-4); c[7] = T(5.0742908e-5); c[8] = T(-2.4281274e-6);
      return 8;
    default:
      return 0;
  }
}

// Derive the per-step constants exactly as the reference forms them (FSLBM.cu:231, 269,
// 599, 624). For T=float this reproduces the reference's float arithmetic on its inputs.
template <class T>
Consts<T> derive(const double* prm) {
  // prm: tblend, pin, nu, d1, blend, gauge, fx, fy, fz, fd_order
  Consts<T> k;
  k.tb = T(prm[0]);
  k.cc = T(1.0 - double(k.tb));                  // float cc=1.0-tblend (double then float)
  k.pin = T(prm[1]);
  const T nu = T(prm[2]);
  k.dtddy = nu - T(0.16666666);                  // FSLBM.cu:599
  k.d1 = int(prm[3]);
  k.m = T(1.0 / double(T(k.d1 * k.d1)));         // 1.0/float(d1*d1), FSLBM.cu:624
  const T blend = T(prm[4]);
  k.K = fd_coefficients<T>(int(prm[9]), blend, k.c);   // FSLBM.cu:231 for orders 0/4
  k.c0 = k.c[0]; k.c1 = k.c[1]; k.c2 = k.c[2];
  k.gauge = T(prm[5]);
  k.fx = T(prm[6]); k.fy = T(prm[7]); k.fz = T(prm[8]);
  return k;
}

template <class T> struct Field {
  const T* p; const T* u; const T* v; const T* w;
};

inline int clampi(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

// One FSLBM sweep + boundary step on the reference layout (buffer planes included).
// io: lx*ly*lz mask, values 0 (fluid), 1 (periodic buffer), 125 (wall); idx = x + lx*(y + ly*z).
template <class T>
void step_ref(const uint8_t* io, int lx, int ly, int lz, int d2, const Consts<T>& K,
              const T* in, T* out, int nthreads) {
  const long n = long(lx) * ly * lz;
  const T* ip = in; const T* iu = in + n; const T* iv = in + 2 * n; const T* iw = in + 3 * n;
  T* op = out; T* ou = out + n; T* ov = out + 2 * n; T* ow = out + 3 * n;
  const long lxy = long(lx) * ly;
  // D3Q27 weights for the x-mid plane (FSLBM.cu:60-63) as exact rationals; x+-1 planes
  // carry the extra factor 0.25 (FSLBM.cu:159, 171).
  const T W[9] = {T(8.0 / 27.0), T(2.0 / 27.0), T(2.0 / 27.0), T(2.0 / 27.0), T(2.0 / 27.0),
                  T(1.0 / 54.0), T(1.0 / 54.0), T(1.0 / 54.0), T(1.0 / 54.0)};
  const int cy[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
  const int cz[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
  auto tex = [&](const T* f, int x, int y, int z) -> T {   // tex3D clamp addressing
    return f[clampi(x, lx) + lx * (long(clampi(y, ly)) + long(ly) * clampi(z, lz))];
  };

  // ---- sweep: new values for fluid cells (FSLBM.cu:130-275); everything else is set by BC
  std::vector<T> sp(n), su(n), sv(n), sw_(n);
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads)
  for (int z = 0; z < lz; ++z)
    for (int y = 0; y < ly; ++y)
      for (int x = 0; x < lx; ++x) {
        const long idx = x + lx * (long(y) + long(ly) * z);
        if (io[idx] != 0) { sp[idx] = ip[idx]; su[idx] = iu[idx]; sv[idx] = iv[idx]; sw_[idx] = iw[idx]; continue; }
        const T rhd1 = ip[idx];
        const T u = iu[idx], v = iv[idx], w = iw[idx];
        T rt1 = 0, uxt1v = 0, uyt1v = 0, uzt1v = 0;
        for (int i = 8; i >= 0; --i) {
          const long id2 = long(lx) * cy[i] + long(cz[i]) * lxy;
          // three x offsets in the reference's order: 0, +1, -1
          for (int xo = 0; xo < 3; ++xo) {
            const int cx = (xo == 0) ? 0 : (xo == 1 ? 1 : -1);
            const long nb = idx + id2 + cx;
            const bool notwall = io[nb] < WALL;                 // FSLBM.cu:138,152,164
            const T pn = notwall ? ip[nb] : rhd1;               // FSLBM.cu:140
            const T un = iu[nb], vn = iv[nb], wn = iw[nb];
            T zet;
            if (cx == 0) zet = (T(cy[i]) * vn + T(cz[i]) * wn) * T(3);
            else if (cx == 1) zet = (un + T(cy[i]) * vn + T(cz[i]) * wn) * T(3);
            else zet = (-un + T(cy[i]) * vn + T(cz[i]) * wn) * T(3);
            const T uu = (un * un + vn * vn + wn * wn) * T(3);
            T rt1v = W[i] * (pn + zet + T(0.5) * (zet * zet - uu));
            if (cx != 0) rt1v = rt1v * T(0.25);
            rt1 += rt1v;
            uyt1v += rt1v * T(cy[i]);
            if (cx == 1) uxt1v += rt1v;
            if (cx == -1) uxt1v -= rt1v;
            uzt1v += rt1v * T(cz[i]);
          }
        }
        // corrector (FSLBM.cu:236-257): reads of the time-n field through clamped addressing
        const int d1 = K.d1;
        T ux2 = u * K.c0, uy2 = v * K.c0, uz2 = w * K.c0;
        {
          const int o = d1;
          const T a0 = tex(iu, x + o, y, z), a1 = tex(iu, x - o, y, z), a2 = tex(iu, x, y + o, z),
                  a3 = tex(iu, x, y - o, z), a4 = tex(iu, x, y, z + o), a5 = tex(iu, x, y, z - o);
          const T b0 = tex(iv, x + o, y, z), b1 = tex(iv, x - o, y, z), b2 = tex(iv, x, y + o, z),
                  b3 = tex(iv, x, y - o, z), b4 = tex(iv, x, y, z + o), b5 = tex(iv, x, y, z - o);
          const T e0 = tex(iw, x + o, y, z), e1 = tex(iw, x - o, y, z), e2 = tex(iw, x, y + o, z),
                  e3 = tex(iw, x, y - o, z), e4 = tex(iw, x, y, z + o), e5 = tex(iw, x, y, z - o);
          ux2 += K.c1 * (a0 + a1 + a2 + a3 + a4 + a5);
          uy2 += K.c1 * (b0 + b1 + b2 + b3 + b4 + b5);
          uz2 += K.c1 * (e0 + e1 + e2 + e3 + e4 + e5);
        }
        for (int kk = 2; kk <= K.K; ++kk) {             // taps at 2*d1 .. K*d1
          const int o = kk * d1;
          const T a0 = tex(iu, x + o, y, z), a1 = tex(iu, x - o, y, z), a2 = tex(iu, x, y + o, z),
                  a3 = tex(iu, x, y - o, z), a4 = tex(iu, x, y, z + o), a5 = tex(iu, x, y, z - o);
          const T b0 = tex(iv, x + o, y, z), b1 = tex(iv, x - o, y, z), b2 = tex(iv, x, y + o, z),
                  b3 = tex(iv, x, y - o, z), b4 = tex(iv, x, y, z + o), b5 = tex(iv, x, y, z - o);
          const T e0 = tex(iw, x + o, y, z), e1 = tex(iw, x - o, y, z), e2 = tex(iw, x, y + o, z),
                  e3 = tex(iw, x, y - o, z), e4 = tex(iw, x, y, z + o), e5 = tex(iw, x, y, z - o);
          ux2 += K.c[kk] * (a0 + a1 + a2 + a3 + a4 + a5);
          uy2 += K.c[kk] * (b0 + b1 + b2 + b3 + b4 + b5);
          uz2 += K.c[kk] * (e0 + e1 + e2 + e3 + e4 + e5);
        }
        // FSLBM.cu:269-273 (+ optional body force, exact +0 when unused)
        sp[idx] = rt1;
        su[idx] = (uxt1v + K.dtddy * ux2 * K.m + K.fx) * K.tb + u * K.cc;
        sv[idx] = (uyt1v + K.dtddy * uy2 * K.m + K.fy) * K.tb + v * K.cc;
        sw_[idx] = (uzt1v + K.dtddy * uz2 * K.m + K.fz) * K.tb + w * K.cc;
      }

  // ---- boundary step (FSLBM.cu:280-303), reading the swept field before any write
  const int L = lz - 2 * d2;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads)
  for (int z = 0; z < lz; ++z)
    for (int y = 0; y < ly; ++y)
      for (int x = 0; x < lx; ++x) {
        const long idx = x + lx * (long(y) + long(ly) * z);
        if (io[idx] == WALL) { op[idx] = 0; ou[idx] = 0; ov[idx] = 0; ow[idx] = 0; continue; }
        if (z < d2) {
          const long s = x + lx * (long(y) + long(ly) * (z + L));
          T pv = sp[s]; pv -= K.gauge; pv += K.pin;
          op[idx] = pv; ou[idx] = su[s]; ov[idx] = sv[s]; ow[idx] = sw_[s];
        } else if (z >= lz - d2) {
          const long s = x + lx * (long(y) + long(ly) * (z - L));
          T pv = sp[s]; pv -= K.pin; pv -= K.gauge;
          op[idx] = pv; ou[idx] = su[s]; ov[idx] = sv[s]; ow[idx] = sw_[s];
        } else {
          op[idx] = sp[idx] - K.gauge; ou[idx] = su[idx]; ov[idx] = sv[idx]; ow[idx] = sw_[idx];
        }
      }
}

// Checks the mask contract the restatement relies on. Returns 0 or a negative code.
int check_ref_mask(const uint8_t* io, int lx, int ly, int lz, int d2) {
  if (lx < 3 || ly < 3 || lz < 2 * d2 + 1 || d2 < 1) return -1;
  for (int z = 0; z < lz; ++z)
    for (int y = 0; y < ly; ++y)
      for (int x = 0; x < lx; ++x) {
        const uint8_t c = io[x + lx * (long(y) + long(ly) * z)];
        if (c != 0 && c != BUF && c != WALL) return -2;
        if (c == 0) {
          if (z < d2 || z >= lz - d2) return -3;                       // fluid only between buffers
          if (x == 0 || y == 0 || x == lx - 1 || y == ly - 1) return -4;  // no fluid on the box rim
        }
      }
  return 0;
}

template <class T>
void pad_core(const uint8_t* mask, int planes, int lx, int ly, int L, int d2, T pin, const T* core,
              std::vector<uint8_t>& io, std::vector<T>& ref) {
  // Builds the reference layout (d2 buffer planes at each streamwise end, FSLBM.cu:291-301)
  // from a periodic core; mask holds one cross-section (planes = 1, extruded along z) or one
  // per core plane (planes = L). Buffer planes carry the mask of the core plane they copy.
  const int lz = L + 2 * d2;
  const long nc = long(lx) * ly * L, nr = long(lx) * ly * lz, lxy = long(lx) * ly;
  io.assign(nr, 0);
  ref.assign(4 * nr, T(0));
  for (int z = 0; z < lz; ++z) {
    int zc = z - d2; int jump = 0;
    if (zc < 0) { zc += L; jump = 1; }
    else if (zc >= L) { zc -= L; jump = -1; }
    const uint8_t* mp = mask + (planes == 1 ? 0 : lxy * zc);
    for (long j = 0; j < lxy; ++j) {
      const long r = j + lxy * z, c = j + lxy * zc;
      const bool wall = mp[j] == WALL;
      io[r] = wall ? WALL : (mp[j] == GHOST ? GHOST : (jump ? BUF : 0));
      if (wall) continue;
      T pv = core[c];
      if (jump == 1) pv += pin;
      if (jump == -1) pv -= pin;
      ref[r] = pv; ref[nr + r] = core[nc + c]; ref[2 * nr + r] = core[2 * nc + c];
      ref[3 * nr + r] = core[3 * nc + c];
    }
  }
}

// Monitor quantities of FSLBM.cu:630-666 on the reference layout, in FP64.
// out: q1, q2, p1, p2, f, sample(w at lx/2,ly/2,lz/2), Re
template <class T>
void monitor_ref(const uint8_t* io, int lx, int ly, int lz, int d2, double nu, double radius,
                 const T* f, double* out) {
  const long n = long(lx) * ly * lz, lxy = long(lx) * ly;
  double l1 = 0;
  for (long i = 0; i < n; ++i) if (io[i] == BUF) l1 += 1.0;
  l1 /= double(2 * d2);                                       // FSLBM.cu:589-591
  double q1 = 0, q2 = 0, p1 = 0, p2 = 0;
  for (long j = 0; j < lxy; ++j) {
    if (io[j + lxy * d2] == GHOST) continue;                   // periodic images are not counted
    q2 += double(f[3 * n + j + lxy * (lz - d2)]); p2 += double(f[j + lxy * (lz - d2)]);
    q1 += double(f[3 * n + j + lxy * d2]);        p1 += double(f[j + lxy * d2]);
  }
  p1 /= l1; p2 /= l1; q1 /= l1; q2 /= l1;                    // FSLBM.cu:647
  const double L = double(lz - 2 * d2);
  out[0] = q1; out[1] = q2; out[2] = p1; out[3] = p2;
  out[4] = (p1 - p2) / q1 / q1 / 3.0 * 4.0 * radius / L;     // FSLBM.cu:660
  out[5] = double(f[3 * n + (lx / 2) + long(lx) * (ly / 2) + lxy * (lz / 2)]);  // FSLBM.cu:653,665
  out[6] = 2.0 * radius * q1 / nu;                            // FSLBM.cu:650
}

// Refills the ghost band (cells marked GHOST, G wide) of a cross-section periodic in x and y
// with the periodic images of the interior, in every plane of the core fields.
template <class T>
void fill_ghosts(const uint8_t* mask2d, int lx, int ly, int L, int G, T* fields) {
  if (G <= 0) return;
  const int nx = lx - 2 * G, ny = ly - 2 * G;
  const long lxy = long(lx) * ly, nc = lxy * L;
  for (int y = 0; y < ly; ++y)
    for (int x = 0; x < lx; ++x) {
      if (mask2d[x + long(lx) * y] != GHOST) continue;
      const int sx = G + ((x - G) % nx + nx) % nx, sy = G + ((y - G) % ny + ny) % ny;
      for (int k = 0; k < 4; ++k)
        for (int z = 0; z < L; ++z)
          fields[k * nc + lxy * z + x + long(lx) * y] = fields[k * nc + lxy * z + sx + long(lx) * sy];
    }
}

template <class T>
int run_core(const uint8_t* mask2d, int planes, int lx, int ly, int L, const double* prm,
             int monitor_every, double radius, long nsteps, T* fields, double* mon_out,
             int nthreads, int ghost = 0) {
  // prm: tblend, pin, nu, d1, blend, fx, fy, fz, fd_order (gauge is driven here)
  const int d1 = int(prm[3]);
  double cdum[9];
  const int K = fd_coefficients<double>(int(prm[8]), 0.0, cdum);
  if (K == 0) return -6;
  const int d2 = std::max(1, K * d1);                         // buffers cover the corrector reach
  if (L < d2 + 1) return -5;
  if (planes != 1 && planes != L) return -1;
  for (int z = 0; z < planes; ++z)
    for (int y = 0; y < ly; ++y)
      for (int x = 0; x < lx; ++x) {
        const uint8_t c = mask2d[x + long(lx) * (y + long(ly) * z)];
        if (c != 0 && c != WALL && !(c == GHOST && ghost > 0)) return -2;
        if (c == 0 && (x == 0 || y == 0 || x == lx - 1 || y == ly - 1)) return -4;
      }
  const long nc = long(lx) * ly * L, lxy = long(lx) * ly;
  const int lz = L + 2 * d2;
  std::vector<uint8_t> io;
  std::vector<T> a, b(4 * long(lx) * ly * lz);
  double gauge = 0.0;
  long nmon = 0;
  for (long c = 1; c <= nsteps; ++c) {
    double p10[10] = {prm[0], prm[1], prm[2], prm[3], prm[4], gauge, prm[5], prm[6], prm[7], prm[8]};
    const Consts<T> K = derive<T>(p10);
    pad_core(mask2d, planes, lx, ly, L, d2, K.pin, fields, io, a);
    step_ref<T>(io.data(), lx, ly, lz, d2, K, a.data(), b.data(), nthreads);
    gauge = 0.0;                                              // FSLBM.cu:628
    const long nr = long(lx) * ly * lz;
    for (int k = 0; k < 4; ++k)
      std::memcpy(fields + k * nc, b.data() + k * nr + lxy * d2, sizeof(T) * nc);
    fill_ghosts(mask2d, lx, ly, L, ghost, fields);
    if (monitor_every > 0 && c % monitor_every == 0) {
      double m[7];
      monitor_ref<T>(io.data(), lx, ly, lz, d2, prm[2], radius, b.data(), m);
      gauge = m[3];                                           // p2 gauges the next step
      if (mon_out) { for (int k = 0; k < 7; ++k) mon_out[7 * nmon + k] = m[k]; }
      ++nmon;
    }
  }
  return int(nmon);
}

}  // namespace

extern "C" {

int oracle_check_ref_mask(const uint8_t* io, int lx, int ly, int lz, int d2) {
  return check_ref_mask(io, lx, ly, lz, d2);
}

// One reference-layout step. prm: tblend, pin, nu, d1, blend, gauge(p2), fx, fy, fz, fd_order.
// in/out: 4*lx*ly*lz values (p block, u block, v block, w block).
int oracle_step_ref_f64(const uint8_t* io, int lx, int ly, int lz, int d2, const double* prm,
                        const double* in, double* out, int nthreads) {
  const int rc = check_ref_mask(io, lx, ly, lz, d2);
  if (rc) return rc;
  step_ref<double>(io, lx, ly, lz, d2, derive<double>(prm), in, out, nthreads);
  return 0;
}
int oracle_step_ref_f32(const uint8_t* io, int lx, int ly, int lz, int d2, const double* prm,
                        const float* in, float* out, int nthreads) {
  const int rc = check_ref_mask(io, lx, ly, lz, d2);
  if (rc) return rc;
  step_ref<float>(io, lx, ly, lz, d2, derive<float>(prm), in, out, nthreads);
  return 0;
}

int oracle_monitor_ref_f64(const uint8_t* io, int lx, int ly, int lz, int d2, double nu,
                           double radius, const double* f, double* out) {
  monitor_ref<double>(io, lx, ly, lz, d2, nu, radius, f, out);
  return 0;
}
int oracle_monitor_ref_f32(const uint8_t* io, int lx, int ly, int lz, int d2, double nu,
                           double radius, const float* f, double* out) {
  monitor_ref<float>(io, lx, ly, lz, d2, nu, radius, f, out);
  return 0;
}

// Periodic-core run: cross-section mask (lx*ly, 0 fluid / 125 wall) extruded over L planes,
// streamwise wrap with the +-pin pressure jump across the seam, realised by padding the core
// with d2 = max(1, K*d1) reference buffer planes each step (K corrector taps). prm: tblend, pin,
// nu, d1, blend, fx, fy, fz, fd_order. Monitor every `monitor_every` steps (0: never); records (7 doubles each) go to
// mon_out. Returns the number of monitor records or a negative code.
int oracle_run_core_f64(const uint8_t* mask2d, int lx, int ly, int L, const double* prm,
                        int monitor_every, double radius, long nsteps, double* fields,
                        double* mon_out, int nthreads) {
  return run_core<double>(mask2d, 1, lx, ly, L, prm, monitor_every, radius, nsteps, fields,
                          mon_out, nthreads);
}
int oracle_run_core_f32(const uint8_t* mask2d, int lx, int ly, int L, const double* prm,
                        int monitor_every, double radius, long nsteps, float* fields,
                        double* mon_out, int nthreads) {
  return run_core<float>(mask2d, 1, lx, ly, L, prm, monitor_every, radius, nsteps, fields,
                         mon_out, nthreads);
}

// The same with a cross-section periodic in x and y (an addition, not in the reference): a band
// of `ghost` cells at the box rim, marked 2 in mask2d, holds the periodic images of the interior
// (period lx - 2*ghost by ly - 2*ghost); ghosts are read as fluid neighbours, never stepped, and
// refilled after every step; monitors skip them.
int oracle_run_core_periodic_f64(const uint8_t* mask2d, int lx, int ly, int L, int ghost,
                                 const double* prm, int monitor_every, double radius, long nsteps,
                                 double* fields, double* mon_out, int nthreads) {
  fill_ghosts(mask2d, lx, ly, L, ghost, fields);
  return run_core<double>(mask2d, 1, lx, ly, L, prm, monitor_every, radius, nsteps, fields,
                          mon_out, nthreads, ghost);
}
int oracle_run_core_periodic_f32(const uint8_t* mask2d, int lx, int ly, int L, int ghost,
                                 const double* prm, int monitor_every, double radius, long nsteps,
                                 float* fields, double* mon_out, int nthreads) {
  fill_ghosts(mask2d, lx, ly, L, ghost, fields);
  return run_core<float>(mask2d, 1, lx, ly, L, prm, monitor_every, radius, nsteps, fields,
                         mon_out, nthreads, ghost);
}

// The same with a mask per core plane (lx*ly*L, 0 fluid / 125 wall): geometry that varies
// along the pipe, such as wall roughness; buffer planes copy the wrapped core planes' masks.
int oracle_run_core3d_f64(const uint8_t* mask3d, int lx, int ly, int L, const double* prm,
                          int monitor_every, double radius, long nsteps, double* fields,
                          double* mon_out, int nthreads) {
  return run_core<double>(mask3d, L, lx, ly, L, prm, monitor_every, radius, nsteps, fields,
                          mon_out, nthreads);
}
int oracle_run_core3d_f32(const uint8_t* mask3d, int lx, int ly, int L, const double* prm,
                          int monitor_every, double radius, long nsteps, float* fields,
                          double* mon_out, int nthreads) {
  return run_core<float>(mask3d, L, lx, ly, L, prm, monitor_every, radius, nsteps, fields,
                         mon_out, nthreads);
}

// Statistics accumulation of FSLBM.cu:715-748 on one sampled plane (n values per field).
// acc: 11 arrays of n doubles in the reference order
//   pav, uxav, uyav, uzav, p2av, ux2av, uy2av, uz2av, uxyav, uxzav, uyzav.
// cnt is the mean-sample count AFTER this sample is included (the reference increments first).
void oracle_stats_accumulate(long n, const double* p, const double* u, const double* v,
                             const double* w, int cnt, double* acc) {
  double* pav = acc; double* uxav = acc + n; double* uyav = acc + 2 * n; double* uzav = acc + 3 * n;
  double* p2av = acc + 4 * n; double* ux2av = acc + 5 * n; double* uy2av = acc + 6 * n;
  double* uz2av = acc + 7 * n; double* uxyav = acc + 8 * n; double* uxzav = acc + 9 * n;
  double* uyzav = acc + 10 * n;
  for (long k = 0; k < n; ++k) {
    pav[k] += p[k];  const double dd1 = pav[k] / double(cnt) - p[k];
    uxav[k] += u[k]; const double dd2 = uxav[k] / double(cnt) - u[k];
    uyav[k] += v[k]; const double dd3 = uyav[k] / double(cnt) - v[k];
    uzav[k] += w[k]; const double dd4 = uzav[k] / double(cnt) - w[k];
    p2av[k] += std::fabs(dd1); ux2av[k] += std::fabs(dd2);
    uy2av[k] += std::fabs(dd3); uz2av[k] += std::fabs(dd4);
    uxyav[k] += dd2 * dd3; uxzav[k] += dd2 * dd4; uyzav[k] += dd4 * dd3;
  }
}

// pipe.m:36-60 restated: mask of (lx0+2d) x (lx0+2d) x (l0+2d) with a circle of radius lx0/2
// whose test uses 1-based indices, d buffer planes (value 1) at both ends, d wall cells of
// padding in x and y. out must hold (lx0+2d)^2*(l0+2d) bytes, x fastest.
int oracle_pipe_m_mask(int lx0, int l0, int d, uint8_t* out) {
  const int lx = lx0 + 2 * d, lz = l0 + 2 * d;
  const double o = lx0 / 2.0, r = o;
  for (int k = 1; k <= lz; ++k)
    for (int j = 1; j <= lx; ++j)
      for (int i = 1; i <= lx; ++i) {
        uint8_t v = WALL;
        const int ii = i - d, jj = j - d;
        if (ii >= 1 && ii <= lx0 && jj >= 1 && jj <= lx0) {
          const bool inside = ((ii - o) * (ii - o) + (jj - o) * (jj - o)) <= r * r;
          v = inside ? 0 : WALL;
          if (inside && (k <= d || k > lz - d)) v = BUF;
        }
        out[(i - 1) + long(lx) * ((j - 1) + long(lx) * (k - 1))] = v;
      }
  return 0;
}

// Corrector coefficients c0..c8 (FP64 forms) of an order; returns the tap count K or 0.
int oracle_fd_coefficients(int order, double blend, double* c) {
  return fd_coefficients<double>(order, blend, c);
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"

// ---- seeded starting fields of the benchmark workloads ----
// The benchmark's CPU arms (the timed CPU baseline and the reference arm) start from the same
// seeded state as the GPU arm but must not load the solver library, so the generator is
// restated here: a circular pipe of radius R centred at (cx, cy) (fluid iff
// (x-cx)^2 + (y-cy)^2 <= R^2), p = 0, stored w = -umax (1 - s^2) with s = r/R, uniform noise
// of amplitude noise*umax on u, v, w, and `modes` random-phase streamwise/azimuthal sinusoids
// of amplitude mode_amp*umax under the envelope 2.6 s (1 - s^2). Random numbers are
// splitmix64 (Steele, Lea and Flood, 2014) of the seed, xor-ed with a counter (4*cell + k,
// cell = x + lx*(y + ly*z)), mapped to [-1, 1) from the top 53 bits. The expressions are
// evaluated in the same order as the library's generator, so the two agree bit for bit (a CPU
// test checks this).
namespace {
uint64_t oracle_splitmix(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double oracle_unit(uint64_t seed, uint64_t counter) {
  return double(oracle_splitmix(oracle_splitmix(seed) ^ counter) >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}
}  // namespace

extern "C" int oracle_init_poiseuille(int lx, int ly, int L, double R, double cx, double cy,
                                      double umax, double noise, int modes, double mode_amp,
                                      uint64_t seed, double* out) {
  if (lx < 1 || ly < 1 || L < 1 || R <= 0 || modes < 0 || modes > 16 || !out) return -1;
  const double pi = 3.14159265358979323846;
  double ph[64];
  for (int m = 0; m < modes; ++m)
    for (int k = 0; k < 4; ++k) ph[4 * m + k] = pi * (1.0 + oracle_unit(seed ^ 0xA5A5A5A5ull, 4ull * m + k));
  const long nc = long(lx) * ly * L;
  const double a = noise * umax, b = mode_amp * umax;
  for (int z = 0; z < L; ++z)
    for (int y = 0; y < ly; ++y)
      for (int x = 0; x < lx; ++x) {
        const long i = x + long(lx) * (y + long(ly) * z);
        const double dx = x - cx, dy = y - cy;
        double f[4] = {0.0, 0.0, 0.0, 0.0};
        if (dx * dx + dy * dy <= R * R) {
          const uint64_t idx = uint64_t(i);
          const double s2 = (dx * dx + dy * dy) / (R * R), s = std::sqrt(s2);
          const double th = std::atan2(dy, dx);
          double du = a * oracle_unit(seed, 4 * idx + 1);
          double dv = a * oracle_unit(seed, 4 * idx + 2);
          double dw = a * oracle_unit(seed, 4 * idx + 3);
          const double env = 2.6 * s * (1.0 - std::fmin(s2, 1.0));
          for (int m = 0; m < modes; ++m) {
            const double kz = 2.0 * pi * double(m + 1) * z / double(L);
            const int n = 1 + m % 4;
            dw += b * env * std::sin(kz + ph[4 * m]) * std::cos(n * th + ph[4 * m + 1]);
            du += b * env * std::cos(kz + ph[4 * m + 2]) * std::sin(n * th + ph[4 * m + 3]);
            dv += b * env * std::sin(kz + ph[4 * m + 2]) * std::cos(n * th + ph[4 * m + 3]);
          }
          f[1] = du; f[2] = dv; f[3] = -umax * std::fmax(0.0, 1.0 - s2) + dw;
        }
        for (int k = 0; k < 4; ++k) out[k * nc + i] = f[k];
      }
  return 0;
}
