// Seeded noise shared by the host and device generators of initial fields.
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define FSLBM_HD __host__ __device__ __forceinline__
#else
#define FSLBM_HD inline
#endif

namespace fslbm {

// splitmix64 (Steele, Lea, Flood 2014): golden-ratio increment, two xor-shift-multiply rounds
FSLBM_HD uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// uniform in [-1, 1) from (seed, counter)
FSLBM_HD double unit_pm(uint64_t seed, uint64_t counter) {
  const uint64_t r = splitmix64(splitmix64(seed) ^ counter);
  return double(r >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

}  // namespace fslbm

namespace fslbm {

constexpr int kMaxInitModes = 16;

// Seeded start of a pipe solve: Poiseuille w = -umax (1 - r^2/R^2) in the stored (negated)
// convention, uniform noise of amplitude noise*umax on u, v, w, and `modes` random-phase
// streamwise/azimuthal sinusoids of amplitude mode_amp*umax under the envelope
// 2.6 s (1 - s^2), s = r/R. Counters of the noise follow the dense index z*lx*ly + y*lx + x.
struct PoiseuilleInit {
  double cx, cy, R, umax, noise, mode_amp;
  uint64_t seed;
  int lx, ly, L, modes;
  double ph[4 * kMaxInitModes];
};

// Mode phases from the seed.
inline void poiseuille_phases(PoiseuilleInit& q) {
  for (int m = 0; m < q.modes; ++m)
    for (int k = 0; k < 4; ++k)
      q.ph[4 * m + k] = 3.14159265358979323846 * (1.0 + unit_pm(q.seed ^ 0xA5A5A5A5ull, 4ull * m + k));
}

// p, u, v, w of fluid cell (x, y, z).
FSLBM_HD void poiseuille_cell(const PoiseuilleInit& q, int x, int y, int z, double out[4]) {
  const uint64_t idx = (uint64_t(z) * q.ly + y) * q.lx + x;
  const double dx = x - q.cx, dy = y - q.cy;
  const double s2 = (dx * dx + dy * dy) / (q.R * q.R), s = sqrt(s2);
  const double th = atan2(dy, dx);
  const double a = q.noise * q.umax, b = q.mode_amp * q.umax;
  double du = a * unit_pm(q.seed, 4 * idx + 1);
  double dv = a * unit_pm(q.seed, 4 * idx + 2);
  double dw = a * unit_pm(q.seed, 4 * idx + 3);
  const double env = 2.6 * s * (1.0 - fmin(s2, 1.0));
  for (int m = 0; m < q.modes; ++m) {
    const double kz = 2.0 * 3.14159265358979323846 * double(m + 1) * z / double(q.L);
    const int n = 1 + m % 4;
    dw += b * env * sin(kz + q.ph[4 * m]) * cos(n * th + q.ph[4 * m + 1]);
    du += b * env * cos(kz + q.ph[4 * m + 2]) * sin(n * th + q.ph[4 * m + 3]);
    dv += b * env * sin(kz + q.ph[4 * m + 2]) * cos(n * th + q.ph[4 * m + 3]);
  }
  out[0] = 0.0;
  out[1] = du;
  out[2] = dv;
  out[3] = -q.umax * fmax(0.0, 1.0 - s2) + dw;
}

}  // namespace fslbm
