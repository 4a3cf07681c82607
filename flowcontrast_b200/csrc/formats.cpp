// Host-side file formats and generators of the drop-in surface: pipe.txt and param.txt
// (written by pipe.m, read by FSLBM.cu), the pipe.m geometry, the reference-layout mask split
// and the seeded initial-field generator.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fslbm.h"
#include "noise.h"

int fslbm_set_error(int code, const char* fmt, ...);

namespace {

constexpr uint8_t kWall = 125, kBuf = 1;

bool read_file(const char* path, std::string& out) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  char buf[1 << 16];
  size_t n;
  out.clear();
  while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, n);
  std::fclose(f);
  return true;
}

// Splits on whitespace.
std::vector<std::string> tokens(const std::string& s) {
  std::vector<std::string> t;
  size_t i = 0;
  while (i < s.size()) {
    while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
    size_t j = i;
    while (j < s.size() && !std::isspace(static_cast<unsigned char>(s[j]))) ++j;
    if (j > i) t.emplace_back(s.substr(i, j - i));
    i = j;
  }
  return t;
}

bool parse_double(const std::string& t, double* v) {
  char* end = nullptr;
  errno = 0;
  *v = std::strtod(t.c_str(), &end);
  return errno == 0 && end && *end == 0;
}

bool parse_int(const std::string& t, int* v) {
  double d;
  if (!parse_double(t, &d) || d != std::floor(d) || std::fabs(d) > 2e9) return false;
  *v = int(d);
  return true;
}

}  // namespace

extern "C" int fslbm_read_pipe_txt(const char* path, int lx, int ly, int lz, uint8_t* out) {
  if (!path || !out || lx <= 0 || ly <= 0 || lz <= 0)
    return fslbm_set_error(FSLBM_ERR_ARG, "read_pipe_txt: bad argument");
  std::string s;
  if (!read_file(path, s)) return fslbm_set_error(FSLBM_ERR_IO, "read_pipe_txt: cannot open %s", path);
  const size_t n = size_t(lx) * ly * lz;
  const std::vector<std::string> t = tokens(s);
  if (t.size() != n)
    return fslbm_set_error(FSLBM_ERR_IO, "read_pipe_txt: %s holds %zu values, expected %zu (%dx%dx%d)",
                           path, t.size(), n, lx, ly, lz);
  for (size_t i = 0; i < n; ++i) {
    int v;
    if (!parse_int(t[i], &v) || v < 0 || v > 255)
      return fslbm_set_error(FSLBM_ERR_IO, "read_pipe_txt: value %zu ('%s') is not a byte", i, t[i].c_str());
    out[i] = uint8_t(v);
  }
  return FSLBM_OK;
}

extern "C" int fslbm_write_pipe_txt(const char* path, int lx, int ly, int lz, const uint8_t* mask) {
  if (!path || !mask) return fslbm_set_error(FSLBM_ERR_ARG, "write_pipe_txt: bad argument");
  FILE* f = std::fopen(path, "w");
  if (!f) return fslbm_set_error(FSLBM_ERR_IO, "write_pipe_txt: cannot create %s", path);
  const size_t n = size_t(lx) * ly * lz;
  for (size_t i = 0; i < n; ++i) std::fprintf(f, "%d\n", int(mask[i]));   // pipe.m:62
  std::fclose(f);
  return FSLBM_OK;
}

extern "C" int fslbm_read_param_txt(const char* path, fslbm_params* prm) {
  if (!path || !prm) return fslbm_set_error(FSLBM_ERR_ARG, "read_param_txt: bad argument");
  std::string s;
  if (!read_file(path, s)) return fslbm_set_error(FSLBM_ERR_IO, "read_param_txt: cannot open %s", path);
  const std::vector<std::string> t = tokens(s);
  // FSLBM.cu:502-507: %e tblend, %e pin, %e nu, %d d1, %d delta, %e blend; trailing lines
  // (the unused save path, :508) are ignored. Floats are read into FP32 as the reference does.
  const int nval = int(std::min<size_t>(t.size(), 6));
  fslbm_params p = *prm;
  for (int k = 0; k < nval; ++k) {
    if (k == 3 || k == 4) {
      int v;
      if (!parse_int(t[k], &v))
        return fslbm_set_error(FSLBM_ERR_IO, "read_param_txt: line %d ('%s') is not an integer", k + 1, t[k].c_str());
      (k == 3 ? p.d1 : p.delta) = v;
    } else {
      double v;
      if (!parse_double(t[k], &v))
        return fslbm_set_error(FSLBM_ERR_IO, "read_param_txt: line %d ('%s') is not a number", k + 1, t[k].c_str());
      const double f = double(float(v));
      if (k == 0) p.tblend = f;
      else if (k == 1) p.pin = f;
      else if (k == 2) p.nu = f;
      else p.blend = f;
    }
  }
  if (nval < 6) return fslbm_set_error(FSLBM_ERR_IO, "read_param_txt: %s holds %d of 6 values", path, nval);
  *prm = p;
  return FSLBM_OK;
}

extern "C" int fslbm_write_param_txt(const char* path, const fslbm_params* prm) {
  if (!path || !prm) return fslbm_set_error(FSLBM_ERR_ARG, "write_param_txt: bad argument");
  FILE* f = std::fopen(path, "w");
  if (!f) return fslbm_set_error(FSLBM_ERR_IO, "write_param_txt: cannot create %s", path);
  // pipe.m:67-68 writes '%f\n%f\n%f\n%d\n%d\n' and recycles '%f\n' for the sixth value
  std::fprintf(f, "%f\n%f\n%f\n%d\n%d\n%f\n", prm->tblend, prm->pin, prm->nu, prm->d1, prm->delta,
               prm->blend);
  std::fclose(f);
  return FSLBM_OK;
}

extern "C" int fslbm_pipe_m_mask(int lx0, int l0, int d, uint8_t* out) {
  if (!out || lx0 < 1 || l0 < 1 || d < 0) return fslbm_set_error(FSLBM_ERR_ARG, "pipe_m_mask: bad argument");
  // pipe.m:38-60. MATLAB indices are 1-based: cell (i,j) of the lx0 x lx0 block is fluid when
  // (i-o)^2 + (j-o)^2 <= r^2 with o = r = lx0/2; planes 1..d and l-d+1..l mark fluid as 1.
  const int lx = lx0 + 2 * d, lz = l0 + 2 * d;
  const double o = lx0 / 2.0;
  for (int k = 0; k < lz; ++k) {
    const bool buffer = k < d || k >= lz - d;
    for (int j = 0; j < lx; ++j)
      for (int i = 0; i < lx; ++i) {
        const int ii = i - d + 1, jj = j - d + 1;   // 1-based inside the unpadded block
        uint8_t v = kWall;
        if (ii >= 1 && ii <= lx0 && jj >= 1 && jj <= lx0 &&
            (ii - o) * (ii - o) + (jj - o) * (jj - o) <= o * o)
          v = buffer ? kBuf : 0;
        out[size_t(i) + size_t(lx) * (j + size_t(lx) * k)] = v;
      }
  }
  return FSLBM_OK;
}

extern "C" int fslbm_ref_mask_to_core(const uint8_t* m, int lx, int ly, int lz_ref, int d2,
                                      uint8_t* core) {
  if (!m || !core || lx < 3 || ly < 3 || d2 < 1 || lz_ref <= 2 * d2)
    return fslbm_set_error(FSLBM_ERR_ARG, "ref_mask_to_core: bad argument");
  const size_t plane = size_t(lx) * ly;
  const int L = lz_ref - 2 * d2;
  if (L < d2)
    return fslbm_set_error(FSLBM_ERR_ARG, "ref_mask_to_core: %d fluid planes shorter than the buffer depth %d", L, d2);
  for (size_t j = 0; j < plane; ++j) {
    const uint8_t v = m[plane * d2 + j];
    if (v != 0 && v != kWall)
      return fslbm_set_error(FSLBM_ERR_ARG, "ref_mask_to_core: value %d in the first fluid plane", int(v));
    const int x = int(j % lx), y = int(j / lx);
    if (v == 0 && (x == 0 || y == 0 || x == lx - 1 || y == ly - 1))
      return fslbm_set_error(FSLBM_ERR_ARG, "ref_mask_to_core: fluid cell (%d,%d) on the box rim", x, y);
    core[j] = v;
  }
  for (int z = 0; z < lz_ref; ++z) {
    const bool buffer = z < d2 || z >= lz_ref - d2;
    for (size_t j = 0; j < plane; ++j) {
      const uint8_t v = m[plane * z + j];
      const uint8_t want = core[j] == kWall ? kWall : (buffer ? kBuf : uint8_t(0));
      if (v != want)
        return fslbm_set_error(FSLBM_ERR_ARG,
                               "ref_mask_to_core: plane %d cell %zu is %d, expected %d (the periodic core "
                               "needs identical planes and buffers that copy them)",
                               z, j, int(v), int(want));
    }
  }
  return FSLBM_OK;
}

extern "C" int fslbm_ref_mask_to_core3d(const uint8_t* m, int lx, int ly, int lz_ref, int d2,
                                        uint8_t* core) {
  if (!m || !core || lx < 3 || ly < 3 || d2 < 1 || lz_ref <= 2 * d2)
    return fslbm_set_error(FSLBM_ERR_ARG, "ref_mask_to_core3d: bad argument");
  const size_t plane = size_t(lx) * ly;
  const int L = lz_ref - 2 * d2;
  if (L < d2)
    return fslbm_set_error(FSLBM_ERR_ARG, "ref_mask_to_core3d: %d fluid planes shorter than the buffer depth %d", L, d2);
  for (int zc = 0; zc < L; ++zc)
    for (size_t j = 0; j < plane; ++j) {
      const uint8_t v = m[plane * (zc + d2) + j];
      if (v != 0 && v != kWall)
        return fslbm_set_error(FSLBM_ERR_ARG, "ref_mask_to_core3d: value %d in fluid plane %d", int(v), zc + d2);
      const int x = int(j % lx), y = int(j / lx);
      if (v == 0 && (x == 0 || y == 0 || x == lx - 1 || y == ly - 1))
        return fslbm_set_error(FSLBM_ERR_ARG, "ref_mask_to_core3d: fluid cell (%d,%d,%d) on the box rim", x, y,
                               zc + d2);
      core[plane * zc + j] = v;
    }
  // buffer planes must be the wrapped core planes (fluid marked 1), as bcond copies them
  for (int z = 0; z < lz_ref; ++z) {
    if (z >= d2 && z < lz_ref - d2) continue;
    const int zc = z < d2 ? z - d2 + L : z - d2 - L;
    for (size_t j = 0; j < plane; ++j) {
      const uint8_t want = core[plane * zc + j] == kWall ? kWall : kBuf;
      if (m[plane * z + j] != want)
        return fslbm_set_error(FSLBM_ERR_ARG,
                               "ref_mask_to_core3d: buffer plane %d cell %zu is %d, expected %d (a copy of "
                               "core plane %d)", z, j, int(m[plane * z + j]), int(want), zc);
    }
  }
  return FSLBM_OK;
}

// Geometry of the seeded start (shared by the host and device generators): fluid cells from the
// mask or the circle; for a mask (or no radius) the centre is the fluid centroid and R the
// largest centre distance plus half a cell.
int fslbm_poiseuille_setup(const fslbm_domain* dom, double umax, double noise, int modes,
                           double mode_amp, uint64_t seed, fslbm::PoiseuilleInit* q,
                           std::vector<uint8_t>* fluid_out) {
  if (!dom || dom->lx < 1 || dom->ly < 1 || dom->lz < 1 || modes < 0 || modes > fslbm::kMaxInitModes)
    return fslbm_set_error(FSLBM_ERR_ARG, "init_poiseuille: bad argument (modes <= %d)", fslbm::kMaxInitModes);
  const int lx = dom->lx, ly = dom->ly;
  const size_t plane = size_t(lx) * ly;
  std::vector<uint8_t>& fluid = *fluid_out;
  fluid.assign(plane, 0);
  double R = dom->radius, cx = dom->cx, cy = dom->cy;
  size_t nf = 0;
  double sx = 0, sy = 0;
  for (size_t j = 0; j < plane; ++j) {
    const int x = int(j % lx), y = int(j / lx);
    bool f;
    if (dom->mask) f = dom->mask[j] == 0;
    else f = (x - cx) * (x - cx) + (y - cy) * (y - cy) <= R * R;
    fluid[j] = f;
    if (f) { ++nf; sx += x; sy += y; }
  }
  if (!nf) return fslbm_set_error(FSLBM_ERR_ARG, "init_poiseuille: no fluid cells");
  if (dom->mask || R <= 0) {
    cx = sx / double(nf); cy = sy / double(nf);
    double r2max = 0;
    for (size_t j = 0; j < plane; ++j)
      if (fluid[j]) {
        const double dx = int(j % lx) - cx, dy = int(j / lx) - cy;
        r2max = std::fmax(r2max, dx * dx + dy * dy);
      }
    R = std::sqrt(r2max) + 0.5;
  }
  std::memset(q, 0, sizeof *q);
  q->cx = cx; q->cy = cy; q->R = R; q->umax = umax; q->noise = noise; q->mode_amp = mode_amp;
  q->seed = seed; q->lx = lx; q->ly = ly; q->L = dom->lz; q->modes = modes;
  fslbm::poiseuille_phases(*q);
  return FSLBM_OK;
}

extern "C" int fslbm_init_poiseuille(const fslbm_domain* dom, double umax, double noise, int modes,
                                     double mode_amp, uint64_t seed, double* p, double* u, double* v,
                                     double* w) {
  if (!p || !u || !v || !w) return fslbm_set_error(FSLBM_ERR_ARG, "init_poiseuille: null output");
  fslbm::PoiseuilleInit q;
  std::vector<uint8_t> fluid;
  if (int r = fslbm_poiseuille_setup(dom, umax, noise, modes, mode_amp, seed, &q, &fluid)) return r;
  const size_t plane = size_t(q.lx) * q.ly;
  for (int z = 0; z < q.L; ++z)
    for (size_t j = 0; j < plane; ++j) {
      const size_t idx = size_t(z) * plane + j;
      if (!fluid[j]) { p[idx] = u[idx] = v[idx] = w[idx] = 0.0; continue; }
      double c[4];
      fslbm::poiseuille_cell(q, int(j % q.lx), int(j / q.lx), z, c);
      p[idx] = c[0]; u[idx] = c[1]; v[idx] = c[2]; w[idx] = c[3];
    }
  return FSLBM_OK;
}
