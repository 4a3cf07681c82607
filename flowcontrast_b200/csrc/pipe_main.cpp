// fslbm_pipe: the drop-in executable. It reads and writes the reference's working-directory files
// (PipeDemoStandalone/FSLBM.cu main, FSLBM.cu:489-905) and runs the time loop on the C ABI.
//
//   inputs   pipe.txt (mask, pipe.m:62), param.txt (FSLBM.cu:499-510), restart set
//            p3Dii ux3Dii uy3Dii uz3Dii qpii.txt (FSLBM.cu:386-427) and
//            _pii.txt ... _uyz2ii.txt _avii.txt (FSLBM.cu:429-468)
//   outputs  qp.txt every 50 steps (FSLBM.cu:663); every 500 steps param.txt is re-read
//            (FSLBM.cu:669-677) and _p.txt ... _uyz2.txt _av.txt (FSLBM.cu:679-768), p.txt
//            ux.txt uy.txt uz.txt IO.txt ux1.txt uy1.txt uz1.txt p1.txt (FSLBM.cu:771-821) are
//            written; every 50000 steps the restart set (FSLBM.cu:825-904).
// The reference box is lx x ly x lz with d2 buffer planes at each streamwise end; its time loop
// runs without end (5e8 steps); here --steps bounds it. Files are validated before the GPU is
// touched.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fslbm.h"

namespace {

struct Options {
  int lx = 120, ly = 120, lz = 320, d2 = 10;
  double radius = 50.0;
  long long steps = 500000000LL;
  int monitor = 50, dump = 500, backup = 50000;
  int dtype = FSLBM_F32, device = 0;
  std::string dir = ".";
  std::string init = "auto";   // auto | restart | initphys
  bool quiet = false;
};

void usage() {
  std::fprintf(stderr,
               "usage: fslbm_pipe [--steps N] [--lx 120] [--ly 120] [--lz 320] [--d2 10]\n"
               "                  [--radius 50] [--dtype f32|f64|f16] [--device 0] [--dir .]\n"
               "                  [--init auto|restart|initphys] [--monitor 50] [--dump 500]\n"
               "                  [--backup 50000] [--quiet]\n");
}

bool parse(int argc, char** argv, Options& o) {
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&](const char* name) -> const char* {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "fslbm_pipe: %s needs a value\n", name);
        return nullptr;
      }
      return argv[++i];
    };
    const char* v = nullptr;
    if (a == "--quiet") { o.quiet = true; continue; }
    if (a == "--help" || a == "-h") return false;
    if (!(v = val(a.c_str()))) return false;
    if (a == "--steps") o.steps = std::atoll(v);
    else if (a == "--lx") o.lx = std::atoi(v);
    else if (a == "--ly") o.ly = std::atoi(v);
    else if (a == "--lz") o.lz = std::atoi(v);
    else if (a == "--d2") o.d2 = std::atoi(v);
    else if (a == "--radius") o.radius = std::atof(v);
    else if (a == "--device") o.device = std::atoi(v);
    else if (a == "--dir") o.dir = v;
    else if (a == "--init") o.init = v;
    else if (a == "--monitor") o.monitor = std::atoi(v);
    else if (a == "--dump") o.dump = std::atoi(v);
    else if (a == "--backup") o.backup = std::atoi(v);
    else if (a == "--dtype") {
      const std::string d = v;
      o.dtype = d == "f64" ? FSLBM_F64 : d == "f16" ? FSLBM_F16 : d == "f32" ? FSLBM_F32 : -1;
      if (o.dtype < 0) { std::fprintf(stderr, "fslbm_pipe: unknown dtype %s\n", v); return false; }
    } else {
      std::fprintf(stderr, "fslbm_pipe: unknown option %s\n", a.c_str());
      return false;
    }
  }
  if (o.lx < 3 || o.ly < 3 || o.lz <= 2 * o.d2 || o.d2 < 0 || o.steps < 0 || o.monitor <= 0 ||
      o.dump <= 0 || o.backup <= 0 || (o.init != "auto" && o.init != "restart" && o.init != "initphys")) {
    std::fprintf(stderr, "fslbm_pipe: invalid sizes, intervals or --init\n");
    return false;
  }
  return true;
}

std::string path(const Options& o, const char* name) { return o.dir + "/" + name; }

bool exists(const std::string& p) {
  FILE* f = std::fopen(p.c_str(), "rb");
  if (!f) return false;
  std::fclose(f);
  return true;
}

int fail(const char* what) {
  char msg[1024];
  fslbm_last_error(msg, sizeof msg);
  std::fprintf(stderr, "fslbm_pipe: %s: %s\n", what, msg);
  return 1;
}

// Text dump, one "%e" value per line (FSLBM.cu:759-769, 784-814).
template <class T>
bool write_lines(const std::string& p, const T* v, size_t n, double scale = 1.0) {
  FILE* f = std::fopen(p.c_str(), "wt");
  if (!f) return false;
  for (size_t k = 0; k < n; ++k) std::fprintf(f, "%e\n", double(v[k]) * scale);
  return std::fclose(f) == 0;
}

bool copy_text(const std::string& from, const std::string& to) {
  FILE* a = std::fopen(from.c_str(), "rb");
  if (!a) return false;
  FILE* b = std::fopen(to.c_str(), "wb");
  if (!b) { std::fclose(a); return false; }
  char buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, a)) > 0) std::fwrite(buf, 1, n, b);
  std::fclose(a);
  return std::fclose(b) == 0;
}

// Raw FP32 file of lx*ly*lz values, x fastest (p3Dii etc., FSLBM.cu:395-422, 832-856).
bool read_raw(const std::string& p, std::vector<float>& v) {
  FILE* f = std::fopen(p.c_str(), "rb");
  if (!f) return false;
  const size_t got = std::fread(v.data(), sizeof(float), v.size(), f);
  const bool extra = std::fgetc(f) != EOF;
  std::fclose(f);
  return got == v.size() && !extra;
}

bool write_raw(const std::string& p, const std::vector<float>& v) {
  FILE* f = std::fopen(p.c_str(), "wb");
  if (!f) return false;
  const size_t put = std::fwrite(v.data(), sizeof(float), v.size(), f);
  return std::fclose(f) == 0 && put == v.size();
}

const char* kStatNames[11] = {"_p", "_ux", "_uy", "_uz", "_p2", "_ux2", "_uy2", "_uz2",
                              "_uxy2", "_uxz2", "_uyz2"};

// The 11 averaged statistics files and the counts file, with `suffix` "" or "ii".
bool write_stats(const Options& o, const std::vector<double>& means, int cnt, int cnt2,
                 const char* suffix) {
  const size_t n = size_t(o.ly) * o.lz;
  for (int k = 0; k < 11; ++k) {
    const std::string name = std::string(kStatNames[k]) + suffix + ".txt";
    if (!write_lines(path(o, name.c_str()), means.data() + k * n, n)) return false;
  }
  const std::string av = std::string("_av") + suffix + ".txt";
  FILE* f = std::fopen(path(o, av.c_str()).c_str(), "wt");
  if (!f) return false;
  std::fprintf(f, "%d %d\n", cnt, cnt2);
  return std::fclose(f) == 0;
}

bool read_stats(const Options& o, std::vector<double>& means, int& cnt, int& cnt2) {
  FILE* f = std::fopen(path(o, "_avii.txt").c_str(), "rt");
  if (!f) return false;
  const bool ok = std::fscanf(f, "%d %d", &cnt, &cnt2) == 2;
  std::fclose(f);
  if (!ok) return false;
  const size_t n = size_t(o.ly) * o.lz;
  means.assign(11 * n, 0.0);
  for (int k = 0; k < 11; ++k) {
    const std::string name = std::string(kStatNames[k]) + "ii.txt";
    FILE* g = std::fopen(path(o, name.c_str()).c_str(), "rt");
    if (!g) return false;
    for (size_t j = 0; j < n; ++j) {
      float t;   // the reference reads each value as a float (FSLBM.cu:454-465)
      if (std::fscanf(g, "%e", &t) != 1) { std::fclose(g); return false; }
      means[k * n + j] = double(t);
    }
    std::fclose(g);
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  if (!parse(argc, argv, o)) {
    usage();
    return 2;
  }
  const size_t cells_ref = size_t(o.lx) * o.ly * o.lz;
  const int L = o.lz - 2 * o.d2;

  // ---- inputs, validated before the GPU is used
  fslbm_params prm{};
  prm.tblend = 1.0; prm.pin = 0.003; prm.nu = 0.004006; prm.d1 = 2; prm.delta = 0; prm.blend = 0.0;
  prm.monitor_every = o.monitor;
  if (fslbm_read_param_txt(path(o, "param.txt").c_str(), &prm)) return fail("param.txt");
  std::vector<uint8_t> mask3d(cells_ref);
  if (fslbm_read_pipe_txt(path(o, "pipe.txt").c_str(), o.lx, o.ly, o.lz, mask3d.data()))
    return fail("pipe.txt");
  // one cross-section extruded along the pipe if every plane has it, else one per plane
  std::vector<uint8_t> core(size_t(o.lx) * o.ly);
  int mask_planes = 1;
  if (fslbm_ref_mask_to_core(mask3d.data(), o.lx, o.ly, o.lz, o.d2, core.data())) {
    core.assign(size_t(o.lx) * o.ly * L, 0);
    if (fslbm_ref_mask_to_core3d(mask3d.data(), o.lx, o.ly, o.lz, o.d2, core.data()))
      return fail("pipe.txt geometry");
    mask_planes = L;
  }
  const bool have_restart = exists(path(o, "p3Dii"));
  if (o.init == "restart" && !have_restart) {
    std::fprintf(stderr, "fslbm_pipe: --init restart but %s is missing\n", path(o, "p3Dii").c_str());
    return 1;
  }
  const bool restart = o.init == "restart" || (o.init == "auto" && have_restart);
  std::vector<float> f[4];
  for (auto& a : f) a.assign(cells_ref, 0.0f);
  if (restart) {
    const char* names[4] = {"p3Dii", "ux3Dii", "uy3Dii", "uz3Dii"};
    for (int k = 0; k < 4; ++k)
      if (!read_raw(path(o, names[k]), f[k])) {
        std::fprintf(stderr, "fslbm_pipe: %s is missing or not %zu floats\n", names[k], cells_ref);
        return 1;
      }
  } else {
    // initphys (FSLBM.cu:374-383): p falls linearly from pin at the inlet, u = 0
    for (int z = 0; z < o.lz; ++z)
      for (size_t j = 0; j < size_t(o.lx) * o.ly; ++j)
        f[0][size_t(z) * o.lx * o.ly + j] = float(prm.pin) * float(o.lz - o.d2 - z) / float(L);
  }
  std::vector<double> means;
  int cnt = 0, cnt2 = 0;
  const bool have_stats = restart && read_stats(o, means, cnt, cnt2);

  // ---- solve
  fslbm_ctx* ctx = nullptr;
  if (fslbm_ctx_create(o.device, &ctx)) return fail("device");
  fslbm_domain dom{};
  dom.lx = o.lx; dom.ly = o.ly; dom.lz = L; dom.mask = core.data(); dom.radius = o.radius;
  dom.buffer_depth = o.d2;
  dom.mask_planes = mask_planes;
  fslbm_solve* s = nullptr;
  if (fslbm_solve_create(ctx, &dom, &prm, fslbm_dtype(o.dtype), &s)) return fail("solve");
  if (fslbm_solve_set_fields_ref(s, f[0].data(), f[1].data(), f[2].data(), f[3].data()))
    return fail("initial fields");
  if (have_stats && fslbm_stats_set(s, means.data(), cnt, cnt2)) return fail("statistics restart");
  if (restart && exists(path(o, "qpii.txt"))) copy_text(path(o, "qpii.txt"), path(o, "qp.txt"));
  { FILE* q = std::fopen(path(o, "qp.txt").c_str(), "a"); if (q) std::fclose(q); }
  if (!o.quiet)
    std::printf("fslbm_pipe: %dx%dx%d (core %d planes), %s start, %s\n", o.lx, o.ly, o.lz, L,
                restart ? "restart" : "initphys",
                o.dtype == FSLBM_F64 ? "FP64" : o.dtype == FSLBM_F16 ? "FP16 storage" : "FP32");

  const size_t nyz = size_t(o.ly) * o.lz, nxy = size_t(o.lx) * o.ly;
  std::vector<float> plane(std::max(nyz, nxy));
  std::vector<double> stats(11 * nyz);
  long long c = 0;
  while (c < o.steps) {
    const long long next = std::min(o.steps, (c / o.monitor + 1) * o.monitor);
    if (fslbm_solve_step(s, next - c)) return fail("step");
    c = next;
    if (c % o.monitor) continue;
    fslbm_monitor m;
    if (fslbm_solve_monitor(s, &m)) return fail("monitor");
    if (!o.quiet)
      std::printf("time step: %lld, dtddy: %e, q1=%e, q2=%e, p1 =%e, p2=%e, f.f.=%e, Re=%e\n", c,
                  float(prm.nu) - 0.16666666f, m.q1, m.q2, m.p1, m.p2, m.f, m.re);
    FILE* q = std::fopen(path(o, "qp.txt").c_str(), "a");
    if (!q) return fail("qp.txt");
    std::fprintf(q, "%e %e %e %e %e %e\n", m.q1, m.q2, m.p1, m.p2, m.f, m.sample);
    std::fclose(q);
    if (c % o.dump == 0) {
      // live parameters (FSLBM.cu:669-677), then the statistics with the new delta policy
      fslbm_params np = prm;
      if (fslbm_read_param_txt(path(o, "param.txt").c_str(), &np) == FSLBM_OK) {
        np.monitor_every = o.monitor;
        if (fslbm_solve_set_params(s, &np) == FSLBM_OK) prm = np;
        else std::fprintf(stderr, "fslbm_pipe: param.txt change rejected, keeping the old values\n");
      }
      if (fslbm_stats_sample(s) || fslbm_stats_get(s, stats.data(), &cnt, &cnt2)) return fail("statistics");
      if (!write_stats(o, stats, cnt, cnt2, "")) return fail("statistics files");
      const char* yz[4] = {"p.txt", "ux.txt", "uy.txt", "uz.txt"};
      for (int k = 0; k < 4; ++k) {
        if (fslbm_solve_get_plane(s, 0, k, plane.data())) return fail("plane");
        if (!write_lines(path(o, yz[k]), plane.data(), nyz)) return fail(yz[k]);
      }
      const char* xy[4] = {"p1.txt", "ux1.txt", "uy1.txt", "uz1.txt"};
      for (int k = 0; k < 4; ++k) {
        if (fslbm_solve_get_plane(s, 1, k, plane.data())) return fail("plane");
        if (!write_lines(path(o, xy[k]), plane.data(), nxy)) return fail(xy[k]);
      }
      FILE* io = std::fopen(path(o, "IO.txt").c_str(), "wt");   // mask, YZ plane x = lx/2
      if (!io) return fail("IO.txt");
      for (int z = 0; z < o.lz; ++z)
        for (int y = 0; y < o.ly; ++y)
          std::fprintf(io, "%d\n", int(mask3d[(size_t(z) * o.ly + y) * o.lx + o.lx / 2]));
      std::fclose(io);
    }
    if (c % o.backup == 0) {
      if (fslbm_solve_get_fields_ref(s, f[0].data(), f[1].data(), f[2].data(), f[3].data()))
        return fail("backup fields");
      const char* names[4] = {"p3Dii", "ux3Dii", "uy3Dii", "uz3Dii"};
      for (int k = 0; k < 4; ++k)
        if (!write_raw(path(o, names[k]), f[k])) return fail(names[k]);
      copy_text(path(o, "qp.txt"), path(o, "qpii.txt"));
      if (fslbm_stats_get(s, stats.data(), &cnt, &cnt2)) return fail("statistics");
      if (!write_stats(o, stats, cnt, cnt2, "ii")) return fail("statistics backup");
    }
  }
  fslbm_solve_destroy(s);
  fslbm_ctx_destroy(ctx);
  return 0;
}
