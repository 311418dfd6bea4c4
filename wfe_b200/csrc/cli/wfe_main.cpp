// wfe: the reference's driver (src/main.cpp) on top of the wfe_b200 C ABI.
//
//   wfe case.ini [key=value ...] [--fp64] [--device N]
//
// Reads the case and its command-line overrides, steps it to t_end and writes
// what the reference writes: <out_dir>/meta.json, zc.bin, run_info.txt and the
// float32 interior snapshots <var>_<step>.bin every out_interval
// (src/io/writer.cpp:12-107), prints the diagnostics line every
// diag_interval and the closing "bitti:" line in the reference's formats
// (src/main.cpp:440-472; tools/run_tests.py parses them), and exits 2 on a
// non-finite state, 3 when |w| exceeds w_abort (the every-10-steps watchdog,
// main.cpp:429-439).  Between those events the steps replay captured CUDA
// graphs (wfe_run).  Only include/wfe_b200.h is used.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "wfe_b200.h"

namespace {

struct Run {
  wfe_ctx* c = nullptr;
  int nx = 0, ny = 0, nz = 0, ng = 3, NX = 0, NY = 0, NZ = 0;
  double dx = 0, dy = 0, dz = 0, dt = 0, t_end = 0, zt = 0;
  int moisture = 0, physics = 0;
  std::string dir;
};

int fail(const Run& r, const char* what) {
  std::fprintf(stderr, "%s: %s\n", what, wfe_last_error(r.c));
  return 1;
}

void mkdirs(const std::string& d) {
  std::string cur;
  for (size_t q = 0; q < d.size(); ++q) {
    cur += d[q];
    if (d[q] == '/' || q + 1 == d.size()) mkdir(cur.c_str(), 0755);
  }
}

bool write_file(const std::string& path, const void* data, size_t bytes) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(data, 1, bytes, f) == bytes;
  std::fclose(f);
  return ok;
}

std::string snap_name(const Run& r, const char* var, int step) {
  char b[64];
  std::snprintf(b, sizeof(b), "/%s_%06d.bin", var, step);
  return r.dir + b;
}

// Writer::write / write_field2d: the interior blocks as float32
int write_snapshot(const Run& r, int step, double t) {
  static const char* names[8] = {"u", "v", "w", "thp", "pip", "qv", "qc", "qr"};
  std::vector<float> buf((size_t)r.nx * r.ny * (r.nz + 1));
  const int nf = r.moisture ? 8 : 5;
  for (int f = 0; f < nf; ++f) {
    if (wfe_field_download(r.c, WFE_ROLE_STATE, f, buf.data(), WFE_DTYPE_F32, WFE_LAYOUT_INTERIOR))
      return fail(r, "download");
    size_t n = (size_t)r.nx * r.ny * (f == WFE_W ? r.nz + 1 : r.nz);
    if (!write_file(snap_name(r, names[f], step), buf.data(), n * sizeof(float))) {
      std::fprintf(stderr, "cannot write %s\n", snap_name(r, names[f], step).c_str());
      return 1;
    }
  }
  std::printf("  cikti yazildi: step %d (t = %.1f s)\n", step, t);
  struct F2 {
    int which;
    const char* name;
    bool on;
  } f2[5] = {{WFE_2D_RAIN, "rain", r.moisture != 0}, {WFE_2D_TSK, "tsk", r.physics != 0},
             {WFE_2D_PBLH, "pblh", r.physics != 0}, {WFE_2D_T2M, "t2m", r.physics != 0},
             {WFE_2D_U10, "u10", r.physics != 0}};
  std::vector<float> b2((size_t)r.nx * r.ny);
  for (const F2& q : f2) {
    if (!q.on) continue;
    if (wfe_field2d_download(r.c, q.which, b2.data(), WFE_DTYPE_F32, WFE_LAYOUT_INTERIOR))
      return fail(r, "download");
    if (!write_file(snap_name(r, q.name, step), b2.data(), b2.size() * sizeof(float))) return 1;
  }
  return 0;
}

struct Diag {
  double wmax = 0, thmin = 0, thmax = 0, pipmax = 0, qcmax = 0, qrmax = 0;
  bool finite = true;
};

// diagnose (src/main.cpp:202-240)
int diagnose(const Run& r, Diag* d) {
  std::vector<double> b((size_t)r.NX * r.NY * r.NZ);
  auto at = [&](int i, int j, int k) {
    return b[((size_t)(k + r.ng) * r.NY + (j + r.ng)) * r.NX + (i + r.ng)];
  };
  auto get = [&](int f) {
    return wfe_field_download(r.c, WFE_ROLE_STATE, f, b.data(), WFE_DTYPE_F64, WFE_LAYOUT_PADDED);
  };
  if (get(WFE_W)) return fail(r, "download");
  for (int k = 0; k <= r.nz; ++k)
    for (int j = 0; j < r.ny; ++j)
      for (int i = 0; i < r.nx; ++i) {
        double v = at(i, j, k);
        if (!std::isfinite(v)) d->finite = false;
        if (std::fabs(v) > d->wmax) d->wmax = std::fabs(v);
      }
  if (get(WFE_THP)) return fail(r, "download");
  for (int k = 0; k < r.nz; ++k)
    for (int j = 0; j < r.ny; ++j)
      for (int i = 0; i < r.nx; ++i) {
        double v = at(i, j, k);
        if (!std::isfinite(v)) d->finite = false;
        if (v < d->thmin) d->thmin = v;
        if (v > d->thmax) d->thmax = v;
      }
  if (get(WFE_PIP)) return fail(r, "download");
  for (int k = 0; k < r.nz; ++k)
    for (int j = 0; j < r.ny; ++j)
      for (int i = 0; i < r.nx; ++i) {
        double v = std::fabs(at(i, j, k));
        if (!std::isfinite(v)) d->finite = false;
        if (v > d->pipmax) d->pipmax = v;
      }
  if (r.moisture) {
    if (get(WFE_QC)) return fail(r, "download");
    for (double v : b)
      if (v > d->qcmax) d->qcmax = v;
    if (get(WFE_QR)) return fail(r, "download");
    for (double v : b) {
      if (!std::isfinite(v)) d->finite = false;
      if (v > d->qrmax) d->qrmax = v;
    }
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  std::string ini = argc > 1 ? argv[1] : "cases/warm_bubble.ini";
  std::vector<const char*> ov;
  int precision = WFE_F32, device = 0;
  for (int a = 2; a < argc; ++a) {
    if (!std::strcmp(argv[a], "--fp64")) precision = WFE_F64;
    else if (!std::strcmp(argv[a], "--device") && a + 1 < argc) device = std::atoi(argv[++a]);
    else if (std::strchr(argv[a], '=')) ov.push_back(argv[a]);
  }
  Run r;
  if (wfe_case_create(ini.c_str(), ov.data(), (int)ov.size(), precision, device, &r.c) != WFE_OK) {
    std::fprintf(stderr, "%s\n", wfe_last_error(nullptr));
    return 1;
  }
  int dims[7];
  double sp[6], rc3[3];
  int fl[10];
  char odir[1024];
  wfe_get_dims(r.c, dims);
  wfe_get_spacing(r.c, sp);
  wfe_get_flags(r.c, fl);
  wfe_get_run_config(r.c, rc3, odir, sizeof(odir));
  r.nx = dims[0], r.ny = dims[1], r.nz = dims[2], r.ng = dims[3], r.NX = dims[4], r.NY = dims[5],
  r.NZ = dims[6];
  r.dx = sp[0], r.dy = sp[1], r.dz = sp[2], r.dt = sp[3], r.t_end = sp[4], r.zt = sp[5];
  r.moisture = fl[0];
  r.physics = fl[7];
  r.dir = odir;
  const double out_every = rc3[0], diag_every = rc3[1], w_abort = rc3[2];
  mkdirs(r.dir);
  {  // Writer::init: meta.json
    FILE* f = std::fopen((r.dir + "/meta.json").c_str(), "w");
    if (!f) {
      std::fprintf(stderr, "cannot write %s/meta.json\n", r.dir.c_str());
      return 1;
    }
    std::fprintf(f,
                 "{\n  \"nx\": %d, \"ny\": %d, \"nz\": %d,\n  \"dx\": %g, \"dy\": %g, \"dz\": %g,\n"
                 "  \"dt\": %g,\n  \"vars\": {\"u\": %d, \"v\": %d, \"w\": %d, \"thp\": %d, \"pip\": %d",
                 r.nx, r.ny, r.nz, r.dx, r.dy, r.dz, r.dt, r.nz, r.nz, r.nz + 1, r.nz, r.nz);
    if (r.moisture)
      std::fprintf(f, ", \"qv\": %d, \"qc\": %d, \"qr\": %d, \"rain\": 1", r.nz, r.nz, r.nz);
    if (r.physics) std::fprintf(f, ", \"tsk\": 1, \"pblh\": 1, \"t2m\": 1, \"u10\": 1");
    std::fprintf(f, "}\n}\n");
    std::fclose(f);
  }
  {  // physical heights of the cell centres (zc.bin, main.cpp:387-395)
    std::vector<double> zc(r.NZ), h((size_t)r.NX * r.NY);
    wfe_get_metric(r.c, 1, zc.data());
    wfe_get_metric(r.c, 4, h.data());
    std::vector<float> z((size_t)r.nx * r.ny * r.nz);
    size_t o = 0;
    for (int k = 0; k < r.nz; ++k)
      for (int j = 0; j < r.ny; ++j)
        for (int i = 0; i < r.nx; ++i) {
          double hh = h[(size_t)(j + r.ng) * r.NX + (i + r.ng)];
          z[o++] = (float)(hh + zc[k + r.ng] * (r.zt - hh) / r.zt);
        }
    write_file(r.dir + "/zc.bin", z.data(), z.size() * sizeof(float));
    FILE* f = std::fopen((r.dir + "/run_info.txt").c_str(), "w");
    if (f) {
      std::fprintf(f, "engine = wfe_b200 (sm_100a)\nprecision = %s\ncase = %s\n",
                   precision == WFE_F64 ? "fp64" : "fp32", ini.c_str());
      for (const char* o2 : ov) std::fprintf(f, "%s\n", o2);
      std::fclose(f);
    }
  }
  if (write_snapshot(r, 0, 0.0)) return 1;

  const int nsteps = (int)std::ceil(r.t_end / r.dt);
  const int diag_steps = std::max(1, (int)std::round(diag_every / r.dt));
  const int out_steps = std::max(1, (int)std::round(out_every / r.dt));
  auto t0 = std::chrono::steady_clock::now();
  int step = 0;
  while (step < nsteps) {
    // replay up to the next watchdog, diagnostic or output step
    int next = std::min(nsteps, (step / 10 + 1) * 10);
    next = std::min(next, (step / diag_steps + 1) * diag_steps);
    next = std::min(next, (step / out_steps + 1) * out_steps);
    if (wfe_run(r.c, next - step, r.dt, step * r.dt) != WFE_OK) return fail(r, "step");
    step = next;
    const double t = step * r.dt;
    if (step % 10 == 0) {
      float wm = 0;
      if (wfe_absmax(r.c, WFE_W, &wm)) return fail(r, "watchdog");
      if (!std::isfinite(wm) || wm > (float)w_abort) {
        std::fprintf(stderr,
                     "HATA: |w|max=%.1f m/s esigi asti (adim %d, t=%.0fs) -- "
                     "acil cikti yazilip durduruluyor\n",
                     wm, step, t);
        write_snapshot(r, step, t);
        return 3;
      }
    }
    if (step % diag_steps == 0 || step == nsteps) {
      Diag d;
      if (diagnose(r, &d)) return 1;
      if (r.moisture)
        std::printf("adim %6d  t=%7.1fs  |w|max=%7.3f  th'=[%+.2f,%+.2f]K  "
                    "qc=%.2fg/kg qr=%.2fg/kg\n",
                    step, t, d.wmax, d.thmin, d.thmax, d.qcmax * 1000, d.qrmax * 1000);
      else
        std::printf("adim %6d  t=%7.1fs  |w|max=%7.3f  th'=[%+.3f,%+.3f]K  |pi'|max=%.2e\n", step,
                    t, d.wmax, d.thmin, d.thmax, d.pipmax);
      if (!d.finite) {
        std::fprintf(stderr, "HATA: NaN/Inf tespit edildi, simulasyon durduruldu.\n");
        return 2;
      }
    }
    if (step % out_steps == 0 || step == nsteps)
      if (write_snapshot(r, step, t)) return 1;
  }
  wfe_sync(r.c);
  double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::printf("bitti: %d adim, %.1f s duvar zamani, %.1f adim/s, gercek-zaman orani %.0fx\n",
              nsteps, wall, nsteps / wall, r.t_end / wall);
  wfe_ctx_destroy(r.c);
  return 0;
}
