// C-ABI of wfe_b200 (include/wfe_b200.h).
#include "wfe_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "model.hpp"
#include "setup.hpp"

using namespace wfe;

struct wfe_ctx {
  CaseSetup cs;
  std::unique_ptr<Model> model;
  std::unique_ptr<Lin> lin;  // declared after model: released first
  std::string err;
  int bdy_idx_hi = 1;  // BdyManager::idx_hi_
  double t_lo = 0, t_hi = 0;
};

namespace {
thread_local std::string g_create_err;

int set_err(wfe_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  else g_create_err = m;
  return code;
}

int model_err(wfe_ctx* c) {
  return set_err(c, WFE_ERR_CUDA, c->model ? c->model->error() : "host-only context");
}

#define NEED_MODEL(c)                                                              \
  do {                                                                             \
    if (!(c)) return WFE_ERR_ARG;                                                  \
    if (!(c)->model)                                                               \
      return set_err((c), WFE_ERR_CUDA, "context was created without a device");  \
  } while (0)

int finish_create(wfe_ctx* c, int precision, int device, wfe_ctx** out) {
  std::string err;
  if (device < 0) {  // host set-up only: no device work, stepping is refused
    *out = c;
    return WFE_OK;
  }
  c->model.reset(Model::create(c->cs, precision == WFE_F64, device, &err));
  if (!c->model) {
    set_err(nullptr, WFE_ERR_CUDA, err);
    delete c;
    return WFE_ERR_CUDA;
  }
  const CaseSetup& cs = c->cs;
  if (cs.bdy.on) {
    // BdyManager::init: weights and the first two target files
    // (src/dynamics/boundary.cpp:9-42)
    std::vector<double> lo[5], hi[5], w;
    bdy_weights(cs.g, cs.p, cs.bdy.width, cs.bdy.tau, cs.bdy.nudge_tau, &w);
    int hi_idx = cs.input.n_bdy - 1 < 1 ? cs.input.n_bdy - 1 : 1;
    if (!bdy_targets(cs, 0, lo, &err) || !bdy_targets(cs, hi_idx, hi, &err)) {
      set_err(nullptr, WFE_ERR_IO, err);
      delete c;
      return WFE_ERR_IO;
    }
    const double* plo[5];
    const double* phi[5];
    for (int v = 0; v < 5; ++v) {
      plo[v] = lo[v].data();
      phi[v] = hi[v].data();
    }
    c->t_lo = 0;
    c->t_hi = cs.input.bdy_interval;
    c->bdy_idx_hi = 1;
    if (c->model->set_boundary(plo, phi, w.data(), c->t_lo, c->t_hi)) {
      set_err(nullptr, WFE_ERR_CUDA, c->model->error());
      delete c;
      return WFE_ERR_CUDA;
    }
  }
  if (cs.sfc.on) {
    const InputData& in = cs.input;
    if (c->model->enable_physics(in.tsk.data(), in.land.data(), in.lat.data(), in.lon.data(),
                                 in.soilw.data(), cs.sfc.start_hour, cs.sfc.doy, cs.sfc.nonlocal)) {
      set_err(nullptr, WFE_ERR_CUDA, c->model->error());
      delete c;
      return WFE_ERR_CUDA;
    }
  }
  *out = c;
  return WFE_OK;
}

int create_from(Config& cfg, const char* const* ov, int nov, int precision, int device,
                wfe_ctx** out) {
  if (!out) return set_err(nullptr, WFE_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (precision != WFE_F32 && precision != WFE_F64)
    return set_err(nullptr, WFE_ERR_ARG, "precision must be WFE_F32 or WFE_F64");
  for (int a = 0; a < nov; ++a) {
    if (!ov || !ov[a]) return set_err(nullptr, WFE_ERR_ARG, "NULL override");
    std::string s = ov[a];
    size_t eq = s.find('=');
    if (eq == std::string::npos)
      return set_err(nullptr, WFE_ERR_ARG, "override without '=': " + s);
    cfg.set(s.substr(0, eq), s.substr(eq + 1));
  }
  auto* c = new wfe_ctx();
  std::string err;
  if (!setup_case(cfg, &c->cs, &err)) {
    delete c;
    bool io = err.find("cannot") != std::string::npos || err.find("corrupt") != std::string::npos;
    return set_err(nullptr, io ? WFE_ERR_IO : WFE_ERR_CONFIG, err);
  }
  return finish_create(c, precision, device, out);
}

// padded <-> interior conversion for the host side
void to_interior(const RefGrid& g, int field, const double* pad, double* in) {
  int nzl = field == WFE_W ? g.nz + 1 : g.nz;
  size_t o = 0;
  for (int k = 0; k < nzl; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) in[o++] = pad[g.idx(i, j, k)];
}
void from_interior(const RefGrid& g, int field, const double* in, double* pad) {
  int nzl = field == WFE_W ? g.nz + 1 : g.nz;
  size_t o = 0;
  for (int k = 0; k < nzl; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) pad[g.idx(i, j, k)] = in[o++];
}
size_t interior_count(const RefGrid& g, int field) {
  return (size_t)g.nx * g.ny * (field == WFE_W ? g.nz + 1 : g.nz);
}

}  // namespace

namespace wfe {
// sets the message wfe_last_error(NULL) returns on this thread
void set_thread_error(const std::string& m) { g_create_err = m; }
}  // namespace wfe

extern "C" {

int wfe_case_create(const char* ini_path, const char* const* overrides, int n_overrides,
                    int precision, int device, wfe_ctx** out) {
  Config cfg;
  if (!ini_path || !cfg.load(ini_path))
    return set_err(nullptr, WFE_ERR_CONFIG,
                   std::string("cannot read case file ") + (ini_path ? ini_path : "(null)"));
  return create_from(cfg, overrides, n_overrides, precision, device, out);
}

int wfe_case_create_text(const char* text, const char* const* overrides, int n_overrides,
                         int precision, int device, wfe_ctx** out) {
  Config cfg;
  if (!text) return set_err(nullptr, WFE_ERR_ARG, "text is NULL");
  cfg.load_text(text);
  return create_from(cfg, overrides, n_overrides, precision, device, out);
}

int wfe_ctx_destroy(wfe_ctx* ctx) {
  delete ctx;
  return WFE_OK;
}

const char* wfe_last_error(const wfe_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_create_err.c_str();
}

int wfe_get_dims(const wfe_ctx* c, int dims[7]) {
  if (!c || !dims) return WFE_ERR_ARG;
  const RefGrid& g = c->cs.g;
  int v[7] = {g.nx, g.ny, g.nz, g.ng, g.NX, g.NY, g.NZ};
  std::memcpy(dims, v, sizeof(v));
  return WFE_OK;
}

int wfe_get_spacing(const wfe_ctx* c, double out[6]) {
  if (!c || !out) return WFE_ERR_ARG;
  const CaseSetup& cs = c->cs;
  double v[6] = {cs.g.dx, cs.g.dy, cs.g.dz, cs.dt, cs.t_end, cs.m.zt};
  std::memcpy(out, v, sizeof(v));
  return WFE_OK;
}

int wfe_get_run_config(const wfe_ctx* c, double out[3], char* out_dir, int out_dir_len) {
  if (!c || !out) return WFE_ERR_ARG;
  const CaseSetup& cs = c->cs;
  out[0] = cs.out_every;
  out[1] = cs.diag_every;
  out[2] = cs.p.w_abort;
  if (out_dir && out_dir_len > 0) {
    std::strncpy(out_dir, cs.out_dir.c_str(), (size_t)out_dir_len - 1);
    out_dir[out_dir_len - 1] = 0;
  }
  return WFE_OK;
}

int wfe_get_flags(const wfe_ctx* c, int flags[10]) {
  if (!c || !flags) return WFE_ERR_ARG;
  const CaseSetup& cs = c->cs;
  int v[10] = {cs.p.moisture,  cs.p.microphysics, cs.p.pd_moist, cs.p.bc_x_open,
               cs.p.bc_y_open, cs.p.w_damping,    cs.file_mode,  cs.sfc.on,
               cs.bdy.on,      cs.p.acoustic_ns};
  std::memcpy(flags, v, sizeof(v));
  return WFE_OK;
}

int wfe_get_metric(const wfe_ctx* c, int which, double* out) {
  if (!c || !out) return WFE_ERR_ARG;
  const HostMetric& m = c->cs.m;
  const std::vector<double>* v[12] = {&m.zeta_w, &m.zeta_c, &m.dzeta_c, &m.dzeta_w, &m.h, &m.hx,
                                      &m.hy, &m.hx_u, &m.hy_v, &m.jac, &m.fcor, &m.mapf};
  if (which < 0 || which >= 12) return WFE_ERR_ARG;
  std::memcpy(out, v[which]->data(), v[which]->size() * sizeof(double));
  return WFE_OK;
}

int wfe_get_base(const wfe_ctx* c, int which, double* out) {
  if (!c || !out) return WFE_ERR_ARG;
  const HostBase& b = c->cs.b;
  const std::vector<double>* v[10] = {&b.thb,   &b.pib,  &b.rhob,  &b.dthbdz, &b.thbw,
                                      &b.rhobw, &b.thvb, &b.thvbw, &b.qvb,    &b.ub};
  if (which < 0 || which >= 10) return WFE_ERR_ARG;
  std::memcpy(out, v[which]->data(), v[which]->size() * sizeof(double));
  return WFE_OK;
}

int wfe_field_upload(wfe_ctx* c, int role, int field, const void* host, int dtype, int layout) {
  NEED_MODEL(c);
  if (host && field >= 0 && field <= 7 && layout == WFE_LAYOUT_INTERIOR)
    return c->model->upload_interior(role, field, host, dtype == WFE_DTYPE_F32) ? model_err(c)
                                                                                : WFE_OK;
  if (!c || !host || field < 0 || field > 7) return set_err(c, WFE_ERR_ARG, "bad argument");
  if (dtype != WFE_DTYPE_F32 && layout != WFE_LAYOUT_INTERIOR)  // FP64 padded: no host copies
    return c->model->upload(role, field, static_cast<const double*>(host)) ? model_err(c) : WFE_OK;
  const RefGrid& g = c->cs.g;
  std::vector<double> pad(g.npts(), 0.0);
  size_t n = layout == WFE_LAYOUT_INTERIOR ? interior_count(g, field) : g.npts();
  std::vector<double> src(n);
  if (dtype == WFE_DTYPE_F32) {
    const float* f = (const float*)host;
    for (size_t q = 0; q < n; ++q) src[q] = f[q];
  } else {
    std::memcpy(src.data(), host, n * sizeof(double));
  }
  if (layout == WFE_LAYOUT_INTERIOR) {
    if (c->model->download(role, field, pad.data())) return model_err(c);
    from_interior(g, field, src.data(), pad.data());
  } else {
    pad.swap(src);
  }
  if (c->model->upload(role, field, pad.data())) return model_err(c);
  return WFE_OK;
}

int wfe_field_download(wfe_ctx* c, int role, int field, void* host, int dtype, int layout) {
  NEED_MODEL(c);
  if (host && field >= 0 && field <= 7 && layout == WFE_LAYOUT_INTERIOR)
    return c->model->download_interior(role, field, host, dtype == WFE_DTYPE_F32) ? model_err(c)
                                                                                  : WFE_OK;
  if (!c || !host || field < 0 || field > 7) return set_err(c, WFE_ERR_ARG, "bad argument");
  if (dtype != WFE_DTYPE_F32 && layout != WFE_LAYOUT_INTERIOR)  // FP64 padded: no host copies
    return c->model->download(role, field, static_cast<double*>(host)) ? model_err(c) : WFE_OK;
  const RefGrid& g = c->cs.g;
  std::vector<double> pad(g.npts());
  if (c->model->download(role, field, pad.data())) return model_err(c);
  std::vector<double> out;
  if (layout == WFE_LAYOUT_INTERIOR) {
    out.resize(interior_count(g, field));
    to_interior(g, field, pad.data(), out.data());
  } else {
    out.swap(pad);
  }
  if (dtype == WFE_DTYPE_F32) {
    float* f = (float*)host;
    for (size_t q = 0; q < out.size(); ++q) f[q] = (float)out[q];
  } else {
    std::memcpy(host, out.data(), out.size() * sizeof(double));
  }
  return WFE_OK;
}

int wfe_field2d_download(wfe_ctx* c, int which, void* host, int dtype, int layout) {
  NEED_MODEL(c);
  if (!c || !host) return set_err(c, WFE_ERR_ARG, "bad argument");
  const RefGrid& g = c->cs.g;
  std::vector<double> pad(g.n2());
  if (c->model->download2d(which, pad.data())) return model_err(c);
  std::vector<double> out;
  if (layout == WFE_LAYOUT_INTERIOR) {
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) out.push_back(pad[g.idx2(i, j)]);
  } else {
    out.swap(pad);
  }
  if (dtype == WFE_DTYPE_F32) {
    float* f = (float*)host;
    for (size_t q = 0; q < out.size(); ++q) f[q] = (float)out[q];
  } else {
    std::memcpy(host, out.data(), out.size() * sizeof(double));
  }
  return WFE_OK;
}

// BdyManager::update (src/dynamics/boundary.cpp:83-89): move to the next
// boundary file once t passes the upper target time
static int boundary_update(wfe_ctx* c, double t) {
  const CaseSetup& cs = c->cs;
  if (!cs.bdy.on) return WFE_OK;
  while (t >= c->t_hi && c->bdy_idx_hi + 1 < cs.input.n_bdy) {
    ++c->bdy_idx_hi;
    std::vector<double> hi[5];
    std::string err;
    if (!bdy_targets(cs, c->bdy_idx_hi, hi, &err)) return set_err(c, WFE_ERR_IO, err);
    const double* phi[5];
    for (int v = 0; v < 5; ++v) phi[v] = hi[v].data();
    c->t_lo = c->t_hi;
    c->t_hi += cs.input.bdy_interval;
    if (c->model->sync() || c->model->set_boundary_hi(phi, c->t_lo, c->t_hi)) return model_err(c);
  }
  return WFE_OK;
}

int wfe_step(wfe_ctx* c, double dt, double t) {
  NEED_MODEL(c);
  if (!c) return WFE_ERR_ARG;
  int rc = boundary_update(c, t);
  if (rc) return rc;
  if (c->model->step(dt, t)) return model_err(c);
  return WFE_OK;
}

int wfe_run(wfe_ctx* c, int nsteps, double dt, double t0) {
  NEED_MODEL(c);
  if (!c || nsteps < 0) return WFE_ERR_ARG;
  int done = 0;
  while (done < nsteps) {
    // run up to the next boundary-file switch with graphs, then switch
    int chunk = nsteps - done;
    const CaseSetup& cs = c->cs;
    double t = t0 + done * dt;
    if (cs.bdy.on && c->bdy_idx_hi + 1 < cs.input.n_bdy) {
      int rc = boundary_update(c, t);
      if (rc) return rc;
      int until = (int)std::ceil((c->t_hi - t) / dt);
      if (until < 1) until = 1;
      if (until < chunk) chunk = until;
    }
    if (c->model->run(chunk, dt, t)) return model_err(c);
    done += chunk;
  }
  return WFE_OK;
}

int wfe_sync(wfe_ctx* c) {
  NEED_MODEL(c);
  if (!c) return WFE_ERR_ARG;
  return c->model->sync() ? model_err(c) : WFE_OK;
}

int wfe_absmax(wfe_ctx* c, int field, float* out) {
  NEED_MODEL(c);
  if (!c || !out) return WFE_ERR_ARG;
  return c->model->absmax(field, out) ? model_err(c) : WFE_OK;
}

int wfe_absmax_begin(wfe_ctx* c, int field, int slot) {
  NEED_MODEL(c);
  return c->model->absmax_begin(field, slot) ? model_err(c) : WFE_OK;
}

int wfe_absmax_end(wfe_ctx* c, int slot, float* out) {
  NEED_MODEL(c);
  if (!out) return set_err(c, WFE_ERR_ARG, "bad argument");
  return c->model->absmax_end(slot, out) ? model_err(c) : WFE_OK;
}

int wfe_dry_mass(wfe_ctx* c, double* out) {
  NEED_MODEL(c);
  if (!c || !out) return WFE_ERR_ARG;
  return c->model->dry_mass(out) ? model_err(c) : WFE_OK;
}

long wfe_launches_per_step(const wfe_ctx* c) {
  return c && c->model ? c->model->launches_per_step() : -1;
}

int wfe_case_variants(const wfe_ctx* c, int out[4]) {
  if (!c || !c->model || !out) return WFE_ERR_ARG;
  c->model->variants(out);
  return WFE_OK;
}

int wfe_time_run(wfe_ctx* c, int nsteps, double dt, double t0, double* ms) {
  NEED_MODEL(c);
  if (!ms || nsteps < 0) return WFE_ERR_ARG;
  return c->model->time_run(nsteps, dt, t0, ms) ? model_err(c) : WFE_OK;
}

int wfe_kernel_times(wfe_ctx* c, double dt, double t, int cap, double* total_ms, int* counts,
                     char* names_csv, int names_len, int* n_out) {
  NEED_MODEL(c);
  if (!total_ms || !counts || !names_csv || !n_out || cap < 1 || names_len < 1)
    return WFE_ERR_ARG;
  std::vector<std::string> names;
  std::vector<double> ms;
  std::vector<int> cnt;
  if (c->model->kernel_times(dt, t, &names, &ms, &cnt)) return model_err(c);
  std::string csv;
  int n = (int)names.size() < cap ? (int)names.size() : cap;
  for (int q = 0; q < n; ++q) {
    total_ms[q] = ms[q];
    counts[q] = cnt[q];
    if (q) csv += ",";
    csv += names[q];
  }
  std::strncpy(names_csv, csv.c_str(), (size_t)names_len - 1);
  names_csv[names_len - 1] = 0;
  *n_out = n;
  return WFE_OK;
}

int wfe_op_apply_bcs(wfe_ctx* c) {
  NEED_MODEL(c);
  if (!c) return WFE_ERR_ARG;
  return c->model->op_apply_bcs() ? model_err(c) : WFE_OK;
}
int wfe_op_tendencies(wfe_ctx* c, double dt, double t) {
  NEED_MODEL(c);
  return c->model->op_tendencies(dt, t) ? model_err(c) : WFE_OK;
}
int wfe_op_acoustic(wfe_ctx* c, double dtau, int nsub) {
  NEED_MODEL(c);
  if (!c || nsub < 1) return WFE_ERR_ARG;
  return c->model->op_acoustic(dtau, nsub) ? model_err(c) : WFE_OK;
}
int wfe_op_moisture_stage(wfe_ctx* c, double dt) {
  NEED_MODEL(c);
  if (!c) return WFE_ERR_ARG;
  return c->model->op_moisture_stage(dt) ? model_err(c) : WFE_OK;
}
int wfe_op_kessler(wfe_ctx* c, double dt) {
  NEED_MODEL(c);
  if (!c) return WFE_ERR_ARG;
  return c->model->op_kessler(dt) ? model_err(c) : WFE_OK;
}
int wfe_op_sfc(wfe_ctx* c, double dt, double t) {
  NEED_MODEL(c);
  if (!c) return WFE_ERR_ARG;
  return c->model->op_sfc(dt, t) ? model_err(c) : WFE_OK;
}

int wfe_set_boundary(wfe_ctx* c, const double* const lo[5], const double* const hi[5],
                     const double* wgt, double t_lo, double t_hi) {
  NEED_MODEL(c);
  if (!c || !lo || !hi || !wgt) return WFE_ERR_ARG;
  for (int v = 0; v < 5; ++v)
    if (!lo[v] || !hi[v]) return WFE_ERR_ARG;
  return c->model->set_boundary(lo, hi, wgt, t_lo, t_hi) ? model_err(c) : WFE_OK;
}

int wfe_bdy_weights(const wfe_ctx* c, int width, double tau, double nudge_tau, double* out) {
  if (!c || !out || width < 0 || (width > 0 && !(tau > 0)) || nudge_tau < 0) return WFE_ERR_ARG;
  std::vector<double> w;
  bdy_weights(c->cs.g, c->cs.p, width, tau, nudge_tau, &w);
  std::memcpy(out, w.data(), w.size() * sizeof(double));
  return WFE_OK;
}

int wfe_clear_boundary(wfe_ctx* c) {
  NEED_MODEL(c);
  return c->model->clear_boundary() ? model_err(c) : WFE_OK;
}

int wfe_set_physics(wfe_ctx* c, const double* tsk, const double* land, const double* lat,
                    const double* lon, const double* soilw, double start_hour, int doy,
                    int nonlocal) {
  NEED_MODEL(c);
  if (!c || !tsk || !land || !lat || !lon || !soilw) return WFE_ERR_ARG;
  return c->model->enable_physics(tsk, land, lat, lon, soilw, start_hour, doy, nonlocal != 0)
             ? model_err(c)
             : WFE_OK;
}

}  // extern "C"

// ------------------------------------------------------------ ensembles
struct wfe_ens {
  std::unique_ptr<Ensemble> e;
  std::vector<wfe_ctx*> members;
};

int wfe_ensemble_create(wfe_ctx* const* members, int n, wfe_ens** out) {
  if (!out || !members || n < 1) return set_err(nullptr, WFE_ERR_ARG, "bad ensemble arguments");
  *out = nullptr;
  std::vector<Model*> ms;
  for (int q = 0; q < n; ++q) {
    if (!members[q] || !members[q]->model)
      return set_err(nullptr, WFE_ERR_ARG, "ensemble member without a device model");
    ms.push_back(members[q]->model.get());
  }
  std::string err;
  Ensemble* e = Ensemble::create(ms, &err);
  if (!e) return set_err(nullptr, WFE_ERR_ARG, err);
  auto* h = new wfe_ens;
  h->e.reset(e);
  h->members.assign(members, members + n);
  *out = h;
  return WFE_OK;
}

int wfe_ensemble_destroy(wfe_ens* ens) {
  delete ens;
  return WFE_OK;
}

int wfe_ensemble_run(wfe_ens* ens, int nsteps, double dt, double t0) {
  if (!ens || nsteps < 0) return set_err(nullptr, WFE_ERR_ARG, "bad ensemble arguments");
  int done = 0;
  while (done < nsteps) {
    // replay up to the earliest boundary-file switch of any member, then switch
    int chunk = nsteps - done;
    const double t = t0 + done * dt;
    for (wfe_ctx* c : ens->members) {
      const CaseSetup& cs = c->cs;
      if (!cs.bdy.on || c->bdy_idx_hi + 1 >= cs.input.n_bdy) continue;
      if (boundary_update(c, t)) return set_err(nullptr, WFE_ERR_IO, c->err);
      int until = (int)std::ceil((c->t_hi - t) / dt);
      if (until < 1) until = 1;
      if (until < chunk) chunk = until;
    }
    if (ens->e->run(chunk, dt, t)) return set_err(nullptr, WFE_ERR_CUDA, ens->e->error());
    done += chunk;
  }
  return WFE_OK;
}

int wfe_ensemble_step(wfe_ens* ens, double dt, double t) {
  if (!ens) return set_err(nullptr, WFE_ERR_ARG, "ensemble is NULL");
  for (wfe_ctx* c : ens->members)
    if (boundary_update(c, t)) return set_err(nullptr, WFE_ERR_IO, c->err);
  if (ens->e->step(dt, t)) return set_err(nullptr, WFE_ERR_CUDA, ens->e->error());
  return WFE_OK;
}

int wfe_ensemble_sync(wfe_ens* ens) {
  if (!ens) return set_err(nullptr, WFE_ERR_ARG, "ensemble is NULL");
  return ens->e->sync() ? set_err(nullptr, WFE_ERR_CUDA, ens->e->error()) : WFE_OK;
}

int wfe_ensemble_time_run(wfe_ens* ens, int nsteps, double dt, double t0, double* ms) {
  if (!ens || !ms || nsteps < 1) return set_err(nullptr, WFE_ERR_ARG, "bad ensemble arguments");
  return ens->e->time_run(nsteps, dt, t0, ms) ? set_err(nullptr, WFE_ERR_CUDA, ens->e->error())
                                              : WFE_OK;
}

long wfe_ensemble_launches_per_step(const wfe_ens* ens) {
  return ens ? ens->e->launches_per_step() : -1;
}

int wfe_ensemble_variants(const wfe_ens* ens, int out[3]) {
  if (!ens || !out) return WFE_ERR_ARG;
  ens->e->variants(&out[0], &out[1], &out[2]);
  return WFE_OK;
}

// ------------------------------------------------- tangent-linear / adjoint
int wfe_lin_enable(wfe_ctx* c) {
  NEED_MODEL(c);
  if (c->lin) return WFE_OK;
  std::string err;
  c->lin.reset(Lin::create(c->model.get(), &err));
  if (!c->lin) return set_err(c, WFE_ERR_CONFIG, err);
  return WFE_OK;
}

int wfe_lin_zero(wfe_ctx* c) {
  NEED_MODEL(c);
  if (!c->lin) return set_err(c, WFE_ERR_ARG, "linearisation not enabled");
  return c->lin->zero() ? set_err(c, WFE_ERR_CUDA, c->lin->error()) : WFE_OK;
}

int wfe_tl_run(wfe_ctx* c, int nsteps, double dt, double t0) {
  NEED_MODEL(c);
  if (!c->lin) return set_err(c, WFE_ERR_ARG, "linearisation not enabled");
  if (nsteps < 0) return set_err(c, WFE_ERR_ARG, "nsteps < 0");
  return c->lin->tl_run(nsteps, dt, t0) ? set_err(c, WFE_ERR_CUDA, c->lin->error()) : WFE_OK;
}

int wfe_ad_run(wfe_ctx* c, int nsteps, double dt, double t0, int checkpoint_every) {
  NEED_MODEL(c);
  if (!c->lin) return set_err(c, WFE_ERR_ARG, "linearisation not enabled");
  if (nsteps < 0) return set_err(c, WFE_ERR_ARG, "nsteps < 0");
  return c->lin->ad_run(nsteps, dt, t0, checkpoint_every) ? set_err(c, WFE_ERR_CUDA, c->lin->error())
                                                           : WFE_OK;
}

// ------------------------------------------------------------- snapshots
int wfe_snapshot_begin(wfe_ctx* c, int n, const int* fields, void* const* host, int dtype) {
  NEED_MODEL(c);
  if (n < 0 || (n > 0 && (!fields || !host))) return set_err(c, WFE_ERR_ARG, "bad snapshot arguments");
  for (int q = 0; q < n; ++q)
    if (!host[q]) return set_err(c, WFE_ERR_ARG, "snapshot host buffer is NULL");
  return c->model->snapshot_begin(n, fields, host, dtype == WFE_DTYPE_F32) ? model_err(c) : WFE_OK;
}

int wfe_snapshot_wait(wfe_ctx* c) {
  NEED_MODEL(c);
  return c->model->snapshot_wait() ? model_err(c) : WFE_OK;
}

void* wfe_host_alloc(size_t bytes) {
  void* p = nullptr;
  return cudaMallocHost(&p, bytes) == cudaSuccess ? p : nullptr;
}

int wfe_host_free(void* p) {
  return cudaFreeHost(p) == cudaSuccess ? WFE_OK : WFE_ERR_CUDA;
}
