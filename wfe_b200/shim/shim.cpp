// Reference-surface shim: the classes a driver written against the
// reference's C++ API uses (Config, GDims, Field3D, State, Metric,
// BaseState, DynParams, Integrator, BdyManager, SfcPBL, InputData, Writer,
// field_absmax; src/core, src/dynamics, src/io, src/physics headers),
// implemented on the wfe_b200 C ABI, so that the reference's src/main.cpp
// compiles unchanged against include/ of this directory and runs on the
// B200 kernels (wfe_b200/shim/Makefile builds it).
//
// Division of labour: the driver keeps doing what it does in the reference
// -- reads the case, builds the grid and DynParams, computes and uploads the
// initial conditions, drives the loop, writes the snapshots -- while the
// set-up the reference does in Metric / BaseState / BdyManager / SfcPBL is
// done by the library from the same configuration (a host-only context for
// the host copies the driver reads, then the device context at
// Integrator::init).  Fatal errors print a message and exit with status 1,
// as the reference's own checks do (src/core/cuda_check.hpp).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <sstream>
#include <string>
#include <vector>

#include "core/base_state.hpp"
#include "core/config.hpp"
#include "core/field3d.hpp"
#include "core/grid.hpp"
#include "core/metric.hpp"
#include "dynamics/boundary.hpp"
#include "dynamics/integrator.hpp"
#include "dynamics/kernels.hpp"
#include "io/input.hpp"
#include "io/writer.hpp"
#include "physics/surface.hpp"
#include "wfe_b200.h"

namespace wfe {

namespace shim {

struct Setup {
  Config cfg;          // the configuration the set-up was built from
  std::string text;    // the same as "key = value" lines
  wfe_ctx* host = nullptr;
  int dims[7] = {};
  double spacing[6] = {};
  ~Setup() {
    if (host) wfe_ctx_destroy(host);
  }
};

constexpr int kDtype = sizeof(real) == 4 ? WFE_DTYPE_F32 : WFE_DTYPE_F64;
constexpr int kPrecision = sizeof(real) == 4 ? WFE_F32 : WFE_F64;

[[noreturn]] void die(const char* what, const wfe_ctx* c) {
  std::fprintf(stderr, "wfe_b200: %s: %s\n", what, wfe_last_error(c));
  std::exit(1);
}

void check(int rc, const char* what, const wfe_ctx* c) {
  if (rc != WFE_OK) die(what, c);
}

std::vector<real> host_array(const Setup& s, bool base, int which, size_t n) {
  std::vector<double> d(n);
  check(base ? wfe_get_base(s.host, which, d.data()) : wfe_get_metric(s.host, which, d.data()),
        "host set-up array", s.host);
  return std::vector<real>(d.begin(), d.end());
}

std::string trim(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  return s.substr(a, s.find_last_not_of(" \t\r\n") - a + 1);
}

}  // namespace shim

// ------------------------------------------------------------------ Config
bool Config::load(const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  char buf[4096];
  while (std::fgets(buf, sizeof(buf), f)) {
    std::string line(buf);
    const size_t c = line.find_first_of("#;");
    if (c != std::string::npos) line.resize(c);
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    const std::string key = shim::trim(line.substr(0, eq));
    if (!key.empty()) kv_[key] = shim::trim(line.substr(eq + 1));
  }
  std::fclose(f);
  return true;
}

real Config::get_real(const std::string& key, real def) const {
  used_.insert(key);
  auto it = kv_.find(key);
  return it == kv_.end() ? def : (real)std::atof(it->second.c_str());
}

int Config::get_int(const std::string& key, int def) const {
  used_.insert(key);
  auto it = kv_.find(key);
  return it == kv_.end() ? def : std::atoi(it->second.c_str());
}

std::string Config::get_str(const std::string& key, const std::string& def) const {
  used_.insert(key);
  auto it = kv_.find(key);
  return it == kv_.end() ? def : it->second;
}

std::vector<std::string> Config::unused() const {
  std::vector<std::string> out;
  for (const auto& kv : kv_)
    if (!used_.count(kv.first) && kv.first.rfind("proj_", 0) != 0 && kv.first != "terrain_source")
      out.push_back(kv.first);
  return out;
}

std::string Config::text() const {
  std::string t;
  for (const auto& kv : kv_) t += kv.first + " = " + kv.second + "\n";
  return t;
}

// ----------------------------------------------------------------- Field3D
void Field3D::upload(const real* h) {
  if (!ctx || field < 0) {
    std::fprintf(stderr, "wfe_b200: upload to a field that is not bound to a context\n");
    std::exit(1);
  }
  shim::check(wfe_field_upload(ctx, role, field, h, shim::kDtype, WFE_LAYOUT_PADDED), "upload", ctx);
}

void Field3D::download(real* h) const {
  if (!ctx) {
    std::fprintf(stderr, "wfe_b200: download of a field that is not bound to a context\n");
    std::exit(1);
  }
  if (plane >= 0)
    shim::check(wfe_field2d_download(ctx, plane, h, shim::kDtype, WFE_LAYOUT_PADDED), "download", ctx);
  else
    shim::check(wfe_field_download(ctx, role, field, h, shim::kDtype, WFE_LAYOUT_PADDED), "download",
                ctx);
}

float field_absmax(const Field3D& f) {
  float out = 0;
  shim::check(wfe_absmax(f.ctx, f.field, &out), "field_absmax", f.ctx);
  return out;
}

// ------------------------------------------------------------------ Metric
void Metric::build(const GDims& g, const Config& cfg, const std::vector<real>*,
                   const std::vector<real>*, const std::vector<real>*) {
  // the keys src/core/metric.cpp reads, so that unused() reports what the
  // reference would report
  for (const char* k : {"coriolis_f", "dz0", "dz_max", "dz_ratio", "mtn_a", "mtn_h0", "mtn_lambda",
                        "mtn_xc", "mtn_ya", "mtn_yc"})
    cfg.get_real(k, 0);
  for (const char* k : {"stretch", "terrain"}) cfg.get_str(k, "");
  auto s = std::make_shared<shim::Setup>();
  s->cfg = cfg;
  s->text = cfg.text();
  if (wfe_case_create_text(s->text.c_str(), nullptr, 0, shim::kPrecision, -1, &s->host) != WFE_OK)
    shim::die("case set-up", nullptr);
  wfe_get_dims(s->host, s->dims);
  wfe_get_spacing(s->host, s->spacing);
  if (s->dims[0] != g.nx || s->dims[1] != g.ny || s->dims[2] != g.nz || g.ng != 3) {
    std::fprintf(stderr, "wfe_b200: the grid does not match the case (ng must be 3)\n");
    std::exit(1);
  }
  const size_t n1 = (size_t)g.NZ, n2 = (size_t)g.NX * g.NY;
  h_zeta_w = shim::host_array(*s, false, 0, n1);
  h_zeta_c = shim::host_array(*s, false, 1, n1);
  h_h = shim::host_array(*s, false, 4, n2);
  h_jac = shim::host_array(*s, false, 9, n2);
  zt_ = (real)s->spacing[5];
  setup_ = s;
}

void Metric::release() { setup_.reset(); }

DevMetric Metric::dev() const {
  DevMetric m;
  m.zt = zt_;
  m.setup = setup_.get();
  return m;
}

// --------------------------------------------------------------- BaseState
void BaseState::build(const GDims& g, const Config& cfg, const Metric& metric,
                      const ProfileTables*) {
  for (const char* k : {"bv_N", "theta0", "wind_offset", "wind_u", "wind_us", "wind_zs"})
    cfg.get_real(k, 0);
  cfg.get_str("wind_profile", "");
  const std::string prof = cfg.get_str("profile", "isentropic");
  setup_ = metric.setup();
  if (!setup_) {
    std::fprintf(stderr, "wfe_b200: BaseState::build before Metric::build\n");
    std::exit(1);
  }
  const size_t n = g.npts();
  h_ub = shim::host_array(*setup_, true, 9, (size_t)g.NZ);
  h_thb3 = shim::host_array(*setup_, true, 0, n);
  h_pib3 = shim::host_array(*setup_, true, 1, n);
  // the reference keeps the moist base profile only for moist soundings and
  // the host copy of qv_b only for wk82 (src/core/base_state.cpp:35, 168)
  has_moisture_ = prof == "wk82" || prof == "file";
  if (prof == "wk82") h_qvb_ = shim::host_array(*setup_, true, 8, n);
  else h_qvb_.clear();
}

void BaseState::release() {
  setup_.reset();
  h_ub.clear();
  h_thb3.clear();
  h_pib3.clear();
  h_qvb_.clear();
}

// --------------------------------------------------------------- InputData
namespace {
bool read_f32(FILE* f, std::vector<real>& dst, size_t n) {
  std::vector<float> tmp(n);
  if (std::fread(tmp.data(), sizeof(float), n, f) != n) return false;
  dst.assign(tmp.begin(), tmp.end());
  return true;
}
}  // namespace

bool InputData::load(const GDims& g, const std::string& dir) {
  dir_ = dir;
  Config meta;
  if (!meta.load(dir + "/wfe_input.ini")) {
    std::fprintf(stderr, "girdi meta okunamadi: %s/wfe_input.ini\n", dir.c_str());
    return false;
  }
  if (meta.get_int("nx", -1) != g.nx || meta.get_int("ny", -1) != g.ny ||
      meta.get_int("nz", -1) != g.nz) {
    std::fprintf(stderr, "girdi grid boyutlari case ile uyusmuyor\n");
    return false;
  }
  if (meta.get_int("version", 1) < 3) {
    std::fprintf(stderr, "girdi surumu 3'ten eski\n");
    return false;
  }
  const int npf = meta.get_int("np_prof", 0);
  bdy_interval = meta.get_real("bdy_interval", 10800);
  n_bdy = meta.get_int("n_bdy", 0);
  start = meta.get_str("start", "");
  FILE* f = std::fopen((dir + "/wfe_init.bin").c_str(), "rb");
  if (!f) {
    std::fprintf(stderr, "wfe_init.bin acilamadi\n");
    return false;
  }
  const size_t n2 = (size_t)g.nx * g.ny, n3 = n2 * g.nz;
  std::vector<real>* order[] = {&prof_z, &prof_th, &prof_qv, &prof_u, &h,  &fcor,
                                &tsk,    &land,    &lat,     &lon,    &soilw, &u,
                                &v,      &th,      &pi,      &qv};
  bool ok = true;
  for (int q = 0; q < 16 && ok; ++q) ok = read_f32(f, *order[q], q < 4 ? (size_t)npf : (q < 11 ? n2 : n3));
  std::fclose(f);
  if (!ok) std::fprintf(stderr, "wfe_init.bin eksik/bozuk\n");
  return ok;
}

bool InputData::load_bdy(const GDims& g, int idx, std::vector<real> fields[5]) const {
  char path[1024];
  std::snprintf(path, sizeof(path), "%s/wfe_bdy_%03d.bin", dir_.c_str(),
                (int)(idx * bdy_interval / 3600));
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    std::fprintf(stderr, "sinir dosyasi acilamadi: %s\n", path);
    return false;
  }
  const size_t n3 = (size_t)g.nx * g.ny * g.nz;
  bool ok = true;
  for (int q = 0; q < 5 && ok; ++q) ok = read_f32(f, fields[q], n3);
  std::fclose(f);
  return ok;
}

// -------------------------------------------------------------- BdyManager
void BdyManager::init(const GDims&, const DynParams&, const InputData* input,
                      const std::vector<real>&, const std::vector<real>&, int bdy_width,
                      real bdy_tau, real nudge_tau) {
  input_ = input;
  width_ = bdy_width;
  tau_ = bdy_tau;
  nudge_tau_ = nudge_tau;
  t_lo_ = 0;
  t_hi_ = input ? input->bdy_interval : 0;
}

void BdyManager::update(real t) {
  // the context switches its own targets inside each step; this copy of the
  // interval only serves tfrac()
  if (!input_ || input_->bdy_interval <= 0) return;
  while (t >= t_hi_ && (int)(t_hi_ / input_->bdy_interval) < input_->n_bdy - 1) {
    t_lo_ = t_hi_;
    t_hi_ += input_->bdy_interval;
  }
}

real BdyManager::tfrac(real t) const {
  if (t_hi_ <= t_lo_) return 0;
  real f = (t - t_lo_) / (t_hi_ - t_lo_);
  return f < 0 ? (real)0 : (f > 1 ? (real)1 : f);
}

// ------------------------------------------------------------------ SfcPBL
void SfcPBL::init(const GDims&, const InputData&, real start_hour_utc, int doy, bool nonlocal) {
  start_hour_ = start_hour_utc;
  doy_ = doy;
  nonlocal_ = nonlocal;
}

void SfcPBL::bind(wfe_ctx* c, size_t n2) {
  tsk_.bind_plane(c, WFE_2D_TSK, n2);
  pblh_.bind_plane(c, WFE_2D_PBLH, n2);
  t2m_.bind_plane(c, WFE_2D_T2M, n2);
  u10_.bind_plane(c, WFE_2D_U10, n2);
}

// -------------------------------------------------------------- Integrator
namespace {
std::string num(double v) {
  char b[64];
  std::snprintf(b, sizeof(b), "%.17g", v);
  return b;
}
}  // namespace

void Integrator::init(const GDims& g, const DevProf&, const DevMetric& m, const DynParams& dp) {
  const shim::Setup* s = m.setup;
  if (!s) {
    std::fprintf(stderr, "wfe_b200: Integrator::init needs the DevMetric of Metric::build\n");
    std::exit(1);
  }
  g_ = g;
  // DynParams the driver changed after reading the case become overrides;
  // values equal to what the case gives are left to the case's own text
  const Config& c = s->cfg;
  std::vector<std::string> ov;
  auto real_key = [&](const char* k, real def, real v) {
    if (c.get_real(k, def) != v) ov.push_back(std::string(k) + "=" + num((double)v));
  };
  auto int_key = [&](const char* k, int def, int v) {
    if (c.get_int(k, def) != v) ov.push_back(std::string(k) + "=" + std::to_string(v));
  };
  auto flag_key = [&](const char* k, const char* def, const char* on, const char* off, bool v) {
    if ((c.get_str(k, def) == on) != v) ov.push_back(std::string(k) + "=" + (v ? on : off));
  };
  real_key("diff_K", 0, dp.diff_K);
  real_key("coriolis_f", 0, dp.coriolis_f);
  real_key("rayleigh_zd", -1, dp.rayleigh_zd);
  real_key("rayleigh_alpha", 0, dp.rayleigh_alpha);
  int_key("acoustic_ns", 6, dp.acoustic_ns);
  real_key("acoustic_beta", (real)0.2, dp.acoustic_beta);
  real_key("acoustic_smdiv", (real)0.1, dp.acoustic_smdiv);
  flag_key("bc_x", "periodic", "open", "periodic", dp.bc_x_open);
  flag_key("bc_y", "periodic", "open", "periodic", dp.bc_y_open);
  real_key("cstar", 30, dp.cstar);
  flag_key("w_damping", "off", "on", "off", dp.w_damping);
  real_key("w_abort", 150, dp.w_abort);
  flag_key("microphysics", "on", "on", "off", dp.microphysics);
  if (dp.moisture) flag_key("pd_moist", "off", "on", "off", dp.pd_moist);
  std::vector<const char*> argv;
  for (const auto& o : ov) argv.push_back(o.c_str());
  int dev = 0;
  WFE_CUDA_CHECK(cudaGetDevice(&dev));
  if (wfe_case_create_text(s->text.c_str(), argv.data(), (int)argv.size(), shim::kPrecision, dev,
                           &ctx_) != WFE_OK)
    shim::die("device context", nullptr);
  int fl[10];
  wfe_get_flags(ctx_, fl);
  if ((fl[0] != 0) != dp.moisture)
    std::fprintf(stderr, "wfe_b200: UYARI: DynParams::moisture differs from the case's (%d); "
                         "the case's is used\n", fl[0]);
  s_n_.bind(ctx_, WFE_ROLE_STATE, g.npts());
  rain_.bind_plane(ctx_, WFE_2D_RAIN, (size_t)g.NX * g.NY);
}

Integrator::~Integrator() {
  if (ctx_) wfe_ctx_destroy(ctx_);
}

void Integrator::step(real dt, real t) {
  shim::check(wfe_run(ctx_, 1, (double)dt, (double)t), "step", ctx_);
  ++steps_;
}

void Integrator::print_profile() const {
  const char* e = std::getenv("WFE_PROF");
  if (!e || e[0] != '1' || !ctx_) return;
  std::printf("profil: %ld adim, adim basina %ld kernel (wfe_b200, CUDA graph)\n", steps_,
              wfe_launches_per_step(ctx_));
}

void Integrator::set_physics(SfcPBL* phys) {
  phys_ = phys;
  if (phys && ctx_) phys->bind(ctx_, (size_t)g_.NX * g_.NY);
}

// ------------------------------------------------------------------ Writer
void Writer::init(const GDims& g, const std::string& out_dir, real dt, bool moisture, bool has_tsk) {
  g_ = g;
  dir_ = out_dir;
  moist_ = moisture;
  std::filesystem::create_directories(dir_);
  out_.resize((size_t)g.nx * g.ny * (g.nz + 1));
  const std::string meta = dir_ + "/meta.json";
  FILE* f = std::fopen(meta.c_str(), "w");
  if (!f) {
    std::fprintf(stderr, "meta.json yazilamadi: %s\n", meta.c_str());
    std::exit(1);
  }
  std::fprintf(f,
               "{\n  \"nx\": %d, \"ny\": %d, \"nz\": %d,\n  \"dx\": %g, \"dy\": %g, \"dz\": %g,\n"
               "  \"dt\": %g,\n  \"vars\": {\"u\": %d, \"v\": %d, \"w\": %d, \"thp\": %d, \"pip\": %d",
               g.nx, g.ny, g.nz, (double)g.dx, (double)g.dy, (double)g.dz, (double)dt, g.nz, g.nz,
               g.nz + 1, g.nz, g.nz);
  if (moist_) std::fprintf(f, ", \"qv\": %d, \"qc\": %d, \"qr\": %d, \"rain\": 1", g.nz, g.nz, g.nz);
  if (has_tsk) std::fprintf(f, ", \"tsk\": 1, \"pblh\": 1, \"t2m\": 1, \"u10\": 1");
  std::fprintf(f, "}\n}\n");
  std::fclose(f);
}

namespace {
void write_floats(const std::string& path, const float* p, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f || std::fwrite(p, sizeof(float), n, f) != n) {
    std::fprintf(stderr, "cikti dosyasi yazilamadi: %s\n", path.c_str());
    std::exit(1);
  }
  std::fclose(f);
}

std::string snap(const std::string& dir, const char* name, int step) {
  char b[64];
  std::snprintf(b, sizeof(b), "/%s_%06d.bin", name, step);
  return dir + b;
}
}  // namespace

void Writer::write_field(const Field3D& f, const char* name, int step, int nzlev) {
  shim::check(wfe_field_download(f.ctx, f.role, f.field, out_.data(), WFE_DTYPE_F32,
                                 WFE_LAYOUT_INTERIOR),
              "snapshot", f.ctx);
  write_floats(snap(dir_, name, step), out_.data(), (size_t)nzlev * g_.ny * g_.nx);
}

void Writer::write(const State& s, int step, real t) {
  write_field(s.u, "u", step, g_.nz);
  write_field(s.v, "v", step, g_.nz);
  write_field(s.w, "w", step, g_.nz + 1);
  write_field(s.thp, "thp", step, g_.nz);
  write_field(s.pip, "pip", step, g_.nz);
  if (moist_) {
    write_field(s.qv, "qv", step, g_.nz);
    write_field(s.qc, "qc", step, g_.nz);
    write_field(s.qr, "qr", step, g_.nz);
  }
  std::printf("  cikti yazildi: step %d (t = %.1f s)\n", step, (double)t);
}

void Writer::write_field2d(const Field3D& f, const char* name, int step) {
  std::vector<float> o((size_t)g_.nx * g_.ny);
  shim::check(wfe_field2d_download(f.ctx, f.plane, o.data(), WFE_DTYPE_F32, WFE_LAYOUT_INTERIOR),
              "snapshot", f.ctx);
  write_floats(snap(dir_, name, step), o.data(), o.size());
}

void Writer::write_static(const char* name, const std::vector<float>& data) {
  write_floats(dir_ + "/" + name + ".bin", data.data(), data.size());
}

}  // namespace wfe
