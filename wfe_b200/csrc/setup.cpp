// Host-side case set-up (see setup.hpp).  FP64 throughout; the arithmetic of
// every stored value follows the reference so that the FP64 set-up is
// bit-identical to the reference's FP64 build.
#include "setup.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <random>
#include <sstream>

namespace wfe {

// ------------------------------------------------------------------ Config
static std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

bool Config::load_text(const std::string& text) {
  // "key = value" lines; '#' or ';' start a comment (src/core/config.cpp:17-31)
  std::istringstream in(text);
  std::string line;
  bool first = true;
  while (std::getline(in, line)) {
    if (first && line.size() >= 3 && (unsigned char)line[0] == 0xEF &&
        (unsigned char)line[1] == 0xBB && (unsigned char)line[2] == 0xBF)
      line = line.substr(3);  // UTF-8 byte-order mark (some reference cases carry one)
    first = false;
    size_t c = line.find_first_of("#;");
    if (c != std::string::npos) line = line.substr(0, c);
    size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    std::string key = trim(line.substr(0, eq)), val = trim(line.substr(eq + 1));
    if (!key.empty()) kv_[key] = val;
  }
  return true;
}

bool Config::load(const std::string& path) {
  std::ifstream f(path);
  if (!f) return false;
  std::stringstream ss;
  ss << f.rdbuf();
  return load_text(ss.str());
}

double Config::real(const std::string& k, double def) const {
  used_.insert(k);
  auto it = kv_.find(k);
  return it == kv_.end() ? def : std::atof(it->second.c_str());
}
int Config::integer(const std::string& k, int def) const {
  used_.insert(k);
  auto it = kv_.find(k);
  return it == kv_.end() ? def : std::atoi(it->second.c_str());
}
std::string Config::str(const std::string& k, const std::string& def) const {
  used_.insert(k);
  auto it = kv_.find(k);
  return it == kv_.end() ? def : it->second;
}
std::vector<std::string> Config::unused() const {
  // keys no getter read, except the ones only the prep tools read
  // (src/core/config.cpp:51-60)
  std::vector<std::string> out;
  for (const auto& kv : kv_) {
    if (used_.count(kv.first)) continue;
    if (kv.first.rfind("proj_", 0) == 0 || kv.first == "terrain_source") continue;
    out.push_back(kv.first);
  }
  return out;
}

RefGrid make_ref_grid(int nx, int ny, int nz, double dx, double dy, double dz) {
  return RefGrid{nx, ny, nz, 3, nx + 6, ny + 6, nz + 7, dx, dy, dz};
}

// ------------------------------------------------------------------ metric
void build_metric(const RefGrid& g, const Config& cfg, const std::vector<double>* h_file,
                  const std::vector<double>* fcor_file, const std::vector<double>* mapf_file,
                  HostMetric* m) {
  const int NZ = g.NZ, nz = g.nz, ng = g.ng;
  const size_t n2 = g.n2();
  // w-level heights, uniform or geometric (src/core/metric.cpp:24-38)
  std::vector<double> zw(nz + 1, 0.0);
  if (cfg.str("stretch", "none") == "geometric") {
    double dz0 = cfg.real("dz0", g.dz), ratio = cfg.real("dz_ratio", 1.05);
    double dzmax = cfg.real("dz_max", g.dz * 4);
    double d = dz0;
    for (int k = 1; k <= nz; ++k) {
      zw[k] = zw[k - 1] + d;
      d = std::min(d * ratio, dzmax);
    }
  } else {
    for (int k = 0; k <= nz; ++k) zw[k] = (double)k * g.dz;
  }
  m->zt = zw[nz];
  auto zw_ext = [&](int k) {  // linear continuation into the ghosts
    if (k < 0) return zw[0] + (double)k * (zw[1] - zw[0]);
    if (k > nz) return zw[nz] + (double)(k - nz) * (zw[nz] - zw[nz - 1]);
    return zw[k];
  };
  m->zeta_w.assign(NZ, 0);
  m->zeta_c.assign(NZ, 0);
  m->dzeta_c.assign(NZ, 0);
  m->dzeta_w.assign(NZ, 0);
  for (int kk = 0; kk < NZ; ++kk) {
    int k = kk - ng;
    m->zeta_w[kk] = zw_ext(k);
    m->zeta_c[kk] = 0.5 * (zw_ext(k) + zw_ext(k + 1));
  }
  for (int kk = 0; kk + 1 < NZ; ++kk) m->dzeta_c[kk] = m->zeta_w[kk + 1] - m->zeta_w[kk];
  m->dzeta_c[NZ - 1] = m->dzeta_c[NZ - 2];
  for (int kk = 1; kk < NZ; ++kk) m->dzeta_w[kk] = m->zeta_c[kk] - m->zeta_c[kk - 1];
  m->dzeta_w[0] = m->dzeta_w[1];

  // terrain at every padded column (src/core/metric.cpp:63-123)
  for (auto* v : {&m->h, &m->hx, &m->hy, &m->hx_u, &m->hy_v, &m->jac}) v->assign(n2, 0.0);
  const std::string terrain = cfg.str("terrain", "none");
  const double h0 = cfg.real("mtn_h0", 250), xa = cfg.real("mtn_a", 5000);
  const double lam = cfg.real("mtn_lambda", 4000);
  const double xc = cfg.real("mtn_xc", g.nx * g.dx / 2), yc = cfg.real("mtn_yc", g.ny * g.dy / 2);
  const double ya = cfg.real("mtn_ya", xa);
  const double pi = 3.14159265358979323846;
  auto height = [&](double x, double y) -> double {
    if (terrain == "schaer") {
      double xr = x - xc;
      double env = std::exp(-(xr / xa) * (xr / xa));
      double c = std::cos(pi * xr / lam);
      return h0 * env * c * c;
    }
    if (terrain == "gauss") {
      double xr = (x - xc) / xa, yr = (y - yc) / ya;
      return h0 * std::exp(-xr * xr - yr * yr);
    }
    return 0.0;
  };
  const double zt = m->zt;
  auto clampi = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
  if (terrain == "file" && h_file) {
    for (int j = -ng; j < g.ny + ng; ++j)
      for (int i = -ng; i < g.nx + ng; ++i)
        m->h[g.idx2(i, j)] = (*h_file)[(size_t)clampi(j, 0, g.ny - 1) * g.nx + clampi(i, 0, g.nx - 1)];
    for (int j = -ng; j < g.ny + ng; ++j)
      for (int i = -ng; i < g.nx + ng; ++i) {
        size_t c = g.idx2(i, j);
        m->jac[c] = (zt - m->h[c]) / zt;
        int im = i > -ng ? i - 1 : i, ip = i < g.nx + ng - 1 ? i + 1 : i;
        int jm = j > -ng ? j - 1 : j, jp = j < g.ny + ng - 1 ? j + 1 : j;
        m->hx[c] = (m->h[g.idx2(ip, j)] - m->h[g.idx2(im, j)]) / ((double)(ip - im) * g.dx);
        m->hy[c] = (m->h[g.idx2(i, jp)] - m->h[g.idx2(i, jm)]) / ((double)(jp - jm) * g.dy);
        m->hx_u[c] = (i == im) ? 0.0 : (m->h[c] - m->h[g.idx2(im, j)]) / g.dx;
        m->hy_v[c] = (j == jm) ? 0.0 : (m->h[c] - m->h[g.idx2(i, jm)]) / g.dy;
      }
  } else {
    for (int j = -ng; j < g.ny + ng; ++j)
      for (int i = -ng; i < g.nx + ng; ++i) {
        double x = ((double)i + 0.5) * g.dx, y = ((double)j + 0.5) * g.dy;
        size_t c = g.idx2(i, j);
        m->h[c] = height(x, y);
        m->jac[c] = (zt - m->h[c]) / zt;
        m->hx[c] = (height(x + g.dx, y) - height(x - g.dx, y)) / (2.0 * g.dx);
        m->hy[c] = (height(x, y + g.dy) - height(x, y - g.dy)) / (2.0 * g.dy);
        m->hx_u[c] = (height(x, y) - height(x - g.dx, y)) / g.dx;
        m->hy_v[c] = (height(x, y) - height(x, y - g.dy)) / g.dy;
      }
  }
  // Coriolis and map factor: constant or clamped copies of interior input
  m->fcor.assign(n2, cfg.real("coriolis_f", 0));
  m->mapf.assign(n2, 1.0);
  for (int j = -ng; j < g.ny + ng; ++j)
    for (int i = -ng; i < g.nx + ng; ++i) {
      size_t src = (size_t)clampi(j, 0, g.ny - 1) * g.nx + clampi(i, 0, g.nx - 1);
      if (fcor_file) m->fcor[g.idx2(i, j)] = (*fcor_file)[src];
      if (mapf_file) m->mapf[g.idx2(i, j)] = (*mapf_file)[src];
    }
}

// -------------------------------------------------------------- base state
namespace {
constexpr double kGrav = 9.81, kCp = 1004.5, kRd = 287.04, kCv = 1004.5 - 287.04, kP00 = 1.0e5;
constexpr double kEps61 = 0.61;
}  // namespace

bool build_base(const RefGrid& g, const Config& cfg, const HostMetric& m, const InputData* tables,
                HostBase* b, std::string* err) {
  const std::string prof = cfg.str("profile", "isentropic");
  const double theta0 = cfg.real("theta0", 300), bvN = cfg.real("bv_N", 0.01);
  const bool constN = prof == "constant_N", wk82 = prof == "wk82", file = prof == "file";
  if (file && (!tables || tables->prof_z.size() < 2)) {
    *err = "profile=file but no profile tables were loaded";
    return false;
  }
  if (!constN && !wk82 && !file && prof != "isentropic") {
    *err = "unknown profile: " + prof;
    return false;
  }
  b->has_moisture = wk82 || file;
  auto lookup = [&](const std::vector<double>& tab, double z) {  // base_state.cpp:104-113
    const std::vector<double>& zt = tables->prof_z;
    double dzt = zt[1] - zt[0];
    double s = (z - zt[0]) / dzt;
    int it = (int)s;
    if (it < 0) it = 0;
    if (it > (int)zt.size() - 2) it = (int)zt.size() - 2;
    double f = s - it;
    return tab[it] * (1 - f) + tab[it + 1] * f;
  };
  const double z_tr = 12000.0, th_tr = 343.0, T_tr = 213.0, qv_max = 0.014;
  auto theta = [&](double z) -> double {  // base_state.cpp:118-126
    if (file) return lookup(tables->prof_th, z);
    if (wk82) {
      if (z <= z_tr) return 300.0 + (th_tr - 300.0) * std::pow(z / z_tr, 1.25);
      return th_tr * std::exp(kGrav * (z - z_tr) / (kCp * T_tr));
    }
    if (constN) return theta0 * std::exp(bvN * bvN * z / kGrav);
    return theta0;
  };
  auto relhum = [&](double z) { return z <= z_tr ? 1.0 - 0.75 * std::pow(z / z_tr, 1.25) : 0.25; };
  auto qsat = [](double p, double T) {  // base_state.cpp:78-81, unclamped
    double es = 610.78 * std::exp(17.269 * (T - 273.16) / (T - 35.86));
    return 0.622 * es / (p - es);
  };

  // 1 m hydrostatic table (base_state.cpp:133-178)
  const double zmin = -(double)(g.ng + 1) * g.dz * 4 - 100.0;
  const double zmax = m.zt + (double)(g.ng + 1) * g.dz * 4 + 100.0;
  const int ntab = (int)((zmax - zmin) / 1.0) + 2, i0 = (int)(-zmin / 1.0);
  std::vector<double> pit(ntab), qvt(ntab, 0.0), thvt(ntab);
  for (int it = 0; it < ntab; ++it) thvt[it] = theta(zmin + it * 1.0);
  auto integrate = [&]() {
    pit[i0] = 1.0;
    for (int it = i0 + 1; it < ntab; ++it)
      pit[it] = pit[it - 1] - kGrav * 1.0 / (kCp * (0.5 * (thvt[it - 1] + thvt[it])));
    for (int it = i0 - 1; it >= 0; --it)
      pit[it] = pit[it + 1] + kGrav * 1.0 / (kCp * (0.5 * (thvt[it] + thvt[it + 1])));
  };
  integrate();
  if (wk82) {
    for (int iter = 0; iter < 5; ++iter) {
      for (int it = 0; it < ntab; ++it) {
        double z = zmin + it * 1.0, th = theta(z), pi = pit[it];
        double T = th * pi, p = kP00 * std::pow(pi, kCp / kRd);
        double qv = std::min(relhum(z) * qsat(p, T), qv_max);
        if (z < 0) qv = qvt[it > 0 ? it : 0];
        qvt[it] = qv;
        thvt[it] = th * (1.0 + kEps61 * qv);
      }
      integrate();
    }
  } else if (file) {
    for (int it = 0; it < ntab; ++it) {
      double z = zmin + it * 1.0;
      qvt[it] = std::max(0.0, lookup(tables->prof_qv, z));
      thvt[it] = theta(z) * (1.0 + kEps61 * qvt[it]);
    }
    integrate();
  }
  auto interp = [&](const std::vector<double>& tab, double z) {  // base_state.cpp:180-187
    double s = (z - zmin) / 1.0;
    int it = (int)s;
    if (it < 0) it = 0;
    if (it > ntab - 2) it = ntab - 2;
    double f = s - it;
    return tab[it] * (1 - f) + tab[it + 1] * f;
  };
  auto rho = [](double pi, double thv) { return kP00 * std::pow(pi, kCv / kRd) / (kRd * thv); };

  const size_t n = g.npts();
  for (auto* v : {&b->thb, &b->pib, &b->rhob, &b->dthbdz, &b->thbw, &b->rhobw, &b->thvb,
                  &b->thvbw, &b->qvb})
    v->assign(n, 0.0);
  for (int k = -g.ng; k < g.nz + 1 + g.ng; ++k)
    for (int j = -g.ng; j < g.ny + g.ng; ++j)
      for (int i = -g.ng; i < g.nx + g.ng; ++i) {
        size_t c = g.idx(i, j, k);
        double hh = m.h[g.idx2(i, j)];
        double zc = hh + m.zeta_c[k + g.ng] * (m.zt - hh) / m.zt;
        double zw = hh + m.zeta_w[k + g.ng] * (m.zt - hh) / m.zt;
        double thc = theta(zc), thw = theta(zw);
        double qvc = b->has_moisture ? interp(qvt, zc) : 0.0;
        double qvw = b->has_moisture ? interp(qvt, zw) : 0.0;
        double thvc = thc * (1.0 + kEps61 * qvc), thvw = thw * (1.0 + kEps61 * qvw);
        double pic = interp(pit, zc), piw = interp(pit, zw);
        b->thb[c] = thc;
        b->pib[c] = pic;
        b->rhob[c] = rho(pic, thvc);
        b->dthbdz[c] = (theta(zc + 1.0) - theta(zc - 1.0)) / 2.0;
        b->thbw[c] = thw;
        b->rhobw[c] = rho(piw, thvw);
        b->thvb[c] = thvc;
        b->thvbw[c] = thvw;
        b->qvb[c] = qvc;
      }
  // base wind: const, tanh, linear shear, or the file table (base_state.cpp:234-252)
  const std::string wprof = cfg.str("wind_profile", "const");
  const double windu = cfg.real("wind_u", 0), us = cfg.real("wind_us", 25);
  const double zs = cfg.real("wind_zs", 3000), uoff = cfg.real("wind_offset", 0);
  b->ub.assign(g.NZ, windu);
  for (int kk = 0; kk < g.NZ; ++kk) {
    double z = m.zeta_c[kk];
    if (z < 0) z = 0;
    if (wprof == "tanh") b->ub[kk] = us * std::tanh(z / zs) + uoff;
    else if (wprof == "linear") b->ub[kk] = us * std::min(z / zs, 1.0) + uoff;
    else if (file && !tables->prof_u.empty()) b->ub[kk] = lookup(tables->prof_u, z);
  }
  return true;
}

// ------------------------------------------------------------- input files
static bool read_f32(FILE* f, std::vector<double>& dst, size_t n) {
  std::vector<float> tmp(n);
  if (std::fread(tmp.data(), sizeof(float), n, f) != n) return false;
  dst.assign(tmp.begin(), tmp.end());
  return true;
}

bool InputData::load(const RefGrid& g, const std::string& d, std::string* err) {
  dir = d;
  Config meta;
  if (!meta.load(d + "/wfe_input.ini")) {
    *err = "cannot read " + d + "/wfe_input.ini";
    return false;
  }
  if (meta.integer("nx", -1) != g.nx || meta.integer("ny", -1) != g.ny ||
      meta.integer("nz", -1) != g.nz) {
    *err = "input grid does not match the case grid";
    return false;
  }
  if (meta.integer("version", 1) < 3) {
    *err = "input version < 3";
    return false;
  }
  int npf = meta.integer("np_prof", 0);
  bdy_interval = meta.real("bdy_interval", 10800);
  n_bdy = meta.integer("n_bdy", 0);
  start = meta.str("start", "");
  FILE* f = std::fopen((d + "/wfe_init.bin").c_str(), "rb");
  if (!f) {
    *err = "cannot open " + d + "/wfe_init.bin";
    return false;
  }
  size_t n2 = (size_t)g.nx * g.ny, n3 = n2 * g.nz;
  bool ok = read_f32(f, prof_z, npf) && read_f32(f, prof_th, npf) && read_f32(f, prof_qv, npf) &&
            read_f32(f, prof_u, npf) && read_f32(f, h, n2) && read_f32(f, fcor, n2) &&
            read_f32(f, tsk, n2) && read_f32(f, land, n2) && read_f32(f, lat, n2) &&
            read_f32(f, lon, n2) && read_f32(f, soilw, n2) && read_f32(f, u, n3) &&
            read_f32(f, v, n3) && read_f32(f, th, n3) && read_f32(f, pi, n3) &&
            read_f32(f, qv, n3);
  std::fclose(f);
  if (!ok) *err = "wfe_init.bin is short or corrupt";
  return ok;
}

bool InputData::load_bdy(const RefGrid& g, int idx, std::vector<double> f[5],
                         std::string* err) const {
  char path[1024];
  std::snprintf(path, sizeof(path), "%s/wfe_bdy_%03d.bin", dir.c_str(),
                (int)(idx * bdy_interval / 3600));
  FILE* fp = std::fopen(path, "rb");
  if (!fp) {
    *err = std::string("cannot open boundary file ") + path;
    return false;
  }
  size_t n3 = (size_t)g.nx * g.ny * g.nz;
  bool ok = true;
  for (int v = 0; v < 5 && ok; ++v) ok = read_f32(fp, f[v], n3);
  std::fclose(fp);
  if (!ok) *err = std::string("boundary file is short or corrupt: ") + path;
  return ok;
}

// ------------------------------------------------------- Davies relaxation
void bdy_weights(const RefGrid& g, const HostParams& p, int width, double tau, double nudge_tau,
                 std::vector<double>* wgt) {
  // cos^2 ramp over `width` rows with 1/tau at the edge, 1/nudge_tau inside
  // (src/dynamics/boundary.cpp:24-42)
  double inner = nudge_tau > 0 ? 1.0 / nudge_tau : 0.0;
  const double pi_half = 1.5707963267948966;
  wgt->assign(g.n2(), 0.0);
  for (int j = 0; j < g.ny; ++j)
    for (int i = 0; i < g.nx; ++i) {
      double w = inner;
      int dist = 1 << 20;
      if (p.bc_x_open) dist = std::min({dist, i, g.nx - 1 - i});
      if (p.bc_y_open) dist = std::min({dist, j, g.ny - 1 - j});
      if (dist < width) {
        double s = std::cos(pi_half * (double)dist / (double)width);
        w = std::max(w, s * s / tau);
      }
      (*wgt)[g.idx2(i, j)] = w;
    }
}

bool bdy_targets(const CaseSetup& cs, int idx, std::vector<double> out[5], std::string* err) {
  // centres -> faces for u, v; full -> perturbation for theta, pi
  // (src/dynamics/boundary.cpp:51-81)
  const RefGrid& g = cs.g;
  std::vector<double> f[5];
  if (!cs.input.load_bdy(g, idx, f, err)) return false;
  auto src = [&](const std::vector<double>& a, int i, int j, int k) {
    return a[((size_t)k * g.ny + j) * g.nx + i];
  };
  for (int v = 0; v < 5; ++v) {
    out[v].assign(g.npts(), 0.0);
    for (int k = 0; k < g.nz; ++k)
      for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx + (v == 0 ? 1 : 0); ++i) {
          size_t c = g.idx(i, j, k);
          double val;
          if (v == 0) {
            int il = i > 0 ? i - 1 : 0, ir = i < g.nx ? i : g.nx - 1;
            val = 0.5 * (src(f[0], il, j, k) + src(f[0], ir, j, k));
          } else if (v == 1) {
            int jl = j > 0 ? j - 1 : 0;
            val = 0.5 * (src(f[1], i, jl, k) + src(f[1], i, j, k));
          } else if (v == 2) {
            val = src(f[2], i, j, k) - cs.b.thb[c];
          } else if (v == 3) {
            val = src(f[3], i, j, k) - cs.b.pib[c];
          } else {
            val = src(f[4], i, j, k);
          }
          out[v][c] = val;
        }
  }
  return true;
}

// ------------------------------------------------------ initial conditions
static void ic_blob(const RefGrid& g, const HostMetric& m, double amp, double xc, double yc,
                    double zc, double xr, double yr, double zr, std::vector<double>* f) {
  // cos^2 blob in physical height (src/main.cpp:28-54, 158-183)
  const double pi = 3.14159265358979323846;
  f->assign(g.npts(), 0.0);
  for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) {
        double x = ((double)i + 0.5) * g.dx, y = ((double)j + 0.5) * g.dy;
        double hh = m.h[g.idx2(i, j)];
        double z = hh + m.zeta_c[k + g.ng] * (m.zt - hh) / m.zt;
        double rx = (x - xc) / xr, ry = (y - yc) / yr, rz = (z - zc) / zr;
        double r = std::sqrt(rx * rx + ry * ry + rz * rz);
        if (r < 1.0) {
          double c = std::cos(pi * r / 2);
          (*f)[g.idx(i, j, k)] = amp * c * c;
        }
      }
}

static void ic_perturbation(const RefGrid& g, double amp, unsigned seed, std::vector<double>* thp) {
  // seeded, box-smoothed theta' noise scaled to an RMS (src/main.cpp:105-144)
  if (amp <= 0) return;
  size_t n = g.npts();
  std::vector<double> p(n, 0.0), tmp;
  std::mt19937 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) p[g.idx(i, j, k)] = (double)nd(rng);
  for (int pass = 0; pass < 6; ++pass) {
    tmp = p;
    for (int k = 1; k < g.nz - 1; ++k)
      for (int j = 1; j < g.ny - 1; ++j)
        for (int i = 1; i < g.nx - 1; ++i) {
          double s6 = tmp[g.idx(i - 1, j, k)] + tmp[g.idx(i + 1, j, k)] + tmp[g.idx(i, j - 1, k)] +
                      tmp[g.idx(i, j + 1, k)] + tmp[g.idx(i, j, k - 1)] + tmp[g.idx(i, j, k + 1)];
          p[g.idx(i, j, k)] = 0.5 * tmp[g.idx(i, j, k)] + s6 / 12.0;
        }
  }
  double ss = 0;
  size_t cnt = 0;
  for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) {
        double v = p[g.idx(i, j, k)];
        ss += v * v;
        ++cnt;
      }
  double rms = std::sqrt(ss / cnt);
  if (rms < 1e-9) return;
  double sc = amp / rms;
  for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) (*thp)[g.idx(i, j, k)] += sc * p[g.idx(i, j, k)];
}

bool setup_case(const Config& cfg_in, CaseSetup* cs, std::string* err) {
  cs->cfg = cfg_in;
  const Config& cfg = cs->cfg;
  // grid and run controls (src/main.cpp:261-273)
  int nx = cfg.integer("nx", 100), ny = cfg.integer("ny", 100), nz = cfg.integer("nz", 50);
  double dx = cfg.real("dx", 200), dy = cfg.real("dy", 200), dz = cfg.real("dz", 200);
  if (nx < 2 || ny < 2 || nz < 4) {
    *err = "grid too small (need nx, ny >= 2 and nz >= 4)";
    return false;
  }
  cs->dt = cfg.real("dt", 0.25);
  cs->t_end = cfg.real("t_end", 1000);
  cs->out_every = cfg.real("out_interval", 100);
  cs->diag_every = cfg.real("diag_interval", 10);
  cs->out_dir = cfg.str("out_dir", "out/warm_bubble");
  const RefGrid g = cs->g = make_ref_grid(nx, ny, nz, dx, dy, dz);
  // dynamics parameters (src/main.cpp:284-298)
  HostParams& p = cs->p;
  p.diff_K = cfg.real("diff_K", 0);
  p.coriolis_f = cfg.real("coriolis_f", 0);
  p.rayleigh_zd = cfg.real("rayleigh_zd", -1);
  p.rayleigh_alpha = cfg.real("rayleigh_alpha", 0);
  p.acoustic_ns = cfg.integer("acoustic_ns", 6);
  p.acoustic_beta = cfg.real("acoustic_beta", 0.2);
  p.acoustic_smdiv = cfg.real("acoustic_smdiv", 0.1);
  p.bc_x_open = cfg.str("bc_x", "periodic") == "open";
  p.bc_y_open = cfg.str("bc_y", "periodic") == "open";
  p.cstar = cfg.real("cstar", 30);
  p.w_damping = cfg.str("w_damping", "off") == "on";
  p.w_abort = cfg.real("w_abort", 150);
  p.pd_moist = cfg.str("pd_moist", "off") == "on";
  p.microphysics = cfg.str("microphysics", "on") == "on";

  cs->file_mode = cfg.str("profile", "isentropic") == "file";
  std::vector<double> mapf;
  if (cs->file_mode) {
    if (!cs->input.load(g, cfg.str("input_dir", ""), err)) return false;
    p.coriolis_use_ub = false;
    // Lambert conformal map factor (src/main.cpp:326-340)
    double phi1 = cfg.real("proj_lat1", 35) * 0.01745329252;
    double phi2 = cfg.real("proj_lat2", 43) * 0.01745329252;
    const double PI4 = 0.78539816339;
    double cn = (std::fabs(phi1 - phi2) < 1e-6)
                    ? std::sin(phi1)
                    : std::log(std::cos(phi1) / std::cos(phi2)) /
                          std::log(std::tan(PI4 + phi2 / 2) / std::tan(PI4 + phi1 / 2));
    double A = std::cos(phi1) * std::pow(std::tan(PI4 + phi1 / 2), cn);
    mapf.resize((size_t)g.nx * g.ny);
    for (size_t q = 0; q < mapf.size(); ++q) {
      double phi = cs->input.lat[q] * 0.01745329252;
      mapf[q] = A / (std::pow(std::tan(PI4 + phi / 2), cn) * std::cos(phi));
    }
  }
  build_metric(g, cfg, cs->file_mode ? &cs->input.h : nullptr,
               cs->file_mode ? &cs->input.fcor : nullptr, cs->file_mode ? &mapf : nullptr, &cs->m);
  if (!build_base(g, cfg, cs->m, cs->file_mode ? &cs->input : nullptr, &cs->b, err)) return false;
  bool qv_blob = cfg.real("qvbub_dq", 0) != 0;
  p.moisture = cs->b.has_moisture || qv_blob;
  if (!p.moisture) p.pd_moist = false;

  for (auto& f : cs->state) f.assign(g.npts(), 0.0);
  if (cs->file_mode) {
    // full fields -> perturbations on the C-grid (src/main.cpp:58-100)
    const InputData& in = cs->input;
    auto src = [&](const std::vector<double>& a, int i, int j, int k) {
      return a[((size_t)k * g.ny + j) * g.nx + i];
    };
    for (int k = 0; k < g.nz; ++k)
      for (int j = 0; j < g.ny; ++j) {
        for (int i = 0; i <= g.nx; ++i) {
          int il = i > 0 ? i - 1 : 0, ir = i < g.nx ? i : g.nx - 1;
          cs->state[0][g.idx(i, j, k)] = 0.5 * (src(in.u, il, j, k) + src(in.u, ir, j, k));
        }
        for (int i = 0; i < g.nx; ++i) {
          int jl = j > 0 ? j - 1 : 0;
          size_t c = g.idx(i, j, k);
          cs->state[1][c] = 0.5 * (src(in.v, i, jl, k) + src(in.v, i, j, k));
          cs->state[3][c] = src(in.th, i, j, k) - cs->b.thb[c];
          cs->state[4][c] = src(in.pi, i, j, k) - cs->b.pib[c];
          cs->state[5][c] = src(in.qv, i, j, k);
        }
      }
    ic_perturbation(g, cfg.real("ic_perturb", 0), (unsigned)cfg.integer("ens_seed", 0),
                    &cs->state[3]);
    cs->bdy.on = true;
    cs->bdy.width = cfg.integer("bdy_width", 8);
    cs->bdy.tau = cfg.real("bdy_tau", 600);
    cs->bdy.nudge_tau = cfg.real("nudge_tau", 0);
    if (cfg.str("physics", "none") == "simple") {
      // start = YYYYMMDDHH: day of year and UTC hour (src/main.cpp:364-377)
      const std::string& st = in.start;
      if (st.size() < 10) {
        *err = "input start time must be YYYYMMDDHH";
        return false;
      }
      int mo = std::atoi(st.substr(4, 2).c_str()), dd = std::atoi(st.substr(6, 2).c_str());
      int hh = std::atoi(st.substr(8, 2).c_str());
      static const int cum[12] = {0, 31, 59, 90, 120, 151, 181, 212, 243, 273, 304, 334};
      if (mo < 1 || mo > 12) {
        *err = "input start month out of range";
        return false;
      }
      cs->sfc.on = true;
      cs->sfc.doy = cum[mo - 1] + dd;
      cs->sfc.start_hour = hh;
      cs->sfc.nonlocal = cfg.str("pbl", "local") == "nonlocal";
    }
  } else {
    // idealised: bubble, base wind, base moisture, qv blob (src/main.cpp:379-382)
    double dth = cfg.real("bubble_dtheta", 0);
    if (dth != 0)
      ic_blob(g, cs->m, dth, cfg.real("bubble_xc", g.nx * g.dx / 2),
              cfg.real("bubble_yc", g.ny * g.dy / 2), cfg.real("bubble_zc", 2000),
              cfg.real("bubble_xr", 2000), cfg.real("bubble_yr", 2000), cfg.real("bubble_zr", 2000),
              &cs->state[3]);
    for (int k = 0; k < g.nz; ++k) {
      double ub = cs->b.ub[k + g.ng];
      if (ub == 0) continue;
      for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i <= g.nx; ++i) cs->state[0][g.idx(i, j, k)] = ub;
    }
    if (cs->b.has_moisture)
      for (int k = 0; k < g.nz; ++k)
        for (int j = 0; j < g.ny; ++j)
          for (int i = 0; i < g.nx; ++i) cs->state[5][g.idx(i, j, k)] = cs->b.qvb[g.idx(i, j, k)];
    double dq = cfg.real("qvbub_dq", 0);
    if (dq != 0)
      ic_blob(g, cs->m, dq, cfg.real("qvbub_xc", g.nx * g.dx / 4),
              cfg.real("qvbub_yc", g.ny * g.dy / 2), cfg.real("qvbub_zc", 2000),
              cfg.real("qvbub_xr", 2000), cfg.real("qvbub_yr", 1e9), cfg.real("qvbub_zr", 2000),
              &cs->state[5]);
  }
  return true;
}

}  // namespace wfe
