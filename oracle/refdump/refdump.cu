// Golden-vector dump driver -- test infrastructure, never shipped.
//
// Links the reference's own objects (built from its sources by oracle/Makefile)
// and drives them through their public C++ API (dynamics/kernels.hpp,
// dynamics/integrator.hpp, physics/*.hpp, core/*.hpp) to write FP64 (or FP32)
// snapshots that pin the CPU oracle and the CUDA path:
//
//   refdump <case.ini> <outdir> mode=run  [nsteps=N] [dump=1,2,5] [key=val...]
//       set-up exactly as src/main.cpp:261-383 (idealised cases only), then
//       Integrator::step N times; dumps metric, base state, initial state and
//       the state after each listed step.
//   refdump <case.ini> <outdir> mode=ops  [nsub=3] [key=val...]
//       deterministic synthetic state -> one call of every operator of the
//       kernel API (apply_bcs, compute_mass_fluxes, compute_divergence,
//       compute_tendencies, bdy_relax, precompute_acoustic_coef,
//       acoustic_substep, update_moisture_stage, kessler_step, SfcPBL).
//   refdump <case.ini> <outdir> mode=bench [warmup=W] [steps=K]
//       same set-up as mode=run, then times K Integrator::step calls with CUDA
//       events on the legacy default stream the reference launches on; prints
//       one line "refbench cells=<n> steps=<K> ms=<elapsed>".
//
// wind_profile=linear (u = wind_us * min(z/wind_zs, 1) + wind_offset, with z
// the cell-centre zeta clamped at 0, as the tanh profile of
// src/core/base_state.cpp:240-245 does) is not expressible in the reference;
// it is applied here after BaseState::build by overwriting the public host
// profile h_ub and the device profile DevProf::ub, so the reference code path
// itself is unchanged.
//
// Output: <outdir>/<name>.bin (little-endian float64, padded reference layout)
// and <outdir>/manifest.txt ("name count" per line).  The initial-condition
// helpers below restate src/main.cpp:28-195 (they live in an anonymous
// namespace there and cannot be linked); the unmodified wfe binary's step-0
// output pins them.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "core/base_state.hpp"
#include "core/config.hpp"
#include "core/field3d.hpp"
#include "core/grid.hpp"
#include "core/metric.hpp"
#include "core/thermo.hpp"
#include "dynamics/integrator.hpp"
#include "dynamics/kernels.hpp"
#include "physics/kessler.hpp"
#include "physics/surface.hpp"

using namespace wfe;

namespace {

struct Dumper {
  std::string dir;
  FILE* man = nullptr;
  explicit Dumper(const std::string& d) : dir(d) {
    std::filesystem::create_directories(dir);
    man = std::fopen((dir + "/manifest.txt").c_str(), "w");
    if (!man) {
      std::fprintf(stderr, "cannot write %s\n", dir.c_str());
      std::exit(1);
    }
  }
  ~Dumper() {
    if (man) std::fclose(man);
  }
  void host(const std::string& name, const std::vector<double>& v) {
    FILE* f = std::fopen((dir + "/" + name + ".bin").c_str(), "wb");
    std::fwrite(v.data(), sizeof(double), v.size(), f);
    std::fclose(f);
    std::fprintf(man, "%s %zu\n", name.c_str(), v.size());
  }
  void dev(const std::string& name, const real* d, size_t n) {
    std::vector<real> h(n);
    WFE_CUDA_CHECK(cudaMemcpy(h.data(), d, n * sizeof(real), cudaMemcpyDeviceToHost));
    std::vector<double> o(h.begin(), h.end());
    host(name, o);
  }
  void field(const std::string& name, const Field3D& f) { dev(name, f.d, f.n); }
  void state(const std::string& pre, const State& s) {
    field(pre + "_u", s.u);
    field(pre + "_v", s.v);
    field(pre + "_w", s.w);
    field(pre + "_thp", s.thp);
    field(pre + "_pip", s.pip);
    field(pre + "_qv", s.qv);
    field(pre + "_qc", s.qc);
    field(pre + "_qr", s.qr);
  }
};

// splitmix64 -> uniform [-1, 1)
double noise(uint64_t f, int i, int j, int k) {
  uint64_t z = (f * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)(i + 64) << 40) ^
               ((uint64_t)(j + 64) << 20) ^ (uint64_t)(k + 64);
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

// ---- idealised initial conditions (restated from src/main.cpp:28-54, 147-195)
void ic_bubble(const GDims& g, const Config& cfg, const Metric& metric, State& s) {
  real dth = cfg.get_real("bubble_dtheta", (real)0);
  if (dth == (real)0) return;
  real xc = cfg.get_real("bubble_xc", g.nx * g.dx / 2);
  real yc = cfg.get_real("bubble_yc", g.ny * g.dy / 2);
  real zc = cfg.get_real("bubble_zc", (real)2000);
  real xr = cfg.get_real("bubble_xr", (real)2000);
  real yr = cfg.get_real("bubble_yr", (real)2000);
  real zr = cfg.get_real("bubble_zr", (real)2000);
  std::vector<real> h(g.npts(), 0);
  const real pi = (real)3.14159265358979323846;
  for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) {
        real x = ((real)i + (real)0.5) * g.dx;
        real y = ((real)j + (real)0.5) * g.dy;
        real z = metric.z_at(g, i, j, metric.h_zeta_c[k + g.ng]);
        real rx = (x - xc) / xr, ry = (y - yc) / yr, rz = (z - zc) / zr;
        real r = std::sqrt(rx * rx + ry * ry + rz * rz);
        if (r < (real)1) {
          real c = std::cos(pi * r / 2);
          h[g.idx(i, j, k)] = dth * c * c;
        }
      }
  s.thp.upload(h.data());
}

void ic_wind(const GDims& g, const BaseState& base, State& s) {
  std::vector<real> h(g.npts(), 0);
  for (int k = 0; k < g.nz; ++k) {
    real ub = base.h_ub[k + g.ng];
    if (ub == (real)0) continue;
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i <= g.nx; ++i) h[g.idx(i, j, k)] = ub;
  }
  s.u.upload(h.data());
}

void ic_moisture(const GDims& g, const BaseState& base, State& s) {
  if (!base.has_moisture()) return;
  std::vector<real> h(g.npts(), 0);
  for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) h[g.idx(i, j, k)] = base.qvb_at(g, i, j, k);
  s.qv.upload(h.data());
}

void ic_qv_blob(const GDims& g, const Config& cfg, const Metric& metric, State& s) {
  real dq = cfg.get_real("qvbub_dq", (real)0);
  if (dq == (real)0) return;
  real xc = cfg.get_real("qvbub_xc", g.nx * g.dx / 4);
  real yc = cfg.get_real("qvbub_yc", g.ny * g.dy / 2);
  real zc = cfg.get_real("qvbub_zc", (real)2000);
  real xr = cfg.get_real("qvbub_xr", (real)2000);
  real yr = cfg.get_real("qvbub_yr", (real)1e9);
  real zr = cfg.get_real("qvbub_zr", (real)2000);
  std::vector<real> h(g.npts(), 0);
  const real pi = (real)3.14159265358979323846;
  for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) {
        real x = ((real)i + (real)0.5) * g.dx;
        real y = ((real)j + (real)0.5) * g.dy;
        real z = metric.z_at(g, i, j, metric.h_zeta_c[k + g.ng]);
        real rx = (x - xc) / xr, ry = (y - yc) / yr, rz = (z - zc) / zr;
        real r = std::sqrt(rx * rx + ry * ry + rz * rz);
        if (r < (real)1) {
          real c = std::cos(pi * r / 2);
          h[g.idx(i, j, k)] = dq * c * c;
        }
      }
  s.qv.upload(h.data());
}

// ---- synthetic operator inputs (ours; values only need to be deterministic)
void synth_state(const GDims& g, const BaseState& base, bool moist, uint64_t seed,
                 State& s) {
  size_t n = g.npts();
  std::vector<real> u(n), v(n), w(n), th(n), pi(n), qv(n, 0), qc(n, 0), qr(n, 0);
  const double tp = 6.283185307179586;
  for (int k = -g.ng; k < g.nz + 1 + g.ng; ++k)
    for (int j = -g.ng; j < g.ny + g.ng; ++j)
      for (int i = -g.ng; i < g.nx + g.ng; ++i) {
        size_t c = g.idx(i, j, k);
        double xi = (i + 0.5) / g.nx, yj = (j + 0.5) / g.ny, zk = (k + 0.5) / g.nz;
        u[c] = (real)(2.0 + 6.0 * std::sin(tp * xi + 1.3 * zk) * std::cos(tp * yj) +
                      2.0 * noise(seed + 1, i, j, k));
        v[c] = (real)(-1.0 + 5.0 * std::cos(tp * yj + 0.7 * zk) * std::sin(tp * xi + 0.4) +
                      2.0 * noise(seed + 2, i, j, k));
        w[c] = (real)(1.5 * std::sin(3.14159 * zk) * std::cos(tp * xi) * std::cos(tp * yj) +
                      0.5 * noise(seed + 3, i, j, k));
        double rr = (xi - 0.5) * (xi - 0.5) + (yj - 0.5) * (yj - 0.5) + (zk - 0.3) * (zk - 0.3);
        th[c] = (real)(1.5 * std::exp(-20.0 * rr) + 0.3 * noise(seed + 4, i, j, k));
        pi[c] = (real)(2e-4 * std::sin(tp * xi) * std::cos(tp * zk) +
                       1e-4 * noise(seed + 5, i, j, k));
        if (moist) {
          double qb = base.qvb_at(g, std::min(std::max(i, 0), g.nx - 1),
                                  std::min(std::max(j, 0), g.ny - 1),
                                  std::min(std::max(k, 0), g.nz - 1));
          qv[c] = (real)std::max(0.0, qb * (1.0 + 0.25 * noise(seed + 6, i, j, k)));
          qc[c] = (real)std::max(0.0, 1.2e-3 * noise(seed + 7, i, j, k) + 3e-4);
          qr[c] = (real)std::max(0.0, 2.0e-3 * noise(seed + 8, i, j, k) + 2e-4);
        }
      }
  s.u.upload(u.data());
  s.v.upload(v.data());
  s.w.upload(w.data());
  s.thp.upload(th.data());
  s.pip.upload(pi.data());
  s.qv.upload(qv.data());
  s.qc.upload(qc.data());
  s.qr.upload(qr.data());
}

std::set<int> parse_list(const std::string& s) {
  std::set<int> out;
  std::stringstream ss(s);
  std::string tok;
  while (std::getline(ss, tok, ','))
    if (!tok.empty()) out.insert(std::atoi(tok.c_str()));
  return out;
}

DynParams params_from(const Config& cfg) {  // src/main.cpp:284-298
  DynParams dp;
  dp.diff_K = cfg.get_real("diff_K", 0);
  dp.coriolis_f = cfg.get_real("coriolis_f", 0);
  dp.rayleigh_zd = cfg.get_real("rayleigh_zd", -1);
  dp.rayleigh_alpha = cfg.get_real("rayleigh_alpha", 0);
  dp.acoustic_ns = cfg.get_int("acoustic_ns", 6);
  dp.acoustic_beta = cfg.get_real("acoustic_beta", (real)0.2);
  dp.acoustic_smdiv = cfg.get_real("acoustic_smdiv", (real)0.1);
  dp.bc_x_open = cfg.get_str("bc_x", "periodic") == "open";
  dp.bc_y_open = cfg.get_str("bc_y", "periodic") == "open";
  dp.cstar = cfg.get_real("cstar", 30);
  dp.w_damping = cfg.get_str("w_damping", "off") == "on";
  dp.w_abort = cfg.get_real("w_abort", 150);
  dp.pd_moist = cfg.get_str("pd_moist", "off") == "on";
  dp.microphysics = cfg.get_str("microphysics", "on") == "on";
  return dp;
}

void dump_setup(Dumper& D, const GDims& g, const Metric& metric, const BaseState& base) {
  DevMetric m = metric.dev();
  size_t n1 = g.NZ, n2 = (size_t)g.NX * g.NY, n = g.npts();
  D.dev("m_zeta_w", m.zeta_w, n1);
  D.dev("m_zeta_c", m.zeta_c, n1);
  D.dev("m_dzeta_c", m.dzeta_c, n1);
  D.dev("m_dzeta_w", m.dzeta_w, n1);
  D.dev("m_h", m.h, n2);
  D.dev("m_hx", m.hx, n2);
  D.dev("m_hy", m.hy, n2);
  D.dev("m_hx_u", m.hx_u, n2);
  D.dev("m_hy_v", m.hy_v, n2);
  D.dev("m_jac", m.jac, n2);
  D.dev("m_fcor", m.fcor, n2);
  D.dev("m_mapf", m.mapf, n2);
  D.host("m_zt", {(double)m.zt});
  DevProf p = base.dev();
  D.dev("b_thb", p.thb, n);
  D.dev("b_pib", p.pib, n);
  D.dev("b_rhob", p.rhob, n);
  D.dev("b_dthbdz", p.dthbdz, n);
  D.dev("b_thbw", p.thbw, n);
  D.dev("b_rhobw", p.rhobw, n);
  D.dev("b_thvb", p.thvb, n);
  D.dev("b_thvbw", p.thvbw, n);
  D.dev("b_qvb", p.qvb, n);
  D.dev("b_ub", p.ub, n1);
  D.host("dims", {(double)g.nx, (double)g.ny, (double)g.nz, (double)g.ng, (double)g.NX,
                  (double)g.NY, (double)g.NZ, (double)g.dx, (double)g.dy, (double)g.dz});
}

// Straight-line shear profile (see header); returns false if not requested.
bool apply_linear_wind(const GDims& g, const Config& cfg, const Metric& metric,
                       BaseState& base) {
  if (cfg.get_str("wind_profile", "const") != "linear") return false;
  real us = cfg.get_real("wind_us", 25);
  real zs = cfg.get_real("wind_zs", 3000);
  real uoff = cfg.get_real("wind_offset", 0);
  for (int kk = 0; kk < g.NZ; ++kk) {
    double z = metric.h_zeta_c[kk];
    if (z < 0) z = 0;
    double f = z / (double)zs;
    if (f > 1) f = 1;
    base.h_ub[kk] = (real)(us * f + uoff);
  }
  WFE_CUDA_CHECK(cudaMemcpy(const_cast<real*>(base.dev().ub), base.h_ub.data(),
                            g.NZ * sizeof(real), cudaMemcpyHostToDevice));
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: refdump case.ini outdir [mode=run|ops] [key=val ...]\n");
    return 1;
  }
  Config cfg;
  if (!cfg.load(argv[1])) {
    std::fprintf(stderr, "cannot read %s\n", argv[1]);
    return 1;
  }
  for (int a = 3; a < argc; ++a) {
    std::string s = argv[a];
    size_t eq = s.find('=');
    if (eq != std::string::npos) cfg.set(s.substr(0, eq), s.substr(eq + 1));
  }
  std::string mode = cfg.get_str("mode", "run");
  int nx = cfg.get_int("nx", 100), ny = cfg.get_int("ny", 100), nz = cfg.get_int("nz", 50);
  real dx = cfg.get_real("dx", 200), dy = cfg.get_real("dy", 200), dz = cfg.get_real("dz", 200);
  real dt = cfg.get_real("dt", (real)0.25);
  GDims g = make_grid(nx, ny, nz, 3, dx, dy, dz);
  DynParams dp = params_from(cfg);

  Metric metric;
  metric.build(g, cfg);
  BaseState base;
  base.build(g, cfg, metric);
  apply_linear_wind(g, cfg, metric, base);
  bool qv_blob = cfg.get_real("qvbub_dq", 0) != (real)0;
  dp.moisture = base.has_moisture() || qv_blob;
  if (!dp.moisture) dp.pd_moist = false;

  if (mode == "bench") {
    Integrator integ;
    integ.init(g, base.dev(), metric.dev(), dp);
    ic_bubble(g, cfg, metric, integ.state());
    ic_wind(g, base, integ.state());
    ic_moisture(g, base, integ.state());
    ic_qv_blob(g, cfg, metric, integ.state());
    int warm = cfg.get_int("warmup", 3), steps = cfg.get_int("steps", 20);
    int step = 0;
    for (int w = 0; w < warm; ++w, ++step) integ.step(dt, step * dt);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    WFE_CUDA_CHECK(cudaDeviceSynchronize());
    cudaEventRecord(e0, 0);
    for (int s = 0; s < steps; ++s, ++step) integ.step(dt, step * dt);
    cudaEventRecord(e1, 0);
    WFE_CUDA_CHECK(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    std::printf("refbench cells=%lld steps=%d ms=%.6f\n", (long long)nx * ny * nz, steps,
                (double)ms);
    return 0;
  }

  Dumper D(argv[2]);
  dump_setup(D, g, metric, base);
  D.host("params", {(double)dp.diff_K, (double)dp.coriolis_f, (double)dp.coriolis_use_ub,
                    (double)dp.rayleigh_zd, (double)dp.rayleigh_alpha,
                    (double)dp.acoustic_ns, (double)dp.acoustic_beta,
                    (double)dp.acoustic_smdiv, (double)dp.bc_x_open, (double)dp.bc_y_open,
                    (double)dp.cstar, (double)dp.moisture, (double)dp.microphysics,
                    (double)dp.pd_moist, (double)dp.w_damping, (double)dt});
  size_t n = g.npts();

  if (mode == "run") {
    Integrator integ;
    integ.init(g, base.dev(), metric.dev(), dp);
    ic_bubble(g, cfg, metric, integ.state());
    ic_wind(g, base, integ.state());
    ic_moisture(g, base, integ.state());
    ic_qv_blob(g, cfg, metric, integ.state());
    D.state("s0", integ.state());
    int nsteps = cfg.get_int("nsteps", 5);
    std::set<int> dumps = parse_list(cfg.get_str("dump", "1,2,5"));
    for (int step = 1; step <= nsteps; ++step) {
      integ.step(dt, (step - 1) * dt);
      if (dumps.count(step)) {
        char pre[32];
        std::snprintf(pre, sizeof(pre), "s%d", step);
        D.state(pre, integ.state());
        if (dp.moisture) D.field(std::string(pre) + "_rain", integ.rain());
      }
    }
    WFE_CUDA_CHECK(cudaDeviceSynchronize());
    std::printf("refdump run: %d steps ok\n", nsteps);
    return 0;
  }

  // ------------------------------------------------------------- mode=ops
  uint64_t seed = (uint64_t)cfg.get_int("seed", 7);
  State s, tend, work, s2;
  s.alloc(n);
  tend.alloc(n);
  work.alloc(n);
  s2.alloc(n);
  synth_state(g, base, dp.moisture, seed, s);
  D.state("in", s);
  apply_bcs(g, dp, s);
  D.state("bc", s);

  Field3D mfx, mfy, mfz, div, piprev, scratch;
  mfx.alloc(n);
  mfy.alloc(n);
  mfz.alloc(n);
  div.alloc(n);
  piprev.alloc(n);
  scratch.alloc(n);
  compute_mass_fluxes(g, base.dev(), metric.dev(), s, mfx, mfy, mfz);
  compute_divergence(g, metric.dev(), mfx, mfy, mfz, div);
  D.field("mfx", mfx);
  D.field("mfy", mfy);
  D.field("mfz", mfz);
  D.field("div", div);
  PDScratch pd;
  if (dp.pd_moist) pd.alloc(n);
  compute_tendencies(g, base.dev(), metric.dev(), dp, dt, s, mfx, mfy, mfz, div, tend,
                     dp.pd_moist ? &pd : nullptr);
  D.state("tend", tend);

  // Davies relaxation onto synthetic targets
  if (cfg.get_int("bdy", 0)) {
    Field3D lo[5], hi[5], wgt;
    std::vector<real> hb(n);
    for (int vv = 0; vv < 5; ++vv) {
      lo[vv].alloc(n);
      hi[vv].alloc(n);
      for (int side = 0; side < 2; ++side) {
        for (size_t c = 0; c < n; ++c)
          hb[c] = (real)((vv == 4 ? 1e-3 : (vv == 3 ? 1e-4 : 1.0)) *
                         noise(seed + 20 + 2 * vv + side, (int)(c % 977), (int)(c / 977), 3));
        (side ? hi[vv] : lo[vv]).upload(hb.data());
      }
    }
    wgt.alloc((size_t)g.NX * g.NY);
    std::vector<real> w2((size_t)g.NX * g.NY, 0);
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i) {
        int dist = std::min(std::min(i, g.nx - 1 - i), std::min(j, g.ny - 1 - j));
        w2[(size_t)(j + g.ng) * g.NX + (i + g.ng)] =
            dist < 3 ? (real)(1.0 / 600.0 / (1 + dist)) : (real)(j % 3 == 0 ? 1e-4 : 0.0);
      }
    wgt.upload(w2.data());
    for (int vv = 0; vv < 5; ++vv) {
      D.field("bdy_lo" + std::to_string(vv), lo[vv]);
      D.field("bdy_hi" + std::to_string(vv), hi[vv]);
    }
    D.field("bdy_wgt", wgt);
    bdy_relax(g, s, lo, hi, (real)0.3, wgt, tend);
    D.state("tendb", tend);
  }

  AcousticCoef ac;
  precompute_acoustic_coef(g, base.dev(), metric.dev(), ac, scratch);
  D.field("ac_rtjx", ac.rtjx);
  D.field("ac_rtjy", ac.rtjy);
  D.field("ac_kt3", ac.kt3);
  D.field("ac_aw", ac.aw);

  // acoustic substeps from the bc-filled state (what Integrator::step does at a stage)
  int nsub = cfg.get_int("nsub", 3);
  real dtau = cfg.get_real("dtau", dt / 6);
  work.copy_from(s);
  piprev.copy_from(s.pip);
  for (int t = 0; t < nsub; ++t) {
    acoustic_substep(g, base.dev(), metric.dev(), dp, dtau, work, tend, piprev, ac);
    if (t == 0) {
      D.state("ac1", work);
      D.field("ac1_piprev", piprev);
    }
  }
  D.state("acn", work);
  D.field("acn_piprev", piprev);
  if (dp.moisture) {
    update_moisture_stage(s, tend, dt, work);
    D.state("mst", work);

    // Kessler on the bc-filled synthetic moist state
    s2.copy_from(s);
    Field3D rain;
    rain.alloc((size_t)g.NX * g.NY);
    kessler_step(g, base.dev(), metric.dev(), dt, s2, rain);
    D.state("kes", s2);
    D.field("kes_rain", rain);

    // Surface layer + PBL + soil + radiation on the same state
    if (cfg.get_int("sfc", 1)) {
      InputData in;
      size_t n2i = (size_t)g.nx * g.ny;
      in.tsk.resize(n2i);
      in.land.resize(n2i);
      in.lat.resize(n2i);
      in.lon.resize(n2i);
      in.soilw.resize(n2i);
      for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx; ++i) {
          size_t c = (size_t)j * g.nx + i;
          in.tsk[c] = (real)(295.0 + 8.0 * noise(seed + 30, i, j, 0));
          in.land[c] = (real)(((i / 3 + j / 2) % 3) != 0 ? 1.0 : 0.0);
          in.lat[c] = (real)(36.0 + 6.0 * (j + 0.5) / g.ny);
          in.lon[c] = (real)(27.0 + 15.0 * (i + 0.5) / g.nx);
          in.soilw[c] = (real)(0.22 + 0.18 * noise(seed + 31, i, j, 0));
        }
      std::vector<double> vin;
      for (auto* vv : {&in.tsk, &in.land, &in.lat, &in.lon, &in.soilw})
        for (real x : *vv) vin.push_back((double)x);
      D.host("sfc_in", vin);
      real hour = cfg.get_real("sfc_hour", 9), tsec = cfg.get_real("sfc_t", 1800);
      int doy = cfg.get_int("sfc_doy", 172);
      for (int rep = 0; rep < 2; ++rep) {
        SfcPBL phys;
        State s3;
        s3.alloc(n);
        s3.copy_from(s);
        phys.init(g, in, hour, doy, rep == 0);
        phys.step(g, base.dev(), metric.dev(), dt, tsec, s3);
        phys.step(g, base.dev(), metric.dev(), dt, tsec + dt, s3);  // soil memory
        std::string pre = rep == 0 ? "sfc" : "sfc2";
        D.state(pre, s3);
        D.field(pre + "_tsk", phys.tsk());
        D.field(pre + "_pblh", phys.pblh());
        D.field(pre + "_t2m", phys.t2m());
        D.field(pre + "_u10", phys.u10());
        phys.release();
      }
    }
  }
  WFE_CUDA_CHECK(cudaDeviceSynchronize());
  std::printf("refdump ops: ok\n");
  return 0;
}
