// Host-side case set-up of wfe_b200, mirroring the reference's drop-in
// surface: the .ini case configs (src/core/config.cpp), the Gal-Chen metric
// (src/core/metric.cpp), the hydrostatic base state (src/core/base_state.cpp),
// the idealised and file-mode initial conditions (src/main.cpp:28-195,
// 313-383), the prep-format input reader (src/io/input.cpp) and the Davies
// weights (src/dynamics/boundary.cpp:24-42).  Everything here is computed in
// FP64 on the reference's padded layout (NX = nx + 6, ng = 3) and converted to
// the device layout by the model.
#pragma once

#include <map>
#include <set>
#include <string>
#include <vector>

namespace wfe {

class Config {
 public:
  bool load(const std::string& path);
  bool load_text(const std::string& text);
  void set(const std::string& k, const std::string& v) { kv_[k] = v; }
  bool has(const std::string& k) const { return kv_.count(k) > 0; }
  double real(const std::string& k, double def) const;
  int integer(const std::string& k, int def) const;
  std::string str(const std::string& k, const std::string& def) const;
  std::vector<std::string> unused() const;
  const std::map<std::string, std::string>& raw() const { return kv_; }

 private:
  std::map<std::string, std::string> kv_;
  mutable std::set<std::string> used_;
};

// Reference padded grid (src/core/grid.hpp:22-36).
struct RefGrid {
  int nx, ny, nz, ng, NX, NY, NZ;
  double dx, dy, dz;
  size_t idx(int i, int j, int k) const {
    return ((size_t)(k + ng) * NY + (j + ng)) * NX + (i + ng);
  }
  size_t idx2(int i, int j) const { return (size_t)(j + ng) * NX + (i + ng); }
  size_t npts() const { return (size_t)NX * NY * NZ; }
  size_t n2() const { return (size_t)NX * NY; }
};
RefGrid make_ref_grid(int nx, int ny, int nz, double dx, double dy, double dz);

struct HostParams {  // src/dynamics/params.hpp:8-25
  double diff_K = 0, coriolis_f = 0;
  bool coriolis_use_ub = true;
  double rayleigh_zd = -1, rayleigh_alpha = 0;
  int acoustic_ns = 6;
  double acoustic_beta = 0.2, acoustic_smdiv = 0.1;
  bool bc_x_open = false, bc_y_open = false;
  double cstar = 30;
  bool moisture = false, microphysics = true, pd_moist = false, w_damping = false;
  double w_abort = 150;
};

// prep-format real-data input (src/io/input.cpp:19-73)
struct InputData {
  std::vector<double> prof_z, prof_th, prof_qv, prof_u;
  std::vector<double> h, fcor, tsk, land, lat, lon, soilw;  // ny*nx
  std::vector<double> u, v, th, pi, qv;                     // nz*ny*nx
  double bdy_interval = 10800;
  int n_bdy = 0;
  std::string start, dir;
  bool load(const RefGrid& g, const std::string& dir, std::string* err);
  bool load_bdy(const RefGrid& g, int idx, std::vector<double> f[5], std::string* err) const;
};

struct HostMetric {
  std::vector<double> zeta_w, zeta_c, dzeta_c, dzeta_w;       // NZ
  std::vector<double> h, hx, hy, hx_u, hy_v, jac, fcor, mapf;  // NX*NY
  double zt = 0;
};

struct HostBase {
  std::vector<double> thb, pib, rhob, dthbdz, thbw, rhobw, thvb, thvbw, qvb;  // npts
  std::vector<double> ub;                                                     // NZ
  bool has_moisture = false;
};

struct SurfaceInit {  // physics=simple (src/main.cpp:364-377)
  bool on = false;
  bool nonlocal = false;
  double start_hour = 0;
  int doy = 1;
};

struct BoundaryInit {  // BdyManager::init (src/dynamics/boundary.cpp:9-42)
  bool on = false;
  int width = 8;
  double tau = 600, nudge_tau = 0;
};

// A fully set-up case: grid, parameters, metric, base state, the initial
// prognostic state (8 fields, padded reference layout) and run controls.
struct CaseSetup {
  Config cfg;
  RefGrid g{};
  HostParams p;
  HostMetric m;
  HostBase b;
  std::vector<double> state[8];  // u v w thp pip qv qc qr
  double dt = 0.25, t_end = 1000, out_every = 100, diag_every = 10;
  std::string out_dir;
  bool file_mode = false;
  InputData input;
  SurfaceInit sfc;
  BoundaryInit bdy;
};

// Builds everything src/main.cpp builds before its time loop.  Returns false
// with a message on a config or input error (the reference exits with 1).
bool setup_case(const Config& cfg, CaseSetup* cs, std::string* err);

void build_metric(const RefGrid& g, const Config& cfg, const std::vector<double>* h_file,
                  const std::vector<double>* fcor_file, const std::vector<double>* mapf_file,
                  HostMetric* m);
bool build_base(const RefGrid& g, const Config& cfg, const HostMetric& m,
                const InputData* tables, HostBase* b, std::string* err);
void bdy_weights(const RefGrid& g, const HostParams& p, int width, double tau, double nudge_tau,
                 std::vector<double>* wgt);
// boundary file idx converted to padded perturbation targets (boundary.cpp:51-81)
bool bdy_targets(const CaseSetup& cs, int idx, std::vector<double> out[5], std::string* err);

}  // namespace wfe
