// Reference-surface shim: the Gal-Chen metric of src/core/metric.hpp.
// Metric::build hands the configuration to the library's host set-up (a
// wfe_b200 context without a device), which computes the metric -- and the
// base state BaseState::build reads -- exactly as the reference does; the
// host copies below come from it.  The terrain, Coriolis and map-factor
// arrays of the prep input are read by the library itself from the same
// input directory, so the pointers passed here are not needed.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "core/config.hpp"
#include "core/grid.hpp"
#include "core/precision.hpp"

namespace wfe {

namespace shim {
struct Setup;  // the host-only context and the configuration it was built from
}

// The reference's by-value metric block.  The library owns the device
// metric, so the pointers stay null; `setup` carries the set-up to
// Integrator::init.
struct DevMetric {
  const real *zeta_w = nullptr, *zeta_c = nullptr, *dzeta_c = nullptr, *dzeta_w = nullptr;
  const real *h = nullptr, *hx = nullptr, *hy = nullptr, *hx_u = nullptr, *hy_v = nullptr;
  const real *jac = nullptr, *fcor = nullptr, *mapf = nullptr;
  real zt = 0;
  const shim::Setup* setup = nullptr;
};

inline size_t idx2(const GDims& g, int i, int j) {
  return (size_t)(j + g.ng) * g.NX + (size_t)(i + g.ng);
}

class Metric {
 public:
  void build(const GDims& g, const Config& cfg, const std::vector<real>* h_file = nullptr,
             const std::vector<real>* fcor_file = nullptr,
             const std::vector<real>* mapf_file = nullptr);
  void release();
  DevMetric dev() const;

  real zt() const { return zt_; }
  std::vector<real> h_zeta_w, h_zeta_c, h_h, h_jac;
  real z_at(const GDims& g, int i, int j, real zeta) const {
    real hh = h_h[idx2(g, i, j)];
    return hh + zeta * (zt_ - hh) / zt_;
  }
  const std::shared_ptr<shim::Setup>& setup() const { return setup_; }

 private:
  std::shared_ptr<shim::Setup> setup_;
  real zt_ = 0;
};

}  // namespace wfe
