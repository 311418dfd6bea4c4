// Reference-surface shim: the hydrostatic base state of
// src/core/base_state.hpp, read from the library's host set-up that
// Metric::build made (the profile tables of file mode come from the same
// input directory there).
#pragma once

#include <memory>
#include <vector>

#include "core/config.hpp"
#include "core/field3d.hpp"
#include "core/grid.hpp"
#include "core/metric.hpp"
#include "core/precision.hpp"

namespace wfe {

struct DevProf {
  const real *thb = nullptr, *pib = nullptr, *rhob = nullptr, *dthbdz = nullptr;
  const real *thbw = nullptr, *rhobw = nullptr, *thvb = nullptr, *thvbw = nullptr;
  const real *qvb = nullptr, *ub = nullptr;
};

struct ProfileTables {
  const std::vector<real>* z = nullptr;
  const std::vector<real>* th = nullptr;
  const std::vector<real>* qv = nullptr;
  const std::vector<real>* u = nullptr;
};

class BaseState {
 public:
  void build(const GDims& g, const Config& cfg, const Metric& metric,
             const ProfileTables* tables = nullptr);
  void release();
  DevProf dev() const { return DevProf{}; }

  std::vector<real> h_ub;
  std::vector<real> h_thb3, h_pib3;
  bool has_moisture() const { return has_moisture_; }
  real qvb_at(const GDims& g, int i, int j, int k) const {
    return h_qvb_.empty() ? (real)0 : h_qvb_[g.idx(i, j, k)];
  }

 private:
  std::shared_ptr<shim::Setup> setup_;
  std::vector<real> h_qvb_;
  bool has_moisture_ = false;
};

}  // namespace wfe
