// Reference-surface shim: the dynamics parameters of
// src/dynamics/params.hpp.  Integrator::init passes each of them to the
// library as a configuration override, so a driver that changes them after
// reading the case is honoured.
#pragma once

#include "core/precision.hpp"

namespace wfe {

struct DynParams {
  real diff_K = 0;
  real coriolis_f = 0;
  bool coriolis_use_ub = true;
  real rayleigh_zd = -1;
  real rayleigh_alpha = 0;
  int acoustic_ns = 6;
  real acoustic_beta = (real)0.2;
  real acoustic_smdiv = (real)0.1;
  bool bc_x_open = false;
  bool bc_y_open = false;
  real cstar = 30;
  bool moisture = false;
  bool microphysics = true;
  bool pd_moist = false;
  bool w_damping = false;
  real w_abort = 150;
};

}  // namespace wfe
