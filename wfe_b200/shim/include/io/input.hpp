// Reference-surface shim: the prep-format real-data input of
// src/io/input.hpp (wfe_input.ini + wfe_init.bin + wfe_bdy_FFF.bin, float32
// interior arrays), read on the host for the driver's initial conditions.
#pragma once

#include <string>
#include <vector>

#include "core/grid.hpp"
#include "core/precision.hpp"

namespace wfe {

class InputData {
 public:
  bool load(const GDims& g, const std::string& dir);
  // boundary file idx: u, v, th, pi, qv (interior)
  bool load_bdy(const GDims& g, int idx, std::vector<real> fields[5]) const;

  std::vector<real> prof_z, prof_th, prof_qv, prof_u;
  std::vector<real> h, fcor;
  std::vector<real> tsk, land, lat, lon, soilw;
  std::vector<real> u, v, th, pi, qv;
  real bdy_interval = 10800;
  int n_bdy = 0;
  std::string start;

 private:
  std::string dir_;
};

}  // namespace wfe
