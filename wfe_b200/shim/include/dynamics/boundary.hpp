// Reference-surface shim: the Davies boundary manager of
// src/dynamics/boundary.hpp.  The library's context reads the boundary
// files of the case's input directory itself and switches them at
// bdy_interval as BdyManager::update does, with the weights the same
// configuration keys give (bdy_width, bdy_tau, nudge_tau); this object
// records the driver's set-up and keeps the reference's accessors.
#pragma once

#include <vector>

#include "core/field3d.hpp"
#include "core/grid.hpp"
#include "dynamics/params.hpp"
#include "io/input.hpp"

namespace wfe {

class BdyManager {
 public:
  void init(const GDims& g, const DynParams& dp, const InputData* input,
            const std::vector<real>& thb3, const std::vector<real>& pib3, int bdy_width,
            real bdy_tau, real nudge_tau);
  void update(real t);
  real tfrac(real t) const;
  bool active() const { return input_ != nullptr; }

  real t_lo_ = 0, t_hi_ = 0;

 private:
  const InputData* input_ = nullptr;
  int width_ = 8;
  real tau_ = 600, nudge_tau_ = 0;
};

}  // namespace wfe
