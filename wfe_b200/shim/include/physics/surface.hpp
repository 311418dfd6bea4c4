// Reference-surface shim: the surface layer / PBL / soil / radiation columns
// of src/physics/surface.hpp.  The library's context sets the physics up
// from the case (physics = simple, pbl, the input's surface fields and start
// time) and runs it inside each step; after Integrator::set_physics the 2D
// diagnostics below are views of the context's fields.
#pragma once

#include "core/base_state.hpp"
#include "core/field3d.hpp"
#include "core/grid.hpp"
#include "core/metric.hpp"
#include "dynamics/state.hpp"
#include "io/input.hpp"

namespace wfe {

class SfcPBL {
 public:
  void init(const GDims& g, const InputData& in, real start_hour_utc, int doy, bool nonlocal);
  void release() {}
  // the context steps the physics with the dynamics (Integrator::step)
  void step(const GDims&, const DevProf&, const DevMetric&, real, real, State&) {}

  const Field3D& tsk() const { return tsk_; }
  const Field3D& pblh() const { return pblh_; }
  const Field3D& t2m() const { return t2m_; }
  const Field3D& u10() const { return u10_; }

  void bind(wfe_ctx* c, size_t n2);

 private:
  Field3D tsk_, pblh_, t2m_, u10_;
  real start_hour_ = 0;
  int doy_ = 1;
  bool nonlocal_ = false;
};

}  // namespace wfe
