// Reference-surface shim: the RK3 integrator of src/dynamics/integrator.hpp
// on a wfe_b200 context.  init() builds the device context from the
// configuration Metric::build recorded, with the DynParams as overrides;
// step() is one large step of the library (replayed from its captured CUDA
// graphs, asynchronous until the next transfer or field_absmax); state()
// and rain() are views of the context's fields.
#pragma once

#include "core/base_state.hpp"
#include "core/field3d.hpp"
#include "core/grid.hpp"
#include "core/metric.hpp"
#include "dynamics/boundary.hpp"
#include "dynamics/kernels.hpp"
#include "dynamics/params.hpp"
#include "dynamics/state.hpp"

namespace wfe {

class SfcPBL;

class Integrator {
 public:
  Integrator() = default;
  Integrator(const Integrator&) = delete;
  Integrator& operator=(const Integrator&) = delete;
  ~Integrator();

  void init(const GDims& g, const DevProf& prof, const DevMetric& m, const DynParams& dp);
  void step(real dt, real t);
  void print_profile() const;

  State& state() { return s_n_; }
  const Field3D& rain() const { return rain_; }
  void set_boundary(BdyManager* bdy) { bdy_ = bdy; }
  void set_physics(SfcPBL* phys);

  wfe_ctx* context() const { return ctx_; }

 private:
  GDims g_{};
  wfe_ctx* ctx_ = nullptr;
  State s_n_;
  Field3D rain_;
  BdyManager* bdy_ = nullptr;
  SfcPBL* phys_ = nullptr;
  long steps_ = 0;
};

}  // namespace wfe
