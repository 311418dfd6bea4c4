// Precision-agnostic interface of a wfe_b200 model instance (one case on one
// GPU).  ModelT<R> in model.cu implements it for float and double.
#pragma once

#include <functional>
#include <string>
#include <utility>
#include <vector>

#include "setup.hpp"

namespace wfe {

// ROLE_LIN: the tangent-linear / adjoint field of the time-n state (Lin)
enum Role { ROLE_STATE = 0, ROLE_TEND = 1, ROLE_WORK = 2, ROLE_PIPREV = 3, ROLE_LIN = 4 };

// One launch of a step recorded instead of issued: its kind (kernels.cuh
// Kind) and argument block.
struct Rec {
  int kind;
  std::vector<unsigned char> args;
};
enum Field2D { F2_RAIN = 0, F2_TSK = 1, F2_PBLH = 2, F2_T2M = 3, F2_U10 = 4, F2_WGT = 5 };

class Model {
 public:
  virtual ~Model() = default;
  // nullptr on failure with *err set
  static Model* create(const CaseSetup& cs, bool fp64, int device, std::string* err);

  virtual const RefGrid& grid() const = 0;
  virtual bool fp64() const = 0;
  const std::string& error() const { return err_; }

  // field transfer in the reference padded layout (NX*NY*NZ doubles)
  virtual int upload(int role, int field, const double* ref_padded) = 0;
  virtual int download(int role, int field, double* ref_padded) = 0;
  // 2D surface fields in the reference padded 2D layout (NX*NY doubles)
  virtual int download2d(int which, double* ref_padded2d) = 0;
  virtual int upload2d(int which, const double* ref_padded2d) = 0;
  // interior (Writer layout) transfers straight between the device and a host
  // buffer of float (dtype_f32) or double, without an FP64 padded copy
  virtual int download_interior(int role, int field, void* host, bool dtype_f32) = 0;
  virtual int upload_interior(int role, int field, const void* host, bool dtype_f32) = 0;
  // raw device-layout transfers of the state (fast path, same precision)
  virtual int upload_state_raw(int field, const void* host_pitched) = 0;
  virtual int download_state_raw(int field, void* host_pitched) = 0;
  virtual size_t pitched_count() const = 0;
  virtual void pitched_dims(int* px, int* py, int* pz) const = 0;

  // Asynchronous snapshot: fields 0..7 (state) and 100 + Field2D (2D fields)
  // packed on the device in step order, copied to the host buffers on a copy
  // stream; the buffers are complete after snapshot_wait (which a new
  // snapshot_begin also does first)
  virtual int snapshot_begin(int n, const int* fields, void* const* host, bool f32) = 0;
  virtual int snapshot_wait() = 0;

  // Integrator::step (src/dynamics/integrator.cpp:71-111): direct launches
  virtual int step(double dt, double t) = 0;
  // nsteps large steps replayed from captured CUDA graphs
  virtual int run(int nsteps, double dt, double t0) = 0;
  virtual int sync() = 0;
  virtual int absmax(int field, float* out) = 0;
  // the same, split: begin enqueues the reduction and its copy into page-locked
  // slot `slot` (0 or 1) on the model's stream; end waits for that slot
  virtual int absmax_begin(int field, int slot) = 0;
  virtual int absmax_end(int slot, float* out) = 0;
  virtual int dry_mass(double* out) = 0;

  // boundary relaxation targets, reference padded layout; t_lo < t_hi
  virtual int set_boundary(const double* const lo[5], const double* const hi[5],
                           const double* wgt_padded2d, double t_lo, double t_hi) = 0;
  virtual int set_boundary_hi(const double* const hi[5], double t_lo, double t_hi) = 0;
  // relaxation off again (targets and weights kept, unused)
  virtual int clear_boundary() = 0;
  virtual int enable_physics(const double* tsk, const double* land, const double* lat,
                             const double* lon, const double* soilw, double start_hour, int doy,
                             bool nonlocal) = 0;

  // operator-level API (src/dynamics/kernels.hpp, physics/*.hpp)
  virtual int op_apply_bcs() = 0;
  virtual int op_tendencies(double dt, double t) = 0;
  virtual int op_acoustic(double dtau, int nsub) = 0;
  virtual int op_moisture_stage(double dt) = 0;
  virtual int op_kessler(double dt) = 0;
  virtual int op_sfc(double dt, double t) = 0;

  // launches made by the last step()/run() call (device kernels only)
  virtual long launches_per_step() const = 0;
  // nsteps graph-replayed steps timed with CUDA events on the model's stream
  virtual int time_run(int nsteps, double dt, double t0, double* ms) = 0;
  // one direct step with CUDA events around every launch: per-kernel totals
  virtual int kernel_times(double dt, double t, std::vector<std::string>* names,
                           std::vector<double>* ms, std::vector<int>* counts) = 0;

  // ------------------------------------- access for batched / linearised steps
  // the launches of one step from the current rotation phase, not issued
  virtual int record_step(double dt, std::vector<Rec>* out) = 0;
  virtual void rotate() = 0;  // what a step does to the buffer roles
  virtual int phase() const = 0;
  // state-like device buffers (states, tendencies, mass fluxes, acoustic
  // scratch): base pointer and element count
  virtual std::vector<std::pair<void*, size_t>> state_buffers() const = 0;
  virtual void* state_field(int field) = 0;  // time-n device buffer of a field
  virtual void* stream_handle() const = 0;
  // a recorded forward u, v (column) launch through the tuned variant: the
  // argument is the launch's AcouArgs
  virtual int replay_uv(const void* args) = 0;
  virtual int replay_column(const void* args) = 0;
  // tendency, acoustic column and u, v variants (-1 before tuning), and
  // whether the column coefficients have per-level tables
  virtual void variants(int out[4]) const = 0;
  // buffer -> linearised buffer map behind ROLE_LIN (empty function: none)
  virtual void set_lin_map(std::function<void*(const void*)> map) = 0;
  // whether the step is one the linearised kernels cover (why not, if not)
  virtual bool linearisable(std::string* why) const = 0;

 protected:
  std::string err_;
};

// Tangent-linear and adjoint runs of a Model's dry dynamics (lin_host.cu).
// The linearised field of the time-n state is the model's ROLE_LIN field.
class Lin {
 public:
  virtual ~Lin() = default;
  static Lin* create(Model* m, std::string* err);
  const std::string& error() const { return err_; }
  // forward and tangent together: state x0 -> xN, ROLE_LIN dx0 -> dxN
  virtual int tl_run(int nsteps, double dt, double t0) = 0;
  // state x0 -> xN (forward with checkpoints every `every` steps), then the
  // adjoint sweep: ROLE_LIN dJ/dxN on entry -> dJ/dx0 on exit
  virtual int ad_run(int nsteps, double dt, double t0, int every) = 0;
  virtual int zero() = 0;  // every linearised buffer to 0

 protected:
  std::string err_;
};

// Members of uneven sizes advancing together: every launch of the RK3 step is
// one batched launch over a member x block work list (kernels.cuh: Batch),
// and the whole step with its acoustic substeps is captured in one CUDA graph
// per rotation phase.  Members are Model instances of one precision on one
// device with the same physics switches and substep count; they stay owned by
// the caller and must outlive the ensemble.  Member state is read and written
// through the members; their streams are ordered after the ensemble's work.
class Ensemble {
 public:
  virtual ~Ensemble() = default;
  // nullptr on failure with *err set
  static Ensemble* create(const std::vector<Model*>& members, std::string* err);
  const std::string& error() const { return err_; }

  // nsteps large steps of every member, t0 the time of the first
  virtual int run(int nsteps, double dt, double t0) = 0;
  // one step with direct batched launches (no graph)
  virtual int step(double dt, double t) = 0;
  virtual int sync() = 0;
  virtual int time_run(int nsteps, double dt, double t0, double* ms) = 0;
  virtual long launches_per_step() const = 0;
  // tuned variants: tendencies variant, acoustic column shape, persistent grid
  virtual void variants(int* tend, int* column, int* persist) const = 0;

 protected:
  std::string err_;
};

}  // namespace wfe
