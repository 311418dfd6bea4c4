// Reference-surface shim: the snapshot writer of src/io/writer.hpp --
// meta.json, float32 interior snapshots <var>_<step>.bin, 2D fields and
// static fields -- reading the context's fields through the C ABI.
#pragma once

#include <string>
#include <vector>

#include "core/field3d.hpp"
#include "core/grid.hpp"
#include "dynamics/state.hpp"

namespace wfe {

class Writer {
 public:
  void init(const GDims& g, const std::string& out_dir, real dt, bool moisture, bool has_tsk);
  void write(const State& s, int step, real t);
  void write_field2d(const Field3D& f, const char* name, int step);
  void write_static(const char* name, const std::vector<float>& data);

 private:
  void write_field(const Field3D& f, const char* name, int step, int nzlev);

  GDims g_{};
  std::string dir_;
  bool moist_ = false;
  std::vector<float> out_;
};

}  // namespace wfe
