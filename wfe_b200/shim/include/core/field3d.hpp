// Reference-surface shim: a field of the reference's Field3D surface
// (src/core/field3d.hpp), as a view of one field of a wfe_b200 context.
// The library keeps its fields in its own pitched device layout, so there
// is no device pointer here (d stays null); upload() and download() move
// the reference's padded layout (NX*NY*NZ values, or NX*NY for the 2D
// fields) through the C ABI with the precision of `real`.
#pragma once

#include <cstddef>

#include "core/cuda_check.hpp"
#include "core/precision.hpp"
#include "wfe_b200.h"

namespace wfe {

struct Field3D {
  real* d = nullptr;
  size_t n = 0;
  // the context field this view reads and writes: a prognostic (field >= 0,
  // role WFE_ROLE_*) or a 2D field (plane = WFE_2D_*)
  wfe_ctx* ctx = nullptr;
  int role = WFE_ROLE_STATE;
  int field = -1;
  int plane = -1;

  Field3D() = default;
  Field3D(const Field3D&) = delete;
  Field3D& operator=(const Field3D&) = delete;

  void bind_field(wfe_ctx* c, int r, int f, size_t count) {
    ctx = c, role = r, field = f, plane = -1, n = count;
  }
  void bind_plane(wfe_ctx* c, int which, size_t count) {
    ctx = c, field = -1, plane = which, n = count;
  }
  void upload(const real* h);
  void download(real* h) const;
};

}  // namespace wfe
