// Reference-surface shim: the prognostic state of src/dynamics/state.hpp as
// views of a context's eight state fields.
#pragma once

#include "core/field3d.hpp"

namespace wfe {

struct State {
  Field3D u, v, w, thp, pip, qv, qc, qr;

  void bind(wfe_ctx* c, int role, size_t n) {
    Field3D* f[8] = {&u, &v, &w, &thp, &pip, &qv, &qc, &qr};
    for (int q = 0; q < 8; ++q) f[q]->bind_field(c, role, q, n);
  }
};

}  // namespace wfe
