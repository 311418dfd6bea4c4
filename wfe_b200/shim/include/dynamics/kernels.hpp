// Reference-surface shim: the part of src/dynamics/kernels.hpp a driver
// calls between steps.  The operators themselves run inside the library
// (wfe_step; operator by operator through wfe_op_* of include/wfe_b200.h).
#pragma once

#include "core/field3d.hpp"
#include "core/grid.hpp"
#include "dynamics/params.hpp"
#include "dynamics/state.hpp"

namespace wfe {

// max |f| over the whole padded field, NaN reported above every finite value
// (src/dynamics/kernels.cu:967-979)
float field_absmax(const Field3D& f);

}  // namespace wfe
