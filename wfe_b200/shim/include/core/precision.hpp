// Reference-surface shim: the arithmetic type of the reference's build
// (src/core/precision.hpp): float, or double with -DWFE_DOUBLE.  A shim
// build with WFE_DOUBLE runs the library in FP64.
#pragma once

namespace wfe {
#ifdef WFE_DOUBLE
using real = double;
#else
using real = float;
#endif
}  // namespace wfe
