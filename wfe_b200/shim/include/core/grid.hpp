// Reference-surface shim: the padded C-grid dimensions of src/core/grid.hpp
// (i fastest, ng ghost cells each side, one extra w level).
#pragma once

#include <cstddef>

#include "core/precision.hpp"

#if defined(__CUDACC__)
#define WFE_HD __host__ __device__
#else
#define WFE_HD
#endif

namespace wfe {

struct GDims {
  int nx, ny, nz;
  int ng;
  int NX, NY, NZ;
  real dx, dy, dz;
  WFE_HD size_t idx(int i, int j, int k) const {
    return ((size_t)(k + ng) * NY + (size_t)(j + ng)) * NX + (size_t)(i + ng);
  }
  size_t npts() const { return (size_t)NX * NY * NZ; }
};

inline GDims make_grid(int nx, int ny, int nz, int ng, real dx, real dy, real dz) {
  GDims g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.ng = ng;
  g.NX = nx + 2 * ng;
  g.NY = ny + 2 * ng;
  g.NZ = nz + 1 + 2 * ng;
  g.dx = dx;
  g.dy = dy;
  g.dz = dz;
  return g;
}

inline constexpr int MAX_COLUMN_LEVELS = 320;

}  // namespace wfe
