// Core device-side data model of wfe_b200: pitched C-grid layout, metric,
// base state, dynamics parameters and the small numerical helpers every
// kernel shares.  Templates on the arithmetic type R (float or double).
//
// Layout.  A field over the Arakawa C-grid of nx*ny*nz cells is stored
// i-fastest with ghost rings, like the reference (src/core/grid.hpp:22-36),
// but pitched for the B200:
//   x: interior i = 0 starts at element OX = 4 (16 B aligned for f32, 32 B
//      for f64); indices -4 .. PX-5 exist; PX = roundup(nx + 8, 8) so every
//      row starts on a 32-byte boundary (TMA global strides must be multiples
//      of 16 B and 128-bit loads need 16-B aligned rows);
//   y: ghosts 3 (j = -3 .. ny+2), z: ghosts 3 below and nz+1+3 above
//      (k = -3 .. nz+3), exactly the reference's NY and NZ.
// 2D fields use the (y, x) part of the same layout, vertical profiles the z
// part.  The reference layout (NX = nx+6) is only used at the C-ABI boundary.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define WFE_HD __host__ __device__ __forceinline__
#else
#define WFE_HD inline
#endif

namespace wfe {

constexpr int kOX = 4, kOY = 3, kOZ = 3;  // interior offsets (ghost widths)
constexpr int kRefNG = 3;                 // reference ghost width

struct Layout {
  int nx, ny, nz;
  int px, py, pz;  // pitched extents (elements)
  WFE_HD size_t at(int i, int j, int k) const {
    return ((size_t)(k + kOZ) * py + (size_t)(j + kOY)) * px + (size_t)(i + kOX);
  }
  WFE_HD size_t at2(int i, int j) const { return (size_t)(j + kOY) * px + (size_t)(i + kOX); }
  WFE_HD int at1(int k) const { return k + kOZ; }
  WFE_HD size_t n3() const { return (size_t)px * py * pz; }
  WFE_HD size_t n2() const { return (size_t)px * py; }
  WFE_HD size_t plane() const { return (size_t)px * py; }
  // 32-bit forms: a padded field holds fewer than 2^31 points (checked when a
  // model is created), and a pointer plus an int offset is one wide
  // multiply-add where a 64-bit offset costs a pair of adds per address
  WFE_HD int ati(int i, int j, int k) const { return ((k + kOZ) * py + (j + kOY)) * px + (i + kOX); }
  WFE_HD int at2i(int i, int j) const { return (j + kOY) * px + (i + kOX); }
  WFE_HD int planei() const { return px * py; }
};

// the largest padded field the 32-bit index forms address
constexpr size_t kMaxIndexedPoints = (size_t)1 << 31;

inline Layout make_layout(int nx, int ny, int nz) {
  Layout L;
  L.nx = nx;
  L.ny = ny;
  L.nz = nz;
  L.px = ((nx + 8) + 7) / 8 * 8;
  L.py = ny + 2 * kOY;
  L.pz = nz + 1 + 2 * kOZ;
  return L;
}

// Gal-Chen metric (src/core/metric.hpp:16-30), device pointers.
template <typename R>
struct DMetric {
  const R *zeta_w, *zeta_c, *dzeta_c, *dzeta_w;       // [pz]
  const R *h, *hx, *hy, *hx_u, *hy_v, *jac, *fcor, *mapf;  // [py*px]
  R zt;
};

// Hydrostatic base state (src/core/base_state.hpp:16-27), device pointers.
template <typename R>
struct DBase {
  const R *thb, *pib, *rhob, *dthbdz, *thbw, *rhobw, *thvb, *thvbw, *qvb;  // 3D
  const R* ub;                                                             // [pz]
  // When the base state is horizontally uniform (its every column holds the
  // same values): thb, pib, rhob and rhobw by level, BL_N x pz values (level
  // index at1(k)), which the mass-flux, Kessler and u, v kernels read instead
  // of the 3D fields -- the same values.  Null otherwise.
  const R* lvl;
};
enum { BL_THB = 0, BL_PIB, BL_RHOB, BL_RHOBW, BL_N };

// Run-constant acoustic coefficients (src/dynamics/kernels.hpp:46-52).
template <typename R>
struct DCoef {
  const R *rtjx, *rtjy, *kt3, *aw;
  // per level (pz entries): 1/dzeta_c, 1/dzeta_w, 1 - zeta_w/zt, 1 - zeta_c/zt,
  // 1/(zeta_c[k+1] - zeta_c[k-1]); the step multiplies by these instead of
  // dividing by the metric in every substep
  const R *inv_dzc, *inv_dzw, *fac_w, *fac_c, *inv_dzc2;
  const R *spg_c, *spg_w;  // Rayleigh coefficient at the cell / w levels
  R inv_dx, inv_dy;
};

// Dynamics parameters (src/dynamics/params.hpp:8-25).
template <typename R>
struct DParams {
  R diff_K;
  R rayleigh_zd, rayleigh_alpha;
  R acoustic_beta, acoustic_smdiv;
  R cstar;
  R w_abort;
  int acoustic_ns;
  int coriolis_use_ub;
  int bc_x_open, bc_y_open;
  int moisture, microphysics, pd_moist, w_damping;
};

// Physical constants (src/core/constants.hpp:7-17).
template <typename R>
struct Phys {
  static constexpr R grav = (R)9.81;
  static constexpr R cp = (R)1004.5;
  static constexpr R Rd = (R)287.04;
  static constexpr R cv = (R)1004.5 - (R)287.04;
  static constexpr R p00 = (R)1.0e5;
  static constexpr R Lv = (R)2.5e6;
  static constexpr R Lf = (R)3.34e5;
  static constexpr R Ls = (R)2.5e6 + (R)3.34e5;
  static constexpr R Rv = (R)461.5;
  static constexpr R eps61 = (R)0.61;
  static constexpr R Tfrz = (R)273.15;
};

// Lateral index maps that reproduce the reference's ghost fill
// (src/dynamics/kernels.cu:725-770): periodic wrap or zero-gradient clamp to
// [0, last].  Valid for the ghost depth the layout stores (3).
WFE_HD int map_lat(int i, int n, int last, int open) {
  if (open) return i < 0 ? 0 : (i > last ? last : i);
  if (i < 0) return i + n;
  if (i > last) return i - n;
  return i;
}
// Vertical zero-gradient map for cell-centred fields (kernels.cu:695-707).
WFE_HD int map_zc(int k, int nz) { return k < 0 ? 0 : (k > nz - 1 ? nz - 1 : k); }

// The lateral ghost columns around the interior, kRefNG wide: the kRefNG rows
// below and above it over the padded width, then the kRefNG columns west and
// east of each interior row.  ring_column maps r in [0, ring_columns) to (i, j).
WFE_HD long ring_columns(const Layout& L) { return 2L * kRefNG * (L.nx + 2 * kRefNG) + 2L * kRefNG * L.ny; }
WFE_HD void ring_column(const Layout& L, long r, int* i, int* j) {
  const long w = L.nx + 2 * kRefNG, band = (long)kRefNG * w;
  if (r < band) {
    *j = (int)(r / w) - kRefNG;
    *i = (int)(r % w) - kRefNG;
  } else if (r < 2 * band) {
    *j = L.ny + (int)((r - band) / w);
    *i = (int)((r - band) % w) - kRefNG;
  } else {
    const long q = r - 2 * band;
    const int m = (int)(q % (2 * kRefNG));
    *j = (int)(q / (2 * kRefNG));
    *i = m < kRefNG ? m - kRefNG : L.nx + (m - kRefNG);
  }
}

}  // namespace wfe
