// Device helpers shared by the forward dynamics kernels and their tangent-
// linear and adjoint counterparts (lin.cu).
#pragma once

#include "core.cuh"
#include "kernels.cuh"

namespace wfe {

template <typename R>
__device__ __forceinline__ R sponge(R zeta, R zt, const DParams<R>& p) {
  // src/dynamics/kernels.cu:42-48
  if (p.rayleigh_zd < (R)0) return 0;
  if (zeta <= p.rayleigh_zd || zt <= p.rayleigh_zd) return 0;
  const R halfpi = (R)1.5707963267948966;
  R s = sin(halfpi * (zeta - p.rayleigh_zd) / (zt - p.rayleigh_zd));
  return p.rayleigh_alpha * s * s;
}

template <typename R>
__device__ __forceinline__ R face5(R qm2, R qm1, R q0, R q1, R q2, R q3, R vel) {
  // 5th-order upwind interface value (src/dynamics/kernels.cu:51-57)
  const R c = (R)(1.0 / 60.0);
  R cen = c * ((R)37 * (q0 + q1) - (R)8 * (qm1 + q2) + (qm2 + q3));
  R upw = c * ((q3 - qm2) - (R)5 * (q2 - qm1) + (R)10 * (q1 - q0));
  return (vel >= (R)0) ? (cen - upw) : (cen + upw);
}

// ------------------------------------------------------ acoustic helpers
template <typename R>
__device__ __forceinline__ R pistar(const AcouArgs<R>& a, int i, int j, int k) {
  // pi* = pi' + smdiv (pi' - pi'_prev)  (kernels.cu:486-489)
  const Layout& L = a.L;
  const bool ghost = i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz;
  R cur, prev;
  if (!ghost) {
    const size_t c = L.at(i, j, k);
    cur = a.pi_cur[c];
    prev = a.pi_prev[c];
  } else {
    const size_t c = L.at(map_lat(i, L.nx, L.nx - 1, a.p.bc_x_open),
                          map_lat(j, L.ny, L.ny - 1, a.p.bc_y_open), map_zc(k, L.nz));
    cur = a.pi_cur[c];
    prev = a.n_pip[c];
  }
  return cur + a.p.acoustic_smdiv * (cur - prev);
}

template <typename R>
__device__ __forceinline__ R theta_v(const AcouArgs<R>& a, int i, int j, int k) {
  // full virtual potential temperature at a cell centre (kernels.cu:490-495)
  const Layout& L = a.L;
  const bool lat = i < 0 || i >= L.nx || j < 0 || j >= L.ny;
  const size_t c = L.at(i, j, k);
  size_t s = c;
  if (lat)
    s = L.at(map_lat(i, L.nx, L.nx - 1, a.p.bc_x_open), map_lat(j, L.ny, L.ny - 1, a.p.bc_y_open), k);
  R t = a.b.thb[c] + (lat ? a.n_thp[s] : a.th_in[c]);
  if (a.p.moisture) t *= (R)1 + Phys<R>::eps61 * a.qv[s];
  return t;
}

}  // namespace wfe
