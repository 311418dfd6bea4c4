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

// a product the compiler may not fuse into a following add: face fluxes are
// rounded once, wherever they are combined (so kernels that keep them in
// registers and kernels that stage them in shared memory agree bit for bit)
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// a fused multiply-add, rounded once in every kernel that calls it
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename R>
__device__ __forceinline__ R face5(R qm2, R qm1, R q0, R q1, R q2, R q3, R vel) {
  // 5th-order upwind interface value (src/dynamics/kernels.cu:51-57).  The
  // reference's centred sum c (37 (q0 + q1) - 8 (q-1 + q2) + (q-2 + q3)) minus
  // (vel >= 0) or plus its upwind correction c ((q3 - q-2) - 5 (q2 - q-1) +
  // 10 (q1 - q0)), c = 1/60, is the one-sided stencil
  // (2 a - 13 b + 47 d + 27 e - 3 f) / 60 over (a, b, d, e, f) = (q-2 .. q2)
  // for vel >= 0 and (q3 .. q-1) otherwise: the same value to rounding in
  // five selects and five rounded multiply-adds instead of seventeen
  // operations, with the explicit roundings every kernel reproduces
  const bool up = vel >= (R)0;
  const R a = up ? qm2 : q3, b = up ? qm1 : q2, d = up ? q0 : q1, e = up ? q1 : q0, f = up ? q2 : qm1;
  R t = mul_rn((R)2, a);
  t = fma_rn((R)-13, b, t);
  t = fma_rn((R)47, d, t);
  t = fma_rn((R)27, e, t);
  t = fma_rn((R)-3, f, t);
  return mul_rn(t, (R)(1.0 / 60.0));
}

// ------------------------------------------------------ Davies relaxation
template <typename R>
__device__ __forceinline__ R time_fraction(const double* clk) {
  // BdyManager::tfrac (src/dynamics/boundary.cpp:91-97)
  double t = clk[CLK_T], lo = clk[CLK_TLO], hi = clk[CLK_THI];
  if (hi <= lo) return 0;
  double f = (t - lo) / (hi - lo);
  return (R)(f < 0 ? 0.0 : (f > 1 ? 1.0 : f));
}

template <typename R>
__device__ __forceinline__ R davies(const TendArgs<R>& a, int v, const R* f, int i, int j, int k) {
  const Layout& L = a.L;
  const R tf = time_fraction<R>(a.clock);
  int iw = i < L.nx ? i : L.nx - 1, jw = j < L.ny ? j : L.ny - 1;
  R w = a.wgt[L.at2i(iw, jw)];
  if (w <= (R)0) return 0;
  const int c = L.ati(i, j, k);
  return w * (((R)1 - tf) * a.lo[v][c] + tf * a.hi[v][c] - f[c]);
}

// ------------------------------------------------------ acoustic helpers
template <typename R>
__device__ __forceinline__ R pistar(const AcouArgs<R>& a, int i, int j, int k) {
  // pi* = pi' + smdiv (pi' - pi'_prev)  (kernels.cu:486-489)
  const Layout& L = a.L;
  const bool ghost = i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz;
  R cur, prev;
  if (!ghost) {
    const int c = L.ati(i, j, k);
    cur = a.pi_cur[c];
    prev = a.pi_prev[c];
  } else {
    const int c = L.ati(map_lat(i, L.nx, L.nx - 1, a.p.bc_x_open),
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
  const int c = L.ati(i, j, k);
  int s = c;
  if (lat)
    s = L.ati(map_lat(i, L.nx, L.nx - 1, a.p.bc_x_open), map_lat(j, L.ny, L.ny - 1, a.p.bc_y_open), k);
  R t = a.b.thb[c] + (lat ? a.n_thp[s] : a.th_in[c]);
  if (a.p.moisture) t *= (R)1 + Phys<R>::eps61 * a.qv[s];
  return t;
}

}  // namespace wfe
