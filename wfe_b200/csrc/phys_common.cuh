// Column-physics arithmetic shared by the Kessler kernel (phys_kessler.cu) and
// its tangent-linear / adjoint (lin.cu): Tetens saturation, the rain fall
// speed, and the per-level conversions written once for a generic value type
// -- the precision R itself, or Dn<R, N>, a value with N directional
// derivatives (forward-mode differentiation of the same expressions, used to
// form the 4 x 5 local Jacobian of a level).
#pragma once

#include "core.cuh"

namespace wfe {

// the CUDA math overloads stay visible beside the dual-number ones below
using ::exp;
using ::pow;

// ------------------------------------------------------ dual numbers
template <typename R, int N>
struct Dn {
  R v;
  R d[N];
};

template <typename R, int N>
__device__ __forceinline__ Dn<R, N> dn_const(R x) {
  Dn<R, N> r;
  r.v = x;
#pragma unroll
  for (int q = 0; q < N; ++q) r.d[q] = 0;
  return r;
}
template <typename R, int N>
__device__ __forceinline__ Dn<R, N> dn_var(R x, int q) {
  Dn<R, N> r = dn_const<R, N>(x);
  r.d[q] = 1;
  return r;
}

#define WFE_DN_OPS(OP, DV)                                                                 \
  template <typename R, int N>                                                             \
  __device__ __forceinline__ Dn<R, N> operator OP(const Dn<R, N>& a, const Dn<R, N>& b) { \
    Dn<R, N> r;                                                                            \
    r.v = a.v OP b.v;                                                                      \
    _Pragma("unroll") for (int q = 0; q < N; ++q) r.d[q] = DV;                            \
    return r;                                                                              \
  }
WFE_DN_OPS(+, a.d[q] + b.d[q])
WFE_DN_OPS(-, a.d[q] - b.d[q])
WFE_DN_OPS(*, a.d[q] * b.v + a.v * b.d[q])
WFE_DN_OPS(/, (a.d[q] * b.v - a.v * b.d[q]) / (b.v * b.v))
#undef WFE_DN_OPS

template <typename R, int N>
__device__ __forceinline__ Dn<R, N> operator+(const Dn<R, N>& a, R b) { return a + dn_const<R, N>(b); }
template <typename R, int N>
__device__ __forceinline__ Dn<R, N> operator+(R a, const Dn<R, N>& b) { return dn_const<R, N>(a) + b; }
template <typename R, int N>
__device__ __forceinline__ Dn<R, N> operator-(const Dn<R, N>& a, R b) { return a - dn_const<R, N>(b); }
template <typename R, int N>
__device__ __forceinline__ Dn<R, N> operator-(R a, const Dn<R, N>& b) { return dn_const<R, N>(a) - b; }
template <typename R, int N>
__device__ __forceinline__ Dn<R, N> operator-(const Dn<R, N>& a) { return dn_const<R, N>((R)0) - a; }
template <typename R, int N>
__device__ __forceinline__ Dn<R, N> operator*(const Dn<R, N>& a, R b) {
  Dn<R, N> r;
  r.v = a.v * b;
#pragma unroll
  for (int q = 0; q < N; ++q) r.d[q] = a.d[q] * b;
  return r;
}
template <typename R, int N>
__device__ __forceinline__ Dn<R, N> operator*(R a, const Dn<R, N>& b) { return b * a; }
template <typename R, int N>
__device__ __forceinline__ Dn<R, N> operator/(const Dn<R, N>& a, R b) { return a / dn_const<R, N>(b); }
template <typename R, int N>
__device__ __forceinline__ Dn<R, N> operator/(R a, const Dn<R, N>& b) { return dn_const<R, N>(a) / b; }

template <typename R, int N>
__device__ __forceinline__ Dn<R, N> exp(const Dn<R, N>& a) {
  Dn<R, N> r;
  r.v = exp(a.v);
#pragma unroll
  for (int q = 0; q < N; ++q) r.d[q] = r.v * a.d[q];
  return r;
}
// x^e for x > 0
template <typename R, int N>
__device__ __forceinline__ Dn<R, N> pow(const Dn<R, N>& a, R e) {
  Dn<R, N> r;
  r.v = pow(a.v, e);
  const R s = e * r.v / a.v;
#pragma unroll
  for (int q = 0; q < N; ++q) r.d[q] = s * a.d[q];
  return r;
}

__device__ __forceinline__ float val(float x) { return x; }
__device__ __forceinline__ double val(double x) { return x; }
template <typename R, int N>
__device__ __forceinline__ R val(const Dn<R, N>& a) { return a.v; }

// the value type's constant
template <typename T, typename R>
struct Const {
  __device__ static T of(R x) { return x; }
};
template <typename R, int N>
struct Const<Dn<R, N>, R> {
  __device__ static Dn<R, N> of(R x) { return dn_const<R, N>(x); }
};

// --------------------------------------------------------- thermodynamics
template <typename R, typename T>
__device__ __forceinline__ T qsat_w_g(T p, T Tk) {  // src/core/thermo.hpp:11-17
  T es = (R)610.78 * exp((R)17.269 * (Tk - (R)273.16) / (Tk - (R)35.86));
  T den = p - es;
  if (val(den) < (R)1) den = Const<T, R>::of((R)1);
  return (R)0.622 * es / den;
}
template <typename R, typename T>
__device__ __forceinline__ T qsat_i_g(T p, T Tk) {  // src/core/thermo.hpp:20-26
  T es = (R)610.78 * exp((R)21.875 * (Tk - (R)273.16) / (Tk - (R)7.66));
  T den = p - es;
  if (val(den) < (R)1) den = Const<T, R>::of((R)1);
  return (R)0.622 * es / den;
}

template <typename R>
__device__ __forceinline__ R fall_speed(R rq, R rho_sfc, R rho, R T) {
  // kessler.cu:195-211: 36.34 (rho qr)^0.1364 sqrt(rho0/rho), x0.35 below freezing
  return rq > (R)1e-9 ? (R)36.34 * pow(rq, (R)0.1364) * sqrt(rho_sfc / rho) *
                            (T < Phys<R>::Tfrz ? (R)0.35 : (R)1)
                      : (R)0;
}

// max(x, 0) / clamp(x, 0, 1) keeping the whole value (with its derivatives)
template <typename T, typename R>
__device__ __forceinline__ T pos(const T& x) {
  return val(x) > (R)0 ? x : Const<T, R>::of((R)0);
}

// Conversions, evaporation and mixed-phase saturation adjustment of one level
// (kessler.cu:239-297).  In: thp, qv, qc, the sedimented qr, pi'; out: thp,
// qv, qc, qr.  rh, thb, pib are the level's reference state.
template <typename R, typename T>
__device__ __forceinline__ void kessler_convert(T& thp, T& qv, T& qc, T& qr, const T& pip, R rh,
                                                R thb, R pib, R dt) {
  const R k1 = (R)0.001, qc0 = (R)0.001;
  T qvk = pos<T, R>(qv);
  T qck = pos<T, R>(qc);
  T qrk = pos<T, R>(qr);
  T pi = pib + pip;
  T th = thb + thp;
  T Tk = th * pi;
  T pres = Phys<R>::p00 * pow(pi, Phys<R>::cp / Phys<R>::Rd);
  T fl = (Tk - (R)233.15) / (R)40;
  if (val(fl) > (R)1) fl = Const<T, R>::of((R)1);
  if (val(fl) < (R)0) fl = Const<T, R>::of((R)0);
  T qsw = qsat_w_g<R, T>(pres, Tk);
  T qs = fl * qsw + ((R)1 - fl) * qsat_i_g<R, T>(pres, Tk);
  T Leff = fl * Phys<R>::Lv + ((R)1 - fl) * Phys<R>::Ls;
  T dqauto = k1 * (val(qck) > qc0 ? qck - qc0 : Const<T, R>::of((R)0));
  T dqacc = (R)2.2 * qck * pow(val(qrk) > (R)1e-9 ? qrk : Const<T, R>::of((R)1e-9), (R)0.875);
  T dqr = dt * (dqauto + dqacc);
  if (val(dqr) > val(qck)) dqr = qck;
  qck = qck - dqr;
  qrk = qrk + dqr;
  if (val(qvk) < val(qs) && val(qrk) > (R)0) {
    T rq = rh * qrk;
    T vent = (R)1.6 + (R)124.9 * pow(rq, (R)0.2046);
    T ern = vent * pow(rq, (R)0.525) / ((R)2.55e8 / (pres * qs) + (R)5.4e5) * (qs - qvk) / (rh * qs);
    T dqe = dt * ern;
    if (val(dqe) > val(qrk)) dqe = qrk;
    if (val(dqe) > val(qs) - val(qvk)) dqe = qs - qvk;
    qrk = qrk - dqe;
    qvk = qvk + dqe;
    thp = thp - Leff * dqe / (Phys<R>::cp * pi);
    th = thb + thp;
    Tk = th * pi;
    T fl2 = (Tk - (R)233.15) / (R)40;
    if (val(fl2) > (R)1) fl2 = Const<T, R>::of((R)1);
    if (val(fl2) < (R)0) fl2 = Const<T, R>::of((R)0);
    qs = fl2 * qsat_w_g<R, T>(pres, Tk) + ((R)1 - fl2) * qsat_i_g<R, T>(pres, Tk);
  }
  T gam = Leff * Leff * qs / (Phys<R>::cp * Phys<R>::Rv * Tk * Tk);
  T dq = (qvk - qs) / ((R)1 + gam);
  if (val(dq) < (R)0) {
    T evap = -dq;
    if (val(evap) > val(qck)) evap = qck;
    dq = -evap;
  }
  qvk = qvk - dq;
  qck = qck + dq;
  thp = thp + Leff * dq / (Phys<R>::cp * pi);
  qv = pos<T, R>(qvk);
  qc = pos<T, R>(qck);
  qr = pos<T, R>(qrk);
}

}  // namespace wfe
