// Tangent-linear (TL) and adjoint (AD) kernels of the dynamics, linearised
// about the forward trajectory (the forward buffers hold the values of the
// step being linearised when these run).
//
// Every kernel mirrors one forward kernel of the step and takes that
// kernel's recorded argument block `a` (forward values) plus the same block
// `d` with the state-like pointers replaced by tangent (TL) or adjoint (AD)
// buffers.  The ghost fill and the mass fluxes are linear, so their TL is the
// forward kernel applied to the tangent buffers.  For the tendencies and the
// forward u, v step one "row" function per output enumerates the nonzeros of
// the output's Jacobian row -- (input array, index, coefficient) -- from the
// forward values; TL gathers sum(coef * dx[index]) and AD scatters
// coef * ybar into the adjoint arrays (atomics), so TL and AD are transposes
// of each other by construction.  The implicit w - pi' column gets its own
// TL (a second Thomas sweep with the same matrix, right-hand side
// dD - dM w) and AD (the transposed tridiagonal solve M^T lambda = wbar,
// then dDbar = lambda, dMbar = -lambda w^T on the three diagonals).
//
// Upwind selections, the radiation-boundary branch and the w(nz) = 0 lid are
// frozen at the trajectory (the derivative of a piecewise-smooth step almost
// everywhere).  Moisture enters as advected species (tendency rows with
// their stage update), through theta_v in the pressure-gradient terms and
// through the moist buoyancy of the column; the Kessler column has its own
// TL/AD (lin_kessler.cu).  The positive-definite limiter, Davies relaxation,
// w damping and the surface physics are not linearised; the host refuses
// cases that use them.
#include <cuda_runtime.h>

#include "core.cuh"
#include "dyn_common.cuh"
#include "kernels.cuh"

namespace wfe {
namespace {

// ----------------------------------------------------------- accumulators
template <typename R, int N>
struct Ptrs {
  R* p[N];
};

template <typename R, int N>
struct TLAcc {  // gathers the row against the tangent inputs
  const Ptrs<R, N>& d;
  R sum;
  __device__ __forceinline__ void operator()(int id, size_t idx, R coef) { sum += coef * d.p[id][idx]; }
};

template <typename R, int N>
struct ADAcc {  // scatters the row, times the output adjoint, into the input adjoints
  const Ptrs<R, N>& b;
  R ybar;
  __device__ __forceinline__ void operator()(int id, size_t idx, R coef) {
    atomicAdd(b.p[id] + idx, coef * ybar);
  }
};

template <typename R>
__device__ __forceinline__ void face5_weights(R vel, R w[6]) {
  // d face5 / d q (src/dynamics/kernels.cu:51-57) for the upwind side of vel
  const R c = (R)(1.0 / 60.0);
  if (vel >= (R)0) {
    w[0] = 2 * c; w[1] = -13 * c; w[2] = 47 * c; w[3] = 27 * c; w[4] = -3 * c; w[5] = 0;
  } else {
    w[0] = 0; w[1] = -3 * c; w[2] = 27 * c; w[3] = 47 * c; w[4] = -13 * c; w[5] = 2 * c;
  }
}

__device__ __forceinline__ size_t off(size_t c, long d) { return (size_t)((long)c + d); }

// ================================================================ tendencies
enum { T_U = 0, T_V, T_W, T_TH, T_MFX, T_MFY, T_MFZ, T_QV, T_QC, T_QR, T_N };

// Contribution cF * dF of one flux F = fv face5(Q[c + (b + n) s], fv): fv is
// 0.5 (MF[ma] + MF[mb]) (avg) or MF[ma].
template <typename R, class Acc>
__device__ __forceinline__ void emit_face(Acc& acc, R cF, const R* MF, int mfid, size_t ma, size_t mb,
                                          bool avg, const R* Q, int qid, size_t c, long s, int b) {
  const R fv = avg ? (R)0.5 * (MF[ma] + MF[mb]) : MF[ma];
  const R* Qc = Q + c;
  const R face = face5(Qc[(long)b * s], Qc[(long)(b + 1) * s], Qc[(long)(b + 2) * s],
                       Qc[(long)(b + 3) * s], Qc[(long)(b + 4) * s], Qc[(long)(b + 5) * s], fv);
  if (avg) {
    acc(mfid, ma, cF * (R)0.5 * face);
    acc(mfid, mb, cF * (R)0.5 * face);
  } else {
    acc(mfid, ma, cF * face);
  }
  R w[6];
  face5_weights(fv, w);
#pragma unroll
  for (int n = 0; n < 6; ++n)
    if (w[n] != (R)0) acc(qid, off(c, (long)(b + n) * s), cF * fv * w[n]);
}

// coef * d divergence(i, j, k) (src/dynamics/kernels.cu:99-110)
template <typename R, class Acc>
__device__ __forceinline__ void emit_div(Acc& acc, const TendArgs<R>& a, int i, int j, int k, R coef) {
  const Layout& L = a.L;
  const size_t c = L.at(i, j, k);
  const R dzc = a.m.dzeta_c[L.at1(k)];
  acc(T_MFX, c + 1, coef / a.dx);
  acc(T_MFX, c, -coef / a.dx);
  acc(T_MFY, c + L.px, coef / a.dy);
  acc(T_MFY, c, -coef / a.dy);
  acc(T_MFZ, c + L.plane(), coef / dzc);
  acc(T_MFZ, c, -coef / dzc);
}

// coef * d laplacian (src/dynamics/kernels.cu:430-443)
template <typename R, class Acc>
__device__ __forceinline__ void emit_lap(Acc& acc, const TendArgs<R>& a, int id, int i, int j, int k,
                                         bool on_w, R coef) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const R dzl = (on_w ? a.m.dzeta_w[kk] : a.m.dzeta_c[kk]) * a.m.jac[L.at2(i, j)];
  const size_t c = L.at(i, j, k);
  const R ax = coef / (a.dx * a.dx), ay = coef / (a.dy * a.dy), az = coef / (dzl * dzl);
  acc(id, c + 1, ax);
  acc(id, c - 1, ax);
  acc(id, c + L.px, ay);
  acc(id, c - L.px, ay);
  acc(id, c + L.plane(), az);
  acc(id, c - L.plane(), az);
  acc(id, c, -2 * (ax + ay + az));
}

template <typename R>
__device__ __forceinline__ R div_value(const TendArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  return (a.mfx[L.at(i + 1, j, k)] - a.mfx[L.at(i, j, k)]) / a.dx +
         (a.mfy[L.at(i, j + 1, k)] - a.mfy[L.at(i, j, k)]) / a.dy +
         (a.mfz[L.at(i, j, k + 1)] - a.mfz[L.at(i, j, k)]) / a.m.dzeta_c[L.at1(k)];
}

// u tendency row (forward: kernels.cu:308-346)
template <typename R, class Acc>
__device__ void row_tu(Acc& acc, const TendArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const size_t c = L.at(i, j, k);
  const long sx = 1, sy = L.px, sz = (long)L.plane();
  const R ru = (R)0.5 * (a.b.rhob[c - sx] * a.m.jac[L.at2(i - 1, j)] + a.b.rhob[c] * a.m.jac[L.at2(i, j)]);
  const R dzc = a.m.dzeta_c[kk];
  emit_face(acc, (R)1 / (a.dx * ru), a.mfx, T_MFX, off(c, -sx), c, true, a.u, T_U, c, sx, -3);
  emit_face(acc, -(R)1 / (a.dx * ru), a.mfx, T_MFX, c, off(c, sx), true, a.u, T_U, c, sx, -2);
  emit_face(acc, (R)1 / (a.dy * ru), a.mfy, T_MFY, off(c, -sx), c, true, a.u, T_U, c, sy, -3);
  emit_face(acc, -(R)1 / (a.dy * ru), a.mfy, T_MFY, off(c, sy - sx), off(c, sy), true, a.u, T_U, c, sy, -2);
  emit_face(acc, (R)1 / (dzc * ru), a.mfz, T_MFZ, off(c, -sx), c, true, a.u, T_U, c, sz, -3);
  emit_face(acc, -(R)1 / (dzc * ru), a.mfz, T_MFZ, off(c, sz - sx), off(c, sz), true, a.u, T_U, c, sz, -2);
  const R dv = (R)0.5 * (div_value(a, i - 1, j, k) + div_value(a, i, j, k));
  const R u0 = a.u[c];
  emit_div(acc, a, i - 1, j, k, u0 * (R)0.5 / ru);
  emit_div(acc, a, i, j, k, u0 * (R)0.5 / ru);
  acc(T_U, c, dv / ru - sponge(a.m.zeta_c[kk], a.m.zt, a.p));
  const R fc = (R)0.5 * (a.m.fcor[L.at2(i - 1, j)] + a.m.fcor[L.at2(i, j)]);
  acc(T_V, off(c, -sx), (R)0.25 * fc);
  acc(T_V, off(c, sy - sx), (R)0.25 * fc);
  acc(T_V, c, (R)0.25 * fc);
  acc(T_V, off(c, sy), (R)0.25 * fc);
  if (a.p.diff_K > (R)0) emit_lap(acc, a, T_U, i, j, k, false, a.p.diff_K);
}

// v tendency row (kernels.cu:348-385)
template <typename R, class Acc>
__device__ void row_tv(Acc& acc, const TendArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const size_t c = L.at(i, j, k);
  const long sx = 1, sy = L.px, sz = (long)L.plane();
  const R rv = (R)0.5 * (a.b.rhob[c - sy] * a.m.jac[L.at2(i, j - 1)] + a.b.rhob[c] * a.m.jac[L.at2(i, j)]);
  const R dzc = a.m.dzeta_c[kk];
  emit_face(acc, (R)1 / (a.dy * rv), a.mfy, T_MFY, off(c, -sy), c, true, a.v, T_V, c, sy, -3);
  emit_face(acc, -(R)1 / (a.dy * rv), a.mfy, T_MFY, c, off(c, sy), true, a.v, T_V, c, sy, -2);
  emit_face(acc, (R)1 / (a.dx * rv), a.mfx, T_MFX, off(c, -sy), c, true, a.v, T_V, c, sx, -3);
  emit_face(acc, -(R)1 / (a.dx * rv), a.mfx, T_MFX, off(c, sx - sy), off(c, sx), true, a.v, T_V, c, sx, -2);
  emit_face(acc, (R)1 / (dzc * rv), a.mfz, T_MFZ, off(c, -sy), c, true, a.v, T_V, c, sz, -3);
  emit_face(acc, -(R)1 / (dzc * rv), a.mfz, T_MFZ, off(c, sz - sy), off(c, sz), true, a.v, T_V, c, sz, -2);
  const R dv = (R)0.5 * (div_value(a, i, j - 1, k) + div_value(a, i, j, k));
  const R v0 = a.v[c];
  emit_div(acc, a, i, j - 1, k, v0 * (R)0.5 / rv);
  emit_div(acc, a, i, j, k, v0 * (R)0.5 / rv);
  acc(T_V, c, dv / rv - sponge(a.m.zeta_c[kk], a.m.zt, a.p));
  const R fc = (R)0.5 * (a.m.fcor[L.at2(i, j - 1)] + a.m.fcor[L.at2(i, j)]);
  acc(T_U, off(c, -sy), -(R)0.25 * fc);
  acc(T_U, off(c, sx - sy), -(R)0.25 * fc);
  acc(T_U, c, -(R)0.25 * fc);
  acc(T_U, off(c, sx), -(R)0.25 * fc);
  if (a.p.diff_K > (R)0) emit_lap(acc, a, T_V, i, j, k, false, a.p.diff_K);
}

// w tendency row, k >= 1 (kernels.cu:387-425; w damping not linearised)
template <typename R, class Acc>
__device__ void row_tw(Acc& acc, const TendArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const size_t c = L.at(i, j, k);
  const long sx = 1, sy = L.px, sz = (long)L.plane();
  const R rw = a.b.rhobw[c] * a.m.jac[L.at2(i, j)];
  const R dzw = a.m.dzeta_w[kk];
  emit_face(acc, (R)1 / (a.dx * rw), a.mfx, T_MFX, off(c, -sz), c, true, a.w, T_W, c, sx, -3);
  emit_face(acc, -(R)1 / (a.dx * rw), a.mfx, T_MFX, off(c, sx - sz), off(c, sx), true, a.w, T_W, c, sx, -2);
  emit_face(acc, (R)1 / (a.dy * rw), a.mfy, T_MFY, off(c, -sz), c, true, a.w, T_W, c, sy, -3);
  emit_face(acc, -(R)1 / (a.dy * rw), a.mfy, T_MFY, off(c, sy - sz), off(c, sy), true, a.w, T_W, c, sy, -2);
  emit_face(acc, (R)1 / (dzw * rw), a.mfz, T_MFZ, off(c, -sz), c, true, a.w, T_W, c, sz, -3);
  emit_face(acc, -(R)1 / (dzw * rw), a.mfz, T_MFZ, c, off(c, sz), true, a.w, T_W, c, sz, -2);
  const R dv = (R)0.5 * (div_value(a, i, j, k - 1) + div_value(a, i, j, k));
  const R w0 = a.w[c];
  emit_div(acc, a, i, j, k - 1, w0 * (R)0.5 / rw);
  emit_div(acc, a, i, j, k, w0 * (R)0.5 / rw);
  acc(T_W, c, dv / rw - sponge(a.m.zeta_w[kk], a.m.zt, a.p));
  if (a.p.diff_K > (R)0) emit_lap(acc, a, T_W, i, j, k, true, a.p.diff_K);
}

// theta' tendency row (kernels.cu:114-146)
template <typename R, class Acc>
__device__ void row_tth(Acc& acc, const TendArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const size_t c = L.at(i, j, k);
  const long sx = 1, sy = L.px, sz = (long)L.plane();
  const R rt = a.b.rhob[c] * a.m.jac[L.at2(i, j)];
  const R dzc = a.m.dzeta_c[kk];
  emit_face(acc, (R)1 / (a.dx * rt), a.mfx, T_MFX, c, c, false, a.thp, T_TH, c, sx, -3);
  emit_face(acc, -(R)1 / (a.dx * rt), a.mfx, T_MFX, off(c, sx), 0, false, a.thp, T_TH, c, sx, -2);
  emit_face(acc, (R)1 / (a.dy * rt), a.mfy, T_MFY, c, c, false, a.thp, T_TH, c, sy, -3);
  emit_face(acc, -(R)1 / (a.dy * rt), a.mfy, T_MFY, off(c, sy), 0, false, a.thp, T_TH, c, sy, -2);
  emit_face(acc, (R)1 / (dzc * rt), a.mfz, T_MFZ, c, c, false, a.thp, T_TH, c, sz, -3);
  emit_face(acc, -(R)1 / (dzc * rt), a.mfz, T_MFZ, off(c, sz), 0, false, a.thp, T_TH, c, sz, -2);
  const R div = div_value(a, i, j, k);
  emit_div(acc, a, i, j, k, a.thp[c] / rt);
  acc(T_TH, c, div / rt - sponge(a.m.zeta_c[kk], a.m.zt, a.p));
  if (a.p.diff_K > (R)0) emit_lap(acc, a, T_TH, i, j, k, false, a.p.diff_K);
}

// moisture species tendency row: flux-form advection only (kernels.cu:886-899)
template <typename R, class Acc>
__device__ void row_tq(Acc& acc, const TendArgs<R>& a, const R* q, int qid, int i, int j, int k) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const size_t c = L.at(i, j, k);
  const long sx = 1, sy = L.px, sz = (long)L.plane();
  const R rt = a.b.rhob[c] * a.m.jac[L.at2(i, j)];
  const R dzc = a.m.dzeta_c[kk];
  emit_face(acc, (R)1 / (a.dx * rt), a.mfx, T_MFX, c, c, false, q, qid, c, sx, -3);
  emit_face(acc, -(R)1 / (a.dx * rt), a.mfx, T_MFX, off(c, sx), 0, false, q, qid, c, sx, -2);
  emit_face(acc, (R)1 / (a.dy * rt), a.mfy, T_MFY, c, c, false, q, qid, c, sy, -3);
  emit_face(acc, -(R)1 / (a.dy * rt), a.mfy, T_MFY, off(c, sy), 0, false, q, qid, c, sy, -2);
  emit_face(acc, (R)1 / (dzc * rt), a.mfz, T_MFZ, c, c, false, q, qid, c, sz, -3);
  emit_face(acc, -(R)1 / (dzc * rt), a.mfz, T_MFZ, off(c, sz), 0, false, q, qid, c, sz, -2);
  emit_div(acc, a, i, j, k, q[c] / rt);
  acc(qid, c, div_value(a, i, j, k) / rt);
}

template <typename R>
__device__ __forceinline__ Ptrs<R, T_N> tend_ptrs(const TendArgs<R>& d) {
  return Ptrs<R, T_N>{{const_cast<R*>(d.u), const_cast<R*>(d.v), const_cast<R*>(d.w),
                       const_cast<R*>(d.thp), const_cast<R*>(d.mfx), const_cast<R*>(d.mfy),
                       const_cast<R*>(d.mfz), const_cast<R*>(d.qv), const_cast<R*>(d.qc),
                       const_cast<R*>(d.qr)}};
}

template <typename R>
__global__ void __launch_bounds__(256) k_tl_tend(TendArgs<R> a, TendArgs<R> d) {
  const Layout& L = a.L;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= L.nx || j >= L.ny || k >= L.nz) return;
  const size_t c = L.at(i, j, k);
  const Ptrs<R, T_N> P = tend_ptrs(d);
  {
    TLAcc<R, T_N> acc{P, 0};
    row_tu(acc, a, i, j, k);
    d.tu[c] = acc.sum;
  }
  {
    TLAcc<R, T_N> acc{P, 0};
    row_tv(acc, a, i, j, k);
    d.tv[c] = acc.sum;
  }
  if (k >= 1) {
    TLAcc<R, T_N> acc{P, 0};
    row_tw(acc, a, i, j, k);
    d.tw[c] = acc.sum;
  }
  {
    TLAcc<R, T_N> acc{P, 0};
    row_tth(acc, a, i, j, k);
    d.tth[c] = acc.sum;
  }
  if (d.tpi) d.tpi[c] = 0;  // pi' has no slow tendency without Davies relaxation
  if (a.p.moisture) {
    const R* qf[3] = {a.qv, a.qc, a.qr};
    R* qo[3] = {d.qo_v, d.qo_c, d.qo_r};
    const R* qn[3] = {d.qn_v, d.qn_c, d.qn_r};
    R* tq[3] = {d.tqv, d.tqc, d.tqr};
    for (int sp = 0; sp < 3; ++sp) {
      TLAcc<R, T_N> acc{P, 0};
      row_tq(acc, a, qf[sp], T_QV + sp, i, j, k);
      if (qo[sp]) qo[sp][c] = qn[sp][c] + a.dt_stage * acc.sum;  // stage value (kernels.cu:268-273)
      else tq[sp][c] = acc.sum;
    }
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_ad_tend(TendArgs<R> a, TendArgs<R> d) {
  const Layout& L = a.L;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= L.nx || j >= L.ny || k >= L.nz) return;
  const size_t c = L.at(i, j, k);
  const Ptrs<R, T_N> P = tend_ptrs(d);
  {
    ADAcc<R, T_N> acc{P, d.tu[c]};
    d.tu[c] = 0;
    if (acc.ybar != (R)0) row_tu(acc, a, i, j, k);
  }
  {
    ADAcc<R, T_N> acc{P, d.tv[c]};
    d.tv[c] = 0;
    if (acc.ybar != (R)0) row_tv(acc, a, i, j, k);
  }
  if (k >= 1) {
    ADAcc<R, T_N> acc{P, d.tw[c]};
    d.tw[c] = 0;
    if (acc.ybar != (R)0) row_tw(acc, a, i, j, k);
  }
  {
    ADAcc<R, T_N> acc{P, d.tth[c]};
    d.tth[c] = 0;
    if (acc.ybar != (R)0) row_tth(acc, a, i, j, k);
  }
  if (d.tpi) d.tpi[c] = 0;
  if (a.p.moisture) {
    const R* qf[3] = {a.qv, a.qc, a.qr};
    R* qo[3] = {d.qo_v, d.qo_c, d.qo_r};
    R* qn[3] = {const_cast<R*>(d.qn_v), const_cast<R*>(d.qn_c), const_cast<R*>(d.qn_r)};
    R* tq[3] = {d.tqv, d.tqc, d.tqr};
    for (int sp = 0; sp < 3; ++sp) {
      R g;
      if (qo[sp]) {
        const R gq = qo[sp][c];
        qo[sp][c] = 0;
        if (gq != (R)0) atomicAdd(qn[sp] + c, gq);
        g = a.dt_stage * gq;
      } else {
        g = tq[sp][c];
        tq[sp][c] = 0;
      }
      ADAcc<R, T_N> acc{P, g};
      if (g != (R)0) row_tq(acc, a, qf[sp], T_QV + sp, i, j, k);
    }
  }
}

// ================================================================ ghost fill
// Adjoint of the ghost fill (forward: dyn_tend.cu fill_body): every written
// ghost value moves its adjoint onto its interior sources and is zeroed.  One
// thread per (padded column, level, field); interior points return at once.
template <typename R>
__global__ void k_ad_fill(FillArgs<R> A, int nk) {
  const Layout& L = A.L;
  const int f = blockIdx.z / nk;
  const int k = (int)(blockIdx.z % nk) - kRefNG;
  if (f >= A.job.n) return;
  R* a = A.job.f[f];
  const int kind = A.job.kind[f];
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) - kRefNG;
  const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y) - kRefNG;
  if (i > L.nx + 2 || j > L.ny + 2) return;
  const int ilast = (kind == 1 && A.open_x) ? L.nx : L.nx - 1;
  const int jlast = (kind == 2 && A.open_y) ? L.ny : L.ny - 1;
  const int si = map_lat(i, L.nx, ilast, A.open_x);
  const int sj = map_lat(j, L.ny, jlast, A.open_y);
  const bool lateral = (si != i) || (sj != j);
  if (!lateral && k >= 0 && k < L.nz) return;  // interior level of an interior column
  const size_t q = L.at(i, j, k);
  const R g = a[q];
  a[q] = 0;
  if (g == (R)0) return;
  if (kind == 3) {
    if (k == L.nz) return;
    if (k >= 0 && k < L.nz) atomicAdd(a + L.at(si, sj, k), g);
    else if (k < 0) {
      atomicAdd(a + L.at(si, sj, 0), (R)2 * g);
      atomicAdd(a + L.at(si, sj, -k), -g);
    } else {
      atomicAdd(a + L.at(si, sj, 2 * L.nz - k), -g);
    }
  } else {
    atomicAdd(a + L.at(si, sj, map_zc(k, L.nz)), g);
  }
}

// =============================================================== mass fluxes
// Adjoint of the mass fluxes (forward: dyn_tend.cu flux_body), same ring.
template <typename R>
__global__ void k_ad_flux(FluxArgs<R> A) {
  const Layout& L = A.L;
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) - 2;
  const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y) - 2;
  const int k = (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (i > L.nx + 2 || j > L.ny + 2 || k > L.nz) return;
  const size_t c = L.at(i, j, k);
  R* ub = const_cast<R*>(A.u);
  R* vb = const_cast<R*>(A.v);
  R* wb = const_cast<R*>(A.w);
  if (k < L.nz) {
    R gx = A.mfx[c], gy = A.mfy[c];
    A.mfx[c] = 0;
    A.mfy[c] = 0;
    R rjx = (R)0.5 * (A.b.rhob[L.at(i - 1, j, k)] * A.m.jac[L.at2(i - 1, j)] +
                      A.b.rhob[c] * A.m.jac[L.at2(i, j)]);
    R rjy = (R)0.5 * (A.b.rhob[L.at(i, j - 1, k)] * A.m.jac[L.at2(i, j - 1)] +
                      A.b.rhob[c] * A.m.jac[L.at2(i, j)]);
    if (gx != (R)0) atomicAdd(ub + c, rjx * gx);
    if (gy != (R)0) atomicAdd(vb + c, rjy * gy);
  }
  if (i > L.nx + 1 || j > L.ny + 1) return;
  R gz = A.mfz[c];
  A.mfz[c] = 0;
  if (k == 0 || k == L.nz || gz == (R)0) return;
  const int kk = L.at1(k);
  R fac = (R)1 - A.m.zeta_w[kk] / A.m.zt;
  R rw = A.b.rhobw[c];
  atomicAdd(wb + c, rw * gz);
  R cu = -rw * gz * (R)0.25 * A.m.hx[L.at2(i, j)] * fac;
  R cv = -rw * gz * (R)0.25 * A.m.hy[L.at2(i, j)] * fac;
  if (cu != (R)0) {
    atomicAdd(ub + L.at(i, j, k - 1), cu);
    atomicAdd(ub + L.at(i + 1, j, k - 1), cu);
    atomicAdd(ub + c, cu);
    atomicAdd(ub + L.at(i + 1, j, k), cu);
  }
  if (cv != (R)0) {
    atomicAdd(vb + L.at(i, j, k - 1), cv);
    atomicAdd(vb + L.at(i, j + 1, k - 1), cv);
    atomicAdd(vb + c, cv);
    atomicAdd(vb + L.at(i, j + 1, k), cv);
  }
}

// ============================================================== acoustic u, v
enum { A_UIN = 0, A_VIN, A_PICUR, A_PIPREV, A_NPIP, A_THIN, A_NTHP, A_TU, A_TV, A_QV, A_N };

template <typename R>
__device__ __forceinline__ Ptrs<R, A_N> acou_ptrs(const AcouArgs<R>& d) {
  return Ptrs<R, A_N>{{const_cast<R*>(d.u_in), const_cast<R*>(d.v_in), const_cast<R*>(d.pi_cur),
                       const_cast<R*>(d.pi_prev), const_cast<R*>(d.n_pip), const_cast<R*>(d.th_in),
                       const_cast<R*>(d.n_thp), const_cast<R*>(d.tu), const_cast<R*>(d.tv),
                       const_cast<R*>(d.qv)}};
}

// coef * d pi*(i, j, k) (dyn_common.cuh pistar)
template <typename R, class Acc>
__device__ __forceinline__ void emit_pistar(Acc& acc, const AcouArgs<R>& a, int i, int j, int k, R coef) {
  const Layout& L = a.L;
  const R sm = a.p.acoustic_smdiv;
  const bool ghost = i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz;
  if (!ghost) {
    const size_t c = L.at(i, j, k);
    acc(A_PICUR, c, coef * ((R)1 + sm));
    acc(A_PIPREV, c, -coef * sm);
  } else {
    const size_t c = L.at(map_lat(i, L.nx, L.nx - 1, a.p.bc_x_open),
                          map_lat(j, L.ny, L.ny - 1, a.p.bc_y_open), map_zc(k, L.nz));
    acc(A_PICUR, c, coef * ((R)1 + sm));
    acc(A_NPIP, c, -coef * sm);
  }
}

// coef * d theta_v(i, j, k) (dyn_common.cuh theta_v): theta' and, moist, qv
template <typename R, class Acc>
__device__ __forceinline__ void emit_thv(Acc& acc, const AcouArgs<R>& a, int i, int j, int k, R coef) {
  const Layout& L = a.L;
  const bool lat = i < 0 || i >= L.nx || j < 0 || j >= L.ny;
  const size_t c = L.at(i, j, k);
  const size_t s =
      lat ? L.at(map_lat(i, L.nx, L.nx - 1, a.p.bc_x_open), map_lat(j, L.ny, L.ny - 1, a.p.bc_y_open), k)
          : c;
  R f = coef;
  if (a.p.moisture) {
    const R th = a.b.thb[c] + (lat ? a.n_thp[s] : a.th_in[c]);
    f = coef * ((R)1 + Phys<R>::eps61 * a.qv[s]);
    acc(A_QV, s, coef * th * Phys<R>::eps61);
  }
  acc(lat ? A_NTHP : A_THIN, s, f);
}

// forward u (is_u) or v step at a face and, when acc is given, coef times
// its Jacobian row (kernels.cu:499-526)
template <typename R, class Acc>
__device__ R uv_face(Acc* acc, const AcouArgs<R>& a, int i, int j, int k, bool is_u, R coef) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const int di = is_u ? 1 : 0, dj = is_u ? 0 : 1;
  const R thf = (R)0.5 * (theta_v(a, i - di, j - dj, k) + theta_v(a, i, j, k));
  const R mf = (R)0.5 * (a.m.mapf[L.at2(i - di, j - dj)] + a.m.mapf[L.at2(i, j)]);
  const R h = is_u ? a.dx : a.dy;
  R grad = (pistar(a, i, j, k) - pistar(a, i - di, j - dj, k)) / h;
  const R slope = (is_u ? a.m.hx_u[L.at2(i, j)] : a.m.hy_v[L.at2(i, j)]) * ((R)1 - a.m.zeta_c[kk] / a.m.zt);
  R dzc2 = 1, jf = 1;
  if (slope != (R)0) {
    dzc2 = a.m.zeta_c[kk + 1] - a.m.zeta_c[kk - 1];
    jf = (R)0.5 * (a.m.jac[L.at2(i - di, j - dj)] + a.m.jac[L.at2(i, j)]);
    R dpdz = (R)0.5 *
             ((pistar(a, i - di, j - dj, k + 1) - pistar(a, i - di, j - dj, k - 1)) +
              (pistar(a, i, j, k + 1) - pistar(a, i, j, k - 1))) /
             dzc2;
    grad -= slope / jf * dpdz;
  }
  const size_t c = L.at(i, j, k);
  const R* tin = is_u ? a.tu : a.tv;
  const R* vin = is_u ? a.u_in : a.v_in;
  const R out = vin[c] + a.dtau * (-Phys<R>::cp * thf * mf * grad + tin[c]);
  if (acc) {
    (*acc)(is_u ? A_UIN : A_VIN, c, coef);
    (*acc)(is_u ? A_TU : A_TV, c, coef * a.dtau);
    const R g1 = -coef * a.dtau * Phys<R>::cp * mf;
    emit_thv(*acc, a, i - di, j - dj, k, g1 * grad * (R)0.5);
    emit_thv(*acc, a, i, j, k, g1 * grad * (R)0.5);
    const R g2 = g1 * thf;
    emit_pistar(*acc, a, i, j, k, g2 / h);
    emit_pistar(*acc, a, i - di, j - dj, k, -g2 / h);
    if (slope != (R)0) {
      const R g3 = -g2 * slope / jf * (R)0.5 / dzc2;
      emit_pistar(*acc, a, i - di, j - dj, k + 1, g3);
      emit_pistar(*acc, a, i - di, j - dj, k - 1, -g3);
      emit_pistar(*acc, a, i, j, k + 1, g3);
      emit_pistar(*acc, a, i, j, k - 1, -g3);
    }
  }
  return out;
}

// coef * d(u_out) row at face (i, j, k), with the radiation faces of open
// boundaries (kernels.cu:654-667, 674-687) and the periodic face
template <typename R, class Acc>
__device__ void row_u_out(Acc& acc, const AcouArgs<R>& a, int i, int j, int k, R coef) {
  const Layout& L = a.L;
  const R cstar = a.p.cstar;
  if (a.p.bc_x_open) {
    if (i == 0) {
      const size_t c0 = L.at(0, j, k);
      const R u0 = a.u_in[c0];
      if (u0 >= (R)0) return;  // out = ub
      const R cb = u0 - cstar;
      const R uf1 = uv_face<R, Acc>(nullptr, a, 1, j, k, true, 0);
      acc(A_UIN, c0, coef * ((R)1 - a.dtau / a.dx * (uf1 - u0 - cb)));
      uv_face(&acc, a, 1, j, k, true, -coef * a.dtau * cb / a.dx);
    } else if (i == L.nx) {
      const size_t cn = L.at(L.nx, j, k);
      const R un = a.u_in[cn];
      if (un <= (R)0) return;
      const R cb = un + cstar;
      const R ufn = uv_face<R, Acc>(nullptr, a, L.nx - 1, j, k, true, 0);
      acc(A_UIN, cn, coef * ((R)1 - a.dtau / a.dx * (un - ufn + cb)));
      uv_face(&acc, a, L.nx - 1, j, k, true, coef * a.dtau * cb / a.dx);
    } else {
      uv_face(&acc, a, i, j, k, true, coef);
    }
  } else {
    uv_face(&acc, a, i == L.nx ? 0 : i, j, k, true, coef);
  }
}

template <typename R, class Acc>
__device__ void row_v_out(Acc& acc, const AcouArgs<R>& a, int i, int j, int k, R coef) {
  const Layout& L = a.L;
  const R cstar = a.p.cstar;
  if (a.p.bc_y_open) {
    if (j == 0) {
      const size_t c0 = L.at(i, 0, k);
      const R v0 = a.v_in[c0];
      if (v0 >= (R)0) return;  // out = 0
      const R cb = v0 - cstar;
      const R vf1 = uv_face<R, Acc>(nullptr, a, i, 1, k, false, 0);
      acc(A_VIN, c0, coef * ((R)1 - a.dtau / a.dy * (vf1 - v0 - cb)));
      uv_face(&acc, a, i, 1, k, false, -coef * a.dtau * cb / a.dy);
    } else if (j == L.ny) {
      const size_t cn = L.at(i, L.ny, k);
      const R vn = a.v_in[cn];
      if (vn <= (R)0) return;
      const R cb = vn + cstar;
      const R vfn = uv_face<R, Acc>(nullptr, a, i, L.ny - 1, k, false, 0);
      acc(A_VIN, cn, coef * ((R)1 - a.dtau / a.dy * (vn - vfn + cb)));
      uv_face(&acc, a, i, L.ny - 1, k, false, coef * a.dtau * cb / a.dy);
    } else {
      uv_face(&acc, a, i, j, k, false, coef);
    }
  } else {
    uv_face(&acc, a, i, j == L.ny ? 0 : j, k, false, coef);
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_tl_uv(AcouArgs<R> a, AcouArgs<R> d) {
  const Layout& L = a.L;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i > L.nx || j > L.ny || k >= L.nz) return;
  const Ptrs<R, A_N> P = acou_ptrs(d);
  if (j < L.ny) {
    TLAcc<R, A_N> acc{P, 0};
    row_u_out(acc, a, i, j, k, (R)1);
    d.u_out[L.at(i, j, k)] = acc.sum;
  }
  if (i < L.nx) {
    TLAcc<R, A_N> acc{P, 0};
    row_v_out(acc, a, i, j, k, (R)1);
    d.v_out[L.at(i, j, k)] = acc.sum;
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_ad_uv(AcouArgs<R> a, AcouArgs<R> d) {
  const Layout& L = a.L;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i > L.nx || j > L.ny || k >= L.nz) return;
  const Ptrs<R, A_N> P = acou_ptrs(d);
  if (j < L.ny) {
    const size_t c = L.at(i, j, k);
    ADAcc<R, A_N> acc{P, (R)1};
    const R g = d.u_out[c];
    d.u_out[c] = 0;
    if (g != (R)0) row_u_out(acc, a, i, j, k, g);
  }
  if (i < L.nx) {
    const size_t c = L.at(i, j, k);
    ADAcc<R, A_N> acc{P, (R)1};
    const R g = d.v_out[c];
    d.v_out[c] = 0;
    if (g != (R)0) row_v_out(acc, a, i, j, k, g);
  }
}

// ================================================================ w - pi' column
// A CTA owns LCX columns of one row with LKL level lanes; the column arrays
// live in shared memory ([level * LCX + column]); the sweeps run in one lane
// per column, everything else in parallel over the levels.
constexpr int LCX = 8, LKL = 16;

// rows 1..n-1 of a tridiagonal system (row 1 without A, row n-1 without C),
// the forward's elimination order (kernels.cu:612-634); arrays strided by LCX
template <typename R>
__device__ void thomas_s(int n, const R* A, const R* B, const R* C, const R* D, R* cs, R* ds, R* x) {
  R cp = 0, dp = 0;
  for (int k = 1; k < n; ++k) {
    const int q = k * LCX;
    if (k == 1) {
      cp = C[q] / B[q];
      dp = D[q] / B[q];
    } else {
      const R m = B[q] - A[q] * cp;
      cp = C[q] / m;
      dp = (D[q] - A[q] * dp) / m;
    }
    cs[q] = cp;
    ds[q] = dp;
  }
  x[n * LCX] = 0;
  R above = 0;
  for (int k = n - 1; k >= 1; --k) {
    above = ds[k * LCX] - cs[k * LCX] * above;
    x[k * LCX] = above;
  }
}

// the transposed system: (M^T)_{k,k-1} = C[k-1], (M^T)_{k,k+1} = A[k+1]
template <typename R>
__device__ void thomas_ts(int n, const R* A, const R* B, const R* C, const R* D, R* cs, R* ds, R* x) {
  R cp = 0, dp = 0;
  for (int k = 1; k < n; ++k) {
    const int q = k * LCX;
    const R sub = k > 1 ? C[q - LCX] : (R)0;
    const R sup = k < n - 1 ? A[q + LCX] : (R)0;
    if (k == 1) {
      cp = sup / B[q];
      dp = D[q] / B[q];
    } else {
      const R m = B[q] - sub * cp;
      cp = sup / m;
      dp = (D[q] - sub * dp) / m;
    }
    cs[q] = cp;
    ds[q] = dp;
  }
  x[n * LCX] = 0;
  x[0] = 0;
  R above = 0;
  for (int k = n - 1; k >= 1; --k) {
    above = ds[k * LCX] - cs[k * LCX] * above;
    x[k * LCX] = above;
  }
}

// shared column arrays: a fixed set of (nz + 1)-level arrays
template <typename R>
struct ColArr {
  R* base;
  int n1;  // nz + 1
  __device__ R* operator[](int q) const { return base + (size_t)q * n1 * LCX; }
};

// Forward values of one column (kernels.cu:552-634) as the column kernel
// computes them, into shared arrays: Av, Sv, P, E on levels; G, A, B, C, D on
// the inner levels; the solution w (with the surface w at level 0).
enum { V_AV, V_SV, V_P, V_E, V_G, V_A, V_B, V_C, V_D, V_W, V_CS, V_DS, V_N };

template <typename R>
__device__ void column_values_s(const AcouArgs<R>& a, int i, int j, bool active, const ColArr<R>& S) {
  const Layout& L = a.L;
  const int nz = L.nz, tx = threadIdx.x, lane = threadIdx.y;
  const R dtau = a.dtau, zt = a.m.zt;
  const R c1 = ((R)1 + a.p.acoustic_beta) * (R)0.5;
  const R c2 = ((R)1 - a.p.acoustic_beta) * (R)0.5;
  const size_t c2d = L.at2(active ? i : 0, j);
  const R J = a.m.jac[c2d], hxc = a.m.hx[c2d], hyc = a.m.hy[c2d], mc = a.m.mapf[c2d];
  const R* u = a.u_out;
  const R* v = a.v_out;
  const long sx = 1, sy = L.px;
  R *Av = S[V_AV] + tx, *Sv = S[V_SV] + tx, *P = S[V_P] + tx, *E = S[V_E] + tx;
  R *G = S[V_G] + tx, *A = S[V_A] + tx, *B = S[V_B] + tx, *C = S[V_C] + tx, *D = S[V_D] + tx;
  if (active)
    for (int k = lane; k <= nz; k += LKL) {
      R av = 0, sv = 0;
      if (k >= 1 && k < nz) {
        const int kk = L.at1(k);
        const size_t c = L.at(i, j, k);
        av = a.co.aw[c];
        R fac = (R)1 - a.m.zeta_w[kk] / zt;
        const size_t cm = c - (size_t)L.plane();
        R uw = (R)0.25 * (u[cm] + u[cm + sx] + u[c] + u[c + sx]);
        R vw = (R)0.25 * (v[cm] + v[cm + sy] + v[c] + v[c + sy]);
        sv = av * (uw * hxc + vw * hyc) * fac;
      }
      Av[k * LCX] = av;
      Sv[k * LCX] = sv;
    }
  __syncthreads();
  if (active)
    for (int k = lane; k < nz; k += LKL) {
      const int kk = L.at1(k);
      const size_t c = L.at(i, j, k);
      R Kt = a.co.kt3[c];
      R Dh = mc * ((a.co.rtjx[c + sx] * u[c + sx] - a.co.rtjx[c] * u[c]) / a.dx +
                   (a.co.rtjy[c + sy] * v[c + sy] - a.co.rtjy[c] * v[c]) / a.dy);
      R dzc = a.m.dzeta_c[kk];
      R wk = a.w_in[c], wkp = a.w_in[c + L.plane()];
      R tpi = a.tpi ? a.tpi[c] : (R)0;
      P[k * LCX] = a.pi_cur[c] + dtau * tpi -
                   dtau * Kt *
                       (Dh - (Sv[(k + 1) * LCX] - Sv[k * LCX]) / dzc +
                        c2 * (Av[(k + 1) * LCX] * wkp - Av[k * LCX] * wk) / dzc);
      E[k * LCX] = dtau * Kt * c1 / dzc;
    }
  __syncthreads();
  if (active)
    for (int k = 1 + lane; k < nz; k += LKL) {
      const int kk = L.at1(k);
      const size_t c = L.at(i, j, k), cm = c - (size_t)L.plane();
      R thc = a.th_in[c], thm = a.th_in[cm];
      R thvw = a.b.thbw[c] + (R)0.5 * (thm + thc);
      if (a.p.moisture) thvw *= (R)1 + Phys<R>::eps61 * (R)0.5 * (a.qv[cm] + a.qv[c]);
      R g = dtau * Phys<R>::cp * thvw * c1 / (J * a.m.dzeta_w[kk]);
      const int q = k * LCX;
      G[q] = g;
      A[q] = -g * E[q - LCX] * Av[q - LCX];
      B[q] = (R)1 + g * Av[q] * (E[q] + E[q - LCX]);
      C[q] = -g * E[q] * Av[q + LCX];
      R buoy = Phys<R>::grav * (R)0.5 * (thm + thc) / a.b.thbw[c];
      if (a.p.moisture) {
        R dqv = (R)0.5 * (a.qv[cm] + a.qv[c]) - (R)0.5 * (a.b.qvb[cm] + a.b.qvb[c]);
        R qcr = (R)0.5 * (a.qc[cm] + a.qc[c]) + (R)0.5 * (a.qr[cm] + a.qr[c]);
        buoy += Phys<R>::grav * (Phys<R>::eps61 * dqv - qcr);
      }
      R RHS = a.w_in[c] + dtau * (buoy + a.tw[c]) -
              dtau * Phys<R>::cp * thvw * c2 * (a.pi_cur[c] - a.pi_cur[cm]) / (J * a.m.dzeta_w[kk]);
      D[q] = RHS - g * (P[q] - P[q - LCX]);
    }
  __syncthreads();
  if (active && lane == 0) {
    R* W = S[V_W] + tx;
    thomas_s(nz, A, B, C, D, S[V_CS] + tx, S[V_DS] + tx, W);
    const size_t c0 = L.at(i, j, 0);
    W[0] = (R)0.5 * (u[c0] + u[c0 + sx]) * hxc + (R)0.5 * (v[c0] + v[c0 + sy]) * hyc;
  }
  __syncthreads();
}

enum { T_DSV = V_N, T_DTH, T_DP, T_DG, T_RHS, T_DW, T_NARR };

template <typename R>
__global__ void __launch_bounds__(LCX * LKL) k_tl_column(AcouArgs<R> a, AcouArgs<R> d) {
  extern __shared__ __align__(16) unsigned char lin_smem[];
  const Layout& L = a.L;
  const int nz = L.nz, tx = threadIdx.x, lane = threadIdx.y;
  const int i = blockIdx.x * LCX + tx, j = blockIdx.y;
  const bool active = i < L.nx;
  const ColArr<R> S{reinterpret_cast<R*>(lin_smem), nz + 1};
  const R dtau = a.dtau, zt = a.m.zt;
  const R c1 = ((R)1 + a.p.acoustic_beta) * (R)0.5;
  const R c2 = ((R)1 - a.p.acoustic_beta) * (R)0.5;
  const size_t c2d = L.at2(active ? i : 0, j);
  const R J = a.m.jac[c2d], hxc = a.m.hx[c2d], hyc = a.m.hy[c2d], mc = a.m.mapf[c2d];
  const R* u = d.u_out;
  const R* v = d.v_out;
  const long sx = 1, sy = L.px;
  R *dSv = S[T_DSV] + tx, *dth = S[T_DTH] + tx, *dP = S[T_DP] + tx, *dG = S[T_DG] + tx;
  R *rhs = S[T_RHS] + tx, *dw = S[T_DW] + tx;
  // the tangent theta' in, before any in-place write of this launch
  if (active)
    for (int k = lane; k < nz; k += LKL) dth[k * LCX] = d.th_in[L.at(i, j, k)];
  column_values_s(a, i, j, active, S);  // ends with a barrier
  const R *Av = S[V_AV] + tx, *P = S[V_P] + tx, *E = S[V_E] + tx, *G = S[V_G] + tx;
  const R *W = S[V_W] + tx;
  if (active)
    for (int k = lane; k <= nz; k += LKL) {
      R s = 0;
      if (k >= 1 && k < nz) {
        const int kk = L.at1(k);
        const size_t c = L.at(i, j, k), cm = c - (size_t)L.plane();
        R fac = (R)1 - a.m.zeta_w[kk] / zt;
        R uw = (R)0.25 * (u[cm] + u[cm + sx] + u[c] + u[c + sx]);
        R vw = (R)0.25 * (v[cm] + v[cm + sy] + v[c] + v[c + sy]);
        s = Av[k * LCX] * (uw * hxc + vw * hyc) * fac;
      }
      dSv[k * LCX] = s;
    }
  __syncthreads();
  if (active)
    for (int k = lane; k < nz; k += LKL) {
      const int kk = L.at1(k);
      const size_t c = L.at(i, j, k);
      R Kt = a.co.kt3[c];
      R dDh = mc * ((a.co.rtjx[c + sx] * u[c + sx] - a.co.rtjx[c] * u[c]) / a.dx +
                    (a.co.rtjy[c + sy] * v[c + sy] - a.co.rtjy[c] * v[c]) / a.dy);
      R dzc = a.m.dzeta_c[kk];
      R dwk = d.w_in[c], dwkp = d.w_in[c + L.plane()];
      R dtpi = d.tpi ? d.tpi[c] : (R)0;
      const int q = k * LCX;
      dP[q] = d.pi_cur[c] + dtau * dtpi -
              dtau * Kt * (dDh - (dSv[q + LCX] - dSv[q]) / dzc + c2 * (Av[q + LCX] * dwkp - Av[q] * dwk) / dzc);
    }
  __syncthreads();
  if (active)
    for (int k = 1 + lane; k < nz; k += LKL) {
      const int kk = L.at1(k);
      const size_t c = L.at(i, j, k), cm = c - (size_t)L.plane();
      const int q = k * LCX;
      const R jdz = J * a.m.dzeta_w[kk];
      const R thd = a.b.thbw[c] + (R)0.5 * (a.th_in[cm] + a.th_in[c]);
      R thvw = thd;
      R dthvw = (R)0.5 * (dth[q - LCX] + dth[q]);
      R dbuoy = Phys<R>::grav * (R)0.5 * (dth[q - LCX] + dth[q]) / a.b.thbw[c];
      if (a.p.moisture) {
        // theta_v = theta (1 + 0.61 qv); buoyancy + g (0.61 qv' - qc - qr)
        const R mq = (R)1 + Phys<R>::eps61 * (R)0.5 * (a.qv[cm] + a.qv[c]);
        const R dqv = (R)0.5 * (d.qv[cm] + d.qv[c]);
        thvw = thd * mq;
        dthvw = dthvw * mq + thd * Phys<R>::eps61 * dqv;
        dbuoy += Phys<R>::grav * (Phys<R>::eps61 * dqv - (R)0.5 * (d.qc[cm] + d.qc[c]) -
                                  (R)0.5 * (d.qr[cm] + d.qr[c]));
      }
      R g = dtau * Phys<R>::cp * dthvw * c1 / jdz;
      R dpi = d.pi_cur[c] - d.pi_cur[cm], pi = a.pi_cur[c] - a.pi_cur[cm];
      R dRHS = d.w_in[c] + dtau * (dbuoy + d.tw[c]) -
               dtau * Phys<R>::cp * c2 * (dthvw * pi + thvw * dpi) / jdz;
      R dD = dRHS - g * (P[q] - P[q - LCX]) - G[q] * (dP[q] - dP[q - LCX]);
      R dA = -g * E[q - LCX] * Av[q - LCX];
      R dB = g * Av[q] * (E[q] + E[q - LCX]);
      R dC = -g * E[q] * Av[q + LCX];
      R mw = dB * W[q];
      if (k > 1) mw += dA * W[q - LCX];
      if (k < nz - 1) mw += dC * W[q + LCX];
      rhs[q] = dD - mw;
      dG[q] = g;
    }
  __syncthreads();
  if (active && lane == 0) {
    thomas_s(nz, S[V_A] + tx, S[V_B] + tx, S[V_C] + tx, rhs, S[V_CS] + tx, S[V_DS] + tx, dw);
    const size_t c0 = L.at(i, j, 0);
    dw[0] = (R)0.5 * (u[c0] + u[c0 + sx]) * hxc + (R)0.5 * (v[c0] + v[c0 + sy]) * hyc;
  }
  __syncthreads();
  if (active)
    for (int k = lane; k <= nz; k += LKL) {
      const size_t c = L.at(i, j, k);
      const int q = k * LCX;
      if (k < nz) {
        d.pi_next[c] = dP[q] - E[q] * (Av[q + LCX] * dw[q + LCX] - Av[q] * dw[q]);
        d.th_out[c] = dth[q] + dtau * (d.tth[c] - (R)0.5 * (dw[q] + dw[q + LCX]) * a.b.dthbdz[c]);
        d.w_out[c] = dw[q];
      } else {
        d.w_out[c] = 0;
      }
    }
}

enum { A_WB = V_N, A_PB, A_TB, A_WS, A_LAM, A_GL, A_PIB, A_THB, A_KTD, A_NARR };

template <typename R>
__global__ void __launch_bounds__(LCX * LKL) k_ad_column(AcouArgs<R> a, AcouArgs<R> d) {
  extern __shared__ __align__(16) unsigned char lin_smem[];
  const Layout& L = a.L;
  const int nz = L.nz, tx = threadIdx.x, lane = threadIdx.y;
  const int i = blockIdx.x * LCX + tx, j = blockIdx.y;
  const bool active = i < L.nx;
  const ColArr<R> S{reinterpret_cast<R*>(lin_smem), nz + 1};
  const R dtau = a.dtau, zt = a.m.zt;
  const R c1 = ((R)1 + a.p.acoustic_beta) * (R)0.5;
  const R c2 = ((R)1 - a.p.acoustic_beta) * (R)0.5;
  const size_t c2d = L.at2(active ? i : 0, j);
  const R J = a.m.jac[c2d], hxc = a.m.hx[c2d], hyc = a.m.hy[c2d], mc = a.m.mapf[c2d];
  R* ub = d.u_out;
  R* vb = d.v_out;
  R* wI = const_cast<R*>(d.w_in);
  R* piC = const_cast<R*>(d.pi_cur);
  R* thI = const_cast<R*>(d.th_in);
  R* twB = const_cast<R*>(d.tw);
  R* tthB = const_cast<R*>(d.tth);
  R* tpiB = const_cast<R*>(d.tpi);
  R* qvI = const_cast<R*>(d.qv);
  R* qcI = const_cast<R*>(d.qc);
  R* qrI = const_cast<R*>(d.qr);
  const bool moist = a.p.moisture != 0;
  const long sx = 1, sy = L.px;
  R *wb = S[A_WB] + tx, *pb = S[A_PB] + tx, *tb = S[A_TB] + tx, *ws = S[A_WS] + tx;
  R *lam = S[A_LAM] + tx, *GL = S[A_GL] + tx, *PIB = S[A_PIB] + tx, *THB = S[A_THB] + tx;
  R *KTD = S[A_KTD] + tx;
  // the sweep's scratch rows, free once the transposed solve is done
  R *QVB = S[V_CS] + tx, *QCB = S[V_DS] + tx;
  // output adjoints, read and cleared before the (possibly aliased) inputs gain theirs
  if (active)
    for (int k = lane; k <= nz; k += LKL) {
      const size_t c = L.at(i, j, k);
      const int q = k * LCX;
      wb[q] = d.w_out[c];
      d.w_out[c] = 0;
      if (k < nz) {
        pb[q] = d.pi_next[c];
        tb[q] = d.th_out[c];
        d.pi_next[c] = 0;
        d.th_out[c] = 0;
      }
    }
  column_values_s(a, i, j, active, S);  // ends with a barrier
  const R *Av = S[V_AV] + tx, *P = S[V_P] + tx, *E = S[V_E] + tx, *G = S[V_G] + tx;
  const R *W = S[V_W] + tx;
  // adjoint of the column solution w (level 0: surface w, level nz: the lid)
  if (active)
    for (int k = lane; k <= nz; k += LKL) {
      const int q = k * LCX;
      R g = 0;
      if (k < nz) {
        const size_t c = L.at(i, j, k);
        g += wb[q] - (R)0.5 * dtau * a.b.dthbdz[c] * tb[q] + E[q] * Av[q] * pb[q];
      }
      if (k >= 1) {
        const size_t cm = L.at(i, j, k - 1);
        g += -(R)0.5 * dtau * a.b.dthbdz[cm] * tb[q - LCX] - E[q - LCX] * Av[q] * pb[q - LCX];
      }
      ws[q] = g;
    }
  __syncthreads();
  if (active && lane == 0) {
    const size_t c0 = L.at(i, j, 0);
    const R g = ws[0];
    if (g != (R)0) {
      atomicAdd(ub + c0, (R)0.5 * hxc * g);
      atomicAdd(ub + c0 + sx, (R)0.5 * hxc * g);
      atomicAdd(vb + c0, (R)0.5 * hyc * g);
      atomicAdd(vb + c0 + sy, (R)0.5 * hyc * g);
    }
    thomas_ts(nz, S[V_A] + tx, S[V_B] + tx, S[V_C] + tx, ws, S[V_CS] + tx, S[V_DS] + tx, lam);
  }
  __syncthreads();
  // per inner level: what its row sends to neighbouring levels
  if (active)
    for (int k = lane; k <= nz; k += LKL) {
      const int q = k * LCX;
      if (k < 1 || k >= nz) {
        GL[q] = 0;
        PIB[q] = 0;
        THB[q] = 0;
        QVB[q] = 0;
        QCB[q] = 0;
        continue;
      }
      const int kk = L.at1(k);
      const size_t c = L.at(i, j, k), cm = c - (size_t)L.plane();
      const R jdz = J * a.m.dzeta_w[kk];
      const R lm = lam[q];
      const R Ab = k > 1 ? -lm * W[q - LCX] : (R)0;
      const R Bb = -lm * W[q];
      const R Cb = k < nz - 1 ? -lm * W[q + LCX] : (R)0;
      const R Gb = Ab * (-E[q - LCX] * Av[q - LCX]) + Bb * (Av[q] * (E[q] + E[q - LCX])) +
                   Cb * (-E[q] * Av[q + LCX]) - lm * (P[q] - P[q - LCX]);
      const R thd = a.b.thbw[c] + (R)0.5 * (a.th_in[cm] + a.th_in[c]);
      const R mq = moist ? (R)1 + Phys<R>::eps61 * (R)0.5 * (a.qv[cm] + a.qv[c]) : (R)1;
      const R thvw = thd * mq;
      const R pi = a.pi_cur[c] - a.pi_cur[cm];
      GL[q] = G[q] * lm;
      PIB[q] = -dtau * Phys<R>::cp * thvw * c2 / jdz * lm;
      const R thvwb = -dtau * Phys<R>::cp * c2 * pi / jdz * lm + Gb * dtau * Phys<R>::cp * c1 / jdz;
      const R bt = Phys<R>::grav * (R)0.5 / a.b.thbw[c] * dtau * lm;
      THB[q] = (R)0.5 * thvwb * mq + bt;
      // per level of the pair (k-1, k): qv through theta_v and buoyancy, qc and qr through buoyancy
      QVB[q] = (R)0.5 * Phys<R>::eps61 * (thvwb * thd + Phys<R>::grav * dtau * lm);
      QCB[q] = -(R)0.5 * Phys<R>::grav * dtau * lm;
      twB[c] += dtau * lm;
    }
  __syncthreads();
  if (active)
    for (int k = lane; k < nz; k += LKL) {
      const int kk = L.at1(k);
      const size_t c = L.at(i, j, k);
      const int q = k * LCX;
      R Pb = pb[q];
      if (k >= 1) Pb -= GL[q];
      if (k + 1 < nz) Pb += GL[q + LCX];
      R pic = Pb;
      if (k >= 1) pic += PIB[q];
      if (k + 1 < nz) pic -= PIB[q + LCX];
      piC[c] += pic;
      if (tpiB) tpiB[c] += dtau * Pb;
      const R Kt = a.co.kt3[c];
      const R Dhb = -dtau * Kt * Pb;
      if (Dhb != (R)0) {
        atomicAdd(ub + c + sx, mc * a.co.rtjx[c + sx] / a.dx * Dhb);
        atomicAdd(ub + c, -mc * a.co.rtjx[c] / a.dx * Dhb);
        atomicAdd(vb + c + sy, mc * a.co.rtjy[c + sy] / a.dy * Dhb);
        atomicAdd(vb + c, -mc * a.co.rtjy[c] / a.dy * Dhb);
      }
      R th = tb[q];
      if (k >= 1) th += THB[q];
      if (k + 1 < nz) th += THB[q + LCX];
      thI[c] += th;
      if (moist) {
        R qvs = 0, qcs = 0;
        if (k >= 1) qvs += QVB[q], qcs += QCB[q];
        if (k + 1 < nz) qvs += QVB[q + LCX], qcs += QCB[q + LCX];
        qvI[c] += qvs;
        qcI[c] += qcs;
        qrI[c] += qcs;
      }
      tthB[c] += dtau * tb[q];
      KTD[q] = Kt / a.m.dzeta_c[kk] * Pb;
    }
  __syncthreads();
  if (active)
    for (int k = lane; k <= nz; k += LKL) {
      const int q = k * LCX;
      const size_t c = L.at(i, j, k);
      R wsum = 0;
      if (k >= 1 && k < nz) wsum += lam[q];
      R kd = (k < nz ? KTD[q] : (R)0) - (k >= 1 ? KTD[q - LCX] : (R)0);
      wsum += dtau * c2 * Av[q] * kd;
      wI[c] += wsum;
      if (k >= 1 && k < nz) {
        const R svb = -dtau * kd;  // adjoint of Sv(k)
        if (svb != (R)0) {
          const int kk = L.at1(k);
          const size_t cm = c - (size_t)L.plane();
          const R fac = (R)1 - a.m.zeta_w[kk] / zt;
          const R cu = (R)0.25 * Av[q] * hxc * fac * svb, cv = (R)0.25 * Av[q] * hyc * fac * svb;
          if (cu != (R)0) {
            atomicAdd(ub + cm, cu);
            atomicAdd(ub + cm + sx, cu);
            atomicAdd(ub + c, cu);
            atomicAdd(ub + c + sx, cu);
          }
          if (cv != (R)0) {
            atomicAdd(vb + cm, cv);
            atomicAdd(vb + cm + sy, cv);
            atomicAdd(vb + c, cv);
            atomicAdd(vb + c + sy, cv);
          }
        }
      }
    }
}

// zero every stored point of a cell field outside the interior cells
template <typename R>
__global__ void k_zero_ring(R* f, Layout L) {
  const size_t n = L.n3();
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % L.px) - kOX;
    const int j = (int)((q / L.px) % L.py) - kOY;
    const int k = (int)(q / L.plane()) - kOZ;
    if (i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz) f[q] = 0;
  }
}

}  // namespace

// ------------------------------------------------------------ host launch
template <typename R>
void zero_ring(R* f, const Layout& L, cudaStream_t st) {
  k_zero_ring<R><<<1184, 256, 0, st>>>(f, L);
}

template <typename R>
void ad_fill(const FillArgs<R>& d, cudaStream_t st) {
  if (d.job.n == 0) return;
  const int nk = d.L.nz + 1 + 2 * kRefNG;  // levels -3 .. nz+3
  dim3 g = grid_fill(d);
  g.z = (unsigned)(d.job.n * nk);
  k_ad_fill<R><<<g, dim3(32, 4), 0, st>>>(d, nk);
}

template <typename R>
void ad_flux(const FluxArgs<R>& d, cudaStream_t st) {
  k_ad_flux<R><<<grid_flux(d), dim3(32, 4, 2), 0, st>>>(d);
}

template <typename R>
void tl_tend(const TendArgs<R>& a, const TendArgs<R>& d, cudaStream_t st) {
  k_tl_tend<R><<<grid_cells<R>(a.L), dim3(32, 4, 2), 0, st>>>(a, d);
}

template <typename R>
void ad_tend(const TendArgs<R>& a, const TendArgs<R>& d, cudaStream_t st) {
  k_ad_tend<R><<<grid_cells<R>(a.L), dim3(32, 4, 2), 0, st>>>(a, d);
}

template <typename R>
void tl_uv(const AcouArgs<R>& a, const AcouArgs<R>& d, cudaStream_t st) {
  k_tl_uv<R><<<grid_uv<R>(a.L), dim3(32, 4, 2), 0, st>>>(a, d);
}

template <typename R>
void ad_uv(const AcouArgs<R>& a, const AcouArgs<R>& d, cudaStream_t st) {
  k_ad_uv<R><<<grid_uv<R>(a.L), dim3(32, 4, 2), 0, st>>>(a, d);
}

int lin_max_levels() { return 160; }  // FP64 adjoint column arrays within 227 KB

template <typename R, int NARR>
static size_t lin_col_smem(int nz) {
  return (size_t)NARR * (nz + 1) * LCX * sizeof(R);
}

// Sets the dynamic shared-memory limits of the column kernels for nz levels,
// once, outside any stream capture.
template <typename R>
int lin_prepare(int nz) {
  if (nz > lin_max_levels()) return 2;
  if (cudaFuncSetAttribute(k_tl_column<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)lin_col_smem<R, T_NARR>(nz)) != cudaSuccess ||
      cudaFuncSetAttribute(k_ad_column<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)lin_col_smem<R, A_NARR>(nz)) != cudaSuccess)
    return 1;
  return lin_kessler_prepare<R>(nz);
}

template <typename R>
int tl_column(const AcouArgs<R>& a, const AcouArgs<R>& d, cudaStream_t st) {
  if (a.L.nz > lin_max_levels()) return 2;
  const size_t sm = lin_col_smem<R, T_NARR>(a.L.nz);
  k_tl_column<R><<<dim3((a.L.nx + LCX - 1) / LCX, a.L.ny), dim3(LCX, LKL), sm, st>>>(a, d);
  return 0;
}

template <typename R>
int ad_column(const AcouArgs<R>& a, const AcouArgs<R>& d, cudaStream_t st) {
  if (a.L.nz > lin_max_levels()) return 2;
  const size_t sm = lin_col_smem<R, A_NARR>(a.L.nz);
  k_ad_column<R><<<dim3((a.L.nx + LCX - 1) / LCX, a.L.ny), dim3(LCX, LKL), sm, st>>>(a, d);
  return 0;
}

#define WFE_INST(R)                                                              \
  template void ad_fill<R>(const FillArgs<R>&, cudaStream_t);                    \
  template void ad_flux<R>(const FluxArgs<R>&, cudaStream_t);                    \
  template void tl_tend<R>(const TendArgs<R>&, const TendArgs<R>&, cudaStream_t); \
  template void ad_tend<R>(const TendArgs<R>&, const TendArgs<R>&, cudaStream_t); \
  template void tl_uv<R>(const AcouArgs<R>&, const AcouArgs<R>&, cudaStream_t);   \
  template void ad_uv<R>(const AcouArgs<R>&, const AcouArgs<R>&, cudaStream_t);   \
  template int tl_column<R>(const AcouArgs<R>&, const AcouArgs<R>&, cudaStream_t); \
  template int ad_column<R>(const AcouArgs<R>&, const AcouArgs<R>&, cudaStream_t);  \
  template void zero_ring<R>(R*, const Layout&, cudaStream_t);                        \
  template int lin_prepare<R>(int);
WFE_INST(float)
WFE_INST(double)
#undef WFE_INST

}  // namespace wfe
