// Tangent-linear (TL) and adjoint (AD) kernels of the dynamics, linearised
// about the forward trajectory (the forward buffers hold the values of the
// step being linearised when these run).
//
// Every kernel mirrors one forward kernel of the step and takes that
// kernel's recorded argument block `a` (forward values) plus the same block
// `d` with the state-like pointers replaced by tangent (TL) or adjoint (AD)
// buffers.  The ghost fill and the mass fluxes are linear, so their TL is the
// forward kernel applied to the tangent buffers.  For the tendencies one
// "row" function per output enumerates the nonzeros of the output's Jacobian
// row -- (input array, index, coefficient) -- from the forward values; TL
// gathers sum(coef * dx[index]) and AD scatters coef * ybar into the adjoint
// arrays (atomics), so TL and AD are transposes of each other by
// construction.  The forward u, v step's TL gathers its rows the same way;
// its AD is gather-form (per-face coefficients, then a per-cell gather, no
// atomics).  The implicit w - pi' column gets its own TL (a second Thomas
// sweep with the same matrix, right-hand side dD - dM w; the launch also
// writes the forward column's outputs) and AD (the transposed tridiagonal
// solve M^T lambda = wbar, then dDbar = lambda, dMbar = -lambda w^T on the
// three diagonals, with the forward solution taken from the launch's outputs
// in the adjoint sweep; its u, v adjoints are gathered per face).
//
// Output adjoints are cleared only after their values have been used: a
// store issued while the load of the same address is in flight stalls the
// memory pipeline.
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
  __device__ __forceinline__ void operator()(int id, int idx, R coef) { sum += coef * d.p[id][idx]; }
};

template <typename R, int N>
struct ADAcc {  // scatters the row, times the output adjoint, into the input adjoints
  const Ptrs<R, N>& b;
  R ybar;
  __device__ __forceinline__ void operator()(int id, int idx, R coef) {
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

__device__ __forceinline__ int off(int c, int d) { return c + d; }

// ================================================================ tendencies
enum { T_U = 0, T_V, T_W, T_TH, T_MFX, T_MFY, T_MFZ, T_QV, T_QC, T_QR, T_N };

// The two faces of one direction of a cell, cL dF_L + cR dF_R, with the
// face-5 stencils (offsets -3..2 of the left face, -2..3 of the right) merged
// into one weight per point: seven q terms instead of up to twelve.  Left
// face mass flux: 0.5 (MF[maL] + MF[mbL]) (avg) or MF[maL]; right likewise.
template <typename R, class Acc>
__device__ __forceinline__ void emit_face_pair(Acc& acc, R cL, R cR, const R* MF, int mfid, int maL,
                                               int mbL, int maR, int mbR, bool avg, const R* Q,
                                               int qid, int c, int s) {
  const R fvL = avg ? (R)0.5 * (MF[maL] + MF[mbL]) : MF[maL];
  const R fvR = avg ? (R)0.5 * (MF[maR] + MF[mbR]) : MF[maR];
  const R* Qc = Q + c;
  R q[7];
#pragma unroll
  for (int n = 0; n < 7; ++n) q[n] = Qc[(int)(n - 3) * s];
  const R faceL = face5(q[0], q[1], q[2], q[3], q[4], q[5], fvL);
  const R faceR = face5(q[1], q[2], q[3], q[4], q[5], q[6], fvR);
  if (avg) {
    acc(mfid, maL, cL * (R)0.5 * faceL);
    acc(mfid, mbL, cL * (R)0.5 * faceL);
    acc(mfid, maR, cR * (R)0.5 * faceR);
    acc(mfid, mbR, cR * (R)0.5 * faceR);
  } else {
    acc(mfid, maL, cL * faceL);
    acc(mfid, maR, cR * faceR);
  }
  R wL[6], wR[6];
  face5_weights(fvL, wL);
  face5_weights(fvR, wR);
  const R gL = cL * fvL, gR = cR * fvR;
#pragma unroll
  for (int n = 0; n < 7; ++n) {
    R wgt = 0;
    if (n < 6) wgt += gL * wL[n];
    if (n >= 1) wgt += gR * wR[n - 1];
    if (wgt != (R)0) acc(qid, off(c, (int)(n - 3) * s), wgt);
  }
}

// coef * d divergence(i, j, k) (src/dynamics/kernels.cu:99-110)
template <typename R, class Acc>
__device__ __forceinline__ void emit_div(Acc& acc, const TendArgs<R>& a, int i, int j, int k, R coef) {
  const Layout& L = a.L;
  const int c = L.ati(i, j, k);
  const R dzc = a.m.dzeta_c[L.at1(k)];
  acc(T_MFX, c + 1, coef / a.dx);
  acc(T_MFX, c, -coef / a.dx);
  acc(T_MFY, c + L.px, coef / a.dy);
  acc(T_MFY, c, -coef / a.dy);
  acc(T_MFZ, c + L.planei(), coef / dzc);
  acc(T_MFZ, c, -coef / dzc);
}

// coef * d laplacian (src/dynamics/kernels.cu:430-443)
template <typename R, class Acc>
__device__ __forceinline__ void emit_lap(Acc& acc, const TendArgs<R>& a, int id, int i, int j, int k,
                                         bool on_w, R coef) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const R dzl = (on_w ? a.m.dzeta_w[kk] : a.m.dzeta_c[kk]) * a.m.jac[L.at2i(i, j)];
  const int c = L.ati(i, j, k);
  const R ax = coef / (a.dx * a.dx), ay = coef / (a.dy * a.dy), az = coef / (dzl * dzl);
  acc(id, c + 1, ax);
  acc(id, c - 1, ax);
  acc(id, c + L.px, ay);
  acc(id, c - L.px, ay);
  acc(id, c + L.planei(), az);
  acc(id, c - L.planei(), az);
  acc(id, c, -2 * (ax + ay + az));
}

template <typename R>
__device__ __forceinline__ R div_value(const TendArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  return (a.mfx[L.ati(i + 1, j, k)] - a.mfx[L.ati(i, j, k)]) / a.dx +
         (a.mfy[L.ati(i, j + 1, k)] - a.mfy[L.ati(i, j, k)]) / a.dy +
         (a.mfz[L.ati(i, j, k + 1)] - a.mfz[L.ati(i, j, k)]) / a.m.dzeta_c[L.at1(k)];
}

// u tendency row (forward: kernels.cu:308-346)
template <typename R, class Acc>
__device__ void row_tu(Acc& acc, const TendArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const int c = L.ati(i, j, k);
  const int sx = 1, sy = L.px, sz = (int)L.planei();
  const R ru = (R)0.5 * (a.b.rhob[c - sx] * a.m.jac[L.at2i(i - 1, j)] + a.b.rhob[c] * a.m.jac[L.at2i(i, j)]);
  const R dzc = a.m.dzeta_c[kk];
  emit_face_pair(acc, (R)1 / (a.dx * ru), -(R)1 / (a.dx * ru), a.mfx, T_MFX, off(c, -sx), c,
                 c, off(c, sx), true, a.u, T_U, c, sx);
  emit_face_pair(acc, (R)1 / (a.dy * ru), -(R)1 / (a.dy * ru), a.mfy, T_MFY, off(c, -sx), c,
                 off(c, sy - sx), off(c, sy), true, a.u, T_U, c, sy);
  emit_face_pair(acc, (R)1 / (dzc * ru), -(R)1 / (dzc * ru), a.mfz, T_MFZ, off(c, -sx), c,
                 off(c, sz - sx), off(c, sz), true, a.u, T_U, c, sz);
  const R dv = (R)0.5 * (div_value(a, i - 1, j, k) + div_value(a, i, j, k));
  const R u0 = a.u[c];
  emit_div(acc, a, i - 1, j, k, u0 * (R)0.5 / ru);
  emit_div(acc, a, i, j, k, u0 * (R)0.5 / ru);
  acc(T_U, c, dv / ru - sponge(a.m.zeta_c[kk], a.m.zt, a.p));
  const R fc = (R)0.5 * (a.m.fcor[L.at2i(i - 1, j)] + a.m.fcor[L.at2i(i, j)]);
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
  const int c = L.ati(i, j, k);
  const int sx = 1, sy = L.px, sz = (int)L.planei();
  const R rv = (R)0.5 * (a.b.rhob[c - sy] * a.m.jac[L.at2i(i, j - 1)] + a.b.rhob[c] * a.m.jac[L.at2i(i, j)]);
  const R dzc = a.m.dzeta_c[kk];
  emit_face_pair(acc, (R)1 / (a.dy * rv), -(R)1 / (a.dy * rv), a.mfy, T_MFY, off(c, -sy), c,
                 c, off(c, sy), true, a.v, T_V, c, sy);
  emit_face_pair(acc, (R)1 / (a.dx * rv), -(R)1 / (a.dx * rv), a.mfx, T_MFX, off(c, -sy), c,
                 off(c, sx - sy), off(c, sx), true, a.v, T_V, c, sx);
  emit_face_pair(acc, (R)1 / (dzc * rv), -(R)1 / (dzc * rv), a.mfz, T_MFZ, off(c, -sy), c,
                 off(c, sz - sy), off(c, sz), true, a.v, T_V, c, sz);
  const R dv = (R)0.5 * (div_value(a, i, j - 1, k) + div_value(a, i, j, k));
  const R v0 = a.v[c];
  emit_div(acc, a, i, j - 1, k, v0 * (R)0.5 / rv);
  emit_div(acc, a, i, j, k, v0 * (R)0.5 / rv);
  acc(T_V, c, dv / rv - sponge(a.m.zeta_c[kk], a.m.zt, a.p));
  const R fc = (R)0.5 * (a.m.fcor[L.at2i(i, j - 1)] + a.m.fcor[L.at2i(i, j)]);
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
  const int c = L.ati(i, j, k);
  const int sx = 1, sy = L.px, sz = (int)L.planei();
  const R rw = a.b.rhobw[c] * a.m.jac[L.at2i(i, j)];
  const R dzw = a.m.dzeta_w[kk];
  emit_face_pair(acc, (R)1 / (a.dx * rw), -(R)1 / (a.dx * rw), a.mfx, T_MFX, off(c, -sz), c,
                 off(c, sx - sz), off(c, sx), true, a.w, T_W, c, sx);
  emit_face_pair(acc, (R)1 / (a.dy * rw), -(R)1 / (a.dy * rw), a.mfy, T_MFY, off(c, -sz), c,
                 off(c, sy - sz), off(c, sy), true, a.w, T_W, c, sy);
  emit_face_pair(acc, (R)1 / (dzw * rw), -(R)1 / (dzw * rw), a.mfz, T_MFZ, off(c, -sz), c,
                 c, off(c, sz), true, a.w, T_W, c, sz);
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
  const int c = L.ati(i, j, k);
  const int sx = 1, sy = L.px, sz = (int)L.planei();
  const R rt = a.b.rhob[c] * a.m.jac[L.at2i(i, j)];
  const R dzc = a.m.dzeta_c[kk];
  emit_face_pair(acc, (R)1 / (a.dx * rt), -(R)1 / (a.dx * rt), a.mfx, T_MFX, c, c,
                 off(c, sx), 0, false, a.thp, T_TH, c, sx);
  emit_face_pair(acc, (R)1 / (a.dy * rt), -(R)1 / (a.dy * rt), a.mfy, T_MFY, c, c,
                 off(c, sy), 0, false, a.thp, T_TH, c, sy);
  emit_face_pair(acc, (R)1 / (dzc * rt), -(R)1 / (dzc * rt), a.mfz, T_MFZ, c, c,
                 off(c, sz), 0, false, a.thp, T_TH, c, sz);
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
  const int c = L.ati(i, j, k);
  const int sx = 1, sy = L.px, sz = (int)L.planei();
  const R rt = a.b.rhob[c] * a.m.jac[L.at2i(i, j)];
  const R dzc = a.m.dzeta_c[kk];
  emit_face_pair(acc, (R)1 / (a.dx * rt), -(R)1 / (a.dx * rt), a.mfx, T_MFX, c, c,
                 off(c, sx), 0, false, q, qid, c, sx);
  emit_face_pair(acc, (R)1 / (a.dy * rt), -(R)1 / (a.dy * rt), a.mfy, T_MFY, c, c,
                 off(c, sy), 0, false, q, qid, c, sy);
  emit_face_pair(acc, (R)1 / (dzc * rt), -(R)1 / (dzc * rt), a.mfz, T_MFZ, c, c,
                 off(c, sz), 0, false, q, qid, c, sz);
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
  const int c = L.ati(i, j, k);
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

// The adjoint runs as one launch per output group (PART: AD_U, AD_V, AD_W,
// AD_TH with the pi' tendency, AD_Q for the three species): each launch is a
// small kernel, where the fused one stalled on instruction fetch.
enum { AD_U = 0, AD_V, AD_W, AD_TH, AD_Q };

template <typename R, int PART>
__global__ void __launch_bounds__(256) k_ad_tend(TendArgs<R> a, TendArgs<R> d) {
  const Layout& L = a.L;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= L.nx || j >= L.ny || k >= L.nz) return;
  const int c = L.ati(i, j, k);
  const Ptrs<R, T_N> P = tend_ptrs(d);
  // each output adjoint is cleared once it has been read and used (a store
  // issued while the load of the same address is in flight stalls the
  // memory pipeline)
  if (PART == AD_U) {
    ADAcc<R, T_N> acc{P, d.tu[c]};
    if (acc.ybar != (R)0) {
      row_tu(acc, a, i, j, k);
      d.tu[c] = 0;
    }
  } else if (PART == AD_V) {
    ADAcc<R, T_N> acc{P, d.tv[c]};
    if (acc.ybar != (R)0) {
      row_tv(acc, a, i, j, k);
      d.tv[c] = 0;
    }
  } else if (PART == AD_W) {
    if (k >= 1) {
      ADAcc<R, T_N> acc{P, d.tw[c]};
      if (acc.ybar != (R)0) {
        row_tw(acc, a, i, j, k);
        d.tw[c] = 0;
      }
    }
  } else if (PART == AD_TH) {
    ADAcc<R, T_N> acc{P, d.tth[c]};
    if (acc.ybar != (R)0) {
      row_tth(acc, a, i, j, k);
      d.tth[c] = 0;
    }
    if (d.tpi && d.tpi[c] != (R)0) d.tpi[c] = 0;
  } else {
    const R* qf[3] = {a.qv, a.qc, a.qr};
    R* qo[3] = {d.qo_v, d.qo_c, d.qo_r};
    R* qn[3] = {const_cast<R*>(d.qn_v), const_cast<R*>(d.qn_c), const_cast<R*>(d.qn_r)};
    R* tq[3] = {d.tqv, d.tqc, d.tqr};
#pragma unroll 1
    for (int sp = 0; sp < 3; ++sp) {
      R* y = qo[sp] ? qo[sp] : tq[sp];
      const R gy = y[c];
      if (gy == (R)0) continue;
      R g = gy;
      if (qo[sp]) {
        // stage value q_n + dt_stage * tq: q_n takes gy (in place: keeps it)
        g = a.dt_stage * gy;
        if (qn[sp] != qo[sp]) {
          atomicAdd(qn[sp] + c, gy);
          y[c] = 0;
        }
      } else {
        y[c] = 0;
      }
      ADAcc<R, T_N> acc{P, g};
      row_tq(acc, a, qf[sp], T_QV + sp, i, j, k);
    }
  }
}

// ================================================================ ghost fill
// Adjoint of the ghost fill (forward: dyn_tend.cu fill_body): every written
// ghost value moves its adjoint onto its sources and is zeroed.  The sources
// are interior points, never other ghosts, so the points can go in any order.
// Threads cover only ghost points: k_ad_fill_levels the ghost levels of the
// interior columns, k_ad_fill_ring every level of the lateral ghost columns.
template <typename R>
__device__ __forceinline__ void ad_fill_point(const FillArgs<R>& A, int f, int i, int j, int k) {
  const Layout& L = A.L;
  R* a = A.job.f[f];
  const int kind = A.job.kind[f];
  const int ilast = (kind == 1 && A.open_x) ? L.nx : L.nx - 1;
  const int jlast = (kind == 2 && A.open_y) ? L.ny : L.ny - 1;
  const int si = map_lat(i, L.nx, ilast, A.open_x);
  const int sj = map_lat(j, L.ny, jlast, A.open_y);
  const bool lateral = (si != i) || (sj != j);
  // an interior level of a column that is not a ghost (the u face nx of an
  // open x boundary, the v face ny of an open y boundary)
  if (!lateral && k >= 0 && k < L.nz) return;
  const int q = L.ati(i, j, k);
  // the ghost's adjoint moves to its sources; it is cleared only once read
  // (a store issued while the load of the same address is in flight stalls
  // the memory pipeline)
  const R g = a[q];
  if (g == (R)0) return;
  a[q] = 0;
  if (kind == 3) {
    if (k == L.nz) return;
    if (k >= 0 && k < L.nz) atomicAdd(a + L.ati(si, sj, k), g);
    else if (k < 0) {
      atomicAdd(a + L.ati(si, sj, 0), (R)2 * g);
      atomicAdd(a + L.ati(si, sj, -k), -g);
    } else {
      atomicAdd(a + L.ati(si, sj, 2 * L.nz - k), -g);
    }
  } else {
    atomicAdd(a + L.ati(si, sj, map_zc(k, L.nz)), g);
  }
}

// grid (nx ny / 256, 7 ghost levels: -3..-1 and nz..nz+3, fields)
template <typename R>
__global__ void __launch_bounds__(256) k_ad_fill_levels(FillArgs<R> A) {
  const Layout& L = A.L;
  const int f = blockIdx.z;
  const int col = (int)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= A.job.n || col >= (int)L.nx * L.ny) return;
  const int m = blockIdx.y;
  const int k = m < kRefNG ? m - kRefNG : L.nz + (m - kRefNG);
  ad_fill_point(A, f, (int)(col % L.nx), (int)(col / L.nx), k);
}

// grid (ring columns / 256, levels -3..nz+3, fields): the lateral ghost
// columns (ring_column)
template <typename R>
__global__ void __launch_bounds__(256) k_ad_fill_ring(FillArgs<R> A) {
  const Layout& L = A.L;
  const int f = blockIdx.z;
  const int r = (int)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= A.job.n || r >= ring_columns(L)) return;
  int i, j;
  ring_column(L, r, &i, &j);
  ad_fill_point(A, f, i, j, (int)blockIdx.y - kRefNG);
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
  const int c = L.ati(i, j, k);
  R* ub = const_cast<R*>(A.u);
  R* vb = const_cast<R*>(A.v);
  R* wb = const_cast<R*>(A.w);
  if (k < L.nz) {
    const R gx = A.mfx[c], gy = A.mfy[c];
    R rjx = (R)0.5 * (A.b.rhob[L.ati(i - 1, j, k)] * A.m.jac[L.at2i(i - 1, j)] +
                      A.b.rhob[c] * A.m.jac[L.at2i(i, j)]);
    R rjy = (R)0.5 * (A.b.rhob[L.ati(i, j - 1, k)] * A.m.jac[L.at2i(i, j - 1)] +
                      A.b.rhob[c] * A.m.jac[L.at2i(i, j)]);
    if (gx != (R)0) {
      atomicAdd(ub + c, rjx * gx);
      A.mfx[c] = 0;
    }
    if (gy != (R)0) {
      atomicAdd(vb + c, rjy * gy);
      A.mfy[c] = 0;
    }
  }
  if (i > L.nx + 1 || j > L.ny + 1) return;
  const R gz = A.mfz[c];
  if (gz == (R)0) return;
  A.mfz[c] = 0;
  if (k == 0 || k == L.nz) return;
  const int kk = L.at1(k);
  R fac = (R)1 - A.m.zeta_w[kk] / A.m.zt;
  R rw = A.b.rhobw[c];
  atomicAdd(wb + c, rw * gz);
  R cu = -rw * gz * (R)0.25 * A.m.hx[L.at2i(i, j)] * fac;
  R cv = -rw * gz * (R)0.25 * A.m.hy[L.at2i(i, j)] * fac;
  if (cu != (R)0) {
    atomicAdd(ub + L.ati(i, j, k - 1), cu);
    atomicAdd(ub + L.ati(i + 1, j, k - 1), cu);
    atomicAdd(ub + c, cu);
    atomicAdd(ub + L.ati(i + 1, j, k), cu);
  }
  if (cv != (R)0) {
    atomicAdd(vb + L.ati(i, j, k - 1), cv);
    atomicAdd(vb + L.ati(i, j + 1, k - 1), cv);
    atomicAdd(vb + c, cv);
    atomicAdd(vb + L.ati(i, j + 1, k), cv);
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
    const int c = L.ati(i, j, k);
    acc(A_PICUR, c, coef * ((R)1 + sm));
    acc(A_PIPREV, c, -coef * sm);
  } else {
    const int c = L.ati(map_lat(i, L.nx, L.nx - 1, a.p.bc_x_open),
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
  const int c = L.ati(i, j, k);
  const int s =
      lat ? L.ati(map_lat(i, L.nx, L.nx - 1, a.p.bc_x_open), map_lat(j, L.ny, L.ny - 1, a.p.bc_y_open), k)
          : c;
  R f = coef;
  if (a.p.moisture) {
    const R th = a.b.thb[c] + (lat ? a.n_thp[s] : a.th_in[c]);
    f = coef * ((R)1 + Phys<R>::eps61 * a.qv[s]);
    acc(A_QV, s, coef * th * Phys<R>::eps61);
  }
  acc(lat ? A_NTHP : A_THIN, s, f);
}

// The pressure-gradient terms of the u (is_u) or v step at a face
// (kernels.cu:499-526): face theta_v and map factor, the horizontal pi*
// gradient with its terrain correction, and what the correction is made of.
template <typename R>
struct UvFace {
  R thf, mf, h, grad, slope, jf, dzc2;
};

template <typename R>
__device__ __forceinline__ UvFace<R> uv_face_terms(const AcouArgs<R>& a, int i, int j, int k, bool is_u) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const int di = is_u ? 1 : 0, dj = is_u ? 0 : 1;
  UvFace<R> f;
  f.thf = (R)0.5 * (theta_v(a, i - di, j - dj, k) + theta_v(a, i, j, k));
  f.mf = (R)0.5 * (a.m.mapf[L.at2i(i - di, j - dj)] + a.m.mapf[L.at2i(i, j)]);
  f.h = is_u ? a.dx : a.dy;
  f.grad = (pistar(a, i, j, k) - pistar(a, i - di, j - dj, k)) / f.h;
  f.slope = (is_u ? a.m.hx_u[L.at2i(i, j)] : a.m.hy_v[L.at2i(i, j)]) * ((R)1 - a.m.zeta_c[kk] / a.m.zt);
  f.dzc2 = 1;
  f.jf = 1;
  if (f.slope != (R)0) {
    f.dzc2 = a.m.zeta_c[kk + 1] - a.m.zeta_c[kk - 1];
    f.jf = (R)0.5 * (a.m.jac[L.at2i(i - di, j - dj)] + a.m.jac[L.at2i(i, j)]);
    R dpdz = (R)0.5 *
             ((pistar(a, i - di, j - dj, k + 1) - pistar(a, i - di, j - dj, k - 1)) +
              (pistar(a, i, j, k + 1) - pistar(a, i, j, k - 1))) /
             f.dzc2;
    f.grad -= f.slope / f.jf * dpdz;
  }
  return f;
}

// forward u (is_u) or v step at a face and, when acc is given, coef times
// its Jacobian row (kernels.cu:499-526)
template <typename R, class Acc>
__device__ R uv_face(Acc* acc, const AcouArgs<R>& a, int i, int j, int k, bool is_u, R coef) {
  const Layout& L = a.L;
  const int di = is_u ? 1 : 0, dj = is_u ? 0 : 1;
  const UvFace<R> f = uv_face_terms(a, i, j, k, is_u);
  const int c = L.ati(i, j, k);
  const R* tin = is_u ? a.tu : a.tv;
  const R* vin = is_u ? a.u_in : a.v_in;
  const R out = vin[c] + a.dtau * (-Phys<R>::cp * f.thf * f.mf * f.grad + tin[c]);
  if (acc) {
    (*acc)(is_u ? A_UIN : A_VIN, c, coef);
    (*acc)(is_u ? A_TU : A_TV, c, coef * a.dtau);
    const R g1 = -coef * a.dtau * Phys<R>::cp * f.mf;
    emit_thv(*acc, a, i - di, j - dj, k, g1 * f.grad * (R)0.5);
    emit_thv(*acc, a, i, j, k, g1 * f.grad * (R)0.5);
    const R g2 = g1 * f.thf;
    emit_pistar(*acc, a, i, j, k, g2 / f.h);
    emit_pistar(*acc, a, i - di, j - dj, k, -g2 / f.h);
    if (f.slope != (R)0) {
      const R g3 = -g2 * f.slope / f.jf * (R)0.5 / f.dzc2;
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
      const int c0 = L.ati(0, j, k);
      const R u0 = a.u_in[c0];
      if (u0 >= (R)0) return;  // out = ub
      const R cb = u0 - cstar;
      const R uf1 = uv_face<R, Acc>(nullptr, a, 1, j, k, true, 0);
      acc(A_UIN, c0, coef * ((R)1 - a.dtau / a.dx * (uf1 - u0 - cb)));
      uv_face(&acc, a, 1, j, k, true, -coef * a.dtau * cb / a.dx);
    } else if (i == L.nx) {
      const int cn = L.ati(L.nx, j, k);
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
      const int c0 = L.ati(i, 0, k);
      const R v0 = a.v_in[c0];
      if (v0 >= (R)0) return;  // out = 0
      const R cb = v0 - cstar;
      const R vf1 = uv_face<R, Acc>(nullptr, a, i, 1, k, false, 0);
      acc(A_VIN, c0, coef * ((R)1 - a.dtau / a.dy * (vf1 - v0 - cb)));
      uv_face(&acc, a, i, 1, k, false, -coef * a.dtau * cb / a.dy);
    } else if (j == L.ny) {
      const int cn = L.ati(i, L.ny, k);
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

// FP32: eight CTAs per SM (32 registers) for the load-bound u, v kernels
template <typename R>
constexpr int kUvLinMinBlocks = sizeof(R) == 4 ? 8 : 1;

template <typename R>
__global__ void __launch_bounds__(256, kUvLinMinBlocks<R>) k_tl_uv(AcouArgs<R> a, AcouArgs<R> d) {
  const Layout& L = a.L;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i > L.nx || j > L.ny || k >= L.nz) return;
  const Ptrs<R, A_N> P = acou_ptrs(d);
  if (j < L.ny) {
    TLAcc<R, A_N> acc{P, 0};
    row_u_out(acc, a, i, j, k, (R)1);
    d.u_out[L.ati(i, j, k)] = acc.sum;
  }
  if (i < L.nx) {
    TLAcc<R, A_N> acc{P, 0};
    row_v_out(acc, a, i, j, k, (R)1);
    d.v_out[L.ati(i, j, k)] = acc.sum;
  }
}

// Adjoint of the u, v step in gather form, two launches and no atomics.
// (1) Per face: the face's own output adjoint, plus what a radiation face
//     (open boundaries) or the periodic face nx adds to the face it was
//     computed from, gives the coefficient of that face's uv_face row; the
//     face writes its u_in / tendency adjoint and three coefficients -- of
//     the pi* difference (gp), of the terrain pi* correction (gs) and of the
//     two theta_v values (gt) -- into scratch.
// (2) Per cell: gathers the coefficients of the faces around the cell (and
//     of the ghost cells the cell is the source of) into pi', pi'_prev /
//     time-n pi', theta' / time-n theta' and qv adjoints, and clears the face
//     output adjoints.
template <typename R>
struct UvScr {
  R *gp_u, *gs_u, *gt_u, *gp_v, *gs_v, *gt_v;
};

template <typename R>
__device__ __forceinline__ void ad_uv_face(const AcouArgs<R>& a, const AcouArgs<R>& d, int i, int j, int k,
                                           bool is_u, R* gp, R* gs, R* gt) {
  const Layout& L = a.L;
  const int n = is_u ? L.nx : L.ny;       // faces 0..n along the face normal
  const int f = is_u ? i : j;             // this face's index along it
  const bool open = is_u ? a.p.bc_x_open : a.p.bc_y_open;
  const R h = is_u ? a.dx : a.dy;
  const R cstar = a.p.cstar;
  const R* yb = is_u ? d.u_out : d.v_out;
  const R* xin = is_u ? a.u_in : a.v_in;
  R* xb = const_cast<R*>(is_u ? d.u_in : d.v_in);
  R* tb = const_cast<R*>(is_u ? d.tu : d.tv);
  auto at_f = [&](int q) { return is_u ? L.ati(q, j, k) : L.ati(i, q, k); };
  const int c = L.ati(i, j, k);
  R ce = 0;  // coefficient of the uv_face row at this face
  if (open) {
    if (f == 0 || f == n) {
      // radiation face (kernels.cu:654-667, 674-687): its own u_in term
      const R x0 = xin[c], g = yb[c];
      if (g != (R)0 && (f == 0 ? x0 < (R)0 : x0 > (R)0)) {
        const R cb = f == 0 ? x0 - cstar : x0 + cstar;
        const R xf = uv_face<R, ADAcc<R, A_N>>(nullptr, a, is_u ? (f == 0 ? 1 : n - 1) : i,
                                                is_u ? j : (f == 0 ? 1 : n - 1), k, is_u, 0);
        const R dd = f == 0 ? (xf - x0 - cb) : (x0 - xf + cb);
        xb[c] += g * ((R)1 - a.dtau / h * dd);
      }
    } else {
      ce = yb[c];
      if (f == 1) {
        const int c0 = at_f(0);
        const R x0 = xin[c0];
        if (x0 < (R)0) ce += -yb[c0] * a.dtau * (x0 - cstar) / h;
      }
      if (f == n - 1) {
        const int cn = at_f(n);
        const R xn = xin[cn];
        if (xn > (R)0) ce += yb[cn] * a.dtau * (xn + cstar) / h;
      }
    }
  } else if (f < n) {
    ce = yb[c];
    if (f == 0) ce += yb[at_f(n)];  // face n repeats face 0
  }
  R p = 0, s = 0, t = 0;
  if (ce != (R)0) {
    const UvFace<R> u = uv_face_terms(a, i, j, k, is_u);
    xb[c] += ce;
    tb[c] += ce * a.dtau;
    const R g1 = -ce * a.dtau * Phys<R>::cp * u.mf;
    t = g1 * u.grad * (R)0.5;
    const R g2 = g1 * u.thf;
    p = g2 / u.h;
    if (u.slope != (R)0) s = -g2 * u.slope / u.jf * (R)0.5 / u.dzc2;
  }
  gp[c] = p;
  gs[c] = s;
  gt[c] = t;
}

template <typename R>
__global__ void __launch_bounds__(256, kUvLinMinBlocks<R>) k_ad_uv_faces(AcouArgs<R> a, AcouArgs<R> d, UvScr<R> w) {
  const Layout& L = a.L;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i > L.nx || j > L.ny || k >= L.nz) return;
  if (j < L.ny) ad_uv_face(a, d, i, j, k, true, w.gp_u, w.gs_u, w.gt_u);
  if (i < L.nx) ad_uv_face(a, d, i, j, k, false, w.gp_v, w.gs_v, w.gt_v);
}

template <typename R>
__global__ void __launch_bounds__(256, kUvLinMinBlocks<R>) k_ad_uv_cells(AcouArgs<R> a, AcouArgs<R> d, UvScr<R> w) {
  const Layout& L = a.L;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  if (i >= nx || j >= ny || k >= nz) return;
  // face coefficients, zero outside the faces that exist
  auto U = [&](const R* g, int fi, int fj, int fk) -> R {
    return (fi >= 0 && fi <= nx && fj >= 0 && fj < ny && fk >= 0 && fk < nz) ? g[L.ati(fi, fj, fk)] : (R)0;
  };
  auto V = [&](const R* g, int fi, int fj, int fk) -> R {
    return (fi >= 0 && fi < nx && fj >= 0 && fj <= ny && fk >= 0 && fk < nz) ? g[L.ati(fi, fj, fk)] : (R)0;
  };
  // adjoint of pi* at cell (ci, cj, ck), interior or ghost (emit_pistar)
  auto pbar = [&](int ci, int cj, int ck) -> R {
    return U(w.gp_u, ci, cj, ck) - U(w.gp_u, ci + 1, cj, ck) + V(w.gp_v, ci, cj, ck) -
           V(w.gp_v, ci, cj + 1, ck) + U(w.gs_u, ci, cj, ck - 1) - U(w.gs_u, ci, cj, ck + 1) +
           U(w.gs_u, ci + 1, cj, ck - 1) - U(w.gs_u, ci + 1, cj, ck + 1) + V(w.gs_v, ci, cj, ck - 1) -
           V(w.gs_v, ci, cj, ck + 1) + V(w.gs_v, ci, cj + 1, ck - 1) - V(w.gs_v, ci, cj + 1, ck + 1);
  };
  const int c = L.ati(i, j, k);
  const R sm = a.p.acoustic_smdiv;
  R* piC = const_cast<R*>(d.pi_cur);
  R* piP = const_cast<R*>(d.pi_prev);
  R* npB = const_cast<R*>(d.n_pip);
  R* thB = const_cast<R*>(d.th_in);
  R* ntB = const_cast<R*>(d.n_thp);
  R* qvB = const_cast<R*>(d.qv);
  // periodic ghosts whose source is this cell: column -1 (row -1) maps to nx - 1 (ny - 1)
  const bool gx = !a.p.bc_x_open && i == nx - 1;
  const bool gy = !a.p.bc_y_open && j == ny - 1;
  {
    const R X = pbar(i, j, k);
    R Xg = 0;
    if (k == 0) Xg += pbar(i, j, -1);
    if (k == nz - 1) Xg += pbar(i, j, nz);
    if (gx) {
      Xg += pbar(-1, j, k);
      if (k == 0) Xg += pbar(-1, j, -1);
      if (k == nz - 1) Xg += pbar(-1, j, nz);
    }
    if (gy) {
      Xg += pbar(i, -1, k);
      if (k == 0) Xg += pbar(i, -1, -1);
      if (k == nz - 1) Xg += pbar(i, -1, nz);
    }
    // pi' and the three pi'_prev / time-n pi' buffers may coincide: one
    // update after another in this thread
    if (X != (R)0) {
      piC[c] += ((R)1 + sm) * X;
      piP[c] += -sm * X;
    }
    if (Xg != (R)0) {
      piC[c] += ((R)1 + sm) * Xg;
      npB[c] += -sm * Xg;
    }
  }
  {
    const bool moist = a.p.moisture != 0;
    const R T = U(w.gt_u, i, j, k) + U(w.gt_u, i + 1, j, k) + V(w.gt_v, i, j, k) + V(w.gt_v, i, j + 1, k);
    if (T != (R)0) {
      if (moist) {
        thB[c] += T * ((R)1 + Phys<R>::eps61 * a.qv[c]);
        qvB[c] += T * (a.b.thb[c] + a.th_in[c]) * Phys<R>::eps61;
      } else {
        thB[c] += T;
      }
    }
    R Tg[2] = {gx ? U(w.gt_u, 0, j, k) : (R)0, gy ? V(w.gt_v, i, 0, k) : (R)0};
    const int gc[2] = {L.ati(-1, j, k), L.ati(i, -1, k)};
    for (int q = 0; q < 2; ++q) {
      if (Tg[q] == (R)0) continue;
      if (moist) {
        ntB[c] += Tg[q] * ((R)1 + Phys<R>::eps61 * a.qv[c]);
        qvB[c] += Tg[q] * (a.b.thb[gc[q]] + a.n_thp[c]) * Phys<R>::eps61;
      } else {
        ntB[c] += Tg[q];
      }
    }
  }
  // the output adjoints are consumed
  d.u_out[c] = 0;
  d.v_out[c] = 0;
  if (i == nx - 1) d.u_out[L.ati(nx, j, k)] = 0;
  if (j == ny - 1) d.v_out[L.ati(i, ny, k)] = 0;
}

// ================================================================ w - pi' column
// A CTA owns kLcx columns of one row with kLkl level lanes; the column arrays
// live in shared memory ([level * kLcx + column]); the sweeps run in one lane
// per column, everything else in parallel over the levels.
// FP32 tiles hold 16 columns x 8 level lanes; FP64 keeps 8 columns x 16 lanes
// so that the adjoint's arrays for lin_max_levels() levels fit in shared memory
template <typename R>
constexpr int kLcx = sizeof(R) == 4 ? 16 : 8;
template <typename R>
constexpr int kLkl = sizeof(R) == 4 ? 8 : 16;

// rows 1..n-1 of a tridiagonal system (row 1 without A, row n-1 without C),
// the forward's elimination (kernels.cu:612-634; dyn_acou.cu phase 4: one
// reciprocal per row); arrays strided by kLcx<R>
template <typename R>
__device__ __forceinline__ void thomas_s(int n, const R* A, const R* B, const R* C, const R* D, R* cs, R* ds,
                                         R* x) {
  R cp = 0, dp = 0;
  for (int k = 1; k < n; ++k) {
    const int q = k * kLcx<R>;
    if (k == 1) {
      const R r = (R)1 / B[q];
      cp = C[q] * r;
      dp = D[q] * r;
    } else {
      const R r = (R)1 / (B[q] - A[q] * cp);
      cp = C[q] * r;
      dp = (D[q] - A[q] * dp) * r;
    }
    cs[q] = cp;
    ds[q] = dp;
  }
  x[n * kLcx<R>] = 0;
  R above = 0;
  for (int k = n - 1; k >= 1; --k) {
    above = ds[k * kLcx<R>] - cs[k * kLcx<R>] * above;
    x[k * kLcx<R>] = above;
  }
}

// the transposed system: (M^T)_{k,k-1} = C[k-1], (M^T)_{k,k+1} = A[k+1]
template <typename R>
__device__ __forceinline__ void thomas_ts(int n, const R* A, const R* B, const R* C, const R* D, R* cs, R* ds,
                                          R* x) {
  R cp = 0, dp = 0;
  for (int k = 1; k < n; ++k) {
    const int q = k * kLcx<R>;
    const R sub = k > 1 ? C[q - kLcx<R>] : (R)0;
    const R sup = k < n - 1 ? A[q + kLcx<R>] : (R)0;
    if (k == 1) {
      const R r = (R)1 / B[q];
      cp = sup * r;
      dp = D[q] * r;
    } else {
      const R r = (R)1 / (B[q] - sub * cp);
      cp = sup * r;
      dp = (D[q] - sub * dp) * r;
    }
    cs[q] = cp;
    ds[q] = dp;
  }
  x[n * kLcx<R>] = 0;
  x[0] = 0;
  R above = 0;
  for (int k = n - 1; k >= 1; --k) {
    above = ds[k * kLcx<R>] - cs[k * kLcx<R>] * above;
    x[k * kLcx<R>] = above;
  }
}

// shared column arrays: a fixed set of (nz + 1)-level arrays
template <typename R>
struct ColArr {
  R* base;
  int n1;  // nz + 1
  __device__ R* operator[](int q) const { return base + (int)q * n1 * kLcx<R>; }
};

// What the TL and AD kernels of one column share: the column's geometry and
// its level k at c0 + k * pl, as the forward column kernel addresses it.
template <typename R>
struct ColGeom {
  int nz;
  R dtau, c1, c2, J, invJ, hxc, hyc, mc, mcx, mcy;
  bool terrain;
  int c0, sx, sy, pl;
  __device__ ColGeom(const AcouArgs<R>& a, int i, int j, bool active) {
    const Layout& L = a.L;
    nz = L.nz;
    dtau = a.dtau;
    c1 = ((R)1 + a.p.acoustic_beta) * (R)0.5;
    c2 = ((R)1 - a.p.acoustic_beta) * (R)0.5;
    const int c2d = L.at2i(active ? i : 0, j);
    J = a.m.jac[c2d];
    hxc = a.m.hx[c2d];
    hyc = a.m.hy[c2d];
    mc = a.m.mapf[c2d];
    invJ = (R)1 / J;
    mcx = mc * a.co.inv_dx;
    mcy = mc * a.co.inv_dy;
    terrain = hxc != (R)0 || hyc != (R)0;
    sx = 1;
    sy = L.px;
    pl = L.planei();
    c0 = L.ati(active ? i : 0, j, 0);
  }
  __device__ int at(int k) const { return c0 + (int)k * pl; }
};

// Forward values of one column (kernels.cu:552-634) with the forward column
// kernel's expressions (dyn_acou.cu phases 1-4), into shared arrays: Av, Sv,
// P, E on levels; G, A, B, C, D on the inner levels; the solution w (with the
// surface w at level 0).  Ends with a barrier.
enum { V_AV, V_SV, V_P, V_E, V_G, V_A, V_B, V_C, V_D, V_W, V_CS, V_DS, V_N };

template <typename R>
__device__ __forceinline__ void column_values_s(const AcouArgs<R>& a, const ColGeom<R>& g, bool active,
                                                const ColArr<R>& S) {
  const Layout& L = a.L;
  const int nz = g.nz, tx = threadIdx.x, lane = threadIdx.y;
  const R dtau = g.dtau, c1 = g.c1, c2 = g.c2;
  const R* __restrict__ u = a.u_out;
  const R* __restrict__ v = a.v_out;
  const int sx = g.sx, sy = g.sy, pl = g.pl;
  R *Av = S[V_AV] + tx, *Sv = S[V_SV] + tx, *P = S[V_P] + tx, *E = S[V_E] + tx;
  R *G = S[V_G] + tx, *A = S[V_A] + tx, *B = S[V_B] + tx, *C = S[V_C] + tx, *D = S[V_D] + tx;
  if (active)
#pragma unroll 4
    for (int k = lane; k <= nz; k += kLkl<R>) {
      R av = 0, sv = 0;
      if (k >= 1 && k < nz) {
        const int c = g.at(k), cm = c - pl;
        av = a.co.aw[c];
        if (g.terrain) {
          R uw = (R)0.25 * (u[cm] + u[cm + sx] + u[c] + u[c + sx]);
          R vw = (R)0.25 * (v[cm] + v[cm + sy] + v[c] + v[c + sy]);
          sv = av * (uw * g.hxc + vw * g.hyc) * a.co.fac_w[L.at1(k)];
        }
      }
      Av[k * kLcx<R>] = av;
      Sv[k * kLcx<R>] = sv;
    }
  __syncthreads();
  if (active)
#pragma unroll 4
    for (int k = lane; k < nz; k += kLkl<R>) {
      const int c = g.at(k);
      R Kt = a.co.kt3[c];
      R Dh = (a.co.rtjx[c + sx] * u[c + sx] - a.co.rtjx[c] * u[c]) * g.mcx +
             (a.co.rtjy[c + sy] * v[c + sy] - a.co.rtjy[c] * v[c]) * g.mcy;
      R idz = a.co.inv_dzc[L.at1(k)];
      R wk = a.w_in[c], wkp = a.w_in[c + pl];
      R tpi = a.tpi ? a.tpi[c] : (R)0;
      const int q = k * kLcx<R>;
      P[q] = a.pi_cur[c] + dtau * tpi -
             dtau * Kt * (Dh - (Sv[q + kLcx<R>] - Sv[q]) * idz + c2 * (Av[q + kLcx<R>] * wkp - Av[q] * wk) * idz);
      E[q] = dtau * Kt * c1 * idz;
    }
  __syncthreads();
  if (active)
#pragma unroll 4
    for (int k = 1 + lane; k < nz; k += kLkl<R>) {
      const int c = g.at(k), cm = c - pl;
      const R iJdz = g.invJ * a.co.inv_dzw[L.at1(k)];
      R thc = a.th_in[c], thm = a.th_in[cm];
      R thbw = a.b.thbw[c];
      R thvw = thbw + (R)0.5 * (thm + thc);
      if (a.p.moisture) thvw *= (R)1 + Phys<R>::eps61 * (R)0.5 * (a.qv[cm] + a.qv[c]);
      R Gk = dtau * Phys<R>::cp * thvw * c1 * iJdz;
      const int q = k * kLcx<R>;
      const R Em = E[q - kLcx<R>], Ek = E[q];
      G[q] = Gk;
      A[q] = -Gk * Em * Av[q - kLcx<R>];
      B[q] = (R)1 + Gk * Av[q] * (Ek + Em);
      C[q] = -Gk * Ek * Av[q + kLcx<R>];
      R buoy = Phys<R>::grav * (R)0.5 * (thm + thc) / thbw;
      if (a.p.moisture) {
        R dqv = (R)0.5 * (a.qv[cm] + a.qv[c]) - (R)0.5 * (a.b.qvb[cm] + a.b.qvb[c]);
        R qcr = (R)0.5 * (a.qc[cm] + a.qc[c]) + (R)0.5 * (a.qr[cm] + a.qr[c]);
        buoy += Phys<R>::grav * (Phys<R>::eps61 * dqv - qcr);
      }
      R RHS = a.w_in[c] + dtau * (buoy + a.tw[c]) -
              dtau * Phys<R>::cp * thvw * c2 * (a.pi_cur[c] - a.pi_cur[cm]) * iJdz;
      D[q] = RHS - Gk * (P[q] - P[q - kLcx<R>]);
    }
  __syncthreads();
  if (active && lane == 0) {
    R* W = S[V_W] + tx;
    thomas_s(nz, A, B, C, D, S[V_CS] + tx, S[V_DS] + tx, W);
    R us = (R)0.5 * (u[g.c0] + u[g.c0 + sx]);
    R vs = (R)0.5 * (v[g.c0] + v[g.c0 + sy]);
    W[0] = us * g.hxc + vs * g.hyc;
  }
  __syncthreads();
}

// The same values from the forward launch's outputs, for the adjoint sweep
// when they are still in place (the adjoint runs before the launch's outputs
// are restored): W is the forward w_out (its level 0 the surface w), P follows
// from pi_next = P - E (Av(k+1) W(k+1) - Av(k) W(k)) up to rounding, and the
// rows A, B, C, G from the inputs as before; no Thomas sweep, no right-hand
// side.  a.w_in and a.th_in must hold the launch's inputs (the undo log's
// copies where the launch updated them in place).  Ends with a barrier.
template <typename R>
__device__ __forceinline__ void column_values_stored_s(const AcouArgs<R>& a, const ColGeom<R>& g, bool active,
                                                       const ColArr<R>& S) {
  const Layout& L = a.L;
  const int nz = g.nz, tx = threadIdx.x, lane = threadIdx.y;
  const R dtau = g.dtau, c1 = g.c1;
  R *Av = S[V_AV] + tx, *P = S[V_P] + tx, *E = S[V_E] + tx, *W = S[V_W] + tx;
  R *G = S[V_G] + tx, *A = S[V_A] + tx, *B = S[V_B] + tx, *C = S[V_C] + tx;
  if (active)
#pragma unroll 4
    for (int k = lane; k <= nz; k += kLkl<R>) {
      const int c = g.at(k);
      Av[k * kLcx<R>] = (k >= 1 && k < nz) ? a.co.aw[c] : (R)0;
      W[k * kLcx<R>] = k < nz ? a.w_out[c] : (R)0;
    }
  __syncthreads();
  if (active)
#pragma unroll 4
    for (int k = lane; k < nz; k += kLkl<R>) {
      const int c = g.at(k);
      const int q = k * kLcx<R>;
      const R e = dtau * a.co.kt3[c] * c1 * a.co.inv_dzc[L.at1(k)];
      E[q] = e;
      P[q] = a.pi_next[c] + e * (Av[q + kLcx<R>] * W[q + kLcx<R>] - Av[q] * W[q]);
    }
  __syncthreads();
  if (active)
#pragma unroll 4
    for (int k = 1 + lane; k < nz; k += kLkl<R>) {
      const int c = g.at(k), cm = c - g.pl;
      const R iJdz = g.invJ * a.co.inv_dzw[L.at1(k)];
      R thvw = a.b.thbw[c] + (R)0.5 * (a.th_in[cm] + a.th_in[c]);
      if (a.p.moisture) thvw *= (R)1 + Phys<R>::eps61 * (R)0.5 * (a.qv[cm] + a.qv[c]);
      const R Gk = dtau * Phys<R>::cp * thvw * c1 * iJdz;
      const int q = k * kLcx<R>;
      const R Em = E[q - kLcx<R>], Ek = E[q];
      G[q] = Gk;
      A[q] = -Gk * Em * Av[q - kLcx<R>];
      B[q] = (R)1 + Gk * Av[q] * (Ek + Em);
      C[q] = -Gk * Ek * Av[q + kLcx<R>];
    }
  __syncthreads();
}

enum { T_DSV = V_N, T_DTH, T_DP, T_RHS, T_DW, T_NARR };

template <typename R>
__global__ void __launch_bounds__(kLcx<R> * kLkl<R>) k_tl_column(AcouArgs<R> a, AcouArgs<R> d, int with_forward) {
  extern __shared__ __align__(16) unsigned char lin_smem[];
  const Layout& L = a.L;
  const int tx = threadIdx.x, lane = threadIdx.y;
  const int i = blockIdx.x * kLcx<R> + tx, j = blockIdx.y;
  const bool active = i < L.nx;
  const ColArr<R> S{reinterpret_cast<R*>(lin_smem), L.nz + 1};
  const ColGeom<R> g(a, i, j, active);
  const int nz = g.nz;
  const R dtau = g.dtau, c1 = g.c1, c2 = g.c2;
  const R* __restrict__ du = d.u_out;
  const R* __restrict__ dv = d.v_out;
  const int sx = g.sx, sy = g.sy, pl = g.pl;
  R *dSv = S[T_DSV] + tx, *dth = S[T_DTH] + tx, *dP = S[T_DP] + tx;
  R *rhs = S[T_RHS] + tx, *dw = S[T_DW] + tx;
  // the tangent theta' in, before any in-place write of this launch
  if (active)
#pragma unroll 4
    for (int k = lane; k < nz; k += kLkl<R>) dth[k * kLcx<R>] = d.th_in[g.at(k)];
  column_values_s(a, g, active, S);
  const R *Av = S[V_AV] + tx, *P = S[V_P] + tx, *E = S[V_E] + tx, *G = S[V_G] + tx;
  const R* W = S[V_W] + tx;
  if (active)
#pragma unroll 4
    for (int k = lane; k <= nz; k += kLkl<R>) {
      R sv = 0;
      if (g.terrain && k >= 1 && k < nz) {
        const int c = g.at(k), cm = c - pl;
        R uw = (R)0.25 * (du[cm] + du[cm + sx] + du[c] + du[c + sx]);
        R vw = (R)0.25 * (dv[cm] + dv[cm + sy] + dv[c] + dv[c + sy]);
        sv = Av[k * kLcx<R>] * (uw * g.hxc + vw * g.hyc) * a.co.fac_w[L.at1(k)];
      }
      dSv[k * kLcx<R>] = sv;
    }
  __syncthreads();
  if (active)
#pragma unroll 4
    for (int k = lane; k < nz; k += kLkl<R>) {
      const int c = g.at(k);
      R Kt = a.co.kt3[c];
      R dDh = (a.co.rtjx[c + sx] * du[c + sx] - a.co.rtjx[c] * du[c]) * g.mcx +
              (a.co.rtjy[c + sy] * dv[c + sy] - a.co.rtjy[c] * dv[c]) * g.mcy;
      R idz = a.co.inv_dzc[L.at1(k)];
      R dwk = d.w_in[c], dwkp = d.w_in[c + pl];
      R dtpi = d.tpi ? d.tpi[c] : (R)0;
      const int q = k * kLcx<R>;
      dP[q] = d.pi_cur[c] + dtau * dtpi -
              dtau * Kt * (dDh - (dSv[q + kLcx<R>] - dSv[q]) * idz + c2 * (Av[q + kLcx<R>] * dwkp - Av[q] * dwk) * idz);
    }
  __syncthreads();
  if (active)
#pragma unroll 4
    for (int k = 1 + lane; k < nz; k += kLkl<R>) {
      const int c = g.at(k), cm = c - pl;
      const int q = k * kLcx<R>;
      const R iJdz = g.invJ * a.co.inv_dzw[L.at1(k)];
      const R thd = a.b.thbw[c] + (R)0.5 * (a.th_in[cm] + a.th_in[c]);
      R thvw = thd;
      R dthvw = (R)0.5 * (dth[q - kLcx<R>] + dth[q]);
      R dbuoy = Phys<R>::grav * (R)0.5 * (dth[q - kLcx<R>] + dth[q]) / a.b.thbw[c];
      if (a.p.moisture) {
        // theta_v = theta (1 + 0.61 qv); buoyancy + g (0.61 qv' - qc - qr)
        const R mq = (R)1 + Phys<R>::eps61 * (R)0.5 * (a.qv[cm] + a.qv[c]);
        const R dqv = (R)0.5 * (d.qv[cm] + d.qv[c]);
        thvw = thd * mq;
        dthvw = dthvw * mq + thd * Phys<R>::eps61 * dqv;
        dbuoy += Phys<R>::grav * (Phys<R>::eps61 * dqv - (R)0.5 * (d.qc[cm] + d.qc[c]) -
                                  (R)0.5 * (d.qr[cm] + d.qr[c]));
      }
      const R dG = dtau * Phys<R>::cp * dthvw * c1 * iJdz;
      R dpi = d.pi_cur[c] - d.pi_cur[cm], pi = a.pi_cur[c] - a.pi_cur[cm];
      R dRHS = d.w_in[c] + dtau * (dbuoy + d.tw[c]) - dtau * Phys<R>::cp * c2 * (dthvw * pi + thvw * dpi) * iJdz;
      R dD = dRHS - dG * (P[q] - P[q - kLcx<R>]) - G[q] * (dP[q] - dP[q - kLcx<R>]);
      R dA = -dG * E[q - kLcx<R>] * Av[q - kLcx<R>];
      R dB = dG * Av[q] * (E[q] + E[q - kLcx<R>]);
      R dC = -dG * E[q] * Av[q + kLcx<R>];
      R mw = dB * W[q];
      if (k > 1) mw += dA * W[q - kLcx<R>];
      if (k < nz - 1) mw += dC * W[q + kLcx<R>];
      rhs[q] = dD - mw;
    }
  __syncthreads();
  if (active && lane == 0) {
    thomas_s(nz, S[V_A] + tx, S[V_B] + tx, S[V_C] + tx, rhs, S[V_CS] + tx, S[V_DS] + tx, dw);
    dw[0] = (R)0.5 * (du[g.c0] + du[g.c0 + sx]) * g.hxc + (R)0.5 * (dv[g.c0] + dv[g.c0 + sy]) * g.hyc;
  }
  __syncthreads();
  if (active)
#pragma unroll 4
    for (int k = lane; k <= nz; k += kLkl<R>) {
      const int c = g.at(k);
      const int q = k * kLcx<R>;
      if (k < nz) {
        d.pi_next[c] = dP[q] - E[q] * (Av[q + kLcx<R>] * dw[q + kLcx<R>] - Av[q] * dw[q]);
        d.th_out[c] = dth[q] + dtau * (d.tth[c] - (R)0.5 * (dw[q] + dw[q + kLcx<R>]) * a.b.dthbdz[c]);
        d.w_out[c] = dw[q];
      } else {
        d.w_out[c] = 0;
      }
      // the forward launch's outputs (dyn_acou.cu phase 5, the same
      // expressions on the same values): the forward column need not run
      if (with_forward) {
        if (k < nz) {
          R wn = W[q], wn1 = W[q + kLcx<R>];
          a.pi_next[c] = P[q] - E[q] * (Av[q + kLcx<R>] * wn1 - Av[q] * wn);
          R wc = (R)0.5 * (wn + wn1);
          a.th_out[c] = a.th_in[c] + dtau * (a.tth[c] - wc * a.b.dthbdz[c]);
          a.w_out[c] = wn;
        } else {
          a.w_out[c] = 0;
        }
      }
    }
}

enum { A_WB = V_N, A_PB, A_TB, A_WS, A_LAM, A_GL, A_PIB, A_THB, A_KTD, A_NARR };

// Adjoint of the column.  dhB (per cell, levels < nz) receives mc times the
// adjoint of the horizontal divergence, svB the u, v weight of level k (the
// surface w at level 0, Sv(k) at levels 1..nz-1); k_ad_column_uv takes both
// to the faces.
// STORED: the forward values from the launch's outputs (column_values_stored_s)
// instead of recomputing the forward column
template <typename R, bool STORED = false>
__global__ void __launch_bounds__(kLcx<R> * kLkl<R>) k_ad_column(AcouArgs<R> a, AcouArgs<R> d, R* dhB, R* svB) {
  extern __shared__ __align__(16) unsigned char lin_smem[];
  const Layout& L = a.L;
  const int tx = threadIdx.x, lane = threadIdx.y;
  const int i = blockIdx.x * kLcx<R> + tx, j = blockIdx.y;
  const bool active = i < L.nx;
  const ColArr<R> S{reinterpret_cast<R*>(lin_smem), L.nz + 1};
  const ColGeom<R> g(a, i, j, active);
  const int nz = g.nz;
  const R dtau = g.dtau, c1 = g.c1, c2 = g.c2;
  const int pl = g.pl;
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
  R *wb = S[A_WB] + tx, *pb = S[A_PB] + tx, *tb = S[A_TB] + tx, *ws = S[A_WS] + tx;
  R *lam = S[A_LAM] + tx, *GL = S[A_GL] + tx, *PIB = S[A_PIB] + tx, *THB = S[A_THB] + tx;
  R* KTD = S[A_KTD] + tx;
  // the sweep's scratch rows, free once the transposed solve is done
  R *QVB = S[V_CS] + tx, *QCB = S[V_DS] + tx;
  // the output adjoints; w and theta' update in place after the first
  // substep (w_out = w_in, th_out = th_in), so the inputs' adjoints replace
  // the outputs' there, and are added to the input's elsewhere while the
  // output's are cleared -- at the end, long after these loads (a store
  // issued while the load of the same address is in flight stalls the
  // memory pipeline)
  const bool w_alias = d.w_out == d.w_in, th_alias = d.th_out == d.th_in;
  if (active)
#pragma unroll 4
    for (int k = lane; k <= nz; k += kLkl<R>) {
      const int c = g.at(k);
      const int q = k * kLcx<R>;
      wb[q] = d.w_out[c];
      if (k < nz) {
        pb[q] = d.pi_next[c];
        tb[q] = d.th_out[c];
      }
    }
  if (STORED)
    column_values_stored_s(a, g, active, S);
  else
    column_values_s(a, g, active, S);
  const R *Av = S[V_AV] + tx, *P = S[V_P] + tx, *E = S[V_E] + tx, *G = S[V_G] + tx;
  const R* W = S[V_W] + tx;
  // adjoint of the column solution w (level 0: surface w, level nz: the lid)
  if (active)
#pragma unroll 4
    for (int k = lane; k <= nz; k += kLkl<R>) {
      const int q = k * kLcx<R>;
      const int c = g.at(k);
      R s = 0;
      if (k < nz) s += wb[q] - (R)0.5 * dtau * a.b.dthbdz[c] * tb[q] + E[q] * Av[q] * pb[q];
      if (k >= 1) s += -(R)0.5 * dtau * a.b.dthbdz[c - pl] * tb[q - kLcx<R>] - E[q - kLcx<R>] * Av[q] * pb[q - kLcx<R>];
      ws[q] = s;
    }
  __syncthreads();
  if (active && lane == 0)
    thomas_ts(nz, S[V_A] + tx, S[V_B] + tx, S[V_C] + tx, ws, S[V_CS] + tx, S[V_DS] + tx, lam);
  __syncthreads();
  // per inner level: what its row sends to neighbouring levels
  if (active)
#pragma unroll 4
    for (int k = lane; k <= nz; k += kLkl<R>) {
      const int q = k * kLcx<R>;
      if (k < 1 || k >= nz) {
        GL[q] = 0;
        PIB[q] = 0;
        THB[q] = 0;
        QVB[q] = 0;
        QCB[q] = 0;
        continue;
      }
      const int c = g.at(k), cm = c - pl;
      const R iJdz = g.invJ * a.co.inv_dzw[L.at1(k)];
      const R lm = lam[q];
      const R Ab = k > 1 ? -lm * W[q - kLcx<R>] : (R)0;
      const R Bb = -lm * W[q];
      const R Cb = k < nz - 1 ? -lm * W[q + kLcx<R>] : (R)0;
      const R Gb = Ab * (-E[q - kLcx<R>] * Av[q - kLcx<R>]) + Bb * (Av[q] * (E[q] + E[q - kLcx<R>])) +
                   Cb * (-E[q] * Av[q + kLcx<R>]) - lm * (P[q] - P[q - kLcx<R>]);
      const R thd = a.b.thbw[c] + (R)0.5 * (a.th_in[cm] + a.th_in[c]);
      const R mq = moist ? (R)1 + Phys<R>::eps61 * (R)0.5 * (a.qv[cm] + a.qv[c]) : (R)1;
      const R thvw = moist ? thd * mq : thd;
      const R pi = a.pi_cur[c] - a.pi_cur[cm];
      GL[q] = G[q] * lm;
      PIB[q] = -dtau * Phys<R>::cp * thvw * c2 * iJdz * lm;
      const R thvwb = -dtau * Phys<R>::cp * c2 * pi * iJdz * lm + Gb * dtau * Phys<R>::cp * c1 * iJdz;
      const R bt = Phys<R>::grav * (R)0.5 / a.b.thbw[c] * dtau * lm;
      THB[q] = (R)0.5 * thvwb * mq + bt;
      // per level of the pair (k-1, k): qv through theta_v and buoyancy, qc and qr through buoyancy
      QVB[q] = (R)0.5 * Phys<R>::eps61 * (thvwb * thd + Phys<R>::grav * dtau * lm);
      QCB[q] = -(R)0.5 * Phys<R>::grav * dtau * lm;
      twB[c] += dtau * lm;
    }
  __syncthreads();
  if (active)
#pragma unroll 4
    for (int k = lane; k < nz; k += kLkl<R>) {
      const int c = g.at(k);
      const int q = k * kLcx<R>;
      // the adjoints this level accumulates into, all read first
      const R pic0 = piC[c];
      const R tpi0 = tpiB ? tpiB[c] : (R)0;
      const R th0 = th_alias ? (R)0 : thI[c];
      const R tth0 = tthB[c];
      R qv0 = 0, qc0 = 0, qr0 = 0;
      if (moist) {
        qv0 = qvI[c];
        qc0 = qcI[c];
        qr0 = qrI[c];
      }
      const R Kt = a.co.kt3[c];
      R Pb = pb[q];
      if (k >= 1) Pb -= GL[q];
      if (k + 1 < nz) Pb += GL[q + kLcx<R>];
      R pic = Pb;
      if (k >= 1) pic += PIB[q];
      if (k + 1 < nz) pic -= PIB[q + kLcx<R>];
      R th = tb[q];
      if (k >= 1) th += THB[q];
      if (k + 1 < nz) th += THB[q + kLcx<R>];
      piC[c] = pic0 + pic;
      if (tpiB) tpiB[c] = tpi0 + dtau * Pb;
      dhB[c] = -dtau * Kt * Pb * g.mc;  // adjoint of the map-factor-scaled divergence
      thI[c] = th0 + th;
      if (!th_alias) d.th_out[c] = 0;
      if (moist) {
        R qvs = 0, qcs = 0;
        if (k >= 1) qvs += QVB[q], qcs += QCB[q];
        if (k + 1 < nz) qvs += QVB[q + kLcx<R>], qcs += QCB[q + kLcx<R>];
        qvI[c] = qv0 + qvs;
        qcI[c] = qc0 + qcs;
        qrI[c] = qr0 + qcs;
      }
      tthB[c] = tth0 + dtau * tb[q];
      d.pi_next[c] = 0;
      KTD[q] = Kt * a.co.inv_dzc[L.at1(k)] * Pb;
    }
  __syncthreads();
  if (active)
#pragma unroll 4
    for (int k = lane; k <= nz; k += kLkl<R>) {
      const int q = k * kLcx<R>;
      const int c = g.at(k);
      const R w0 = w_alias ? (R)0 : wI[c];
      R wsum = 0;
      if (k >= 1 && k < nz) wsum += lam[q];
      R kd = (k < nz ? KTD[q] : (R)0) - (k >= 1 ? KTD[q - kLcx<R>] : (R)0);
      wsum += dtau * c2 * Av[q] * kd;
      wI[c] = w0 + wsum;
      if (!w_alias) d.w_out[c] = 0;
      // the u, v weight of level k: surface w (level 0) or Sv(k) over the
      // faces of levels k - 1 and k (k_ad_column_uv takes them to the faces)
      if (k == 0)
        svB[c] = (R)0.5 * ws[0];
      else if (k < nz)
        svB[c] = (R)0.25 * Av[q] * a.co.fac_w[L.at1(k)] * (-dtau * kd);
    }
}

// The u, v adjoints the column sends to the faces around it, gathered per
// face from the two columns beside it (no atomics): dh holds mc * (adjoint
// of the horizontal divergence) per cell, sv the weight of the surface w
// (level 0) or of Sv(k) (levels 1..nz-1), which reaches the faces of levels
// k - 1 and k times the column's terrain slope hx (hy).
template <typename R>
__global__ void __launch_bounds__(256) k_ad_column_uv(AcouArgs<R> a, AcouArgs<R> d, const R* __restrict__ dh,
                                                      const R* __restrict__ sv) {
  const Layout& L = a.L;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  if (i > nx || j > ny || k >= nz) return;
  const int c = L.ati(i, j, k), pl = L.planei();
  // a column's weight at level k for the faces of level k: its own level and the one above
  auto wsv = [&](int cc) { return sv[cc] + (k + 1 < nz ? sv[cc + pl] : (R)0); };
  if (j < ny) {  // u face i: columns i - 1 and i
    R g = 0;
    const R rj = a.co.rtjx[c] * a.co.inv_dx;
    if (i >= 1) {
      const int cl = c - 1;
      g += rj * dh[cl] + a.m.hx[L.at2i(i - 1, j)] * wsv(cl);
    }
    if (i < nx) g += -rj * dh[c] + a.m.hx[L.at2i(i, j)] * wsv(c);
    if (g != (R)0) d.u_out[c] += g;
  }
  if (i < nx) {  // v face j: rows j - 1 and j
    R g = 0;
    const R rj = a.co.rtjy[c] * a.co.inv_dy;
    if (j >= 1) {
      const int cl = c - L.px;
      g += rj * dh[cl] + a.m.hy[L.at2i(i, j - 1)] * wsv(cl);
    }
    if (j < ny) g += -rj * dh[c] + a.m.hy[L.at2i(i, j)] * wsv(c);
    if (g != (R)0) d.v_out[c] += g;
  }
}

// Undo-log copies: up to kCopyMax whole fields (n elements each) in one
// launch, 16-byte vectors; blockIdx.y picks the field, a grid-stride loop
// over it with four loads in flight per thread before their stores.
template <typename R>
__global__ void __launch_bounds__(256) k_copy_fields(CopyJob<R> job, size_t n) {
  const size_t nv = n * sizeof(R) / 16;  // n * sizeof(R) is a multiple of 16 (copy_fields)
  const int f = blockIdx.y;
  const uint4* __restrict__ src = reinterpret_cast<const uint4*>(job.src[f]);
  uint4* __restrict__ dst = reinterpret_cast<uint4*>(job.dst[f]);
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; e + 3 * stride < nv; e += 4 * stride) {
    const uint4 v0 = src[e], v1 = src[e + stride], v2 = src[e + 2 * stride], v3 = src[e + 3 * stride];
    dst[e] = v0;
    dst[e + stride] = v1;
    dst[e + 2 * stride] = v2;
    dst[e + 3 * stride] = v3;
  }
  for (; e < nv; e += stride) dst[e] = src[e];
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
int copy_fields(const CopyJob<R>& job, size_t n, cudaStream_t st) {
  if (job.count < 1) return 0;
  if (job.count > kCopyMax || (n * sizeof(R)) % 16) return 1;
  for (int f = 0; f < job.count; ++f)
    if ((reinterpret_cast<uintptr_t>(job.src[f]) | reinterpret_cast<uintptr_t>(job.dst[f])) % 16) return 1;
  k_copy_fields<R><<<dim3((148 * 8 + job.count - 1) / job.count, job.count), 256, 0, st>>>(job, n);
  return 0;
}

template <typename R>
void zero_ring(R* f, const Layout& L, cudaStream_t st) {
  k_zero_ring<R><<<1184, 256, 0, st>>>(f, L);
}

template <typename R>
void ad_fill(const FillArgs<R>& d, cudaStream_t st) {
  if (d.job.n == 0) return;
  const int nk = d.L.nz + 1 + 2 * kRefNG;  // levels -3 .. nz+3
  const long cols = (long)d.L.nx * d.L.ny, ring = ring_columns(d.L);
  k_ad_fill_levels<R><<<dim3((unsigned)((cols + 255) / 256), 2 * kRefNG + 1, d.job.n), 256, 0, st>>>(d);
  k_ad_fill_ring<R><<<dim3((unsigned)((ring + 255) / 256), nk, d.job.n), 256, 0, st>>>(d);
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
  const dim3 g = grid_cells<R>(a.L), b(32, 4, 2);
  k_ad_tend<R, AD_U><<<g, b, 0, st>>>(a, d);
  k_ad_tend<R, AD_V><<<g, b, 0, st>>>(a, d);
  k_ad_tend<R, AD_W><<<g, b, 0, st>>>(a, d);
  k_ad_tend<R, AD_TH><<<g, b, 0, st>>>(a, d);
  if (a.p.moisture) k_ad_tend<R, AD_Q><<<g, b, 0, st>>>(a, d);
}

template <typename R>
void tl_uv(const AcouArgs<R>& a, const AcouArgs<R>& d, cudaStream_t st) {
  k_tl_uv<R><<<grid_uv<R>(a.L), dim3(32, 4, 2), 0, st>>>(a, d);
}

template <typename R>
void ad_uv(const AcouArgs<R>& a, const AcouArgs<R>& d, const LinScratch<R>& scr, cudaStream_t st) {
  const UvScr<R> w{scr.f[0], scr.f[1], scr.f[2], scr.f[3], scr.f[4], scr.f[5]};
  k_ad_uv_faces<R><<<grid_uv<R>(a.L), dim3(32, 4, 2), 0, st>>>(a, d, w);
  k_ad_uv_cells<R><<<grid_cells<R>(a.L), dim3(32, 4, 2), 0, st>>>(a, d, w);
}

int lin_max_levels() { return 160; }  // FP64 adjoint column arrays within 227 KB

template <typename R, int NARR>
static size_t lin_col_smem(int nz) {
  return (size_t)NARR * (nz + 1) * kLcx<R> * sizeof(R);
}

// Sets the dynamic shared-memory limits of the column kernels for nz levels,
// once, outside any stream capture.
template <typename R>
int lin_prepare(int nz) {
  if (nz > lin_max_levels()) return 2;
  if (raise_smem_limit(k_tl_column<R>, lin_col_smem<R, T_NARR>(nz)) != cudaSuccess ||
      raise_smem_limit(k_ad_column<R>, lin_col_smem<R, A_NARR>(nz)) != cudaSuccess ||
      raise_smem_limit(k_ad_column<R, true>, lin_col_smem<R, A_NARR>(nz)) != cudaSuccess)
    return 1;
  return lin_kessler_prepare<R>(nz);
}

template <typename R>
int tl_column(const AcouArgs<R>& a, const AcouArgs<R>& d, bool with_forward, cudaStream_t st) {
  if (a.L.nz > lin_max_levels()) return 2;
  const size_t sm = lin_col_smem<R, T_NARR>(a.L.nz);
  k_tl_column<R><<<dim3((a.L.nx + kLcx<R> - 1) / kLcx<R>, a.L.ny), dim3(kLcx<R>, kLkl<R>), sm, st>>>(
      a, d, with_forward ? 1 : 0);
  return 0;
}

template <typename R>
int ad_column(const AcouArgs<R>& a, const AcouArgs<R>& d, const LinScratch<R>& scr, cudaStream_t st) {
  if (a.L.nz > lin_max_levels()) return 2;
  const size_t sm = lin_col_smem<R, A_NARR>(a.L.nz);
  k_ad_column<R><<<dim3((a.L.nx + kLcx<R> - 1) / kLcx<R>, a.L.ny), dim3(kLcx<R>, kLkl<R>), sm, st>>>(a, d, scr.f[0], scr.f[1]);
  k_ad_column_uv<R><<<grid_uv<R>(a.L), dim3(32, 4, 2), 0, st>>>(a, d, scr.f[0], scr.f[1]);
  return 0;
}

template <typename R>
int ad_column_stored(const AcouArgs<R>& a, const AcouArgs<R>& d, const LinScratch<R>& scr, cudaStream_t st) {
  if (a.L.nz > lin_max_levels()) return 2;
  const size_t sm = lin_col_smem<R, A_NARR>(a.L.nz);
  k_ad_column<R, true><<<dim3((a.L.nx + kLcx<R> - 1) / kLcx<R>, a.L.ny), dim3(kLcx<R>, kLkl<R>), sm, st>>>(
      a, d, scr.f[0], scr.f[1]);
  k_ad_column_uv<R><<<grid_uv<R>(a.L), dim3(32, 4, 2), 0, st>>>(a, d, scr.f[0], scr.f[1]);
  return 0;
}

#define WFE_INST(R)                                                              \
  template void ad_fill<R>(const FillArgs<R>&, cudaStream_t);                    \
  template void ad_flux<R>(const FluxArgs<R>&, cudaStream_t);                    \
  template void tl_tend<R>(const TendArgs<R>&, const TendArgs<R>&, cudaStream_t); \
  template void ad_tend<R>(const TendArgs<R>&, const TendArgs<R>&, cudaStream_t); \
  template void tl_uv<R>(const AcouArgs<R>&, const AcouArgs<R>&, cudaStream_t);   \
  template void ad_uv<R>(const AcouArgs<R>&, const AcouArgs<R>&, const LinScratch<R>&, cudaStream_t); \
  template int tl_column<R>(const AcouArgs<R>&, const AcouArgs<R>&, bool, cudaStream_t); \
  template int ad_column<R>(const AcouArgs<R>&, const AcouArgs<R>&, const LinScratch<R>&, cudaStream_t); \
  template int ad_column_stored<R>(const AcouArgs<R>&, const AcouArgs<R>&, const LinScratch<R>&, cudaStream_t); \
  template void zero_ring<R>(R*, const Layout&, cudaStream_t);                        \
  template int copy_fields<R>(const CopyJob<R>&, size_t, cudaStream_t);               \
  template int lin_prepare<R>(int);
WFE_INST(float)
WFE_INST(double)
#undef WFE_INST

}  // namespace wfe
