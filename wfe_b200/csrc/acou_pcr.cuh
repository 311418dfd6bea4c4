// The parallel tridiagonal solve of the vertically implicit w equation
// (src/dynamics/kernels.cu:612-634 solve the same rows by a Thomas sweep),
// shared by the parallel-solve column kernel (dyn_acou.cu) and its pipelined
// form (dyn_acou_pipe.cu).
//
// Level lane p of KL owns KCH consecutive rows in registers (slots
// 1..KCH); the column is padded with identity rows (x = 0) where a lane's
// slots run past the inner levels, which leaves the solution unchanged.
//   1. the lane eliminates its first KCH - 1 rows with its last row's unknown
//      y_p and the previous lane's y_{p-1} as parameters:
//      x_q = G_q + A_q y_{p-1} + B_q y_p (one Thomas pass, three right-hand
//      sides);
//   2. its last row, with the first-row expression of the lane above, is one
//      row L y_{p-1} + M y_p + U y_{p+1} = F of a system in the lanes' y;
//   3. that system is solved by parallel cyclic reduction over the lanes
//      through shared memory (ceil(log2(KL)) steps).
// The quotients are products with IEEE reciprocals; the solution equals the
// Thomas sweep's to rounding.
#pragma once

#include "core.cuh"

namespace wfe {

__device__ __forceinline__ float pcr_rcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double pcr_rcp(double x) { return __drcp_rn(x); }

// per-lane result: rows 1..KCH-1 as x_q = Gx[q] + Ax[q] y_{p-1} + Bx[q] y_p,
// the first row of the lane above as gn + an y_p + bn y_{p+1}, and the
// unknowns of this lane and its neighbours
template <typename R, int KCH>
struct PcrLane {
  R Gx[KCH + 1], Ax[KCH + 1], Bx[KCH + 1];
  R gn, an, bn;
  R y, yprev, ynext;
};

// shared values the solve needs per (level lane, column): the first-row
// expressions (3), the reduced rows double-buffered (8), the unknowns (1)
constexpr int kPcrWork = 12;

// Every thread of the CX x KL group calls this with its lane's rows; the
// group's work area holds kPcrWork * KL * CX values; sync() is a barrier of
// exactly the calling threads (the CTA, or the consumer warps of a
// warp-specialised CTA).  Ends after the last shared read of the area.
template <typename R, int CX, int KL, int KCH, class Sync>
__device__ __forceinline__ void pcr_solve(const R (&Ar)[KCH + 1], const R (&Br)[KCH + 1],
                                          const R (&Cr)[KCH + 1], const R (&Dr)[KCH + 1], R* work, int tx,
                                          int lane, Sync sync, PcrLane<R, KCH>& o) {
  static_assert(KCH >= 2, "every lane needs an interior row");
  constexpr int NL = KL * CX;
  R* fG = work;
  R* fA = fG + NL;
  R* fB = fA + NL;
  R* red = fB + NL;
  R* yv = red + 8 * NL;
  const int me = lane * CX + tx;
  // ---- 1. rows 1 .. KCH-1 in terms of (y_{p-1}, y_p)
  {
    R cp[KCH], gp[KCH], ap[KCH], bp[KCH];
#pragma unroll
    for (int q = 1; q < KCH; ++q) {
      const R r = pcr_rcp(Br[q] - Ar[q] * (q > 1 ? cp[q - 1] : (R)0));
      cp[q] = q == KCH - 1 ? (R)0 : Cr[q] * r;
      gp[q] = (Dr[q] - Ar[q] * (q > 1 ? gp[q - 1] : (R)0)) * r;
      ap[q] = ((q == 1 ? -Ar[q] : (R)0) - Ar[q] * (q > 1 ? ap[q - 1] : (R)0)) * r;
      bp[q] = ((q == KCH - 1 ? -Cr[q] : (R)0) - Ar[q] * (q > 1 ? bp[q - 1] : (R)0)) * r;
    }
#pragma unroll
    for (int q = KCH - 1; q >= 1; --q) {
      if (q == KCH - 1) {
        o.Gx[q] = gp[q], o.Ax[q] = ap[q], o.Bx[q] = bp[q];
      } else {
        o.Gx[q] = gp[q] - cp[q] * o.Gx[q + 1];
        o.Ax[q] = ap[q] - cp[q] * o.Ax[q + 1];
        o.Bx[q] = bp[q] - cp[q] * o.Bx[q + 1];
      }
    }
  }
  fG[me] = o.Gx[1];
  fA[me] = o.Ax[1];
  fB[me] = o.Bx[1];
  sync();
  // ---- 2. the lane's row of the reduced system: its last row with x of the
  // row below it (this lane's row KCH - 1) and of the row above it (the
  // first row of the lane above; none above the top lane)
  o.gn = 0, o.an = 0, o.bn = 0;
  if (lane + 1 < KL) {
    o.gn = fG[me + CX];
    o.an = fA[me + CX];
    o.bn = fB[me + CX];
  }
  R Lr = Ar[KCH] * o.Ax[KCH - 1];
  R Mr = Br[KCH] + Ar[KCH] * o.Bx[KCH - 1] + Cr[KCH] * o.an;
  R Ur = Cr[KCH] * o.bn;
  R Fr = Dr[KCH] - Ar[KCH] * o.Gx[KCH - 1] - Cr[KCH] * o.gn;
  // ---- 3. parallel cyclic reduction over the lanes
  R* buf = red;
  buf[me] = Lr;
  buf[NL + me] = Mr;
  buf[2 * NL + me] = Ur;
  buf[3 * NL + me] = Fr;
  sync();
#pragma unroll
  for (int h = 1; h < KL; h *= 2) {
    R* nb = buf == red ? red + 4 * NL : red;
    R al = 0, ga = 0, Lm = 0, Um = 0, Fm = 0, Lp = 0, Up = 0, Fp = 0;
    if (lane - h >= 0) {
      const int q = me - h * CX;
      al = -Lr * pcr_rcp(buf[NL + q]);
      Lm = buf[q];
      Um = buf[2 * NL + q];
      Fm = buf[3 * NL + q];
    }
    if (lane + h < KL) {
      const int q = me + h * CX;
      ga = -Ur * pcr_rcp(buf[NL + q]);
      Lp = buf[q];
      Up = buf[2 * NL + q];
      Fp = buf[3 * NL + q];
    }
    Mr = Mr + al * Um + ga * Lp;
    Fr = Fr + al * Fm + ga * Fp;
    Lr = al * Lm;
    Ur = ga * Up;
    nb[me] = Lr;
    nb[NL + me] = Mr;
    nb[2 * NL + me] = Ur;
    nb[3 * NL + me] = Fr;
    buf = nb;
    sync();
  }
  o.y = Fr * pcr_rcp(Mr);
  yv[me] = o.y;
  sync();
  o.yprev = lane > 0 ? yv[me - CX] : (R)0;
  o.ynext = lane + 1 < KL ? yv[me + CX] : (R)0;
}

}  // namespace wfe
