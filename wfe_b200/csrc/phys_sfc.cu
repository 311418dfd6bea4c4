// Surface layer (Louis 1979), two-stream radiation, 4-layer soil, local-Ri or
// Troen-Mahrt nonlocal PBL and implicit column mixing on the B200
// (src/physics/surface.cu:28-514).
//
// Two implementations of the same columns.  The level-parallel kernels
// (k_sfc_*_cols, used whenever a column fits in shared memory) run the
// per-level work over the level lanes of a CTA and the recurrences along the
// column from shared memory.  The scratch kernels (any column depth) run one
// thread per column as the reference does, with the per-column work arrays
// (the reference keeps 21 KB of them on the thread stack) in a scratch buffer
// laid out column-fastest.  The momentum columns on u and v faces run in one
// launch.  Every value follows the reference's expressions.
#include <cuda_runtime.h>

#include "core.cuh"
#include "kernels.cuh"

namespace wfe {

namespace {

template <typename R>
__device__ __forceinline__ R qsat_tet(R p, R T) {  // src/core/thermo.hpp:11-17
  R es = (R)610.78 * exp((R)17.269 * (T - (R)273.16) / (T - (R)35.86));
  R den = p - es;
  if (den < (R)1) den = (R)1;
  return (R)0.622 * es / den;
}

template <typename R>
__device__ __forceinline__ R psi_m(R zeta) {  // surface.cu:30-36
  if (zeta >= (R)0) return (R)-5 * fmin(zeta, (R)2);
  R x = pow((R)1 - (R)16 * zeta, (R)0.25);
  const R halfpi = (R)1.5707963267948966;
  return (R)2 * log(((R)1 + x) * (R)0.5) + log(((R)1 + x * x) * (R)0.5) - (R)2 * atan(x) + halfpi;
}
template <typename R>
__device__ __forceinline__ R psi_h(R zeta) {  // surface.cu:37-41
  if (zeta >= (R)0) return (R)-5 * fmin(zeta, (R)2);
  R x = pow((R)1 - (R)16 * zeta, (R)0.25);
  return (R)2 * log(((R)1 + x * x) * (R)0.5);
}

// One column of a scratch array: element k at p[k * s].
template <typename R>
struct Col {
  R* p;
  size_t s;
  __device__ __forceinline__ R& operator[](int k) const { return p[(size_t)k * s]; }
};

// implicit column diffusion (Thomas), surface.cu:61-84; A..D are work columns
template <typename R>
__device__ void diffuse_col(int nz, R dt, Col<R> rho, Col<R> rhow, Col<R> dzc, Col<R> dzw,
                            Col<R> Kw, R src0, Col<R> phi, const Col<R>* fcg, Col<R> A, Col<R> B,
                            Col<R> C, Col<R> D) {
  for (int k = 0; k < nz; ++k) {
    R a = (k > 0) ? rhow[k] * Kw[k] / dzw[k] : (R)0;
    R c = (k < nz - 1) ? rhow[k + 1] * Kw[k + 1] / dzw[k + 1] : (R)0;
    R m = rho[k] * dzc[k] / dt;
    A[k] = -a;
    B[k] = m + a + c;
    C[k] = -c;
    D[k] = m * phi[k];
    if (fcg) D[k] += (*fcg)[k] - (*fcg)[k + 1];
  }
  D[0] += src0;
  for (int k = 1; k < nz; ++k) {
    R w = A[k] / B[k - 1];
    B[k] -= w * C[k - 1];
    D[k] -= w * D[k - 1];
  }
  phi[nz - 1] = D[nz - 1] / B[nz - 1];
  for (int k = nz - 2; k >= 0; --k) phi[k] = (D[k] - C[k] * phi[k + 1]) / B[k];
}

}  // namespace

// scratch columns of the mass-column kernel
enum { SC_RHO, SC_RHOW, SC_DZC, SC_DZW, SC_THV, SC_KW, SC_TH, SC_QV, SC_KLOC, SC_SH2, SC_TLEV,
       SC_EPS, SC_FUP, SC_FDN, SC_RAD, SC_SW, SC_FCGT, SC_FCGQ, SC_A, SC_B, SC_C, SC_D, SC_N };
// scratch columns of a momentum column
enum { SM_RHO, SM_RHOW, SM_DZC, SM_DZW, SM_KW, SM_PHI, SM_A, SM_B, SM_C, SM_D, SM_N };

template <typename R>
__device__ __forceinline__ void sfc_scalar_body(const SfcArgs<R>& a, int bx, int by) {
  const Layout& L = a.L;
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  if (i >= L.nx || j >= L.ny) return;
  const int nz = L.nz;
  using P = Phys<R>;
  const R KAPPA = (R)0.4, SIGMA = (R)5.67e-8, S0 = (R)1361, KM_MAX = (R)1000, KM_MIN = (R)0.1;
  const R SOIL_DZ[4] = {(R)0.1, (R)0.3, (R)0.6, (R)1.0};
  const size_t c2 = L.at2(i, j);
  const size_t n2 = L.n2();
  const R J = a.m.jac[c2];
  double tend_s = a.clock[CLK_T] + a.clock[CLK_DT];  // end of the step
  R utc = (R)(a.start_hour + tend_s / 3600.0);
  utc = utc - (R)24 * floor(utc / (R)24);

  // work columns: array q of this column at scratch[(q * (nz + 1) + k) * ncol + col]
  const size_t ncol = (size_t)L.nx * L.ny, col = (size_t)j * L.nx + i;
  auto C_ = [&](int q) { return Col<R>{a.scratch + (size_t)q * (nz + 1) * ncol + col, ncol}; };
  Col<R> rho = C_(SC_RHO), rhow = C_(SC_RHOW), dzc = C_(SC_DZC), dzw = C_(SC_DZW), thv = C_(SC_THV);
  Col<R> Kw = C_(SC_KW), thcol = C_(SC_TH), qvcol = C_(SC_QV), Kloc = C_(SC_KLOC);
  Col<R> shear2 = C_(SC_SH2);
  R lwp = 0;
  for (int k = 0; k < nz; ++k) {
    const int kk = L.at1(k);
    const size_t c = L.at(i, j, k);
    rho[k] = a.b.rhob[c];
    rhow[k] = a.b.rhobw[c];
    dzc[k] = a.m.dzeta_c[kk] * J;
    dzw[k] = a.m.dzeta_w[kk] * J;
    thcol[k] = a.b.thb[c] + a.thp[c];
    qvcol[k] = a.qv[c];
    thv[k] = thcol[k] * ((R)1 + P::eps61 * qvcol[k]);
    lwp += rho[k] * (a.qc[c] > (R)0 ? a.qc[c] : (R)0) * dzc[k] * (R)1000;
  }
  // The local-Ri diffusivity (surface.cu:285-298) and the bulk-Richardson shear
  // of the PBL-height search (surface.cu:321) depend only on the column loaded
  // above; they are evaluated here, with the reference's expressions, so that
  // the wind columns are dead before the radiation arrays are live.
  auto ucen = [&](int k) {  // cell-centre winds (surface.cu:112-113)
    const size_t c = L.at(i, j, k);
    return (R)0.5 * (a.u[c] + a.u[c + 1]);
  };
  auto vcen = [&](int k) {
    const size_t c = L.at(i, j, k);
    return (R)0.5 * (a.v[c] + a.v[c + L.px]);
  };
  for (int k = 1; k < nz; ++k) {
    R dz = dzw[k];
    R uk = ucen(k), vk = vcen(k);
    R du = (uk - ucen(k - 1)) / dz, dv = (vk - vcen(k - 1)) / dz;
    R S2 = du * du + dv * dv + (R)1e-8;
    R thvw = (R)0.5 * (thv[k - 1] + thv[k]);
    R N2 = P::grav / thvw * (thv[k] - thv[k - 1]) / dz;
    R Ri = N2 / S2;
    R zw = a.m.zeta_w[L.at1(k)] * J;
    R l = KAPPA * zw / ((R)1 + KAPPA * zw / (R)150);
    if (Ri < (R)0) {
      Kloc[k] = l * l * sqrt(S2) * sqrt((R)1 - (R)16 * Ri);
    } else {
      R d = (R)1 + (R)5 * Ri;
      Kloc[k] = l * l * sqrt(S2) / (d * d);
    }
    shear2[k] = uk * uk + vk * vk + (R)0.1;
  }
  // surface layer (surface.cu:120-161)
  const bool onland = a.land[c2] > (R)0.5;
  const R z0 = onland ? (R)0.1 : (R)2e-4;
  const R alb = onland ? (R)0.2 : (R)0.08;
  R beta;
  if (onland) {
    R f = (a.soilw[c2] - (R)0.08) / ((R)0.32 - (R)0.08);
    f = fmin((R)1, fmax((R)0, f));
    beta = fmax((R)0.05, f * f);
  } else {
    beta = (R)1;
  }
  R z1 = (R)0.5 * dzc[0];
  const R u0 = ucen(0), v0 = vcen(0);
  R V1 = sqrt(u0 * u0 + v0 * v0);
  if (V1 < (R)0.5) V1 = (R)0.5;
  const size_t c0 = L.at(i, j, 0);
  R pi1 = a.b.pib[c0] + a.pip[c0];
  R p1 = P::p00 * pow(pi1, P::cp / P::Rd);
  R Ts = a.tsk[c2];
  R pis = pi1 + P::grav * z1 / (P::cp * thv[0]);
  R ths = Ts / pis;
  R qs_s = qsat_tet(p1, Ts);
  R thvs = ths * ((R)1 + P::eps61 * (beta * qs_s + ((R)1 - beta) * qvcol[0]));
  R Rib = P::grav * z1 * (thv[0] - thvs) / (thvs * V1 * V1);
  R a2 = KAPPA / log(z1 / z0);
  a2 *= a2;
  R Fm, Fh;
  if (Rib < (R)0) {
    R sq = sqrt(-Rib * z1 / z0);
    Fm = (R)1 - (R)9.4 * Rib / ((R)1 + (R)7.4 * (R)9.4 * a2 * sq);
    Fh = (R)1 - (R)9.4 * Rib / ((R)1 + (R)5.3 * (R)9.4 * a2 * sq);
  } else {
    R d = (R)1 + (R)4.7 * Rib;
    Fm = Fh = (R)1 / (d * d);
  }
  R Cd = a2 * Fm, Ch = a2 * Fh;
  a.cdv[c2] = Cd * V1;
  // 2 m / 10 m diagnostics (surface.cu:163-182)
  R z0h = z0 * (R)0.1;
  R lnz1z0 = log(z1 / z0);
  R zeta1 = (Rib >= (R)0) ? Rib * lnz1z0 / ((R)1 - (R)5 * fmin(Rib, (R)0.19)) : Rib * lnz1z0;
  zeta1 = fmax((R)-8, fmin((R)2, zeta1));
  R zol = zeta1 / z1;
  R den_m = lnz1z0 - psi_m(zeta1) + psi_m(z0 * zol);
  R num_m = log((R)10 / z0) - psi_m((R)10 * zol) + psi_m(z0 * zol);
  R r10 = fmax((R)0, fmin((R)1.2, num_m / fmax(den_m, (R)0.1)));
  a.u10[c2] = V1 * r10;
  R den_h = log(z1 / z0h) - psi_h(zeta1) + psi_h(z0h * zol);
  R num_h = log((R)2 / z0h) - psi_h((R)2 * zol) + psi_h(z0h * zol);
  R r2 = fmax((R)0, fmin((R)1.2, num_h / fmax(den_h, (R)0.1)));
  R th2 = ths + (thcol[0] - ths) * r2;
  a.t2m[c2] = th2 * pi1;
  R shf = Ch * V1 * (ths - thcol[0]);
  R qflx = Ch * V1 * beta * (qs_s - qvcol[0]);
  if (!onland && qflx < (R)0) qflx = 0;
  // two-stream radiation (surface.cu:188-243)
  R decl = (R)0.40928 * sin((R)6.2832 * ((R)284 + a.doy) / (R)365);
  R latr = a.lat[c2] * (R)0.0174533;
  R hsol = utc + a.lon[c2] / (R)15;
  R H = (R)0.2618 * (hsol - (R)12);
  R cosz = sin(latr) * sin(decl) + cos(latr) * cos(decl) * cos(H);
  if (cosz < (R)0) cosz = 0;
  Col<R> Tlev = C_(SC_TLEV), epslw = C_(SC_EPS), Fup = C_(SC_FUP), Fdn = C_(SC_FDN);
  Col<R> radht = C_(SC_RAD);
  for (int k = 0; k < nz; ++k) {
    const size_t c = L.at(i, j, k);
    R pik = a.b.pib[c] + a.pip[c];
    Tlev[k] = thcol[k] * pik;
    R du = rho[k] * qvcol[k] * dzc[k];
    R dl = rho[k] * (a.qc[c] > (R)0 ? a.qc[c] : (R)0) * dzc[k] * (R)1000;
    epslw[k] = (R)1 - exp(-((R)0.22 * du + (R)0.30 * dl));
  }
  Fdn[nz] = (R)0;
  for (int k = nz - 1; k >= 0; --k)
    Fdn[k] = Fdn[k + 1] * ((R)1 - epslw[k]) + epslw[k] * SIGMA * Tlev[k] * Tlev[k] * Tlev[k] * Tlev[k];
  R lwd = Fdn[0];
  Fup[0] = (R)0.97 * SIGMA * Ts * Ts * Ts * Ts + (R)0.03 * Fdn[0];
  for (int k = 0; k < nz; ++k)
    Fup[k + 1] = Fup[k] * ((R)1 - epslw[k]) + epslw[k] * SIGMA * Tlev[k] * Tlev[k] * Tlev[k] * Tlev[k];
  R mu = fmax(cosz, (R)0.05);
  R cldalb = lwp / (lwp + (R)60);
  R Sdn = S0 * cosz * (R)0.95 * ((R)1 - cldalb);
  Col<R> swabs = C_(SC_SW);
  for (int k = nz - 1; k >= 0; --k) {
    const size_t c = L.at(i, j, k);
    R du = rho[k] * qvcol[k] * dzc[k];
    R dl = rho[k] * (a.qc[c] > (R)0 ? a.qc[c] : (R)0) * dzc[k] * (R)1000;
    R tau = exp(-((R)0.008 * du + (R)0.15 * dl) / mu);
    R ab = Sdn * ((R)1 - tau);
    swabs[k] = ab;
    Sdn *= tau;
  }
  R swn = Sdn * ((R)1 - alb);
  for (int k = 0; k < nz; ++k) {
    const size_t c = L.at(i, j, k);
    R pik = a.b.pib[c] + a.pip[c];
    R lwconv = (Fdn[k + 1] - Fdn[k]) + (Fup[k] - Fup[k + 1]);
    R net = lwconv + swabs[k];
    radht[k] = net / (rho[k] * P::cp * dzc[k]) / pik;
  }
  // 4-layer soil (surface.cu:245-282)
  R lwu = (R)0.97 * SIGMA * Ts * Ts * Ts * Ts;
  R G = swn + (R)0.97 * lwd - lwu - rho[0] * P::cp * shf * pi1 - rho[0] * P::Lv * qflx;
  if (onland) {
    R w = a.soilw[c2];
    R Cso = (R)1.2e6 + (R)3.2e6 * fmin(fmax(w, (R)0), (R)0.4);
    R Kso = (R)0.25 + (R)3.0 * fmin(fmax(w, (R)0), (R)0.4);
    R Tso[4], A[4], B[4], C[4], D[4];
    for (int l = 0; l < 4; ++l) Tso[l] = a.soilt[(size_t)l * n2 + c2];
    for (int l = 0; l < 4; ++l) {
      R cap = Cso * SOIL_DZ[l] / a.dt;
      R ku = (l > 0) ? Kso / ((R)0.5 * (SOIL_DZ[l - 1] + SOIL_DZ[l])) : (R)0;
      R kl = (l < 3) ? Kso / ((R)0.5 * (SOIL_DZ[l] + SOIL_DZ[l + 1])) : Kso / SOIL_DZ[l];
      A[l] = -ku;
      C[l] = (l < 3) ? -kl : (R)0;
      B[l] = cap + ku + kl;
      D[l] = cap * Tso[l];
    }
    D[0] += G;
    D[3] += (Kso / SOIL_DZ[3]) * a.tdeep[c2];
    for (int l = 1; l < 4; ++l) {
      R ww = A[l] / B[l - 1];
      B[l] -= ww * C[l - 1];
      D[l] -= ww * D[l - 1];
    }
    Tso[3] = D[3] / B[3];
    for (int l = 2; l >= 0; --l) Tso[l] = (D[l] - C[l] * Tso[l + 1]) / B[l];
    for (int l = 0; l < 4; ++l) {
      if (Tso[l] < (R)200) Tso[l] = 200;
      if (Tso[l] > (R)350) Tso[l] = 350;
      a.soilt[(size_t)l * n2 + c2] = Tso[l];
    }
    a.tsk[c2] = Tso[0];
  }
  // eddy diffusivity: local Ri or nonlocal Troen-Mahrt (surface.cu:300-371)
  Col<R> fcg_th = C_(SC_FCGT), fcg_qv = C_(SC_FCGQ);
  Kw[0] = 0;
  fcg_th[0] = fcg_qv[0] = fcg_th[nz] = fcg_qv[nz] = 0;
  if (a.nonlocal) {
    R ust = sqrt(Cd) * V1;
    R thv1 = thv[0];
    R wthv0 = shf * ((R)1 + P::eps61 * qvcol[0]) + P::eps61 * thcol[0] * qflx;
    const R Ric = (R)0.25;
    R hpbl = a.m.zeta_c[L.at1(nz - 1)] * J;
    R ws = ust > (R)0.1 ? ust : (R)0.1;
    for (int it = 0; it < 3; ++it) {
      R exc = (wthv0 > (R)0) ? (R)6.8 * wthv0 / ws : (R)0;
      R thv_s = thv1 + exc;
      R prevRb = 0;
      hpbl = a.m.zeta_c[L.at1(nz - 1)] * J;
      for (int k = 1; k < nz; ++k) {
        R zc = a.m.zeta_c[L.at1(k)] * J;
        R Rbk = P::grav * (thv[k] - thv_s) * zc / (thv1 * shear2[k]);
        if (Rbk >= Ric) {
          R zcm = a.m.zeta_c[L.at1(k - 1)] * J;
          R f = (Ric - prevRb) / (Rbk - prevRb + (R)1e-9);
          f = fmin((R)1, fmax((R)0, f));
          hpbl = zcm + f * (zc - zcm);
          break;
        }
        prevRb = Rbk;
      }
      R zc0 = a.m.zeta_c[L.at1(0)] * J;
      if (hpbl < zc0) hpbl = zc0;
      R wstar = (wthv0 > (R)0) ? cbrt(P::grav / thv1 * wthv0 * hpbl) : (R)0;
      ws = cbrt(ust * ust * ust + (R)0.6 * wstar * wstar * wstar);
      if (ws < (R)0.1) ws = (R)0.1;
    }
    a.pblh[c2] = hpbl;
    R gth = (wthv0 > (R)0) ? (R)6.8 * shf / (ws * hpbl) : (R)0;
    R gqv = (wthv0 > (R)0) ? (R)6.8 * qflx / (ws * hpbl) : (R)0;
    for (int k = 1; k < nz; ++k) {
      R zw = a.m.zeta_w[L.at1(k)] * J;
      R Kv;
      if (wthv0 > (R)0 && zw < hpbl) {
        R zf = zw / hpbl;
        Kv = KAPPA * ws * zw * (1 - zf) * (1 - zf);
        fcg_th[k] = rhow[k] * Kv * gth;
        fcg_qv[k] = rhow[k] * Kv * gqv;
      } else {
        Kv = Kloc[k];
        fcg_th[k] = fcg_qv[k] = 0;
      }
      if (Kv < KM_MIN) Kv = KM_MIN;
      if (Kv > KM_MAX) Kv = KM_MAX;
      Kw[k] = Kv;
      a.km[L.at(i, j, k)] = Kv;
    }
  } else {
    a.pblh[c2] = 0;
    for (int k = 1; k < nz; ++k) {
      R Kv = Kloc[k];
      if (Kv < KM_MIN) Kv = KM_MIN;
      if (Kv > KM_MAX) Kv = KM_MAX;
      Kw[k] = Kv;
      a.km[L.at(i, j, k)] = Kv;
      fcg_th[k] = fcg_qv[k] = 0;
    }
  }
  Col<R> tA = C_(SC_A), tB = C_(SC_B), tC = C_(SC_C), tD = C_(SC_D);
  diffuse_col<R>(nz, a.dt, rho, rhow, dzc, dzw, Kw, rho[0] * shf, thcol, &fcg_th, tA, tB, tC, tD);
  diffuse_col<R>(nz, a.dt, rho, rhow, dzc, dzw, Kw, rho[0] * qflx, qvcol, &fcg_qv, tA, tB, tC, tD);
  for (int k = 0; k < nz; ++k) {
    const size_t c = L.at(i, j, k);
    R dth = a.dt * radht[k];
    if (dth > (R)0.02) dth = (R)0.02;
    if (dth < (R)-0.02) dth = (R)-0.02;
    a.thp[c] = thcol[k] - a.b.thb[c] + dth;
    R q = qvcol[k];
    a.qv[c] = q > (R)0 ? q : (R)0;
  }
}

// ------------------------------------------------ level-parallel columns
// A CTA owns kSfcCX columns with kSfcKL level lanes; the column arrays live
// in shared memory, level-major ([k][column]).  The per-level work (loading,
// local-Ri diffusivities, emissivities, heating rates, nonlocal K and the
// rows of the implicit mixing) runs over the lanes; the recurrences along
// the column (radiative fluxes, the shortwave path, the PBL-height search,
// the Thomas sweeps, the soil) run in lane 0 of each column from shared
// memory.  The theta' and qv mixing share one matrix, so one forward
// elimination serves both right-hand sides (the matrix is rebuilt and
// eliminated identically for each in the scratch kernels).  Expressions as
// in the scratch kernels above.
constexpr int kSfcCX = 16, kSfcKL = 8;
enum { SS_TH, SS_QV, SS_THV, SS_SH2, SS_KW, SS_FCT, SS_FCQ, SS_RAD, SS_TMP,
       SS_EPS, SS_TLEV, SS_FDN, SS_FUP, SS_SWA, SS_N };  // A, B, C, D alias EPS .. FDN
enum { SSM_A, SSM_B, SSM_C, SSM_D, SSM_PHI, SSM_N };
constexpr int kSfcScal = 12;  // per-column scalars after the column arrays

template <typename R>
size_t sfc_cols_smem(int nz, int sub) {
  const size_t n1 = (size_t)(nz + 1) * kSfcCX;
  return sub == 0 ? (SS_N * n1 + (size_t)kSfcScal * kSfcCX) * sizeof(R) : SSM_N * n1 * sizeof(R);
}

template <typename R>
__device__ __forceinline__ void sfc_scalar_cols(const SfcArgs<R>& a, int bx, int by, R* sm) {
  const Layout& L = a.L;
  const int nz = L.nz;
  const int tx = threadIdx.x, lane = threadIdx.y;
  const int i = bx * kSfcCX + tx, j = by;
  const bool active = i < L.nx && j < L.ny;
  using P = Phys<R>;
  const R KAPPA = (R)0.4, SIGMA = (R)5.67e-8, S0 = (R)1361, KM_MAX = (R)1000, KM_MIN = (R)0.1;
  const int n1 = (nz + 1) * kSfcCX;
  auto X = [&](int q, int k) -> R& { return sm[q * n1 + k * kSfcCX + tx]; };
  R* scal = sm + SS_N * n1;
  auto S = [&](int q) -> R& { return scal[q * kSfcCX + tx]; };
  enum { SC_SHF, SC_QFLX, SC_HPBL, SC_WS, SC_GTH, SC_GQV, SC_POS, SC_RHO0 };
  const int c2 = L.at2i(active ? i : 0, j);
  const int n2 = L.planei();
  const R J = a.m.jac[c2];
  double tend_s = a.clock[CLK_T] + a.clock[CLK_DT];  // end of the step
  R utc = (R)(a.start_hour + tend_s / 3600.0);
  utc = utc - (R)24 * floor(utc / (R)24);
  // solar geometry (surface.cu:188-196), the same in every lane of the column
  R decl = (R)0.40928 * sin((R)6.2832 * ((R)284 + a.doy) / (R)365);
  R latr = a.lat[c2] * (R)0.0174533;
  R hsol = utc + a.lon[c2] / (R)15;
  R H = (R)0.2618 * (hsol - (R)12);
  R cosz = sin(latr) * sin(decl) + cos(latr) * cos(decl) * cos(H);
  if (cosz < (R)0) cosz = 0;
  const R mu = fmax(cosz, (R)0.05);
  auto ucen = [&](int k) {
    const int c = L.ati(i, j, k);
    return (R)0.5 * (a.u[c] + a.u[c + 1]);
  };
  auto vcen = [&](int k) {
    const int c = L.ati(i, j, k);
    return (R)0.5 * (a.v[c] + a.v[c + L.px]);
  };
  // ---- per level: the column, lwp terms, emissivity, temperature, the
  // shortwave transmission
  if (active)
    for (int k = lane; k < nz; k += kSfcKL) {
      const int kk = L.at1(k);
      const int c = L.ati(i, j, k);
      const R rho = a.b.rhob[c];
      const R dzc = a.m.dzeta_c[kk] * J;
      const R th = a.b.thb[c] + a.thp[c];
      const R qv = a.qv[c];
      X(SS_TH, k) = th;
      X(SS_QV, k) = qv;
      X(SS_THV, k) = th * ((R)1 + P::eps61 * qv);
      const R qcp = a.qc[c] > (R)0 ? a.qc[c] : (R)0;
      X(SS_TMP, k) = rho * qcp * dzc * (R)1000;
      const R pik = a.b.pib[c] + a.pip[c];
      X(SS_TLEV, k) = th * pik;
      R du = rho * qv * dzc;
      R dl = rho * qcp * dzc * (R)1000;
      X(SS_EPS, k) = (R)1 - exp(-((R)0.22 * du + (R)0.30 * dl));
      X(SS_SWA, k) = exp(-((R)0.008 * du + (R)0.15 * dl) / mu);  // transmission
    }
  __syncthreads();
  // ---- per level: local-Ri diffusivity and bulk-Richardson shear
  if (active)
    for (int k = 1 + lane; k < nz; k += kSfcKL) {
      const int kk = L.at1(k);
      R dz = a.m.dzeta_w[kk] * J;
      R uk = ucen(k), vk = vcen(k);
      R du = (uk - ucen(k - 1)) / dz, dv = (vk - vcen(k - 1)) / dz;
      R S2 = du * du + dv * dv + (R)1e-8;
      R thvw = (R)0.5 * (X(SS_THV, k - 1) + X(SS_THV, k));
      R N2 = P::grav / thvw * (X(SS_THV, k) - X(SS_THV, k - 1)) / dz;
      R Ri = N2 / S2;
      R zw = a.m.zeta_w[kk] * J;
      R l = KAPPA * zw / ((R)1 + KAPPA * zw / (R)150);
      R Kl;
      if (Ri < (R)0) {
        Kl = l * l * sqrt(S2) * sqrt((R)1 - (R)16 * Ri);
      } else {
        R d = (R)1 + (R)5 * Ri;
        Kl = l * l * sqrt(S2) / (d * d);
      }
      X(SS_KW, k) = Kl;  // the local K; the nonlocal scheme replaces it below
      X(SS_SH2, k) = uk * uk + vk * vk + (R)0.1;
    }
  __syncthreads();
  // ---- along the column, lane 0: surface layer, radiation, soil, PBL height
  if (active && lane == 0) {
    R lwp = 0;
    for (int k = 0; k < nz; ++k) lwp += X(SS_TMP, k);
    const bool onland = a.land[c2] > (R)0.5;
    const R z0 = onland ? (R)0.1 : (R)2e-4;
    const R alb = onland ? (R)0.2 : (R)0.08;
    R beta;
    if (onland) {
      R f = (a.soilw[c2] - (R)0.08) / ((R)0.32 - (R)0.08);
      f = fmin((R)1, fmax((R)0, f));
      beta = fmax((R)0.05, f * f);
    } else {
      beta = (R)1;
    }
    const int c0 = L.ati(i, j, 0);
    const R rho0 = a.b.rhob[c0];
    const R dzc0 = a.m.dzeta_c[L.at1(0)] * J;
    R z1 = (R)0.5 * dzc0;
    const R u0 = ucen(0), v0 = vcen(0);
    R V1 = sqrt(u0 * u0 + v0 * v0);
    if (V1 < (R)0.5) V1 = (R)0.5;
    R pi1 = a.b.pib[c0] + a.pip[c0];
    R p1 = P::p00 * pow(pi1, P::cp / P::Rd);
    R Ts = a.tsk[c2];
    const R thv0 = X(SS_THV, 0), th0 = X(SS_TH, 0), qv0 = X(SS_QV, 0);
    R pis = pi1 + P::grav * z1 / (P::cp * thv0);
    R ths = Ts / pis;
    R qs_s = qsat_tet(p1, Ts);
    R thvs = ths * ((R)1 + P::eps61 * (beta * qs_s + ((R)1 - beta) * qv0));
    R Rib = P::grav * z1 * (thv0 - thvs) / (thvs * V1 * V1);
    R a2 = KAPPA / log(z1 / z0);
    a2 *= a2;
    R Fm, Fh;
    if (Rib < (R)0) {
      R sq = sqrt(-Rib * z1 / z0);
      Fm = (R)1 - (R)9.4 * Rib / ((R)1 + (R)7.4 * (R)9.4 * a2 * sq);
      Fh = (R)1 - (R)9.4 * Rib / ((R)1 + (R)5.3 * (R)9.4 * a2 * sq);
    } else {
      R d = (R)1 + (R)4.7 * Rib;
      Fm = Fh = (R)1 / (d * d);
    }
    R Cd = a2 * Fm, Ch = a2 * Fh;
    a.cdv[c2] = Cd * V1;
    R z0h = z0 * (R)0.1;
    R lnz1z0 = log(z1 / z0);
    R zeta1 = (Rib >= (R)0) ? Rib * lnz1z0 / ((R)1 - (R)5 * fmin(Rib, (R)0.19)) : Rib * lnz1z0;
    zeta1 = fmax((R)-8, fmin((R)2, zeta1));
    R zol = zeta1 / z1;
    R den_m = lnz1z0 - psi_m(zeta1) + psi_m(z0 * zol);
    R num_m = log((R)10 / z0) - psi_m((R)10 * zol) + psi_m(z0 * zol);
    R r10 = fmax((R)0, fmin((R)1.2, num_m / fmax(den_m, (R)0.1)));
    a.u10[c2] = V1 * r10;
    R den_h = log(z1 / z0h) - psi_h(zeta1) + psi_h(z0h * zol);
    R num_h = log((R)2 / z0h) - psi_h((R)2 * zol) + psi_h(z0h * zol);
    R r2 = fmax((R)0, fmin((R)1.2, num_h / fmax(den_h, (R)0.1)));
    R th2 = ths + (th0 - ths) * r2;
    a.t2m[c2] = th2 * pi1;
    R shf = Ch * V1 * (ths - th0);
    R qflx = Ch * V1 * beta * (qs_s - qv0);
    if (!onland && qflx < (R)0) qflx = 0;
    // two-stream radiation (surface.cu:198-243)
    R Fdn = 0;
    X(SS_FDN, nz) = 0;
    for (int k = nz - 1; k >= 0; --k) {
      const R e = X(SS_EPS, k), T = X(SS_TLEV, k);
      Fdn = Fdn * ((R)1 - e) + e * SIGMA * T * T * T * T;
      X(SS_FDN, k) = Fdn;
    }
    R lwd = Fdn;
    R Fup = (R)0.97 * SIGMA * Ts * Ts * Ts * Ts + (R)0.03 * Fdn;
    X(SS_FUP, 0) = Fup;
    for (int k = 0; k < nz; ++k) {
      const R e = X(SS_EPS, k), T = X(SS_TLEV, k);
      Fup = Fup * ((R)1 - e) + e * SIGMA * T * T * T * T;
      X(SS_FUP, k + 1) = Fup;
    }
    R cldalb = lwp / (lwp + (R)60);
    R Sdn = S0 * cosz * (R)0.95 * ((R)1 - cldalb);
    for (int k = nz - 1; k >= 0; --k) {
      R tau = X(SS_SWA, k);
      R ab = Sdn * ((R)1 - tau);
      X(SS_SWA, k) = ab;
      Sdn *= tau;
    }
    R swn = Sdn * ((R)1 - alb);
    // 4-layer soil (surface.cu:245-282)
    const R SOIL_DZ[4] = {(R)0.1, (R)0.3, (R)0.6, (R)1.0};
    R lwu = (R)0.97 * SIGMA * Ts * Ts * Ts * Ts;
    R G = swn + (R)0.97 * lwd - lwu - rho0 * P::cp * shf * pi1 - rho0 * P::Lv * qflx;
    if (onland) {
      R w = a.soilw[c2];
      R Cso = (R)1.2e6 + (R)3.2e6 * fmin(fmax(w, (R)0), (R)0.4);
      R Kso = (R)0.25 + (R)3.0 * fmin(fmax(w, (R)0), (R)0.4);
      R Tso[4], A[4], B[4], C[4], D[4];
      for (int l = 0; l < 4; ++l) Tso[l] = a.soilt[l * n2 + c2];
      for (int l = 0; l < 4; ++l) {
        R cap = Cso * SOIL_DZ[l] / a.dt;
        R ku = (l > 0) ? Kso / ((R)0.5 * (SOIL_DZ[l - 1] + SOIL_DZ[l])) : (R)0;
        R kl = (l < 3) ? Kso / ((R)0.5 * (SOIL_DZ[l] + SOIL_DZ[l + 1])) : Kso / SOIL_DZ[l];
        A[l] = -ku;
        C[l] = (l < 3) ? -kl : (R)0;
        B[l] = cap + ku + kl;
        D[l] = cap * Tso[l];
      }
      D[0] += G;
      D[3] += (Kso / SOIL_DZ[3]) * a.tdeep[c2];
      for (int l = 1; l < 4; ++l) {
        R ww = A[l] / B[l - 1];
        B[l] -= ww * C[l - 1];
        D[l] -= ww * D[l - 1];
      }
      Tso[3] = D[3] / B[3];
      for (int l = 2; l >= 0; --l) Tso[l] = (D[l] - C[l] * Tso[l + 1]) / B[l];
      for (int l = 0; l < 4; ++l) {
        if (Tso[l] < (R)200) Tso[l] = 200;
        if (Tso[l] > (R)350) Tso[l] = 350;
        a.soilt[l * n2 + c2] = Tso[l];
      }
      a.tsk[c2] = Tso[0];
    }
    // PBL height (surface.cu:300-337)
    R hpbl = 0, ws = 0, gth = 0, gqv = 0;
    R pos = 0;
    if (a.nonlocal) {
      R ust = sqrt(Cd) * V1;
      R wthv0 = shf * ((R)1 + P::eps61 * qv0) + P::eps61 * th0 * qflx;
      const R Ric = (R)0.25;
      ws = ust > (R)0.1 ? ust : (R)0.1;
      for (int it = 0; it < 3; ++it) {
        R exc = (wthv0 > (R)0) ? (R)6.8 * wthv0 / ws : (R)0;
        R thv_s = thv0 + exc;
        R prevRb = 0;
        hpbl = a.m.zeta_c[L.at1(nz - 1)] * J;
        for (int k = 1; k < nz; ++k) {
          R zc = a.m.zeta_c[L.at1(k)] * J;
          R Rbk = P::grav * (X(SS_THV, k) - thv_s) * zc / (thv0 * X(SS_SH2, k));
          if (Rbk >= Ric) {
            R zcm = a.m.zeta_c[L.at1(k - 1)] * J;
            R f = (Ric - prevRb) / (Rbk - prevRb + (R)1e-9);
            f = fmin((R)1, fmax((R)0, f));
            hpbl = zcm + f * (zc - zcm);
            break;
          }
          prevRb = Rbk;
        }
        R zc0 = a.m.zeta_c[L.at1(0)] * J;
        if (hpbl < zc0) hpbl = zc0;
        R wstar = (wthv0 > (R)0) ? cbrt(P::grav / thv0 * wthv0 * hpbl) : (R)0;
        ws = cbrt(ust * ust * ust + (R)0.6 * wstar * wstar * wstar);
        if (ws < (R)0.1) ws = (R)0.1;
      }
      a.pblh[c2] = hpbl;
      gth = (wthv0 > (R)0) ? (R)6.8 * shf / (ws * hpbl) : (R)0;
      gqv = (wthv0 > (R)0) ? (R)6.8 * qflx / (ws * hpbl) : (R)0;
      pos = wthv0 > (R)0 ? (R)1 : (R)0;
    } else {
      a.pblh[c2] = 0;
    }
    S(SC_SHF) = shf;
    S(SC_QFLX) = qflx;
    S(SC_HPBL) = hpbl;
    S(SC_WS) = ws;
    S(SC_GTH) = gth;
    S(SC_GQV) = gqv;
    S(SC_POS) = pos;
    S(SC_RHO0) = rho0;
  }
  __syncthreads();
  // ---- per level: heating rates, K, countergradient fluxes
  if (active) {
    const R hpbl = S(SC_HPBL), ws = S(SC_WS), gth = S(SC_GTH), gqv = S(SC_GQV);
    const bool pos = S(SC_POS) > (R)0;
    for (int k = lane; k < nz; k += kSfcKL) {
      const int kk = L.at1(k);
      const int c = L.ati(i, j, k);
      const R rho = a.b.rhob[c];
      const R dzc = a.m.dzeta_c[kk] * J;
      R pik = a.b.pib[c] + a.pip[c];
      R lwconv = (X(SS_FDN, k + 1) - X(SS_FDN, k)) + (X(SS_FUP, k) - X(SS_FUP, k + 1));
      R net = lwconv + X(SS_SWA, k);
      X(SS_RAD, k) = net / (rho * P::cp * dzc) / pik;
      R Kv, ft = 0, fq = 0;
      if (k == 0) {
        Kv = 0;
      } else {
        if (a.nonlocal) {
          R zw = a.m.zeta_w[kk] * J;
          if (pos && zw < hpbl) {
            R zf = zw / hpbl;
            R rhow = a.b.rhobw[c];
            Kv = KAPPA * ws * zw * (1 - zf) * (1 - zf);
            ft = rhow * Kv * gth;
            fq = rhow * Kv * gqv;
          } else {
            Kv = X(SS_KW, k);
          }
        } else {
          Kv = X(SS_KW, k);
        }
        if (Kv < KM_MIN) Kv = KM_MIN;
        if (Kv > KM_MAX) Kv = KM_MAX;
        a.km[c] = Kv;
      }
      X(SS_KW, k) = Kv;
      X(SS_FCT, k) = ft;
      X(SS_FCQ, k) = fq;
    }
    if (lane == 0) X(SS_FCT, nz) = X(SS_FCQ, nz) = 0;
  }
  __syncthreads();
  // ---- per level: rows of the implicit mixing (surface.cu:61-76), one
  // matrix, two right-hand sides (A, B, C, D of theta' alias the radiation
  // arrays, now dead; D of qv reuses the lwp terms)
  const int SA = SS_EPS, SB = SS_TLEV, SCC = SS_FDN, SD = SS_FUP, SQ = SS_TMP;
  if (active)
    for (int k = lane; k < nz; k += kSfcKL) {
      const int kk = L.at1(k);
      const int c = L.ati(i, j, k);
      R av = (k > 0) ? a.b.rhobw[c] * X(SS_KW, k) / (a.m.dzeta_w[kk] * J) : (R)0;
      R cv = (k < nz - 1) ? a.b.rhobw[c + L.planei()] * X(SS_KW, k + 1) / (a.m.dzeta_w[kk + 1] * J)
                          : (R)0;
      R m = a.b.rhob[c] * (a.m.dzeta_c[kk] * J) / a.dt;
      X(SA, k) = -av;
      X(SB, k) = m + av + cv;
      X(SCC, k) = -cv;
      R dt_ = m * X(SS_TH, k);
      dt_ += X(SS_FCT, k) - X(SS_FCT, k + 1);
      R dq_ = m * X(SS_QV, k);
      dq_ += X(SS_FCQ, k) - X(SS_FCQ, k + 1);
      X(SD, k) = dt_;
      X(SQ, k) = dq_;
    }
  __syncthreads();
  if (active && lane == 0) {
    X(SD, 0) += S(SC_RHO0) * S(SC_SHF);
    X(SQ, 0) += S(SC_RHO0) * S(SC_QFLX);
    for (int k = 1; k < nz; ++k) {
      R w = X(SA, k) / X(SB, k - 1);
      X(SB, k) -= w * X(SCC, k - 1);
      X(SD, k) -= w * X(SD, k - 1);
      X(SQ, k) -= w * X(SQ, k - 1);
    }
    R pt = X(SD, nz - 1) / X(SB, nz - 1), pq = X(SQ, nz - 1) / X(SB, nz - 1);
    X(SS_TH, nz - 1) = pt;
    X(SS_QV, nz - 1) = pq;
    for (int k = nz - 2; k >= 0; --k) {
      pt = (X(SD, k) - X(SCC, k) * pt) / X(SB, k);
      pq = (X(SQ, k) - X(SCC, k) * pq) / X(SB, k);
      X(SS_TH, k) = pt;
      X(SS_QV, k) = pq;
    }
  }
  __syncthreads();
  if (active)
    for (int k = lane; k < nz; k += kSfcKL) {
      const int c = L.ati(i, j, k);
      R dth = a.dt * X(SS_RAD, k);
      if (dth > (R)0.02) dth = (R)0.02;
      if (dth < (R)-0.02) dth = (R)-0.02;
      a.thp[c] = X(SS_TH, k) - a.b.thb[c] + dth;
      R q = X(SS_QV, k);
      a.qv[c] = q > (R)0 ? q : (R)0;
    }
}

// momentum columns on u faces (z = 0, i = 1..nx-1) and v faces (z = 1,
// j = 1..ny-1): surface drag + implicit mixing (surface.cu:390-436)
template <typename R>
__device__ __forceinline__ void sfc_momentum_cols(const SfcArgs<R>& a, int bx, int by, int bz, R* sm) {
  const Layout& L = a.L;
  const int nz = L.nz;
  const bool on_v = bz == 1;
  const int tx = threadIdx.x, lane = threadIdx.y;
  const int i = bx * kSfcCX + tx + (on_v ? 0 : 1);
  const int j = by + (on_v ? 1 : 0);
  const bool active = i < L.nx && j < L.ny;
  const int di = on_v ? 0 : 1, dj = on_v ? 1 : 0;
  R* f = on_v ? a.v : a.u;
  const int n1 = (nz + 1) * kSfcCX;
  auto X = [&](int q, int k) -> R& { return sm[q * n1 + k * kSfcCX + tx]; };
  const R J = active ? (R)0.5 * (a.m.jac[L.at2i(i - di, j - dj)] + a.m.jac[L.at2i(i, j)]) : (R)1;
  auto Kw = [&](int k) {
    return (R)0.5 * (a.km[L.ati(i - di, j - dj, k)] + a.km[L.ati(i, j, k)]);
  };
  if (active)
    for (int k = lane; k < nz; k += kSfcKL) {
      const int kk = L.at1(k);
      const int c = L.ati(i, j, k), cb = L.ati(i - di, j - dj, k);
      R av = 0, cv = 0;
      if (k > 0) {
        R rhow = (R)0.5 * (a.b.rhobw[cb] + a.b.rhobw[c]);
        av = rhow * Kw(k) / (a.m.dzeta_w[kk] * J);
      }
      if (k < nz - 1) {
        const int pl = L.planei();
        R rhow = (R)0.5 * (a.b.rhobw[cb + pl] + a.b.rhobw[c + pl]);
        cv = rhow * Kw(k + 1) / (a.m.dzeta_w[kk + 1] * J);
      }
      R rho = (R)0.5 * (a.b.rhob[cb] + a.b.rhob[c]);
      R m = rho * (a.m.dzeta_c[kk] * J) / a.dt;
      X(SSM_A, k) = -av;
      X(SSM_B, k) = m + av + cv;
      X(SSM_C, k) = -cv;
      X(SSM_D, k) = m * f[c];
    }
  __syncthreads();
  if (active && lane == 0) {
    const int c0 = L.ati(i, j, 0), cb0 = L.ati(i - di, j - dj, 0);
    R cdva = (R)0.5 * (a.cdv[L.at2i(i - di, j - dj)] + a.cdv[L.at2i(i, j)]);
    R rho0 = (R)0.5 * (a.b.rhob[cb0] + a.b.rhob[c0]);
    X(SSM_D, 0) += -rho0 * cdva * f[c0];
    for (int k = 1; k < nz; ++k) {
      R w = X(SSM_A, k) / X(SSM_B, k - 1);
      X(SSM_B, k) -= w * X(SSM_C, k - 1);
      X(SSM_D, k) -= w * X(SSM_D, k - 1);
    }
    R phi = X(SSM_D, nz - 1) / X(SSM_B, nz - 1);
    X(SSM_PHI, nz - 1) = phi;
    for (int k = nz - 2; k >= 0; --k) {
      phi = (X(SSM_D, k) - X(SSM_C, k) * phi) / X(SSM_B, k);
      X(SSM_PHI, k) = phi;
    }
  }
  __syncthreads();
  if (active)
    for (int k = lane; k < nz; k += kSfcKL) f[L.ati(i, j, k)] = X(SSM_PHI, k);
}

template <typename R>
__global__ void __launch_bounds__(kSfcCX * kSfcKL) k_sfc_scalar_cols(SfcArgs<R> a) {
  extern __shared__ __align__(16) unsigned char smem_sfc[];
  sfc_scalar_cols(a, blockIdx.x, blockIdx.y, reinterpret_cast<R*>(smem_sfc));
}
template <typename R>
__global__ void __launch_bounds__(kSfcCX * kSfcKL) k_sfc_scalar_cols_batch(Batch<SfcArgs<R>> b) {
  extern __shared__ __align__(16) unsigned char smem_sfc[];
  for_each_work(b, [](const SfcArgs<R>& a, int x, int y, int) {
    sfc_scalar_cols(a, x, y, reinterpret_cast<R*>(smem_sfc));
  });
}
template <typename R>
__global__ void __launch_bounds__(kSfcCX * kSfcKL) k_sfc_momentum_cols(SfcArgs<R> a) {
  extern __shared__ __align__(16) unsigned char smem_sfc[];
  sfc_momentum_cols(a, blockIdx.x, blockIdx.y, blockIdx.z, reinterpret_cast<R*>(smem_sfc));
}
template <typename R>
__global__ void __launch_bounds__(kSfcCX * kSfcKL) k_sfc_momentum_cols_batch(Batch<SfcArgs<R>> b) {
  extern __shared__ __align__(16) unsigned char smem_sfc[];
  for_each_work(b, [](const SfcArgs<R>& a, int x, int y, int z) {
    sfc_momentum_cols(a, x, y, z, reinterpret_cast<R*>(smem_sfc));
  });
}

template <typename R>
__global__ void __launch_bounds__(128) k_sfc_scalar(SfcArgs<R> a) {
  sfc_scalar_body(a, blockIdx.x, blockIdx.y);
}
template <typename R>
__global__ void __launch_bounds__(128) k_sfc_scalar_batch(Batch<SfcArgs<R>> b) {
  for_each_work(b, [](const SfcArgs<R>& a, int x, int y, int) { sfc_scalar_body(a, x, y); });
}

// momentum columns: block z = 0 for u faces i = 1..nx-1, 1 for v faces
// j = 1..ny-1: surface drag + implicit mixing (surface.cu:390-436)
template <typename R>
__device__ __forceinline__ void sfc_momentum_body(const SfcArgs<R>& a, int bx, int by, int bz) {
  const Layout& L = a.L;
  const bool on_v = bz == 1;
  const int i = bx * blockDim.x + threadIdx.x + (on_v ? 0 : 1);
  const int j = by * blockDim.y + threadIdx.y + (on_v ? 1 : 0);
  if (i >= L.nx || j >= L.ny) return;
  const int nz = L.nz;
  const int di = on_v ? 0 : 1, dj = on_v ? 1 : 0;
  R* f = on_v ? a.v : a.u;
  R J = (R)0.5 * (a.m.jac[L.at2(i - di, j - dj)] + a.m.jac[L.at2(i, j)]);
  const size_t ncol = (size_t)L.nx * L.ny, col = (size_t)j * L.nx + i;
  R* base = a.scratch + (on_v ? (size_t)SM_N * (nz + 1) * ncol : 0);
  auto C_ = [&](int q) { return Col<R>{base + (size_t)q * (nz + 1) * ncol + col, ncol}; };
  Col<R> rho = C_(SM_RHO), rhow = C_(SM_RHOW), dzc = C_(SM_DZC), dzw = C_(SM_DZW), Kw = C_(SM_KW);
  Col<R> phi = C_(SM_PHI);
  for (int k = 0; k < nz; ++k) {
    const int kk = L.at1(k);
    const size_t c = L.at(i, j, k), cb = L.at(i - di, j - dj, k);
    rho[k] = (R)0.5 * (a.b.rhob[cb] + a.b.rhob[c]);
    rhow[k] = (R)0.5 * (a.b.rhobw[cb] + a.b.rhobw[c]);
    dzc[k] = a.m.dzeta_c[kk] * J;
    dzw[k] = a.m.dzeta_w[kk] * J;
    Kw[k] = (k > 0) ? (R)0.5 * (a.km[cb] + a.km[c]) : (R)0;
    phi[k] = f[c];
  }
  R cdva = (R)0.5 * (a.cdv[L.at2(i - di, j - dj)] + a.cdv[L.at2(i, j)]);
  R src0 = -rho[0] * cdva * phi[0];
  diffuse_col<R>(nz, a.dt, rho, rhow, dzc, dzw, Kw, src0, phi, (const Col<R>*)nullptr, C_(SM_A),
                 C_(SM_B), C_(SM_C), C_(SM_D));
  for (int k = 0; k < nz; ++k) f[L.at(i, j, k)] = phi[k];
}

template <typename R>
__global__ void __launch_bounds__(128) k_sfc_momentum(SfcArgs<R> a) {
  sfc_momentum_body(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename R>
__global__ void __launch_bounds__(128) k_sfc_momentum_batch(Batch<SfcArgs<R>> b) {
  for_each_work(b, [](const SfcArgs<R>& a, int x, int y, int z) { sfc_momentum_body(a, x, y, z); });
}

template <typename R>
size_t sfc_scratch_count(const Layout& L) {
  // the mass columns and, afterwards, two sets of momentum columns reuse it
  size_t per = (size_t)(L.nz + 1) * L.nx * L.ny;
  return per * (SC_N > 2 * SM_N ? SC_N : 2 * SM_N);
}

// The level-parallel kernels hold a column in shared memory; deeper columns
// than the shared memory takes run the scratch kernels.
template <typename R>
bool sfc_cols_fit(int nz) {
  return sfc_cols_smem<R>(nz, 0) <= 200 * 1024 && sfc_cols_smem<R>(nz, 1) <= 200 * 1024;
}

template <typename R>
int prepare_sfc(int nz) {
  if (!sfc_cols_fit<R>(nz)) return 0;
  cudaError_t e = raise_smem_limit(k_sfc_scalar_cols<R>, sfc_cols_smem<R>(nz, 0));
  if (e == cudaSuccess) e = raise_smem_limit(k_sfc_scalar_cols_batch<R>, sfc_cols_smem<R>(nz, 0));
  if (e == cudaSuccess) e = raise_smem_limit(k_sfc_momentum_cols<R>, sfc_cols_smem<R>(nz, 1));
  if (e == cudaSuccess) e = raise_smem_limit(k_sfc_momentum_cols_batch<R>, sfc_cols_smem<R>(nz, 1));
  return e == cudaSuccess ? 0 : 1;
}

// sub 0: scalar columns; sub 1: u and v momentum columns (after sub 0).
// nz_max: the deepest column of the launch (the ensemble's deepest member)
template <typename R>
dim3 grid_sfc(const Layout& L, int sub, int nz_max) {
  if (sfc_cols_fit<R>(nz_max)) return dim3((L.nx + kSfcCX - 1) / kSfcCX, L.ny, sub == 0 ? 1 : 2);
  return dim3((L.nx + 31) / 32, (L.ny + 3) / 4, sub == 0 ? 1 : 2);
}

template <typename R>
int launch_sfc(const SfcArgs<R>& a, cudaStream_t st) {
  const int nz = a.L.nz;
  if (sfc_cols_fit<R>(nz)) {
    const dim3 b(kSfcCX, kSfcKL);
    k_sfc_scalar_cols<R><<<grid_sfc<R>(a.L, 0, nz), b, sfc_cols_smem<R>(nz, 0), st>>>(a);
    k_sfc_momentum_cols<R><<<grid_sfc<R>(a.L, 1, nz), b, sfc_cols_smem<R>(nz, 1), st>>>(a);
    return 0;
  }
  if (!a.scratch) return 2;
  dim3 b(32, 4);
  k_sfc_scalar<R><<<grid_sfc<R>(a.L, 0, nz), b, 0, st>>>(a);
  k_sfc_momentum<R><<<grid_sfc<R>(a.L, 1, nz), b, 0, st>>>(a);
  return 0;
}

template <typename R>
void batch_sfc(const Batch<SfcArgs<R>>& b, int sub, int nblocks, int nz_max, cudaStream_t st) {
  if (sfc_cols_fit<R>(nz_max)) {
    const dim3 blk(kSfcCX, kSfcKL);
    if (sub == 0) k_sfc_scalar_cols_batch<R><<<nblocks, blk, sfc_cols_smem<R>(nz_max, 0), st>>>(b);
    else k_sfc_momentum_cols_batch<R><<<nblocks, blk, sfc_cols_smem<R>(nz_max, 1), st>>>(b);
    return;
  }
  if (sub == 0) k_sfc_scalar_batch<R><<<nblocks, dim3(32, 4), 0, st>>>(b);
  else k_sfc_momentum_batch<R><<<nblocks, dim3(32, 4), 0, st>>>(b);
}

// whether the scratch buffer is needed (columns too deep for shared memory)
template <typename R>
bool sfc_needs_scratch(int nz) {
  return !sfc_cols_fit<R>(nz);
}

template int launch_sfc<float>(const SfcArgs<float>&, cudaStream_t);
template int launch_sfc<double>(const SfcArgs<double>&, cudaStream_t);
template dim3 grid_sfc<float>(const Layout&, int, int);
template dim3 grid_sfc<double>(const Layout&, int, int);
template void batch_sfc<float>(const Batch<SfcArgs<float>>&, int, int, int, cudaStream_t);
template void batch_sfc<double>(const Batch<SfcArgs<double>>&, int, int, int, cudaStream_t);
template int prepare_sfc<float>(int);
template int prepare_sfc<double>(int);
template bool sfc_needs_scratch<float>(int);
template bool sfc_needs_scratch<double>(int);
template size_t sfc_scratch_count<float>(const Layout&);
template size_t sfc_scratch_count<double>(const Layout&);

}  // namespace wfe
