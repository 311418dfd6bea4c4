// Tangent-linear (TL) and adjoint (AD) of the Kessler column (forward:
// phys_kessler.cu, after src/physics/kessler.cu:22-149), linearised about the
// state the forward kernel reads.
//
// Sedimentation.  The subcycle count and the below-freezing fall-speed factor
// are frozen at the trajectory.  The flux F_k = rho_k q_k v_k with
// v ~ (rho q)^0.1364 gives dF_k = 1.1364 rho_k v_k dq_k (zero where v_k = 0,
// i.e. where rho q <= 1e-9 or q <= 0).  TL steps the tangent beside the
// forward subcycles.  AD recomputes the forward subcycles, applies the
// conversions' adjoint, then walks the subcycles backwards, replaying the
// forward from the column's start up to each subcycle for its fall speeds
// (nsub (nsub - 1) / 2 replayed subcycles; nsub is 1-3 on the usual grids).
//
// Conversions.  kessler_convert (phys_common.cuh) evaluated on dual numbers:
// one direction, the tangent itself, for TL; five directions (theta', qv,
// qc, the sedimented qr, pi') for the 4 x 5 local Jacobian whose transpose AD
// applies.  Branches (autoconversion threshold, evaporation, the saturation
// clip, the ice fraction clamps, max(q, 0)) are frozen at the trajectory.
//
// The rain accumulator is a diagnostic and is not linearised.  A CTA owns KCX
// columns with KKL level lanes and the column arrays in shared memory, as the
// forward kernel does; every forward value is computed with the forward's
// expressions, so subcycle counts and branch decisions agree with it.
#include <cuda_runtime.h>

#include "core.cuh"
#include "kernels.cuh"
#include "phys_common.cuh"

namespace wfe {
namespace {

constexpr int KCX = 8, KKL = 32;

#define KS(X, k) X[(size_t)(k) * KCX + tx]

// dF/dq / (rho v) of the sedimentation flux: 1 + the fall-speed exponent
template <typename R>
__device__ __forceinline__ R flux_slope() {
  return (R)1.1364;
}

// Column set-up of the forward (phys_kessler.cu phase 1): q = max(qr, 0),
// rho, the level depths and the first fall speeds; the column's subcycle
// count and length land in ns_s / dts_s.  Ends with a barrier.
template <typename R>
__device__ void kes_setup(const KesArgs<R>& a, int i, int j, bool active, R rho_sfc, R* q, R* rho, R* dz,
                          R* v, R* red, int* ns_s, R* dts_s) {
  const Layout& L = a.L;
  const int nz = L.nz, tx = threadIdx.x, lane = threadIdx.y;
  const R J = active ? a.m.jac[L.at2(i, j)] : (R)1;
  R vmax = 0, dmin = (R)1e30;
  if (active)
    for (int k = lane; k < nz; k += KKL) {
      const size_t c = L.at(i, j, k);
      R qq = a.qr[c];
      R qk = qq > (R)0 ? qq : (R)0;
      R rh = a.b.rhob[c];
      R h = a.m.dzeta_c[L.at1(k)] * J;
      R T = (a.b.thb[c] + a.thp[c]) * (a.b.pib[c] + a.pip[c]);
      R vk = fall_speed(rh * qk, rho_sfc, rh, T);
      KS(q, k) = qk;
      KS(rho, k) = rh;
      KS(dz, k) = h;
      KS(v, k) = vk;
      if (vk > vmax) vmax = vk;
      if (h < dmin) dmin = h;
    }
  red[(size_t)lane * KCX + tx] = vmax;
  red[(size_t)(KKL + lane) * KCX + tx] = dmin;
  __syncthreads();
  if (lane == 0) {
    R vm = 0, dm = (R)1e30;
    for (int l = 0; l < KKL; ++l) {
      R x = red[(size_t)l * KCX + tx], y = red[(size_t)(KKL + l) * KCX + tx];
      if (x > vm) vm = x;
      if (y < dm) dm = y;
    }
    int ns = active ? 1 + (int)(vm * a.dt / ((R)0.8 * dm)) : 0;
    ns_s[tx] = ns;
    dts_s[tx] = active ? a.dt / (R)ns : (R)0;
  }
  __syncthreads();
}

// fall speeds of the current q (phys_kessler.cu phase 2, between subcycles)
template <typename R>
__device__ void kes_speeds(const KesArgs<R>& a, int i, int j, R rho_sfc, const R* q, const R* rho, R* v) {
  const Layout& L = a.L;
  const int tx = threadIdx.x;
  for (int k = threadIdx.y; k < L.nz; k += KKL) {
    const size_t c = L.at(i, j, k);
    R qq = KS(q, k);
    R rq = KS(rho, k) * (qq > (R)0 ? qq : (R)0);
    R T = (a.b.thb[c] + a.thp[c]) * (a.b.pib[c] + a.pip[c]);
    KS(v, k) = fall_speed(rq, rho_sfc, KS(rho, k), T);
  }
}

// one forward upwind subcycle of an active column (phys_kessler.cu phase 2);
// the caller keeps the block's barriers uniform
template <typename R>
__device__ void kes_fluxes(int nz, const R* q, const R* rho, const R* v, R* F) {
  const int tx = threadIdx.x;
  for (int k = threadIdx.y; k <= nz; k += KKL) KS(F, k) = (k < nz) ? KS(rho, k) * KS(q, k) * KS(v, k) : (R)0;
}
template <typename R>
__device__ void kes_update(int nz, R dts, R* q, const R* rho, const R* dz, const R* F) {
  const int tx = threadIdx.x;
  for (int k = threadIdx.y; k < nz; k += KKL)
    KS(q, k) += dts * (KS(F, k + 1) - KS(F, k)) / (KS(rho, k) * KS(dz, k));
}

template <typename R>
__global__ void __launch_bounds__(KCX * KKL) k_tl_kessler(KesArgs<R> a, KesArgs<R> d) {
  extern __shared__ __align__(16) unsigned char kes_lin_smem[];
  const Layout& L = a.L;
  const int nz = L.nz, tx = threadIdx.x, lane = threadIdx.y;
  const int i = blockIdx.x * KCX + tx, j = blockIdx.y;
  const bool active = i < L.nx;
  R* q = reinterpret_cast<R*>(kes_lin_smem);
  R* rho = q + (size_t)nz * KCX;
  R* dz = rho + (size_t)nz * KCX;
  R* v = dz + (size_t)nz * KCX;
  R* dq = v + (size_t)nz * KCX;
  R* F = dq + (size_t)nz * KCX;       // nz + 1
  R* dF = F + (size_t)(nz + 1) * KCX;  // nz + 1
  R* red = dF + (size_t)(nz + 1) * KCX;
  __shared__ int ns_s[KCX];
  __shared__ R dts_s[KCX];
  const R rho_sfc = active ? a.b.rhob[L.at(i, j, 0)] : (R)1;
  if (active)
    for (int k = lane; k < nz; k += KKL) {
      const size_t c = L.at(i, j, k);
      KS(dq, k) = a.qr[c] > (R)0 ? d.qr[c] : (R)0;
    }
  kes_setup(a, i, j, active, rho_sfc, q, rho, dz, v, red, ns_s, dts_s);
  int nmax = 0;
  for (int x = 0; x < KCX; ++x) nmax = max(nmax, ns_s[x]);
  const int nsub = ns_s[tx];
  const R dts = dts_s[tx];

  for (int s = 0; s < nmax; ++s) {
    const bool on = active && s < nsub;
    if (on) {
      kes_fluxes(nz, q, rho, v, F);
      for (int k = lane; k <= nz; k += KKL)
        KS(dF, k) = (k < nz) ? flux_slope<R>() * KS(rho, k) * KS(v, k) * KS(dq, k) : (R)0;
    }
    __syncthreads();
    if (on) {
      kes_update(nz, dts, q, rho, dz, F);
      for (int k = lane; k < nz; k += KKL)
        KS(dq, k) += dts * (KS(dF, k + 1) - KS(dF, k)) / (KS(rho, k) * KS(dz, k));
    }
    __syncthreads();
    if (on && s + 1 < nsub) kes_speeds(a, i, j, rho_sfc, q, rho, v);
    __syncthreads();
  }

  if (active)
    for (int k = lane; k < nz; k += KKL) {
      const size_t c = L.at(i, j, k);
      using D1 = Dn<R, 1>;
      D1 thp{a.thp[c], {d.thp[c]}}, qv{a.qv[c], {d.qv[c]}}, qc{a.qc[c], {d.qc[c]}};
      D1 qr{KS(q, k), {KS(dq, k)}};
      const D1 pip{a.pip[c], {d.pip[c]}};
      kessler_convert<R, D1>(thp, qv, qc, qr, pip, KS(rho, k), a.b.thb[c], a.b.pib[c], a.dt);
      d.thp[c] = thp.d[0];
      d.qv[c] = qv.d[0];
      d.qc[c] = qc.d[0];
      d.qr[c] = qr.d[0];
    }
}

template <typename R>
__global__ void __launch_bounds__(KCX * KKL) k_ad_kessler(KesArgs<R> a, KesArgs<R> d) {
  extern __shared__ __align__(16) unsigned char kes_lin_smem[];
  const Layout& L = a.L;
  const int nz = L.nz, tx = threadIdx.x, lane = threadIdx.y;
  const int i = blockIdx.x * KCX + tx, j = blockIdx.y;
  const bool active = i < L.nx;
  R* q = reinterpret_cast<R*>(kes_lin_smem);
  R* rho = q + (size_t)nz * KCX;
  R* dz = rho + (size_t)nz * KCX;
  R* v = dz + (size_t)nz * KCX;
  R* q0 = v + (size_t)nz * KCX;
  R* v0 = q0 + (size_t)nz * KCX;
  R* qb = v0 + (size_t)nz * KCX;
  R* F = qb + (size_t)nz * KCX;        // nz + 1
  R* Fb = F + (size_t)(nz + 1) * KCX;  // nz + 1
  R* red = Fb + (size_t)(nz + 1) * KCX;
  __shared__ int ns_s[KCX];
  __shared__ R dts_s[KCX];
  R* thpB = d.thp;
  R* qvB = d.qv;
  R* qcB = d.qc;
  R* qrB = d.qr;
  R* pipB = const_cast<R*>(d.pip);
  const R rho_sfc = active ? a.b.rhob[L.at(i, j, 0)] : (R)1;
  kes_setup(a, i, j, active, rho_sfc, q, rho, dz, v, red, ns_s, dts_s);
  int nmax = 0;
  for (int x = 0; x < KCX; ++x) nmax = max(nmax, ns_s[x]);
  const int nsub = ns_s[tx];
  const R dts = dts_s[tx];
  if (active)
    for (int k = lane; k < nz; k += KKL) {
      KS(q0, k) = KS(q, k);
      KS(v0, k) = KS(v, k);
    }

  // 1) the forward subcycles: the sedimented qr the conversions start from
  for (int s = 0; s < nmax; ++s) {
    const bool on = active && s < nsub;
    if (on) kes_fluxes(nz, q, rho, v, F);
    __syncthreads();
    if (on) kes_update(nz, dts, q, rho, dz, F);
    __syncthreads();
    if (on && s + 1 < nsub) kes_speeds(a, i, j, rho_sfc, q, rho, v);
    __syncthreads();
  }

  // 2) the conversions' adjoint: xbar = J^T ybar per level (thp, qv, qc in place)
  if (active)
    for (int k = lane; k < nz; k += KKL) {
      const size_t c = L.at(i, j, k);
      using D5 = Dn<R, 5>;
      D5 thp = dn_var<R, 5>(a.thp[c], 0), qv = dn_var<R, 5>(a.qv[c], 1), qc = dn_var<R, 5>(a.qc[c], 2);
      D5 qr = dn_var<R, 5>(KS(q, k), 3);
      const D5 pip = dn_var<R, 5>(a.pip[c], 4);
      kessler_convert<R, D5>(thp, qv, qc, qr, pip, KS(rho, k), a.b.thb[c], a.b.pib[c], a.dt);
      const R y0 = thpB[c], y1 = qvB[c], y2 = qcB[c], y3 = qrB[c];
      R x[5];
#pragma unroll
      for (int m = 0; m < 5; ++m) x[m] = thp.d[m] * y0 + qv.d[m] * y1 + qc.d[m] * y2 + qr.d[m] * y3;
      thpB[c] = x[0];
      qvB[c] = x[1];
      qcB[c] = x[2];
      KS(qb, k) = x[3];
      pipB[c] += x[4];
    }
  __syncthreads();

  // 3) the subcycles backwards; subcycle s needs the fall speeds v^s, replayed
  //    from the column's start
  for (int s = nmax - 1; s >= 0; --s) {
    const bool on = active && s < nsub;
    if (on)
      for (int k = lane; k < nz; k += KKL) {
        KS(q, k) = KS(q0, k);
        KS(v, k) = KS(v0, k);
      }
    __syncthreads();
    for (int r = 0; r < s; ++r) {
      if (on) kes_fluxes(nz, q, rho, v, F);
      __syncthreads();
      if (on) kes_update(nz, dts, q, rho, dz, F);
      __syncthreads();
      if (on) kes_speeds(a, i, j, rho_sfc, q, rho, v);
      __syncthreads();
    }
    // q_k += dts (F_{k+1} - F_k) / (rho_k dz_k): F_k feeds levels k and k-1
    if (on)
      for (int k = lane; k < nz; k += KKL) {
        R fb = -dts * KS(qb, k) / (KS(rho, k) * KS(dz, k));
        if (k >= 1) fb += dts * KS(qb, k - 1) / (KS(rho, k - 1) * KS(dz, k - 1));
        KS(Fb, k) = fb;
      }
    __syncthreads();
    if (on)
      for (int k = lane; k < nz; k += KKL) KS(qb, k) += flux_slope<R>() * KS(rho, k) * KS(v, k) * KS(Fb, k);
    __syncthreads();
  }

  // 4) q = max(qr, 0) at the start
  if (active)
    for (int k = lane; k < nz; k += KKL) {
      const size_t c = L.at(i, j, k);
      qrB[c] = a.qr[c] > (R)0 ? KS(qb, k) : (R)0;
    }
}

#undef KS

template <typename R>
size_t tl_kessler_smem(int nz) {
  return ((size_t)5 * nz + 2 * (nz + 1) + 2 * KKL) * KCX * sizeof(R);
}
template <typename R>
size_t ad_kessler_smem(int nz) {
  return ((size_t)7 * nz + 2 * (nz + 1) + 2 * KKL) * KCX * sizeof(R);
}

}  // namespace

template <typename R>
int lin_kessler_prepare(int nz) {
  if (raise_smem_limit(k_tl_kessler<R>, tl_kessler_smem<R>(nz)) != cudaSuccess ||
      raise_smem_limit(k_ad_kessler<R>, ad_kessler_smem<R>(nz)) != cudaSuccess)
    return 1;
  return 0;
}

template <typename R>
void tl_kessler(const KesArgs<R>& a, const KesArgs<R>& d, cudaStream_t st) {
  k_tl_kessler<R><<<dim3((a.L.nx + KCX - 1) / KCX, a.L.ny), dim3(KCX, KKL), tl_kessler_smem<R>(a.L.nz), st>>>(
      a, d);
}

template <typename R>
void ad_kessler(const KesArgs<R>& a, const KesArgs<R>& d, cudaStream_t st) {
  k_ad_kessler<R><<<dim3((a.L.nx + KCX - 1) / KCX, a.L.ny), dim3(KCX, KKL), ad_kessler_smem<R>(a.L.nz), st>>>(
      a, d);
}

#define WFE_INST(R)                                                                  \
  template int lin_kessler_prepare<R>(int);                                          \
  template void tl_kessler<R>(const KesArgs<R>&, const KesArgs<R>&, cudaStream_t); \
  template void ad_kessler<R>(const KesArgs<R>&, const KesArgs<R>&, cudaStream_t);
WFE_INST(float)
WFE_INST(double)
#undef WFE_INST

}  // namespace wfe
