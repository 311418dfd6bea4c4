// Slow-tendency path of one RK3 stage on the B200: one ghost-fill launch,
// one mass-flux launch, an optional positive-definite-limiter launch and one
// fused tendency launch that evaluates every prognostic tendency of a cell
// (5th-order flux-form advection of u, v, w, theta', qv, qc, qr with the
// Gal-Chen metric, Coriolis, Rayleigh sponge, w damping, constant-K diffusion
// and Davies relaxation) and, in the integrator, writes the moisture stage
// value q_n + dt_m * tq directly instead of storing tq.
//
// The arithmetic of every output value follows the reference expression by
// expression (src/dynamics/kernels.cu:42-443, 292-304, 268-273) so that the
// FP64 build agrees with the reference FP64 build to rounding.
#include <cuda_runtime.h>

#include "core.cuh"
#include "kernels.cuh"
#include "dyn_common.cuh"

namespace wfe {

// -------------------------------------------------------------- ghost fill
// One launch fills the ghost rings of up to 8 fields with the composition of
// the reference's fill order z -> x -> y (kernels.cu:692-835): a ghost value
// is the z rule applied to the laterally mapped source column.  kind: 0 cell
// scalar, 1 u (x faces 0..nx), 2 v (y faces 0..ny), 3 w (levels 0..nz,
// w(nz) = 0, odd reflection about w(0) below, about w(nz) above).
// ghost value of (i, j, k) from the mapped source column (si, sj)
template <typename R>
__device__ __forceinline__ R ghost_value(const Layout& L, const R* a, int kind, int si, int sj,
                                         int k) {
  if (kind == 3) {  // w: rigid top, odd reflections (kernels.cu:710-723)
    if (k == L.nz) return 0;
    if (k >= 0 && k < L.nz) return a[L.at(si, sj, k)];
    if (k < 0) return (R)2 * a[L.at(si, sj, 0)] - a[L.at(si, sj, -k)];
    return -a[L.at(si, sj, 2 * L.nz - k)];
  }
  return a[L.at(si, sj, map_zc(k, L.nz))];
}

// levels of a lateral ghost column one thread fills (one batch of loads)
constexpr int kFillChunk = 8;
__host__ __device__ inline int fill_chunks(int nz) {
  return (nz + 2 * kRefNG + 1 + kFillChunk - 1) / kFillChunk;
}

template <typename R>
__device__ __forceinline__ void fill_body(const FillArgs<R>& A, int bx, int by, int bz) {
  // one thread per padded column (i, j) of one field and part: part 0 fills
  // the ghost levels of the interior columns, part p >= 1 the p-th chunk of
  // kFillChunk levels of the lateral ghost columns (so that no thread walks a
  // whole column)
  const Layout& L = A.L;
  const int open_x = A.open_x, open_y = A.open_y;
  const int nparts = 1 + fill_chunks(L.nz);
  const int f = bz / nparts, part = bz % nparts;
  if (f >= A.job.n) return;
  R* a = A.job.f[f];
  const int kind = A.job.kind[f];
  const int i = (int)(bx * blockDim.x + threadIdx.x) - kRefNG;
  const int j = (int)(by * blockDim.y + threadIdx.y) - kRefNG;
  if (i > L.nx + 2 || j > L.ny + 2) return;
  const int ilast = (kind == 1 && open_x) ? L.nx : L.nx - 1;
  const int jlast = (kind == 2 && open_y) ? L.ny : L.ny - 1;
  const int si = map_lat(i, L.nx, ilast, open_x);
  const int sj = map_lat(j, L.ny, jlast, open_y);
  const int k0 = -kRefNG, k1 = L.nz + kRefNG;  // inclusive
  if ((si != i) || (sj != j)) {
    // lateral ghost column, levels of this part; the sources are another
    // column, so the loads are issued before the stores
    if (part == 0) return;
    const int kb = k0 + (part - 1) * kFillChunk;
    R v[kFillChunk];
#pragma unroll
    for (int u = 0; u < kFillChunk; ++u)
      if (kb + u <= k1) v[u] = ghost_value(L, a, kind, si, sj, kb + u);
#pragma unroll
    for (int u = 0; u < kFillChunk; ++u)
      if (kb + u <= k1) a[L.at(i, j, kb + u)] = v[u];
    return;
  }
  if (part != 0) return;
  // interior column: the levels below 0 and from nz up (w(nz) is the rigid lid)
  R lo[kRefNG], hi[kRefNG + 1];
#pragma unroll
  for (int m = 1; m <= kRefNG; ++m) lo[m - 1] = ghost_value(L, a, kind, i, j, -m);
#pragma unroll
  for (int m = 0; m <= kRefNG; ++m) hi[m] = ghost_value(L, a, kind, i, j, L.nz + m);
#pragma unroll
  for (int m = 1; m <= kRefNG; ++m) a[L.at(i, j, -m)] = lo[m - 1];
#pragma unroll
  for (int m = 0; m <= kRefNG; ++m) a[L.at(i, j, L.nz + m)] = hi[m];
}

template <typename R>
__global__ void k_fill_ghosts(FillArgs<R> a) {
  fill_body(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename R>
__global__ void k_fill_ghosts_batch(Batch<FillArgs<R>> b) {
  for_each_work(b, [](const FillArgs<R>& a, int x, int y, int z) { fill_body(a, x, y, z); });
}

// ------------------------------------------------------------- mass fluxes
// rho_b J weighted horizontal fluxes on the ring -2..n+2 and the
// contravariant vertical flux on -2..n+1 (kernels.cu:68-97); w levels 0 and
// nz carry Omega = 0.
template <typename R>
__device__ __forceinline__ void flux_body(const FluxArgs<R>& A, int bx, int by, int bz) {
  const Layout& L = A.L;
  const DBase<R>& b = A.b;
  const DMetric<R>& m = A.m;
  const R* __restrict__ u = A.u;
  const R* __restrict__ v = A.v;
  const R* __restrict__ w = A.w;
  R* __restrict__ mfx = A.mfx;
  R* __restrict__ mfy = A.mfy;
  R* __restrict__ mfz = A.mfz;
  const int i = (int)(bx * blockDim.x + threadIdx.x) - 2;
  const int j = (int)(by * blockDim.y + threadIdx.y) - 2;
  const int k = (int)(bz * blockDim.z + threadIdx.z);
  if (i > L.nx + 2 || j > L.ny + 2 || k > L.nz) return;
  const size_t c = L.at(i, j, k);
  if (k < L.nz) {
    R rjx = (R)0.5 * (b.rhob[L.at(i - 1, j, k)] * m.jac[L.at2(i - 1, j)] + b.rhob[c] * m.jac[L.at2(i, j)]);
    mfx[c] = rjx * u[c];
    R rjy = (R)0.5 * (b.rhob[L.at(i, j - 1, k)] * m.jac[L.at2(i, j - 1)] + b.rhob[c] * m.jac[L.at2(i, j)]);
    mfy[c] = rjy * v[c];
  }
  if (i > L.nx + 1 || j > L.ny + 1) return;
  if (k == 0 || k == L.nz) {
    mfz[c] = 0;
    return;
  }
  const int kk = L.at1(k);
  R fac = (R)1 - m.zeta_w[kk] / m.zt;
  R uw = (R)0.25 * (u[L.at(i, j, k - 1)] + u[L.at(i + 1, j, k - 1)] + u[c] + u[L.at(i + 1, j, k)]);
  R vw = (R)0.25 * (v[L.at(i, j, k - 1)] + v[L.at(i, j + 1, k - 1)] + v[c] + v[L.at(i, j + 1, k)]);
  R cross = (uw * m.hx[L.at2(i, j)] + vw * m.hy[L.at2(i, j)]) * fac;
  mfz[c] = b.rhobw[c] * (w[c] - cross);
}

template <typename R>
__global__ void k_mass_flux(FluxArgs<R> a) {
  flux_body(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename R>
__global__ void k_mass_flux_batch(Batch<FluxArgs<R>> b) {
  for_each_work(b, [](const FluxArgs<R>& a, int x, int y, int z) { flux_body(a, x, y, z); });
}

// divergence of the mass flux at cell (i,j,k) (kernels.cu:99-110), evaluated
// where needed instead of being stored
template <typename R>
__device__ __forceinline__ R divergence(const TendArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  const size_t c = L.at(i, j, k);
  return (a.mfx[c + 1] - a.mfx[c]) * a.co.inv_dx + (a.mfy[c + L.px] - a.mfy[c]) * a.co.inv_dy +
         (a.mfz[c + L.plane()] - a.mfz[c]) * a.co.inv_dzc[L.at1(k)];
}

// Flux-form advection of a cell-centred scalar (kernels.cu:114-179).
template <typename R>
__device__ __forceinline__ R scalar_adv(const TendArgs<R>& a, const R* __restrict__ q, int i, int j,
                                        int k, R div) {
  const Layout& L = a.L;
  const size_t c = L.at(i, j, k);
  const size_t sx = 1, sy = L.px, sz = L.plane();
  const R* Q = q + c;
  R fxL = a.mfx[c], fxR = a.mfx[c + sx];
  R fyL = a.mfy[c], fyR = a.mfy[c + sy];
  R fzB = a.mfz[c], fzT = a.mfz[c + sz];
  R FxL = mul_rn(fxL, face5(Q[-3 * (long)sx], Q[-2 * (long)sx], Q[-1 * (long)sx], Q[0], Q[sx], Q[2 * sx], fxL));
  R FxR = mul_rn(fxR, face5(Q[-2 * (long)sx], Q[-1 * (long)sx], Q[0], Q[sx], Q[2 * sx], Q[3 * sx], fxR));
  R FyL = mul_rn(fyL, face5(Q[-3 * (long)sy], Q[-2 * (long)sy], Q[-1 * (long)sy], Q[0], Q[sy], Q[2 * sy], fyL));
  R FyR = mul_rn(fyR, face5(Q[-2 * (long)sy], Q[-1 * (long)sy], Q[0], Q[sy], Q[2 * sy], Q[3 * sy], fyR));
  R FzB = mul_rn(fzB, face5(Q[-3 * (long)sz], Q[-2 * (long)sz], Q[-1 * (long)sz], Q[0], Q[sz], Q[2 * sz], fzB));
  R FzT = mul_rn(fzT, face5(Q[-2 * (long)sz], Q[-1 * (long)sz], Q[0], Q[sz], Q[2 * sz], Q[3 * sz], fzT));
  R fdiv = (FxR - FxL) * a.co.inv_dx + (FyR - FyL) * a.co.inv_dy + (FzT - FzB) * a.co.inv_dzc[L.at1(k)];
  R rt = a.b.rhob[c] * a.m.jac[L.at2(i, j)];
  return (-fdiv + Q[0] * div) / rt;
}

// Face fluxes of a scalar used by the positive-definite limiter
// (kernels.cu:187-218): F on the left/lower face of cell (i,j,k).
template <typename R>
__device__ __forceinline__ R qflux_x(const TendArgs<R>& a, const R* q, int i, int j, int k) {
  const size_t c = a.L.at(i, j, k);
  R f = a.mfx[c];
  const R* Q = q + c;
  return f * face5(Q[-3], Q[-2], Q[-1], Q[0], Q[1], Q[2], f);
}
template <typename R>
__device__ __forceinline__ R qflux_y(const TendArgs<R>& a, const R* q, int i, int j, int k) {
  const size_t c = a.L.at(i, j, k);
  const long s = a.L.px;
  R f = a.mfy[c];
  const R* Q = q + c;
  return f * face5(Q[-3 * s], Q[-2 * s], Q[-s], Q[0], Q[s], Q[2 * s], f);
}
template <typename R>
__device__ __forceinline__ R qflux_z(const TendArgs<R>& a, const R* q, int i, int j, int k) {
  const size_t c = a.L.at(i, j, k);
  const long s = (long)a.L.plane();
  R f = a.mfz[c];
  const R* Q = q + c;
  return f * face5(Q[-3 * s], Q[-2 * s], Q[-s], Q[0], Q[s], Q[2 * s], f);
}

// Outflow ratio min(1, available / outgoing) per species (kernels.cu:221-238).
template <typename R>
__device__ __forceinline__ void pd_body(const PdArgs<R>& P, int bx, int by, int bz) {
  const TendArgs<R>& a = P.t;
  R* __restrict__ rv = P.rv;
  R* __restrict__ rc = P.rc;
  R* __restrict__ rr = P.rr;
  const Layout& L = a.L;
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz * blockDim.z + threadIdx.z;
  if (i >= L.nx || j >= L.ny || k >= L.nz) return;
  const R dzc = a.m.dzeta_c[L.at1(k)];
  const R rt = a.b.rhob[L.at(i, j, k)] * a.m.jac[L.at2(i, j)];
  const R* qs[3] = {a.qv, a.qc, a.qr};
  R* outs[3] = {rv, rc, rr};
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const R* q = qs[s];
    R out = fmax((R)0, qflux_x(a, q, i + 1, j, k)) / a.dx + fmax((R)0, -qflux_x(a, q, i, j, k)) / a.dx +
            fmax((R)0, qflux_y(a, q, i, j + 1, k)) / a.dy + fmax((R)0, -qflux_y(a, q, i, j, k)) / a.dy +
            fmax((R)0, qflux_z(a, q, i, j, k + 1)) / dzc + fmax((R)0, -qflux_z(a, q, i, j, k)) / dzc;
    R avail = rt * fmax((R)0, q[L.at(i, j, k)]);
    R r = (a.dt * out > (R)1e-20) ? avail / (a.dt * out) : (R)1;
    outs[s][L.at(i, j, k)] = fmin((R)1, r);
  }
}

template <typename R>
__global__ void k_pd_ratio(PdArgs<R> a) {
  pd_body(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename R>
__global__ void k_pd_ratio_batch(Batch<PdArgs<R>> b) {
  for_each_work(b, [](const PdArgs<R>& a, int x, int y, int z) { pd_body(a, x, y, z); });
}

// ratio at a possibly-ghost cell: lateral periodic / zero-gradient map
// (kernels.cu:864-866); vertical neighbours only multiply a zero flux.
template <typename R>
__device__ __forceinline__ R ratio_at(const TendArgs<R>& a, const R* ratio, int i, int j, int k) {
  const Layout& L = a.L;
  int si = map_lat(i, L.nx, L.nx - 1, a.p.bc_x_open);
  int sj = map_lat(j, L.ny, L.ny - 1, a.p.bc_y_open);
  int sk = map_zc(k, L.nz);
  return ratio[L.at(si, sj, sk)];
}

// Renormalised positive-definite advection (kernels.cu:241-264).
template <typename R>
__device__ __forceinline__ R pd_adv(const TendArgs<R>& a, const R* q, const R* ratio, int i, int j,
                                    int k, R div) {
  const Layout& L = a.L;
  R fxl = qflux_x(a, q, i, j, k), fxr = qflux_x(a, q, i + 1, j, k);
  R fyl = qflux_y(a, q, i, j, k), fyr = qflux_y(a, q, i, j + 1, k);
  R fzl = qflux_z(a, q, i, j, k), fzr = qflux_z(a, q, i, j, k + 1);
  R sxl, sxr, syl, syr, szl, szr;
  if (i > 0 && i < L.nx - 1 && j > 0 && j < L.ny - 1 && k > 0 && k < L.nz - 1) {
    // every upwind cell is interior: plain offsets from the cell
    const R* r0 = ratio + L.at(i, j, k);
    const int sy = L.px, sz = (int)L.plane();
    sxl = fxl * r0[fxl >= (R)0 ? -1 : 0];
    sxr = fxr * r0[fxr >= (R)0 ? 0 : 1];
    syl = fyl * r0[fyl >= (R)0 ? -sy : 0];
    syr = fyr * r0[fyr >= (R)0 ? 0 : sy];
    szl = fzl * r0[fzl >= (R)0 ? -sz : 0];
    szr = fzr * r0[fzr >= (R)0 ? 0 : sz];
  } else {
    sxl = fxl * ratio_at(a, ratio, fxl >= (R)0 ? i - 1 : i, j, k);
    sxr = fxr * ratio_at(a, ratio, fxr >= (R)0 ? i : i + 1, j, k);
    syl = fyl * ratio_at(a, ratio, i, fyl >= (R)0 ? j - 1 : j, k);
    syr = fyr * ratio_at(a, ratio, i, fyr >= (R)0 ? j : j + 1, k);
    szl = fzl * ratio_at(a, ratio, i, j, fzl >= (R)0 ? k - 1 : k);
    szr = fzr * ratio_at(a, ratio, i, j, fzr >= (R)0 ? k : k + 1);
  }
  R fdiv = (sxr - sxl) * a.co.inv_dx + (syr - syl) * a.co.inv_dy + (szr - szl) * a.co.inv_dzc[L.at1(k)];
  R rt = a.b.rhob[L.at(i, j, k)] * a.m.jac[L.at2(i, j)];
  return (-fdiv + q[L.at(i, j, k)] * div) / rt;
}

// Constant-K Laplacian (kernels.cu:430-443).
template <typename R>
__device__ __forceinline__ R laplacian(const TendArgs<R>& a, const R* f, int i, int j, int k,
                                       bool on_w) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  R dzl = (on_w ? a.m.dzeta_w[kk] : a.m.dzeta_c[kk]) * a.m.jac[L.at2(i, j)];
  const size_t c = L.at(i, j, k);
  R cc = f[c];
  return (f[c + 1] - 2 * cc + f[c - 1]) / (a.dx * a.dx) +
         (f[c + L.px] - 2 * cc + f[c - L.px]) / (a.dy * a.dy) +
         (f[c + L.plane()] - 2 * cc + f[c - L.plane()]) / (dzl * dzl);
}


// One moisture species: tendency (op API) or stage value (integrator).
template <typename R>
__device__ __forceinline__ R moist_species(const TendArgs<R>& a, const R* q, const R* ratio,
                                           const R* qn, const R* qo, bool davies_qv, int i, int j,
                                           int k, size_t c, R div0) {
  R t = (a.p.pd_moist && ratio) ? pd_adv(a, q, ratio, i, j, k, div0)
                                : scalar_adv(a, q, i, j, k, div0);
  if (davies_qv) t += davies(a, 4, q, i, j, k);
  return qo ? qn[c] + a.dt_stage * t : t;
}

// The outputs of one cell, computed before any of them is stored (so that a
// thread computing two cells reads all its inputs before its first store).
template <typename R>
struct TendOut {
  R tu, tv, tw, tth, tpi, q[3];
};

// ------------------------------------------------------ fused tendencies
// PART selects the prognostics a launch computes: 1 = momentum (u, v, w),
// 2 = scalars (theta', pi' relaxation, qv, qc, qr), 3 = all of them.  The
// split variants need fewer registers (higher occupancy); the autotuner picks.
enum { TEND_MOM = 1, TEND_SCAL = 2, TEND_ALL = 3 };

template <typename R, int PART>
__device__ __forceinline__ void tend_cell(const TendArgs<R>& a, int i, int j, int k, TendOut<R>& o) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const size_t c = L.at(i, j, k);
  const long sx = 1, sy = L.px, sz = (long)L.plane();
  const bool bdy = a.lo[0] != nullptr;
  const R* MX = a.mfx + c;
  const R* MY = a.mfy + c;
  const R* MZ = a.mfz + c;
  const R div0 = divergence(a, i, j, k);

  // ---- u on the x face i (kernels.cu:308-346)
  if (PART & TEND_MOM) {
    const R* U = a.u + c;
    R fcL = (R)0.5 * (MX[-sx] + MX[0]), fcR = (R)0.5 * (MX[0] + MX[sx]);
    R FxL = fcL * face5(U[-3 * sx], U[-2 * sx], U[-sx], U[0], U[sx], U[2 * sx], fcL);
    R FxR = fcR * face5(U[-2 * sx], U[-sx], U[0], U[sx], U[2 * sx], U[3 * sx], fcR);
    R fyB = (R)0.5 * (MY[-sx] + MY[0]), fyT = (R)0.5 * (MY[sy - sx] + MY[sy]);
    R FyB = fyB * face5(U[-3 * sy], U[-2 * sy], U[-sy], U[0], U[sy], U[2 * sy], fyB);
    R FyT = fyT * face5(U[-2 * sy], U[-sy], U[0], U[sy], U[2 * sy], U[3 * sy], fyT);
    R fzB = (R)0.5 * (MZ[-sx] + MZ[0]), fzT = (R)0.5 * (MZ[sz - sx] + MZ[sz]);
    R FzB = fzB * face5(U[-3 * sz], U[-2 * sz], U[-sz], U[0], U[sz], U[2 * sz], fzB);
    R FzT = fzT * face5(U[-2 * sz], U[-sz], U[0], U[sz], U[2 * sz], U[3 * sz], fzT);
    R fdiv = (FxR - FxL) * a.co.inv_dx + (FyT - FyB) * a.co.inv_dy + (FzT - FzB) * a.co.inv_dzc[kk];
    R dv = (R)0.5 * (divergence(a, i - 1, j, k) + div0);
    R ru = (R)0.5 * (a.b.rhob[c - sx] * a.m.jac[L.at2(i - 1, j)] + a.b.rhob[c] * a.m.jac[L.at2(i, j)]);
    const R* V = a.v + c;
    R vavg = (R)0.25 * (V[-sx] + V[sy - sx] + V[0] + V[sy]);
    R fc = (R)0.5 * (a.m.fcor[L.at2(i - 1, j)] + a.m.fcor[L.at2(i, j)]);
    R relax = -a.co.spg_c[kk] * (U[0] - a.b.ub[kk]);
    R t = (-fdiv + U[0] * dv) / ru + fc * vavg + relax;
    if (a.p.diff_K > (R)0) t += a.p.diff_K * laplacian(a, a.u, i, j, k, false);
    if (bdy) t += davies(a, 0, a.u, i, j, k);
    o.tu = t;
  }
  // ---- v on the y face j (kernels.cu:348-385)
  if (PART & TEND_MOM) {
    const R* V = a.v + c;
    R fcB = (R)0.5 * (MY[-sy] + MY[0]), fcT = (R)0.5 * (MY[0] + MY[sy]);
    R FyB = fcB * face5(V[-3 * sy], V[-2 * sy], V[-sy], V[0], V[sy], V[2 * sy], fcB);
    R FyT = fcT * face5(V[-2 * sy], V[-sy], V[0], V[sy], V[2 * sy], V[3 * sy], fcT);
    R fxL = (R)0.5 * (MX[-sy] + MX[0]), fxR = (R)0.5 * (MX[sx - sy] + MX[sx]);
    R FxL = fxL * face5(V[-3 * sx], V[-2 * sx], V[-sx], V[0], V[sx], V[2 * sx], fxL);
    R FxR = fxR * face5(V[-2 * sx], V[-sx], V[0], V[sx], V[2 * sx], V[3 * sx], fxR);
    R fzB = (R)0.5 * (MZ[-sy] + MZ[0]), fzT = (R)0.5 * (MZ[sz - sy] + MZ[sz]);
    R FzB = fzB * face5(V[-3 * sz], V[-2 * sz], V[-sz], V[0], V[sz], V[2 * sz], fzB);
    R FzT = fzT * face5(V[-2 * sz], V[-sz], V[0], V[sz], V[2 * sz], V[3 * sz], fzT);
    R fdiv = (FxR - FxL) * a.co.inv_dx + (FyT - FyB) * a.co.inv_dy + (FzT - FzB) * a.co.inv_dzc[kk];
    R dv = (R)0.5 * (divergence(a, i, j - 1, k) + div0);
    R rv = (R)0.5 * (a.b.rhob[c - sy] * a.m.jac[L.at2(i, j - 1)] + a.b.rhob[c] * a.m.jac[L.at2(i, j)]);
    const R* U = a.u + c;
    R uavg = (R)0.25 * (U[-sy] + U[sx - sy] + U[0] + U[sx]);
    R fc = (R)0.5 * (a.m.fcor[L.at2(i, j - 1)] + a.m.fcor[L.at2(i, j)]);
    R uref = a.p.coriolis_use_ub ? a.b.ub[kk] : (R)0;
    R relax = -a.co.spg_c[kk] * V[0];
    R t = (-fdiv + V[0] * dv) / rv - fc * (uavg - uref) + relax;
    if (a.p.diff_K > (R)0) t += a.p.diff_K * laplacian(a, a.v, i, j, k, false);
    if (bdy) t += davies(a, 1, a.v, i, j, k);
    o.tv = t;
  }
  // ---- w on the inner level k >= 1 (kernels.cu:387-425)
  if ((PART & TEND_MOM) && k >= 1) {
    const R* W = a.w + c;
    R fxL = (R)0.5 * (MX[-sz] + MX[0]), fxR = (R)0.5 * (MX[sx - sz] + MX[sx]);
    R FxL = fxL * face5(W[-3 * sx], W[-2 * sx], W[-sx], W[0], W[sx], W[2 * sx], fxL);
    R FxR = fxR * face5(W[-2 * sx], W[-sx], W[0], W[sx], W[2 * sx], W[3 * sx], fxR);
    R fyB = (R)0.5 * (MY[-sz] + MY[0]), fyT = (R)0.5 * (MY[sy - sz] + MY[sy]);
    R FyB = fyB * face5(W[-3 * sy], W[-2 * sy], W[-sy], W[0], W[sy], W[2 * sy], fyB);
    R FyT = fyT * face5(W[-2 * sy], W[-sy], W[0], W[sy], W[2 * sy], W[3 * sy], fyT);
    R fzB = (R)0.5 * (MZ[-sz] + MZ[0]), fzT = (R)0.5 * (MZ[0] + MZ[sz]);
    R FzB = fzB * face5(W[-3 * sz], W[-2 * sz], W[-sz], W[0], W[sz], W[2 * sz], fzB);
    R FzT = fzT * face5(W[-2 * sz], W[-sz], W[0], W[sz], W[2 * sz], W[3 * sz], fzT);
    R fdiv = (FxR - FxL) * a.co.inv_dx + (FyT - FyB) * a.co.inv_dy + (FzT - FzB) * a.co.inv_dzw[kk];
    R dv = (R)0.5 * (divergence(a, i, j, k - 1) + div0);
    R rw = a.b.rhobw[c] * a.m.jac[L.at2(i, j)];
    R relax = -a.co.spg_w[kk] * W[0];
    R wk = W[0];
    if (a.p.w_damping) {
      R cr = fabs(wk) * a.dt / (a.m.dzeta_w[kk] * a.m.jac[L.at2(i, j)]);
      if (cr > (R)1) relax -= (R)0.3 * (cr - (R)1) * wk / a.dt;
    }
    R t = (-fdiv + wk * dv) / rw + relax;
    if (a.p.diff_K > (R)0) t += a.p.diff_K * laplacian(a, a.w, i, j, k, true);
    o.tw = t;
  }
  if (!(PART & TEND_SCAL)) return;
  // ---- theta' (kernels.cu:114-146)
  {
    R t = scalar_adv(a, a.thp, i, j, k, div0) - a.co.spg_c[kk] * a.thp[c];
    if (a.p.diff_K > (R)0) t += a.p.diff_K * laplacian(a, a.thp, i, j, k, false);
    if (bdy) t += davies(a, 2, a.thp, i, j, k);
    o.tth = t;
  }
  // ---- pi': no slow advection; Davies only (kernels.cu:900-901)
  if (a.tpi) o.tpi = bdy ? davies(a, 3, a.pip, i, j, k) : (R)0;
  // ---- moisture (kernels.cu:886-899) and its stage update (kernels.cu:268-273)
  if (a.p.moisture) {
    o.q[0] = moist_species(a, a.qv, a.ratio_v, a.qn_v, a.qo_v, bdy, i, j, k, c, div0);
    o.q[1] = moist_species(a, a.qc, a.ratio_c, a.qn_c, a.qo_c, false, i, j, k, c, div0);
    o.q[2] = moist_species(a, a.qr, a.ratio_r, a.qn_r, a.qo_r, false, i, j, k, c, div0);
  }
}

template <typename R, int PART>
__device__ __forceinline__ void tend_store(const TendArgs<R>& a, int i, int j, int k, const TendOut<R>& o) {
  const size_t c = a.L.at(i, j, k);
  if (PART & TEND_MOM) {
    a.tu[c] = o.tu;
    a.tv[c] = o.tv;
    if (k >= 1) a.tw[c] = o.tw;
  }
  if (!(PART & TEND_SCAL)) return;
  a.tth[c] = o.tth;
  if (a.tpi) a.tpi[c] = o.tpi;
  if (a.p.moisture) {
    (a.qo_v ? a.qo_v : a.tqv)[c] = o.q[0];
    (a.qo_c ? a.qo_c : a.tqc)[c] = o.q[1];
    (a.qo_r ? a.qo_r : a.tqr)[c] = o.q[2];
  }
}

template <typename R, int PART>
__device__ __forceinline__ void tend_body(const TendArgs<R>& a, int bx, int by, int bz) {
  const Layout& L = a.L;
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz * blockDim.z + threadIdx.z;
  if (i >= L.nx || j >= L.ny || k >= L.nz) return;
  TendOut<R> o;
  tend_cell<R, PART>(a, i, j, k, o);
  tend_store<R, PART>(a, i, j, k, o);
}

// Two neighbouring cells along x per thread, both computed before either is
// stored: the cells' stencils share most of their loads and all of their
// row and level offsets (the same values as tend_body).
template <typename R, int PART>
__device__ __forceinline__ void tend_body2(const TendArgs<R>& a, int bx, int by, int bz) {
  const Layout& L = a.L;
  const int i = 2 * (bx * blockDim.x + threadIdx.x);
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz * blockDim.z + threadIdx.z;
  if (i >= L.nx || j >= L.ny || k >= L.nz) return;
  TendOut<R> o0;
  if (i + 1 < L.nx) {
    TendOut<R> o1;
    tend_cell<R, PART>(a, i, j, k, o0);
    tend_cell<R, PART>(a, i + 1, j, k, o1);
    tend_store<R, PART>(a, i, j, k, o0);
    tend_store<R, PART>(a, i + 1, j, k, o1);
  } else {
    tend_cell<R, PART>(a, i, j, k, o0);
    tend_store<R, PART>(a, i, j, k, o0);
  }
}

template <typename R, int PART>
__global__ void __launch_bounds__(256) k_tendencies(TendArgs<R> a) {
  tend_body<R, PART>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename R, int PART>
__global__ void __launch_bounds__(128) k_tendencies2(TendArgs<R> a) {
  tend_body2<R, PART>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename R, int PART>
__global__ void __launch_bounds__(256) k_tendencies_batch(Batch<TendArgs<R>> b) {
  for_each_work(b, [](const TendArgs<R>& a, int x, int y, int z) { tend_body<R, PART>(a, x, y, z); });
}

// ------------------------------------------------------- small utilities
__device__ __forceinline__ void clock_body(const ClockArgs& a) {
  if (threadIdx.x != 0) return;
  double* clk = a.clk;
  if (a.advance) {
    clk[CLK_T] += clk[CLK_DT];
  } else {
    clk[CLK_T] = a.t;
    clk[CLK_TLO] = a.t_lo;
    clk[CLK_THI] = a.t_hi;
    clk[CLK_DT] = a.dt;
  }
}

__global__ void k_clock(ClockArgs a) { clock_body(a); }
__global__ void k_clock_batch(Batch<ClockArgs> b) {
  for_each_work(b, [](const ClockArgs& a, int, int, int) { clock_body(a); });
}

void launch_clock(double* clock, double t, double t_lo, double t_hi, double dt, int advance,
                  cudaStream_t st) {
  k_clock<<<1, 32, 0, st>>>(ClockArgs{clock, t, t_lo, t_hi, dt, advance});
}

dim3 grid_clock() { return dim3(1, 1, 1); }

void batch_clock(const Batch<ClockArgs>& b, int nblocks, cudaStream_t st) {
  k_clock_batch<<<nblocks, 32, 0, st>>>(b);
}

// out = x + a * y over every stored point (src/dynamics/kernels.cu:268-273)
template <typename R>
__global__ void k_axpy(const R* __restrict__ x, const R* __restrict__ y, R a, R* __restrict__ out,
                       size_t n) {
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x)
    out[q] = x[q] + a * y[q];
}

template <typename R>
void launch_axpy(const R* x, const R* y, R a, R* out, size_t n, cudaStream_t st) {
  int grd = (int)((n + 255) / 256);
  if (grd > 148 * 16) grd = 148 * 16;
  k_axpy<R><<<grd, 256, 0, st>>>(x, y, a, out, n);
}

// ------------------------------------------------------------ host launch
template <typename R>
dim3 grid_fill(const FillArgs<R>& a) {
  return dim3((a.L.nx + 6 + 31) / 32, (a.L.ny + 6 + 3) / 4, a.job.n * (1 + fill_chunks(a.L.nz)));
}

template <typename R>
void launch_fill_ghosts(const Layout& L, const GhostJob<R>& job, int open_x, int open_y,
                        cudaStream_t st) {
  if (job.n == 0) return;
  FillArgs<R> a{L, job, open_x, open_y};
  k_fill_ghosts<R><<<grid_fill(a), dim3(32, 4), 0, st>>>(a);
}

template <typename R>
void batch_fill(const Batch<FillArgs<R>>& b, int nblocks, cudaStream_t st) {
  k_fill_ghosts_batch<R><<<nblocks, dim3(32, 4), 0, st>>>(b);
}

template <typename R>
dim3 grid_flux(const FluxArgs<R>& a) {
  return dim3((a.L.nx + 5 + 31) / 32, (a.L.ny + 5 + 3) / 4, (a.L.nz + 1 + 1) / 2);
}

template <typename R>
void launch_mass_flux(const Layout& L, const DBase<R>& b, const DMetric<R>& m, const R* u,
                      const R* v, const R* w, R* mfx, R* mfy, R* mfz, cudaStream_t st) {
  FluxArgs<R> a{L, b, m, u, v, w, mfx, mfy, mfz};
  k_mass_flux<R><<<grid_flux(a), dim3(32, 4, 2), 0, st>>>(a);
}

template <typename R>
void batch_flux(const Batch<FluxArgs<R>>& b, int nblocks, cudaStream_t st) {
  k_mass_flux_batch<R><<<nblocks, dim3(32, 4, 2), 0, st>>>(b);
}

template <typename R>
dim3 grid_cells(const Layout& L) {
  return dim3((L.nx + 31) / 32, (L.ny + 3) / 4, (L.nz + 1) / 2);
}

template <typename R>
void launch_pd_ratio(const TendArgs<R>& a, R* rv, R* rc, R* rr, cudaStream_t st) {
  k_pd_ratio<R><<<grid_cells<R>(a.L), dim3(32, 4, 2), 0, st>>>(PdArgs<R>{a, rv, rc, rr});
}

template <typename R>
void batch_pd(const Batch<PdArgs<R>>& b, int nblocks, cudaStream_t st) {
  k_pd_ratio_batch<R><<<nblocks, dim3(32, 4, 2), 0, st>>>(b);
}

template <typename R>
void launch_tendencies(const TendArgs<R>& a, int variant, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  dim3 grd = grid_cells<R>(a.L);
  if (variant == 4) {  // two cells per thread along x
    dim3 b2(16, 4, 2);
    dim3 g2((a.L.nx + 31) / 32, (a.L.ny + 3) / 4, (a.L.nz + 1) / 2);
    k_tendencies2<R, TEND_ALL><<<g2, b2, 0, st>>>(a);
  } else if (variant == 3) {  // momentum only (beside the TMA-staged scalar kernel)
    k_tendencies<R, TEND_MOM><<<grd, blk, 0, st>>>(a);
  } else if (variant == 1) {
    k_tendencies<R, TEND_MOM><<<grd, blk, 0, st>>>(a);
    k_tendencies<R, TEND_SCAL><<<grd, blk, 0, st>>>(a);
  } else {
    k_tendencies<R, TEND_ALL><<<grd, blk, 0, st>>>(a);
  }
}

// variant 1 runs two subs (momentum, scalars); variant 0 one fused sub
template <typename R>
void batch_tend(const Batch<TendArgs<R>>& b, int variant, int sub, int nblocks, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  if (variant == 1) {
    if (sub == 0) k_tendencies_batch<R, TEND_MOM><<<nblocks, blk, 0, st>>>(b);
    else k_tendencies_batch<R, TEND_SCAL><<<nblocks, blk, 0, st>>>(b);
  } else {
    k_tendencies_batch<R, TEND_ALL><<<nblocks, blk, 0, st>>>(b);
  }
}

template <typename R>
int occupancy_tend(int variant, int sub) {
  int n = 0;
  cudaError_t e;
  if (variant == 1 && sub == 0)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tendencies_batch<R, TEND_MOM>, 256, 0);
  else if (variant == 1)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tendencies_batch<R, TEND_SCAL>, 256, 0);
  else
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tendencies_batch<R, TEND_ALL>, 256, 0);
  return e == cudaSuccess && n > 0 ? n : 1;
}

#define WFE_INST(R)                                                                               \
  template void launch_fill_ghosts<R>(const Layout&, const GhostJob<R>&, int, int, cudaStream_t); \
  template void launch_mass_flux<R>(const Layout&, const DBase<R>&, const DMetric<R>&, const R*,  \
                                    const R*, const R*, R*, R*, R*, cudaStream_t);                \
  template void launch_pd_ratio<R>(const TendArgs<R>&, R*, R*, R*, cudaStream_t);                 \
  template void launch_tendencies<R>(const TendArgs<R>&, int, cudaStream_t);                         \
  template void launch_axpy<R>(const R*, const R*, R, R*, size_t, cudaStream_t);              \
  template dim3 grid_fill<R>(const FillArgs<R>&);                                              \
  template dim3 grid_flux<R>(const FluxArgs<R>&);                                              \
  template dim3 grid_cells<R>(const Layout&);                                                   \
  template void batch_fill<R>(const Batch<FillArgs<R>>&, int, cudaStream_t);                   \
  template void batch_flux<R>(const Batch<FluxArgs<R>>&, int, cudaStream_t);                   \
  template void batch_pd<R>(const Batch<PdArgs<R>>&, int, cudaStream_t);                       \
  template void batch_tend<R>(const Batch<TendArgs<R>>&, int, int, int, cudaStream_t);         \
  template int occupancy_tend<R>(int, int);
WFE_INST(float)
WFE_INST(double)
#undef WFE_INST

}  // namespace wfe
