// Slow-tendency path of one RK3 stage on the B200: one ghost-fill launch,
// one mass-flux launch, an optional positive-definite-limiter launch and one
// fused tendency launch that evaluates every prognostic tendency of a cell
// (5th-order flux-form advection of u, v, w, theta', qv, qc, qr with the
// Gal-Chen metric, Coriolis, Rayleigh sponge, w damping, constant-K diffusion
// and Davies relaxation) and, in the integrator, writes the moisture stage
// value q_n + dt_m * tq directly instead of storing tq.
//
// The arithmetic of every output value follows the reference expression by
// expression (src/dynamics/kernels.cu:42-443, 292-304, 268-273), the face5
// stencil in its expanded one-sided form (dyn_common.cuh), so that the FP64
// build agrees with the reference FP64 build to rounding.
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
  // one thread per work item of field bz: items [0, nx ny) fill the ghost
  // levels of one interior column; the rest fill one chunk of kFillChunk
  // levels of one lateral ghost column (ring_column), chunk by chunk over the
  // ring -- no thread walks a whole column and none idles on a point that is
  // not a ghost
  const Layout& L = A.L;
  const int open_x = A.open_x, open_y = A.open_y;
  const int f = bz;
  if (f >= A.job.n) return;
  R* a = A.job.f[f];
  const int kind = A.job.kind[f];
  const long item = (long)bx * blockDim.x + threadIdx.x;
  const long ncol = (long)L.nx * L.ny, nring = ring_columns(L);
  int i, j, part;  // part 0: ghost levels of an interior column; p >= 1: chunk p - 1
  if (item < ncol) {
    i = (int)(item % L.nx);
    j = (int)(item / L.nx);
    part = 0;
  } else {
    const long r = item - ncol;
    if (r >= nring * fill_chunks(L.nz)) return;
    ring_column(L, r % nring, &i, &j);
    part = 1 + (int)(r / nring);
  }
  const int ilast = (kind == 1 && open_x) ? L.nx : L.nx - 1;
  const int jlast = (kind == 2 && open_y) ? L.ny : L.ny - 1;
  const int si = map_lat(i, L.nx, ilast, open_x);
  const int sj = map_lat(j, L.ny, jlast, open_y);
  const int k0 = -kRefNG, k1 = L.nz + kRefNG;  // inclusive
  if ((si != i) || (sj != j)) {
    // lateral ghost column, levels of this chunk; the sources are another
    // column, so the loads are issued before the stores
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
  // a column that is its own source: an interior column, or a ring column
  // that is not a ghost (the u faces nx of an open x boundary, the v faces ny
  // of an open y boundary; its first chunk's item fills it)
  if (part > 1) return;
  // the levels below 0 and from nz up (w(nz) is the rigid lid)
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
// nz carry Omega = 0.  HB: the base state from its level tables (DBase::lvl).
template <typename R, bool HB = false>
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
  const int c = L.ati(i, j, k);
  const int kk = L.at1(k);
  if (k < L.nz) {
    const R rb = HB ? b.lvl[BL_RHOB * L.pz + kk] : b.rhob[c];
    const R rbx = HB ? rb : b.rhob[L.ati(i - 1, j, k)];
    const R rby = HB ? rb : b.rhob[L.ati(i, j - 1, k)];
    R rjx = (R)0.5 * (rbx * m.jac[L.at2i(i - 1, j)] + rb * m.jac[L.at2i(i, j)]);
    mfx[c] = rjx * u[c];
    R rjy = (R)0.5 * (rby * m.jac[L.at2i(i, j - 1)] + rb * m.jac[L.at2i(i, j)]);
    mfy[c] = rjy * v[c];
  }
  if (i > L.nx + 1 || j > L.ny + 1) return;
  if (k == 0 || k == L.nz) {
    mfz[c] = 0;
    return;
  }
  // the terrain cross flux, where the column has a slope (flat columns skip
  // the eight velocity loads: the product with a zero slope is zero)
  const R hx = m.hx[L.at2i(i, j)], hy = m.hy[L.at2i(i, j)];
  R cross = 0;
  if (hx != (R)0 || hy != (R)0) {
    R fac = (R)1 - m.zeta_w[kk] / m.zt;
    R uw = (R)0.25 * (u[L.ati(i, j, k - 1)] + u[L.ati(i + 1, j, k - 1)] + u[c] + u[L.ati(i + 1, j, k)]);
    R vw = (R)0.25 * (v[L.ati(i, j, k - 1)] + v[L.ati(i, j + 1, k - 1)] + v[c] + v[L.ati(i, j + 1, k)]);
    cross = (uw * hx + vw * hy) * fac;
  }
  mfz[c] = (HB ? b.lvl[BL_RHOBW * L.pz + kk] : b.rhobw[c]) * (w[c] - cross);
}

template <typename R, bool HB>
__global__ void k_mass_flux(FluxArgs<R> a) {
  flux_body<R, HB>(a, blockIdx.x, blockIdx.y, blockIdx.z);
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
  const int c = L.ati(i, j, k);
  return (a.mfx[c + 1] - a.mfx[c]) * a.co.inv_dx + (a.mfy[c + L.px] - a.mfy[c]) * a.co.inv_dy +
         (a.mfz[c + L.planei()] - a.mfz[c]) * a.co.inv_dzc[L.at1(k)];
}

// ------------------------------------------------------------ face fluxes
// Every advective face flux is one exactly rounded product (mul_rn) of its
// mass flux and its face5 value, and every output combines the differences
// of its opposite faces in one expression: a kernel that evaluates each face
// once and shares it gets the bits of one that evaluates the faces per cell.

// The lower face (west, south or bottom, by the stride s) of the momentum
// point at offset o (its upper face: o = s): mass flux averaged over the two
// faces M[o + m0], M[o] beside it, the point's field Q on o - 3s .. o + 2s
// (kernels.cu:308-425).
template <typename R>
__device__ __forceinline__ R face_mom(const R* M, int m0, const R* Q, int s, int o = 0) {
  const R f = (R)0.5 * (M[o + m0] + M[o]);
  return mul_rn(f, face5(Q[o - 3 * s], Q[o - 2 * s], Q[o - s], Q[o], Q[o + s], Q[o + 2 * s], f));
}

// The lower face of a cell-centred scalar: the face's mass flux M[0]
// (kernels.cu:114-179, 187-218).
template <typename R>
__device__ __forceinline__ R face_sc(const R* M, const R* Q, int s) {
  const R f = M[0];
  return mul_rn(f, face5(Q[-3 * s], Q[-2 * s], Q[-s], Q[0], Q[s], Q[2 * s], f));
}

// Flux-form tendency of a scalar cell (value q0, level index kk) from the
// face-flux differences east - west, north - south, top - bottom.
template <typename R>
__device__ __forceinline__ R scalar_tend(const TendArgs<R>& a, R q0, int c, int i, int j, int kk, R dX,
                                         R dY, R dZ, R div) {
  R fdiv = dX * a.co.inv_dx + dY * a.co.inv_dy + dZ * a.co.inv_dzc[kk];
  R rt = a.b.rhob[c] * a.m.jac[a.L.at2i(i, j)];
  return (-fdiv + q0 * div) / rt;
}

// Face fluxes of a scalar used by the positive-definite limiter
// (kernels.cu:187-218): F on the left/lower face of cell (i,j,k).
template <typename R>
__device__ __forceinline__ R qflux_x(const TendArgs<R>& a, const R* q, int i, int j, int k) {
  const int c = a.L.ati(i, j, k);
  return face_sc(a.mfx + c, q + c, 1);
}
template <typename R>
__device__ __forceinline__ R qflux_y(const TendArgs<R>& a, const R* q, int i, int j, int k) {
  const int c = a.L.ati(i, j, k);
  return face_sc(a.mfy + c, q + c, a.L.px);
}
template <typename R>
__device__ __forceinline__ R qflux_z(const TendArgs<R>& a, const R* q, int i, int j, int k) {
  const int c = a.L.ati(i, j, k);
  return face_sc(a.mfz + c, q + c, a.L.planei());
}

// Outflow ratio min(1, available / outgoing) per species (kernels.cu:221-238),
// one thread per cell.  The outgoing flux sums each direction's two faces and
// scales the sum by the precomputed reciprocal spacing (the reference divides
// each face by the spacing: the same value to rounding), one division per
// species instead of seven.
template <typename R>
__device__ __forceinline__ void pd_body(const PdArgs<R>& P, int bx, int by, int bz) {
  const TendArgs<R>& a = P.t;
  const Layout& L = a.L;
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz * blockDim.z + threadIdx.z;
  if (i >= L.nx || j >= L.ny || k >= L.nz) return;
  const int c = L.ati(i, j, k);
  const R idz = a.co.inv_dzc[L.at1(k)];
  const R rt = a.b.rhob[c] * a.m.jac[L.at2i(i, j)];
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const R* q = s == 0 ? a.qv : (s == 1 ? a.qc : a.qr);
    R* outp = s == 0 ? P.rv : (s == 1 ? P.rc : P.rr);
    const R ox = fmax((R)0, qflux_x(a, q, i + 1, j, k)) + fmax((R)0, -qflux_x(a, q, i, j, k));
    const R oy = fmax((R)0, qflux_y(a, q, i, j + 1, k)) + fmax((R)0, -qflux_y(a, q, i, j, k));
    const R oz = fmax((R)0, qflux_z(a, q, i, j, k + 1)) + fmax((R)0, -qflux_z(a, q, i, j, k));
    const R out = ox * a.co.inv_dx + oy * a.co.inv_dy + oz * idz;
    const R avail = rt * fmax((R)0, q[c]);
    const R r = (a.dt * out > (R)1e-20) ? avail / (a.dt * out) : (R)1;
    outp[c] = fmin((R)1, r);
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_pd_ratio(PdArgs<R> a) {
  pd_body(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename R>
__global__ void __launch_bounds__(256) k_pd_ratio_batch(Batch<PdArgs<R>> b) {
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
  return ratio[L.ati(si, sj, sk)];
}

// Limited face fluxes of the renormalised positive-definite advection
// (kernels.cu:241-264): the flux on the lower face of cell (i, j, k) times
// the outflow ratio of its upwind cell (read at its own index when that cell
// is interior, through ratio_at's ghost map otherwise).
template <typename R>
__device__ __forceinline__ R pd_face_x(const TendArgs<R>& a, const R* q, const R* ratio, int i, int j, int k) {
  const int c = a.L.ati(i, j, k);
  const R F = face_sc(a.mfx + c, q + c, 1);
  const int u = F >= (R)0 ? i - 1 : i;
  return mul_rn(F, (u >= 0 && u < a.L.nx) ? ratio[c + (u - i)] : ratio_at(a, ratio, u, j, k));
}
template <typename R>
__device__ __forceinline__ R pd_face_y(const TendArgs<R>& a, const R* q, const R* ratio, int i, int j, int k) {
  const int c = a.L.ati(i, j, k);
  const int sy = a.L.px;
  const R F = face_sc(a.mfy + c, q + c, sy);
  const int u = F >= (R)0 ? j - 1 : j;
  return mul_rn(F, (u >= 0 && u < a.L.ny) ? ratio[c + (u - j) * sy] : ratio_at(a, ratio, i, u, k));
}
template <typename R>
__device__ __forceinline__ R pd_face_z(const TendArgs<R>& a, const R* q, const R* ratio, int i, int j, int k) {
  const int c = a.L.ati(i, j, k);
  const int sz = a.L.planei();
  const R F = face_sc(a.mfz + c, q + c, sz);
  const int u = F >= (R)0 ? k - 1 : k;
  return mul_rn(F, (u >= 0 && u < a.L.nz) ? ratio[c + (u - k) * sz] : ratio_at(a, ratio, i, j, u));
}

// Constant-K Laplacian (kernels.cu:430-443).
template <typename R>
__device__ __forceinline__ R laplacian(const TendArgs<R>& a, const R* f, int i, int j, int k,
                                       bool on_w) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  R dzl = (on_w ? a.m.dzeta_w[kk] : a.m.dzeta_c[kk]) * a.m.jac[L.at2i(i, j)];
  const int c = L.ati(i, j, k);
  R cc = f[c];
  return (f[c + 1] - 2 * cc + f[c - 1]) / (a.dx * a.dx) +
         (f[c + L.px] - 2 * cc + f[c - L.px]) / (a.dy * a.dy) +
         (f[c + L.planei()] - 2 * cc + f[c - L.planei()]) / (dzl * dzl);
}


// One moisture species: tendency (op API) or stage value (integrator) from
// its face-flux differences (limited fluxes under the positive-definite
// option).
template <typename R>
__device__ __forceinline__ R moist_out(const TendArgs<R>& a, const R* q, const R* qn, const R* qo, bool davies_qv,
                                       int i, int j, int k, int c, R dX, R dY, R dZ, R div0) {
  R t = scalar_tend(a, q[c], c, i, j, a.L.at1(k), dX, dY, dZ, div0);
  if (davies_qv) t += davies(a, 4, q, i, j, k);
  return qo ? qn[c] + a.dt_stage * t : t;
}

// A species' stage value or tendency at cell (i, j, k), its faces evaluated
// per cell.
template <typename R>
__device__ __forceinline__ R species_cell(const TendArgs<R>& a, const R* q, const R* ratio, const R* qn,
                                          const R* qo, bool davies_qv, int i, int j, int k, int c, R div0) {
  if (a.p.pd_moist && ratio)
    return moist_out(a, q, qn, qo, davies_qv, i, j, k, c,
                     pd_face_x(a, q, ratio, i + 1, j, k) - pd_face_x(a, q, ratio, i, j, k),
                     pd_face_y(a, q, ratio, i, j + 1, k) - pd_face_y(a, q, ratio, i, j, k),
                     pd_face_z(a, q, ratio, i, j, k + 1) - pd_face_z(a, q, ratio, i, j, k), div0);
  const int sx = 1, sy = a.L.px, sz = a.L.planei();
  const R* MX = a.mfx + c;
  const R* MY = a.mfy + c;
  const R* MZ = a.mfz + c;
  const R* Q = q + c;
  return moist_out(a, q, qn, qo, davies_qv, i, j, k, c, face_sc(MX + sx, Q + sx, sx) - face_sc(MX, Q, sx),
                   face_sc(MY + sy, Q + sy, sy) - face_sc(MY, Q, sy),
                   face_sc(MZ + sz, Q + sz, sz) - face_sc(MZ, Q, sz), div0);
}

// u tendency on the x face i from its face-flux differences and the
// divergences of the cells west of and at it (kernels.cu:308-346); the
// neighbours' divergence comes from a callable, evaluated where the sum needs
// it (fewer registers live across the face evaluations).
template <typename R, class Div>
__device__ __forceinline__ R u_out(const TendArgs<R>& a, int i, int j, int k, R dX, R dY, R dZ, Div div_w,
                                   R div0, bool bdy) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const int c = L.ati(i, j, k);
  const int sx = 1, sy = L.px;
  const R* U = a.u + c;
  const R* V = a.v + c;
  R fdiv = dX * a.co.inv_dx + dY * a.co.inv_dy + dZ * a.co.inv_dzc[kk];
  R dv = (R)0.5 * (div_w() + div0);
  R ru = (R)0.5 * (a.b.rhob[c - sx] * a.m.jac[L.at2i(i - 1, j)] + a.b.rhob[c] * a.m.jac[L.at2i(i, j)]);
  R vavg = (R)0.25 * (V[-sx] + V[sy - sx] + V[0] + V[sy]);
  R fc = (R)0.5 * (a.m.fcor[L.at2i(i - 1, j)] + a.m.fcor[L.at2i(i, j)]);
  R relax = -a.co.spg_c[kk] * (U[0] - a.b.ub[kk]);
  R t = (-fdiv + U[0] * dv) / ru + fc * vavg + relax;
  if (a.p.diff_K > (R)0) t += a.p.diff_K * laplacian(a, a.u, i, j, k, false);
  if (bdy) t += davies(a, 0, a.u, i, j, k);
  return t;
}

// v tendency on the y face j (kernels.cu:348-385); div_s: the cell south of it.
template <typename R, class Div>
__device__ __forceinline__ R v_out(const TendArgs<R>& a, int i, int j, int k, R dX, R dY, R dZ, Div div_s,
                                   R div0, bool bdy) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const int c = L.ati(i, j, k);
  const int sx = 1, sy = L.px;
  const R* U = a.u + c;
  const R* V = a.v + c;
  R fdiv = dX * a.co.inv_dx + dY * a.co.inv_dy + dZ * a.co.inv_dzc[kk];
  R dv = (R)0.5 * (div_s() + div0);
  R rv = (R)0.5 * (a.b.rhob[c - sy] * a.m.jac[L.at2i(i, j - 1)] + a.b.rhob[c] * a.m.jac[L.at2i(i, j)]);
  R uavg = (R)0.25 * (U[-sy] + U[sx - sy] + U[0] + U[sx]);
  R fc = (R)0.5 * (a.m.fcor[L.at2i(i, j - 1)] + a.m.fcor[L.at2i(i, j)]);
  R uref = a.p.coriolis_use_ub ? a.b.ub[kk] : (R)0;
  R relax = -a.co.spg_c[kk] * V[0];
  R t = (-fdiv + V[0] * dv) / rv - fc * (uavg - uref) + relax;
  if (a.p.diff_K > (R)0) t += a.p.diff_K * laplacian(a, a.v, i, j, k, false);
  if (bdy) t += davies(a, 1, a.v, i, j, k);
  return t;
}

// w tendency on the inner level k >= 1 (kernels.cu:387-425); div_b: the cell
// below it.
template <typename R, class Div>
__device__ __forceinline__ R w_out(const TendArgs<R>& a, int i, int j, int k, R dX, R dY, R dZ, Div div_b,
                                   R div0) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const int c = L.ati(i, j, k);
  const R* W = a.w + c;
  R fdiv = dX * a.co.inv_dx + dY * a.co.inv_dy + dZ * a.co.inv_dzw[kk];
  R dv = (R)0.5 * (div_b() + div0);
  R rw = a.b.rhobw[c] * a.m.jac[L.at2i(i, j)];
  R relax = -a.co.spg_w[kk] * W[0];
  R wk = W[0];
  if (a.p.w_damping) {
    R cr = fabs(wk) * a.dt / (a.m.dzeta_w[kk] * a.m.jac[L.at2i(i, j)]);
    if (cr > (R)1) relax -= (R)0.3 * (cr - (R)1) * wk / a.dt;
  }
  R t = (-fdiv + wk * dv) / rw + relax;
  if (a.p.diff_K > (R)0) t += a.p.diff_K * laplacian(a, a.w, i, j, k, true);
  return t;
}

// theta' tendency (kernels.cu:114-146).
template <typename R>
__device__ __forceinline__ R th_out(const TendArgs<R>& a, int i, int j, int k, R dX, R dY, R dZ, R div0,
                                    bool bdy) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const int c = L.ati(i, j, k);
  R t = scalar_tend(a, a.thp[c], c, i, j, kk, dX, dY, dZ, div0) - a.co.spg_c[kk] * a.thp[c];
  if (a.p.diff_K > (R)0) t += a.p.diff_K * laplacian(a, a.thp, i, j, k, false);
  if (bdy) t += davies(a, 2, a.thp, i, j, k);
  return t;
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
  const int c = L.ati(i, j, k);
  const int sx = 1, sy = L.px, sz = L.planei();
  const bool bdy = a.lo[0] != nullptr;
  const R* MX = a.mfx + c;
  const R* MY = a.mfy + c;
  const R* MZ = a.mfz + c;
  const R div0 = divergence(a, i, j, k);

  if (PART & TEND_MOM) {
    const R* U = a.u + c;
    const R dX = face_mom(MX, -sx, U, sx, sx) - face_mom(MX, -sx, U, sx);
    const R dY = face_mom(MY, -sx, U, sy, sy) - face_mom(MY, -sx, U, sy);
    const R dZ = face_mom(MZ, -sx, U, sz, sz) - face_mom(MZ, -sx, U, sz);
    o.tu = u_out(a, i, j, k, dX, dY, dZ, [&] { return divergence(a, i - 1, j, k); }, div0, bdy);
  }
  if (PART & TEND_MOM) {
    const R* V = a.v + c;
    const R dX = face_mom(MX, -sy, V, sx, sx) - face_mom(MX, -sy, V, sx);
    const R dY = face_mom(MY, -sy, V, sy, sy) - face_mom(MY, -sy, V, sy);
    const R dZ = face_mom(MZ, -sy, V, sz, sz) - face_mom(MZ, -sy, V, sz);
    o.tv = v_out(a, i, j, k, dX, dY, dZ, [&] { return divergence(a, i, j - 1, k); }, div0, bdy);
  }
  if ((PART & TEND_MOM) && k >= 1) {
    const R* W = a.w + c;
    const R dX = face_mom(MX, -sz, W, sx, sx) - face_mom(MX, -sz, W, sx);
    const R dY = face_mom(MY, -sz, W, sy, sy) - face_mom(MY, -sz, W, sy);
    const R dZ = face_mom(MZ, -sz, W, sz, sz) - face_mom(MZ, -sz, W, sz);
    o.tw = w_out(a, i, j, k, dX, dY, dZ, [&] { return divergence(a, i, j, k - 1); }, div0);
  }
  if (!(PART & TEND_SCAL)) return;
  {
    const R* T = a.thp + c;
    const R dX = face_sc(MX + sx, T + sx, sx) - face_sc(MX, T, sx);
    const R dY = face_sc(MY + sy, T + sy, sy) - face_sc(MY, T, sy);
    const R dZ = face_sc(MZ + sz, T + sz, sz) - face_sc(MZ, T, sz);
    o.tth = th_out(a, i, j, k, dX, dY, dZ, div0, bdy);
  }
  // pi': no slow advection; Davies only (kernels.cu:900-901)
  if (a.tpi) o.tpi = bdy ? davies(a, 3, a.pip, i, j, k) : (R)0;
  // moisture (kernels.cu:886-899) and its stage update (kernels.cu:268-273)
  if (a.p.moisture) {
    o.q[0] = species_cell(a, a.qv, a.ratio_v, a.qn_v, a.qo_v, bdy, i, j, k, c, div0);
    o.q[1] = species_cell(a, a.qc, a.ratio_c, a.qn_c, a.qo_c, false, i, j, k, c, div0);
    o.q[2] = species_cell(a, a.qr, a.ratio_r, a.qn_r, a.qo_r, false, i, j, k, c, div0);
  }
}

template <typename R, int PART>
__device__ __forceinline__ void tend_store(const TendArgs<R>& a, int i, int j, int k, const TendOut<R>& o) {
  const int c = a.L.ati(i, j, k);
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
// the fused FP32 kernel held to 64 registers (4 blocks per SM): its
// unconstrained allocation takes 80 and runs 3
template <typename R>
__global__ void __launch_bounds__(256, 4) k_tendencies_occ4(TendArgs<R> a) {
  tend_body<R, TEND_ALL>(a, blockIdx.x, blockIdx.y, blockIdx.z);
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
// 256-thread blocks over the interior columns and the ring's chunks, one z
// slice per field
template <typename R>
dim3 grid_fill(const FillArgs<R>& a) {
  const long items = (long)a.L.nx * a.L.ny + ring_columns(a.L) * fill_chunks(a.L.nz);
  return dim3((unsigned)((items + 255) / 256), 1, a.job.n);
}

template <typename R>
void launch_fill_ghosts(const Layout& L, const GhostJob<R>& job, int open_x, int open_y,
                        cudaStream_t st) {
  if (job.n == 0) return;
  FillArgs<R> a{L, job, open_x, open_y};
  k_fill_ghosts<R><<<grid_fill(a), 256, 0, st>>>(a);
}

template <typename R>
void batch_fill(const Batch<FillArgs<R>>& b, int nblocks, cudaStream_t st) {
  k_fill_ghosts_batch<R><<<nblocks, 256, 0, st>>>(b);
}

template <typename R>
dim3 grid_flux(const FluxArgs<R>& a) {
  return dim3((a.L.nx + 5 + 31) / 32, (a.L.ny + 5 + 3) / 4, (a.L.nz + 1 + 1) / 2);
}

template <typename R>
void launch_mass_flux(const Layout& L, const DBase<R>& b, const DMetric<R>& m, const R* u,
                      const R* v, const R* w, R* mfx, R* mfy, R* mfz, cudaStream_t st) {
  FluxArgs<R> a{L, b, m, u, v, w, mfx, mfy, mfz};
  if (b.lvl) k_mass_flux<R, true><<<grid_flux(a), dim3(32, 4, 2), 0, st>>>(a);
  else k_mass_flux<R, false><<<grid_flux(a), dim3(32, 4, 2), 0, st>>>(a);
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
dim3 grid_pd(const Layout& L) {
  return grid_cells<R>(L);
}

template <typename R>
void launch_pd_ratio(const TendArgs<R>& a, R* rv, R* rc, R* rr, cudaStream_t st) {
  k_pd_ratio<R><<<grid_pd<R>(a.L), dim3(32, 4, 2), 0, st>>>(PdArgs<R>{a, rv, rc, rr});
}

template <typename R>
void batch_pd(const Batch<PdArgs<R>>& b, int nblocks, cudaStream_t st) {
  k_pd_ratio_batch<R><<<nblocks, dim3(32, 4, 2), 0, st>>>(b);
}

// the fused and split tendency kernels' blocks
constexpr int kTdBx = 32, kTdBy = 4, kTdBz = 2;

template <typename R>
dim3 grid_tend(const Layout& L) {
  return dim3((L.nx + kTdBx - 1) / kTdBx, (L.ny + kTdBy - 1) / kTdBy, (L.nz + kTdBz - 1) / kTdBz);
}

template <typename R>
void launch_tendencies(const TendArgs<R>& a, int variant, cudaStream_t st) {
  dim3 blk(kTdBx, kTdBy, kTdBz);
  dim3 grd = grid_tend<R>(a.L);
  if (variant == 4) {  // two cells per thread along x
    dim3 b2(16, 4, 2);
    dim3 g2((a.L.nx + 31) / 32, (a.L.ny + 3) / 4, (a.L.nz + 1) / 2);
    k_tendencies2<R, TEND_ALL><<<g2, b2, 0, st>>>(a);
  } else if (variant == 3) {  // momentum only (beside the TMA-staged scalar kernel)
    k_tendencies<R, TEND_MOM><<<grd, blk, 0, st>>>(a);
  } else if (variant == 1) {
    k_tendencies<R, TEND_MOM><<<grd, blk, 0, st>>>(a);
    k_tendencies<R, TEND_SCAL><<<grd, blk, 0, st>>>(a);
  } else if constexpr (sizeof(R) == 4) {
    k_tendencies_occ4<R><<<grd, blk, 0, st>>>(a);
  } else {
    k_tendencies<R, TEND_ALL><<<grd, blk, 0, st>>>(a);
  }
}

// variant 1 runs two subs (momentum, scalars); variant 0 one fused sub
template <typename R>
void batch_tend(const Batch<TendArgs<R>>& b, int variant, int sub, int nblocks, cudaStream_t st) {
  dim3 blk(kTdBx, kTdBy, kTdBz);
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
  template dim3 grid_tend<R>(const Layout&);                                                    \
  template dim3 grid_pd<R>(const Layout&);                                                      \
  template void batch_fill<R>(const Batch<FillArgs<R>>&, int, cudaStream_t);                   \
  template void batch_flux<R>(const Batch<FluxArgs<R>>&, int, cudaStream_t);                   \
  template void batch_pd<R>(const Batch<PdArgs<R>>&, int, cudaStream_t);                       \
  template void batch_tend<R>(const Batch<TendArgs<R>>&, int, int, int, cudaStream_t);         \
  template int occupancy_tend<R>(int, int);
WFE_INST(float)
WFE_INST(double)
#undef WFE_INST

}  // namespace wfe
