// Split-explicit acoustic substep on the B200 (src/dynamics/kernels.cu:445-688).
//
// Two launches per substep replace the reference's 9-11:
//   k_acoustic_uv      forward u, v update with divergence damping, full
//                      theta_v PGF, terrain cross term and map factor, plus the
//                      Klemp-Wilhelmson radiation faces (open) or the periodic
//                      face (u(nx) = u(0)) computed in the same thread;
//   k_acoustic_column  the vertically implicit w - pi' system of a column
//                      (off-centred, Thomas), theta' stratification update and
//                      diagnostic surface w.  A CTA owns CX whole columns; the
//                      column coefficients live in shared memory, the per-level
//                      phases run in parallel over k and the Thomas sweep runs
//                      in one lane per column (the reference keeps seven
//                      320-deep arrays per thread in local memory).
//
// No ghost-fill launch is needed inside the acoustic loop: pi' at a ghost point
// is read from the mapped interior point of the current buffer (the reference
// refreshes pi' ghosts after every substep), while pi'_prev, theta' and qv at
// lateral ghosts come from the time-n state (the reference's copies are made at
// the stage start and never refreshed: kernels.cu:946-963, integrator.cpp:93-94).
// u, v, theta' and pi' are double buffered by the integrator, so the column
// kernel may read neighbours while the next substep's buffers are written.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

#include "core.cuh"
#include "kernels.cuh"
#include "acou_pcr.cuh"
#include "dyn_common.cuh"
#include "tma.cuh"

namespace wfe {

// ---------------------------------------------------- run-constant coefficients
template <typename R>
__global__ void k_coef_centre(Layout L, DBase<R> b, DMetric<R> m, R* rtjc, R* kt3, R* aw) {
  // kernels.cu:452-464 over the whole padded grid
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) - kOX;
  const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y) - kOY;
  const int k = (int)(blockIdx.z * blockDim.z + threadIdx.z) - kOZ;
  if (i + kOX >= L.px || j + kOY >= L.py || k + kOZ >= L.pz) return;
  const size_t c = L.at(i, j, k);
  R J = m.jac[L.at2(i, j)];
  rtjc[c] = b.rhob[c] * b.thvb[c] * J;
  kt3[c] = Phys<R>::Rd * b.pib[c] / (Phys<R>::cv * b.rhob[c] * b.thvb[c] * J);
  aw[c] = b.rhobw[c] * b.thvbw[c];
}

template <typename R>
__global__ void k_coef_face(Layout L, const R* rtjc, R* rtjx, R* rtjy) {
  // kernels.cu:466-474: face averages; the first padded row/column of the
  // reference layout (i = -3, j = -3) keeps the centre value
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) - kOX;
  const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y) - kOY;
  const int k = (int)(blockIdx.z * blockDim.z + threadIdx.z) - kOZ;
  if (i + kOX >= L.px || j + kOY >= L.py || k + kOZ >= L.pz) return;
  const size_t c = L.at(i, j, k);
  rtjx[c] = (i > -kRefNG) ? (R)0.5 * (rtjc[c - 1] + rtjc[c]) : rtjc[c];
  rtjy[c] = (j > -kRefNG) ? (R)0.5 * (rtjc[c - L.px] + rtjc[c]) : rtjc[c];
}

// ------------------------------------------------------------ forward u, v
// Interior points: every neighbour the forward step reads is an interior
// point, so pi* and theta_v are plain offsets from the face (no ghost maps).
template <typename R>
__device__ __forceinline__ bool uv_interior(const Layout& L, int i, int j, int k) {
  return i >= 1 && i < L.nx && j >= 1 && j < L.ny && k >= 1 && k < L.nz - 1;
}

template <typename R>
__device__ __forceinline__ R pistar_at(const AcouArgs<R>& a, int c) {
  R cur = a.pi_cur[c];
  return cur + a.p.acoustic_smdiv * (cur - a.pi_prev[c]);
}

// theta_v from the cell's base theta thb
template <typename R>
__device__ __forceinline__ R theta_v_with(const AcouArgs<R>& a, int c, R thb) {
  R t = thb + a.th_in[c];
  if (a.p.moisture) t *= (R)1 + Phys<R>::eps61 * a.qv[c];
  return t;
}

template <typename R>
__device__ __forceinline__ R theta_v_at(const AcouArgs<R>& a, int c) {
  return theta_v_with(a, c, a.b.thb[c]);
}

// u (d = 1) or v (d = L.px) forward step at an interior face, with the
// reference's expressions (kernels.cu:499-526)
template <typename R>
__device__ __forceinline__ R uv_forward_interior(const AcouArgs<R>& a, int i, int j, int k, bool is_u) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const int c = L.ati(i, j, k);
  const int c2 = L.at2i(i, j);
  const int d = is_u ? 1 : L.px;
  const int pl = L.planei();
  R thb_f = (R)0.5 * (theta_v_at(a, c - d) + theta_v_at(a, c));
  R mf = (R)0.5 * (a.m.mapf[c2 - d] + a.m.mapf[c2]);
  R p0 = pistar_at(a, c), pm = pistar_at(a, c - d);
  R grad = (p0 - pm) / (is_u ? a.dx : a.dy);
  R slope = (is_u ? a.m.hx_u[c2] : a.m.hy_v[c2]) * ((R)1 - a.m.zeta_c[kk] / a.m.zt);
  if (slope != (R)0) {
    R dzc2 = a.m.zeta_c[kk + 1] - a.m.zeta_c[kk - 1];
    R jf = (R)0.5 * (a.m.jac[c2 - d] + a.m.jac[c2]);
    R dpdz = (R)0.5 *
             ((pistar_at(a, c - d + pl) - pistar_at(a, c - d - pl)) +
              (pistar_at(a, c + pl) - pistar_at(a, c - pl))) /
             dzc2;
    grad -= slope / jf * dpdz;
  }
  const R* tin = is_u ? a.tu : a.tv;
  const R* vin = is_u ? a.u_in : a.v_in;
  return vin[c] + a.dtau * (-Phys<R>::cp * thb_f * mf * grad + tin[c]);
}

template <typename R>
__device__ __forceinline__ R u_forward(const AcouArgs<R>& a, int i, int j, int k) {
  // kernels.cu:499-512
  const Layout& L = a.L;
  if (uv_interior<R>(L, i, j, k)) return uv_forward_interior(a, i, j, k, true);
  const int kk = L.at1(k);
  const R zt = a.m.zt;
  R thbu = (R)0.5 * (theta_v(a, i - 1, j, k) + theta_v(a, i, j, k));
  R mu = (R)0.5 * (a.m.mapf[L.at2i(i - 1, j)] + a.m.mapf[L.at2i(i, j)]);
  R grad = (pistar(a, i, j, k) - pistar(a, i - 1, j, k)) / a.dx;
  R zxu = a.m.hx_u[L.at2i(i, j)] * ((R)1 - a.m.zeta_c[kk] / zt);
  if (zxu != (R)0) {
    R dzc2 = a.m.zeta_c[kk + 1] - a.m.zeta_c[kk - 1];
    R ju = (R)0.5 * (a.m.jac[L.at2i(i - 1, j)] + a.m.jac[L.at2i(i, j)]);
    R dpdz = (R)0.5 *
             ((pistar(a, i - 1, j, k + 1) - pistar(a, i - 1, j, k - 1)) +
              (pistar(a, i, j, k + 1) - pistar(a, i, j, k - 1))) /
             dzc2;
    grad -= zxu / ju * dpdz;
  }
  const int c = L.ati(i, j, k);
  return a.u_in[c] + a.dtau * (-Phys<R>::cp * thbu * mu * grad + a.tu[c]);
}

template <typename R>
__device__ __forceinline__ R v_forward(const AcouArgs<R>& a, int i, int j, int k) {
  // kernels.cu:513-526
  const Layout& L = a.L;
  if (uv_interior<R>(L, i, j, k)) return uv_forward_interior(a, i, j, k, false);
  const int kk = L.at1(k);
  const R zt = a.m.zt;
  R thbv = (R)0.5 * (theta_v(a, i, j - 1, k) + theta_v(a, i, j, k));
  R mv = (R)0.5 * (a.m.mapf[L.at2i(i, j - 1)] + a.m.mapf[L.at2i(i, j)]);
  R grad = (pistar(a, i, j, k) - pistar(a, i, j - 1, k)) / a.dy;
  R zyv = a.m.hy_v[L.at2i(i, j)] * ((R)1 - a.m.zeta_c[kk] / zt);
  if (zyv != (R)0) {
    R dzc2 = a.m.zeta_c[kk + 1] - a.m.zeta_c[kk - 1];
    R jv = (R)0.5 * (a.m.jac[L.at2i(i, j - 1)] + a.m.jac[L.at2i(i, j)]);
    R dpdz = (R)0.5 *
             ((pistar(a, i, j - 1, k + 1) - pistar(a, i, j - 1, k - 1)) +
              (pistar(a, i, j, k + 1) - pistar(a, i, j, k - 1))) /
             dzc2;
    grad -= zyv / jv * dpdz;
  }
  const int c = L.ati(i, j, k);
  return a.v_in[c] + a.dtau * (-Phys<R>::cp * thbv * mv * grad + a.tv[c]);
}

// u (v) at an interior face from the cell values beside it: theta_v and pi*
// at the face's two cells (kernels.cu:499-526).  pz(p) gives the pi* values
// the terrain term needs, p = {pi*(west/south, k+1), pi*(west/south, k-1),
// pi*(k+1), pi*(k-1)}, from global or from shared memory.
// The face's metric factors: the map factor averaged over the face's two
// cells and the terrain slope term (zero on flat ground).
template <typename R>
struct FaceMetric {
  R mf, slope;
};
template <typename R>
__device__ __forceinline__ FaceMetric<R> u_metric(const AcouArgs<R>& a, int c2, int kk) {
  return {(R)0.5 * (a.m.mapf[c2 - 1] + a.m.mapf[c2]), a.m.hx_u[c2] * a.co.fac_c[kk]};
}
template <typename R>
__device__ __forceinline__ FaceMetric<R> v_metric(const AcouArgs<R>& a, int c2, int kk) {
  const int sy = a.L.px;
  return {(R)0.5 * (a.m.mapf[c2 - sy] + a.m.mapf[c2]), a.m.hy_v[c2] * a.co.fac_c[kk]};
}

template <typename R, typename PZ>
__device__ __forceinline__ R u_interior_core_m(const AcouArgs<R>& a, int c2, int kk, FaceMetric<R> g, R tv0,
                                               R tvx, R ps0, R psx, R uin, R tin, PZ pz) {
  R thb_f = (R)0.5 * (tvx + tv0);
  R mf = g.mf;
  R grad = (ps0 - psx) * a.co.inv_dx;
  R slope = g.slope;
  if (slope != (R)0) {
    R jf = (R)0.5 * (a.m.jac[c2 - 1] + a.m.jac[c2]);
    R q[4];
    pz(q);
    R dpdz = (R)0.5 * ((q[0] - q[1]) + (q[2] - q[3])) * a.co.inv_dzc2[kk];
    grad -= slope / jf * dpdz;
  }
  return uin + a.dtau * (-Phys<R>::cp * thb_f * mf * grad + tin);
}

template <typename R, typename PZ>
__device__ __forceinline__ R v_interior_core_m(const AcouArgs<R>& a, int c2, int kk, FaceMetric<R> g, R tv0,
                                               R tvy, R ps0, R psy, R vin, R tin, PZ pz) {
  const int sy = a.L.px;
  R thb_f = (R)0.5 * (tvy + tv0);
  R mf = g.mf;
  R grad = (ps0 - psy) * a.co.inv_dy;
  R slope = g.slope;
  if (slope != (R)0) {
    R jf = (R)0.5 * (a.m.jac[c2 - sy] + a.m.jac[c2]);
    R q[4];
    pz(q);
    R dpdz = (R)0.5 * ((q[0] - q[1]) + (q[2] - q[3])) * a.co.inv_dzc2[kk];
    grad -= slope / jf * dpdz;
  }
  return vin + a.dtau * (-Phys<R>::cp * thb_f * mf * grad + tin);
}

template <typename R, typename PZ>
__device__ __forceinline__ R u_interior_core(const AcouArgs<R>& a, int c2, int kk, R tv0, R tvx, R ps0,
                                             R psx, R uin, R tin, PZ pz) {
  return u_interior_core_m(a, c2, kk, u_metric(a, c2, kk), tv0, tvx, ps0, psx, uin, tin, pz);
}

template <typename R, typename PZ>
__device__ __forceinline__ R v_interior_core(const AcouArgs<R>& a, int c2, int kk, R tv0, R tvy, R ps0,
                                             R psy, R vin, R tin, PZ pz) {
  return v_interior_core_m(a, c2, kk, v_metric(a, c2, kk), tv0, tvy, ps0, psy, vin, tin, pz);
}

template <typename R>
__device__ __forceinline__ R u_interior_from_m(const AcouArgs<R>& a, int c, int c2, int kk, FaceMetric<R> g,
                                               R tv0, R tvx, R ps0, R psx, R uin, R tin) {
  const int pl = a.L.planei();
  return u_interior_core_m(a, c2, kk, g, tv0, tvx, ps0, psx, uin, tin, [&](R* q) {
    q[0] = pistar_at(a, c - 1 + pl);
    q[1] = pistar_at(a, c - 1 - pl);
    q[2] = pistar_at(a, c + pl);
    q[3] = pistar_at(a, c - pl);
  });
}

template <typename R>
__device__ __forceinline__ R u_interior_from(const AcouArgs<R>& a, int c, int c2, int kk, R tv0, R tvx,
                                             R ps0, R psx, R uin, R tin) {
  return u_interior_from_m(a, c, c2, kk, u_metric(a, c2, kk), tv0, tvx, ps0, psx, uin, tin);
}

template <typename R>
__device__ __forceinline__ R u_interior_val(const AcouArgs<R>& a, int c, int c2, int kk, R tv0, R tvx,
                                            R ps0, R psx) {
  return u_interior_from(a, c, c2, kk, tv0, tvx, ps0, psx, a.u_in[c], a.tu[c]);
}

template <typename R>
__device__ __forceinline__ R v_interior_from_m(const AcouArgs<R>& a, int c, int c2, int kk, FaceMetric<R> g,
                                               R tv0, R tvy, R ps0, R psy, R vin, R tin) {
  const int sy = a.L.px, pl = a.L.planei();
  return v_interior_core_m(a, c2, kk, g, tv0, tvy, ps0, psy, vin, tin, [&](R* q) {
    q[0] = pistar_at(a, c - sy + pl);
    q[1] = pistar_at(a, c - sy - pl);
    q[2] = pistar_at(a, c + pl);
    q[3] = pistar_at(a, c - pl);
  });
}

template <typename R>
__device__ __forceinline__ R v_interior_from(const AcouArgs<R>& a, int c, int c2, int kk, R tv0, R tvy,
                                             R ps0, R psy, R vin, R tin) {
  return v_interior_from_m(a, c, c2, kk, v_metric(a, c2, kk), tv0, tvy, ps0, psy, vin, tin);
}

template <typename R>
__device__ __forceinline__ R v_interior_val(const AcouArgs<R>& a, int c, int c2, int kk, R tv0, R tvy,
                                            R ps0, R psy) {
  return v_interior_from(a, c, c2, kk, tv0, tvy, ps0, psy, a.v_in[c], a.tv[c]);
}

// Both faces of an interior point: the cell values at (i,j), (i-1,j) and
// (i,j-1) are loaded once for the u and the v face.
template <typename R>
__device__ __forceinline__ void uv_pair_interior(const AcouArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const int c = L.ati(i, j, k), c2 = L.at2i(i, j);
  const int sy = L.px;
  const R tv0 = theta_v_at(a, c), tvx = theta_v_at(a, c - 1), tvy = theta_v_at(a, c - sy);
  const R ps0 = pistar_at(a, c), psx = pistar_at(a, c - 1), psy = pistar_at(a, c - sy);
  a.u_out[c] = u_interior_val(a, c, c2, kk, tv0, tvx, ps0, psx);
  a.v_out[c] = v_interior_val(a, c, c2, kk, tv0, tvy, ps0, psy);
}

// u on an x face (0..nx) of a row j < ny that is not an interior point:
// radiation faces (open) or the periodic face u(nx) = u(0)
template <typename R>
__device__ __forceinline__ R u_face_edge(const AcouArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  const int kk = L.at1(k);
  const R cstar = a.p.cstar;
  if (a.p.bc_x_open) {
    if (i == 0) {  // kernels.cu:654-660
      R u0 = a.u_in[L.ati(0, j, k)];
      if (u0 >= (R)0) return a.b.ub[kk];
      R cb = u0 - cstar;
      return u0 - a.dtau * cb * (u_forward(a, 1, j, k) - u0) / a.dx;
    }
    if (i == L.nx) {  // kernels.cu:661-667
      R un = a.u_in[L.ati(L.nx, j, k)];
      if (un <= (R)0) return a.b.ub[kk];
      R cb = un + cstar;
      return un - a.dtau * cb * (un - u_forward(a, L.nx - 1, j, k)) / a.dx;
    }
    return u_forward(a, i, j, k);
  }
  return u_forward(a, i == L.nx ? 0 : i, j, k);  // periodic face u(nx) = u(0)
}

// v on a y face (0..ny) of a column i < nx that is not an interior point
template <typename R>
__device__ __forceinline__ R v_face_edge(const AcouArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  const R cstar = a.p.cstar;
  if (a.p.bc_y_open) {
    if (j == 0) {  // kernels.cu:674-680
      R v0 = a.v_in[L.ati(i, 0, k)];
      if (v0 >= (R)0) return 0;
      R cb = v0 - cstar;
      return v0 - a.dtau * cb * (v_forward(a, i, 1, k) - v0) / a.dy;
    }
    if (j == L.ny) {  // kernels.cu:681-687
      R vn = a.v_in[L.ati(i, L.ny, k)];
      if (vn <= (R)0) return 0;
      R cb = vn + cstar;
      return vn - a.dtau * cb * (vn - v_forward(a, i, L.ny - 1, k)) / a.dy;
    }
    return v_forward(a, i, j, k);
  }
  return v_forward(a, i, j == L.ny ? 0 : j, k);
}

// Launched as BX x BY x BZ blocks (kUvBx x kUvBy x kUvBz, or kUvShapes[1]
// where the grid has few rows).  Each thread computes theta_v and pi* of
// its own cell once and shares them through shared memory: an interior
// point takes its x (y) neighbour's values from the thread beside it in the
// block when there is one, instead of loading the neighbour's five fields.
constexpr int kUvBx = 16, kUvBy = 16, kUvBz = 1;
// the block shapes of launch_acoustic_uv: square tiles of faces, and tiles
// two rows high and four levels deep for slabs of a few rows (a 16-row block
// over the 5 face rows of a 4-row slab idles two thirds of its threads)
constexpr int kUvShapes[2][3] = {{kUvBx, kUvBy, kUvBz}, {32, 2, 4}};

// HB: the base theta of the block's level from its level table (DBase::lvl)
template <typename R, bool HB = false, int BX = kUvBx, int BY = kUvBy, int BZ = kUvBz>
__device__ __forceinline__ void uv_body(const AcouArgs<R>& a, int bx, int by, int bz) {
  __shared__ R s_tv[BZ][BY][BX], s_ps[BZ][BY][BX];
  const Layout& L = a.L;
  const int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
  const int i = bx * BX + tx;
  const int j = by * BY + ty;
  const int k = bz * BZ + tz;
  const bool has_cell = i < L.nx && j < L.ny && k < L.nz;
  const int c = has_cell ? L.ati(i, j, k) : 0;
  const int sy = L.px;
  // an interior point's own inputs and face metric, and its x (y)
  // neighbour's values when the neighbour is not in the block, are loaded
  // before the barrier so that their latency overlaps the shared values'
  // (the same values either way)
  const bool inner = uv_interior<R>(L, i, j, k);
  R tv0 = 0, ps0 = 0, uin = 0, tun = 0, vin = 0, tvn = 0, tvx = 0, psx = 0, tvy = 0, psy = 0;
  FaceMetric<R> gu{}, gv{};
  const int kk = L.at1(k);
  const int c2 = L.at2i(i, j);
  // theta_v of a cell of this level (the base theta from the table when HB)
  auto thv = [&](int cc) { return HB ? theta_v_with(a, cc, a.b.lvl[BL_THB * L.pz + kk]) : theta_v_at(a, cc); };
  if (has_cell) {
    tv0 = thv(c);
    ps0 = pistar_at(a, c);
  }
  if (inner) {
    uin = a.u_in[c];
    tun = a.tu[c];
    vin = a.v_in[c];
    tvn = a.tv[c];
    gu = u_metric(a, c2, kk);
    gv = v_metric(a, c2, kk);
    if (tx == 0) {
      tvx = thv(c - 1);
      psx = pistar_at(a, c - 1);
    }
    if (ty == 0) {
      tvy = thv(c - sy);
      psy = pistar_at(a, c - sy);
    }
  }
  s_tv[tz][ty][tx] = tv0;
  s_ps[tz][ty][tx] = ps0;
  __syncthreads();
  if (i > L.nx || j > L.ny || k >= L.nz) return;
  if (inner) {
    // the same values uv_pair_interior loads (kernels.cu:499-526)
    if (tx > 0) {
      tvx = s_tv[tz][ty][tx - 1];
      psx = s_ps[tz][ty][tx - 1];
    }
    if (ty > 0) {
      tvy = s_tv[tz][ty - 1][tx];
      psy = s_ps[tz][ty - 1][tx];
    }
    a.u_out[c] = u_interior_from_m(a, c, c2, kk, gu, tv0, tvx, ps0, psx, uin, tun);
    a.v_out[c] = v_interior_from_m(a, c, c2, kk, gv, tv0, tvy, ps0, psy, vin, tvn);
    return;
  }
  if (j < L.ny) a.u_out[L.ati(i, j, k)] = u_face_edge(a, i, j, k);
  if (i < L.nx) a.v_out[L.ati(i, j, k)] = v_face_edge(a, i, j, k);
}

// One face with uv_body's arithmetic (the fused substep kernel computes a
// tile's faces itself)
template <typename R>
__device__ __forceinline__ R u_face(const AcouArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  if (uv_interior<R>(L, i, j, k)) {
    const int c = L.ati(i, j, k);
    return u_interior_val(a, c, L.at2i(i, j), L.at1(k), theta_v_at(a, c), theta_v_at(a, c - 1),
                          pistar_at(a, c), pistar_at(a, c - 1));
  }
  return u_face_edge(a, i, j, k);
}

template <typename R>
__device__ __forceinline__ R v_face(const AcouArgs<R>& a, int i, int j, int k) {
  const Layout& L = a.L;
  if (uv_interior<R>(L, i, j, k)) {
    const int c = L.ati(i, j, k), sy = L.px;
    return v_interior_val(a, c, L.at2i(i, j), L.at1(k), theta_v_at(a, c), theta_v_at(a, c - sy),
                          pistar_at(a, c), pistar_at(a, c - sy));
  }
  return v_face_edge(a, i, j, k);
}

// FP32: 32 registers, eight CTAs per SM -- the kernel waits on loads, and the
// extra resident warps hide more of that than the few spills cost
template <typename R>
constexpr int kUvMinBlocks = sizeof(R) == 4 ? 8 : 1;

template <typename R, bool HB, int S>
__global__ void __launch_bounds__(256, kUvMinBlocks<R>) k_acoustic_uv(AcouArgs<R> a) {
  uv_body<R, HB, kUvShapes[S][0], kUvShapes[S][1], kUvShapes[S][2]>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename R>
__global__ void __launch_bounds__(256, kUvMinBlocks<R>) k_acoustic_uv_batch(Batch<AcouArgs<R>> b) {
  for_each_work(b, [](const AcouArgs<R>& a, int x, int y, int z) { uv_body(a, x, y, z); });
}

// ------------------------------------------ pipelined forward u, v
// Persistent CTAs over tiles of kUvpX x kUvpY x kUvpZ faces.  One producer
// warp streams each tile's boxes into a ring of kUvpStages shared-memory
// stages (cp.async.bulk.tensor, no multicast, this GPU's own fields): pi',
// pi'_prev, theta', theta_b and qv with one cell toward -x and -y and one
// level below and above, and u, tu, v, tv of the tile.  Consumer thread
// (tx, ty, tz) owns the u and v faces of cell (i0+tx, j0+ty, k0+tz):
//   * interior faces from shared memory with uv_body's expressions;
//   * the faces uv_body computes with the generic expressions (levels 0 and
//     nz-1, u at j = 0, v at i = 0) from shared memory when the column has no
//     terrain slope there (those expressions, with the same values);
//   * every other face -- lateral edges with the radiation or periodic
//     condition, sloped non-interior faces -- and u(nx), v(ny) by the
//     thread of the cell beside them, with uv_body's global-memory path.
// Every stage wait is bounded in wall time; on a timeout *err is set.
constexpr int kUvpStages = 3;
constexpr int kUvpThreads = kUvpX * kUvpY * kUvpZ;
constexpr uint64_t kUvpWaitNs = 4000000000ull;

template <typename R>
struct UvpLayout {
  size_t field[UV_N];
  size_t stage0, stage_bytes, total;
  uint32_t tx_bytes;
  __host__ __device__ UvpLayout(bool moist) {
    size_t o = 0;
    tx_bytes = 0;
    for (int f = 0; f < UV_N; ++f) {
      field[f] = 0;
      if (f == UV_QV && !moist) continue;
      int bx, by, bz;
      uv_pipe_box(f, &bx, &by, &bz);
      const size_t b = (size_t)bx * by * bz * sizeof(R);
      field[f] = o;
      o += (b + 127) / 128 * 128;
      tx_bytes += (uint32_t)b;
    }
    stage_bytes = o;
    stage0 = 128;
    total = stage0 + (size_t)kUvpStages * stage_bytes;
  }
};

template <typename R>
__global__ void __launch_bounds__(kUvpThreads + 32, 1)
    k_acoustic_uv_pipe(const __grid_constant__ PipeUvParams<R> p) {
  extern __shared__ __align__(128) unsigned char smem_uvp[];
  const AcouArgs<R>& a = p.a;
  const Layout& L = a.L;
  const bool moist = a.p.moisture != 0;
  const UvpLayout<R> lay(moist);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_uvp);
  uint64_t* empty = full + kUvpStages;
  const int tid = threadIdx.x;
  const int ntx = (L.nx + kUvpX - 1) / kUvpX, nty = (L.ny + kUvpY - 1) / kUvpY;
  const int ntz = (L.nz + kUvpZ - 1) / kUvpZ;
  const int ntiles = ntx * nty * ntz;
  if (tid == 0) {
    for (int s = 0; s < kUvpStages; ++s) {
      tma::mbar_init(&full[s], 1);
      tma::mbar_init(&empty[s], 1);
    }
    tma::fence_barrier_init();
  }
  __syncthreads();
  if (tid >= kUvpThreads) {
    // ------------------------------------------------------------ producer
    if (tid != kUvpThreads) return;
    int n = 0, armed[kUvpStages];
    for (int s = 0; s < kUvpStages; ++s) armed[s] = -1;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++n) {
      const int s = n % kUvpStages, use = n / kUvpStages;
      if (use > 0 && !tma::mbar_wait_for(&empty[s], (use - 1) & 1, kUvpWaitNs)) {
        atomicExch(p.err, 1u);
        break;
      }
      tma::mbar_arrive_expect_tx(&full[s], lay.tx_bytes);
      armed[s] = use;
      unsigned char* stg = smem_uvp + lay.stage0 + (size_t)s * lay.stage_bytes;
      const int i0 = (t % ntx) * kUvpX, j0 = (t / ntx % nty) * kUvpY, k0 = t / (ntx * nty) * kUvpZ;
      for (int f = 0; f < UV_N; ++f) {
        if (f == UV_QV && !moist) continue;
        const bool halo = f <= UV_QV;
        tma::load_3d(stg + lay.field[f], &p.map[f], i0 + kOX - (halo ? 4 : 0),
                     j0 + kOY - (halo ? 1 : 0), k0 + kOZ - (halo ? 1 : 0), &full[s]);
      }
    }
    for (int s = 0; s < kUvpStages; ++s)
      if (armed[s] >= 0) tma::mbar_wait_for(&full[s], armed[s] & 1, kUvpWaitNs);
    return;
  }
  // -------------------------------------------------------------- consumers
  const int tx = tid % kUvpX, ty = tid / kUvpX % kUvpY, tz = tid / (kUvpX * kUvpY);
  constexpr int HX = kUvpX + 4, HY = kUvpY + 1;
  int n = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++n) {
    const int s = n % kUvpStages, use = n / kUvpStages;
    const bool ok = tma::mbar_wait_for(&full[s], use & 1, kUvpWaitNs);
    if (tma::named_or(1, kUvpThreads, !ok)) {
      if (tid == 0) atomicExch(p.err, 1u);
      break;
    }
    const unsigned char* stg = smem_uvp + lay.stage0 + (size_t)s * lay.stage_bytes;
    auto fld = [&](int f) { return reinterpret_cast<const R*>(stg + lay.field[f]); };
    const R* sPI = fld(UV_PI);
    const R* sPP = fld(UV_PIP);
    const R* sTH = fld(UV_TH);
    const R* sTB = fld(UV_THB);
    const R* sQV = fld(UV_QV);
    const int i0 = (t % ntx) * kUvpX, j0 = (t / ntx % nty) * kUvpY, k0 = t / (ntx * nty) * kUvpZ;
    const int i = i0 + tx, j = j0 + ty, k = k0 + tz;
    // halo-box index of cell (i + dx, j + dy, k + dz)
    auto hix = [&](int dx, int dy, int dz) { return ((tz + 1 + dz) * HY + (ty + 1 + dy)) * HX + tx + 4 + dx; };
    auto thv = [&](int h) {  // theta_v_at from shared memory
      R tv = sTB[h] + sTH[h];
      if (moist) tv *= (R)1 + Phys<R>::eps61 * sQV[h];
      return tv;
    };
    auto pst = [&](int h) {  // pistar_at from shared memory
      R cur = sPI[h];
      return cur + a.p.acoustic_smdiv * (cur - sPP[h]);
    };
    R uo = 0, vo = 0;
    bool u_done = false, v_done = false;
    const bool cell = i < L.nx && j < L.ny && k < L.nz;
    if (cell) {
      const int kk = L.at1(k);
      const int c2 = L.at2i(i, j);
      const int t0 = (tz * kUvpY + ty) * kUvpX + tx;  // tile-box index
      const int h0 = hix(0, 0, 0);
      const R tv0 = thv(h0), ps0 = pst(h0);
      if (uv_interior<R>(L, i, j, k)) {
        const R tvx = thv(h0 - 1), psx = pst(h0 - 1);
        const R tvy = thv(h0 - HX), psy = pst(h0 - HX);
        uo = u_interior_core(a, c2, kk, tv0, tvx, ps0, psx, fld(UV_U)[t0], fld(UV_TU)[t0], [&](R* q) {
          q[0] = pst(hix(-1, 0, 1));
          q[1] = pst(hix(-1, 0, -1));
          q[2] = pst(hix(0, 0, 1));
          q[3] = pst(hix(0, 0, -1));
        });
        vo = v_interior_core(a, c2, kk, tv0, tvy, ps0, psy, fld(UV_V)[t0], fld(UV_TV)[t0], [&](R* q) {
          q[0] = pst(hix(0, -1, 1));
          q[1] = pst(hix(0, -1, -1));
          q[2] = pst(hix(0, 0, 1));
          q[3] = pst(hix(0, 0, -1));
        });
        u_done = v_done = true;
      } else {
        // uv_body's generic expressions (u_forward / v_forward) where they
        // read only this tile's cells and no terrain term
        if (i >= 1 && a.m.hx_u[c2] * ((R)1 - a.m.zeta_c[kk] / a.m.zt) == (R)0) {
          R thbu = (R)0.5 * (thv(h0 - 1) + tv0);
          R mu = (R)0.5 * (a.m.mapf[c2 - 1] + a.m.mapf[c2]);
          R grad = (ps0 - pst(h0 - 1)) / a.dx;
          uo = fld(UV_U)[t0] + a.dtau * (-Phys<R>::cp * thbu * mu * grad + fld(UV_TU)[t0]);
          u_done = true;
        }
        if (j >= 1 && a.m.hy_v[c2] * ((R)1 - a.m.zeta_c[kk] / a.m.zt) == (R)0) {
          R thbv = (R)0.5 * (thv(h0 - HX) + tv0);
          R mv = (R)0.5 * (a.m.mapf[c2 - L.px] + a.m.mapf[c2]);
          R grad = (ps0 - pst(h0 - HX)) / a.dy;
          vo = fld(UV_V)[t0] + a.dtau * (-Phys<R>::cp * thbv * mv * grad + fld(UV_TV)[t0]);
          v_done = true;
        }
      }
    }
    // every input of the tile has been read from shared memory: the producer
    // may refill the stage
    tma::named_sync(1, kUvpThreads);
    if (tid == 0) tma::mbar_arrive(&empty[s]);
    if (cell) {
      const int c = L.ati(i, j, k);
      a.u_out[c] = u_done ? uo : u_face_edge(a, i, j, k);
      a.v_out[c] = v_done ? vo : v_face_edge(a, i, j, k);
      if (i == L.nx - 1) a.u_out[L.ati(L.nx, j, k)] = u_face_edge(a, L.nx, j, k);
      if (j == L.ny - 1) a.v_out[L.ati(i, L.ny, k)] = v_face_edge(a, i, L.ny, k);
    }
  }
}

// ------------------------------------------------- implicit w - pi' columns
// Shared-memory column arrays, level-major so that the CX lanes of a level
// hit distinct banks: X(k, col) = base[k * CX + col].
template <typename R, int CX>
struct ColSmem {
  R *Av, *Sv, *P, *E, *A, *B, *C, *D, *Wn;
  __device__ ColSmem(R* s, int nz1) {
    size_t n = (size_t)nz1 * CX;
    Av = s; Sv = Av + n; P = Sv + n; E = P + n; A = E + n; B = A + n; C = B + n; D = C + n;
    Wn = D + n;
  }
};

// Where a column reads the new u, v: the substep's output fields, or the
// fused kernel's shared tiles.  u_at(k, 0|1): the column's west | east face
// at level k; v_at(k, 0|1): its south | north face.
template <typename R>
struct UvGlobal {
  const R* __restrict__ u;
  const R* __restrict__ v;
  int c0, pl, sy;
  __device__ R u_at(int k, int dx) const { return u[c0 + k * pl + dx]; }
  __device__ R v_at(int k, int dy) const { return v[c0 + k * pl + dy * sy]; }
};

// tiles: us[k * (CX + 1) + face], vs[(k * 2 + row) * CX + column]
template <typename R, int CX>
struct UvTile {
  const R* us;
  const R* vs;
  int tx;
  __device__ R u_at(int k, int dx) const { return us[k * (CX + 1) + tx + dx]; }
  __device__ R v_at(int k, int dy) const { return vs[(k * 2 + dy) * CX + tx]; }
};

template <typename R, int CX, int KL, typename UV>
__device__ __forceinline__ void column_core(const AcouArgs<R>& a, int bx, int by, R* smem, const UV& uv) {
  const Layout& L = a.L;
  const int nz = L.nz;
  ColSmem<R, CX> S(smem, nz + 1);
  const int tx = threadIdx.x;           // column within the CTA
  const int lane_k = threadIdx.y;       // level lane
  const int i = bx * CX + tx;
  const int j = by;
  const bool active = i < L.nx;
  const R dtau = a.dtau;
  const R c1 = ((R)1 + a.p.acoustic_beta) * (R)0.5;
  const R c2 = ((R)1 - a.p.acoustic_beta) * (R)0.5;
  const int c2d = L.at2i(active ? i : 0, j);
  const R J = a.m.jac[c2d], hxc = a.m.hx[c2d], hyc = a.m.hy[c2d], mc = a.m.mapf[c2d];
  const R invJ = (R)1 / J;
  const R mcx = mc * a.co.inv_dx, mcy = mc * a.co.inv_dy;
  const bool terrain = hxc != (R)0 || hyc != (R)0;
  const int sx = 1, sy = L.px, pl = L.planei();
  const int c0 = L.ati(active ? i : 0, j, 0);  // level k at c0 + k * pl
#define SM(X, k) S.X[(k) * CX + tx]

  // phase 1: Av = rho^w theta_v^w (0 at the rigid levels) and the explicit
  // terrain cross flux Sv with the new u, v (kernels.cu:552-568)
  if (active)
#pragma unroll 4
    for (int k = lane_k; k <= nz; k += KL) {
      R av = 0, sv = 0;
      if (k >= 1 && k < nz) {
        const int c = c0 + k * pl, cm = c - pl;
        av = a.co.aw[c];
        if (terrain) {
          R uw = (R)0.25 * (uv.u_at(k - 1, 0) + uv.u_at(k - 1, 1) + uv.u_at(k, 0) + uv.u_at(k, 1));
          R vw = (R)0.25 * (uv.v_at(k - 1, 0) + uv.v_at(k - 1, 1) + uv.v_at(k, 0) + uv.v_at(k, 1));
          sv = av * (uw * hxc + vw * hyc) * a.co.fac_w[L.at1(k)];
        }
      }
      SM(Av, k) = av;
      SM(Sv, k) = sv;
    }
  __syncthreads();
  // phase 2: explicit part of the pi' equation (kernels.cu:570-587)
  if (active)
#pragma unroll 4
    for (int k = lane_k; k < nz; k += KL) {
      const int kk = L.at1(k);
      const int c = c0 + k * pl;
      R Kt = a.co.kt3[c];
      R Dh = (a.co.rtjx[c + sx] * uv.u_at(k, 1) - a.co.rtjx[c] * uv.u_at(k, 0)) * mcx +
             (a.co.rtjy[c + sy] * uv.v_at(k, 1) - a.co.rtjy[c] * uv.v_at(k, 0)) * mcy;
      R idz = a.co.inv_dzc[kk];
      R wk = a.w_in[c], wkp = a.w_in[c + pl];
      R tpi = a.tpi ? a.tpi[c] : (R)0;
      SM(P, k) = a.pi_cur[c] + dtau * tpi -
                 dtau * Kt *
                     (Dh - (SM(Sv, k + 1) - SM(Sv, k)) * idz +
                      c2 * (SM(Av, k + 1) * wkp - SM(Av, k) * wk) * idz);
      SM(E, k) = dtau * Kt * c1 * idz;
    }
  __syncthreads();
  // phase 3: tridiagonal rows for w at inner levels (kernels.cu:589-611)
  if (active)
#pragma unroll 4
    for (int k = 1 + lane_k; k < nz; k += KL) {
      const int kk = L.at1(k);
      const int c = c0 + k * pl, cm = c - pl;
      const R iJdz = invJ * a.co.inv_dzw[kk];
      R thc = a.th_in[c], thm = a.th_in[cm];
      R thbw = a.b.thbw[c];
      R thvw = thbw + (R)0.5 * (thm + thc);
      if (a.p.moisture) thvw *= (R)1 + Phys<R>::eps61 * (R)0.5 * (a.qv[cm] + a.qv[c]);
      R G = dtau * Phys<R>::cp * thvw * c1 * iJdz;
      R Em = SM(E, k - 1), Ek = SM(E, k);
      SM(A, k) = -G * Em * SM(Av, k - 1);
      SM(B, k) = (R)1 + G * SM(Av, k) * (Ek + Em);
      SM(C, k) = -G * Ek * SM(Av, k + 1);
      R buoy = Phys<R>::grav * (R)0.5 * (thm + thc) / thbw;
      if (a.p.moisture) {
        R dqv = (R)0.5 * (a.qv[cm] + a.qv[c]) - (R)0.5 * (a.b.qvb[cm] + a.b.qvb[c]);
        R qcr = (R)0.5 * (a.qc[cm] + a.qc[c]) + (R)0.5 * (a.qr[cm] + a.qr[c]);
        buoy += Phys<R>::grav * (Phys<R>::eps61 * dqv - qcr);
      }
      R RHS = a.w_in[c] + dtau * (buoy + a.tw[c]) -
              dtau * Phys<R>::cp * thvw * c2 * (a.pi_cur[c] - a.pi_cur[cm]) * iJdz;
      SM(D, k) = RHS - G * (SM(P, k) - SM(P, k - 1));
    }
  __syncthreads();
  // phase 4: Thomas sweep, one lane per column (kernels.cu:612-634), one
  // reciprocal per level; the next level's row is read before this level's
  // results are stored
  if (active && lane_k == 0) {
    R cprev = 0, dprev = 0;
    R Ak = SM(A, 1), Bk = SM(B, 1), Ck = SM(C, 1), Dk = SM(D, 1);
    for (int k = 1; k < nz; ++k) {
      R An = 0, Bn = 1, Cn = 0, Dn = 0;
      if (k + 1 < nz) {
        An = SM(A, k + 1);
        Bn = SM(B, k + 1);
        Cn = SM(C, k + 1);
        Dn = SM(D, k + 1);
      }
      R r, ck, dk;
      if (k == 1) {
        r = (R)1 / Bk;
        ck = Ck * r;
        dk = Dk * r;
      } else {
        r = (R)1 / (Bk - Ak * cprev);
        ck = Ck * r;
        dk = (Dk - Ak * dprev) * r;
      }
      SM(C, k) = ck;
      SM(D, k) = dk;
      cprev = ck;
      dprev = dk;
      Ak = An, Bk = Bn, Ck = Cn, Dk = Dn;
    }
    SM(Wn, nz) = 0;
    R wabove = 0;
    for (int k = nz - 1; k >= 1; --k) {
      R wk = SM(D, k) - SM(C, k) * wabove;
      SM(Wn, k) = wk;
      wabove = wk;
    }
    R us = (R)0.5 * (uv.u_at(0, 0) + uv.u_at(0, 1));
    R vs = (R)0.5 * (uv.v_at(0, 0) + uv.v_at(0, 1));
    SM(Wn, 0) = us * hxc + vs * hyc;
  }
  __syncthreads();
  // phase 5: pi', theta', w (kernels.cu:636-644)
  if (active)
#pragma unroll 4
    for (int k = lane_k; k <= nz; k += KL) {
      const int c = c0 + k * pl;
      if (k < nz) {
        R wn = SM(Wn, k), wn1 = SM(Wn, k + 1);
        a.pi_next[c] = SM(P, k) - SM(E, k) * (SM(Av, k + 1) * wn1 - SM(Av, k) * wn);
        R wc = (R)0.5 * (wn + wn1);
        a.th_out[c] = a.th_in[c] + dtau * (a.tth[c] - wc * a.b.dthbdz[c]);
        a.w_out[c] = wn;
      } else {
        a.w_out[c] = 0;
      }
    }
#undef SM
}

template <typename R, int CX, int KL>
__device__ __forceinline__ void column_body(const AcouArgs<R>& a, int bx, int by) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Layout& L = a.L;
  const int i = bx * CX + (int)threadIdx.x;
  const UvGlobal<R> uv{a.u_out, a.v_out, L.ati(i < L.nx ? i : 0, by, 0), L.planei(), L.px};
  column_core<R, CX, KL>(a, bx, by, reinterpret_cast<R*>(smem_raw), uv);
}

template <typename R, int CX, int KL>
__global__ void __launch_bounds__(CX * KL) k_acoustic_column(AcouArgs<R> a) {
  column_body<R, CX, KL>(a, blockIdx.x, blockIdx.y);
}

// Column variant with contiguous level chunks: level lane l owns levels
// l*ch .. l*ch+ch-1 (ch = ceil((nz+1)/KL)) and runs phases 1-3 of column_core
// for them in registers without barriers, recomputing Av, Sv, P and E of the
// level below its chunk (its first row needs them) and Av, Sv of the level
// above; it loads phase 5's inputs before the sweep, so their latency
// overlaps it, and keeps theta' of its levels.  Only the rows A, B, C, D and
// the solution pass through shared memory (two barriers instead of four).
// The same expressions on the same values as column_core: bit-identical.
// KCH: the largest chunk (nz + 1 <= KL * KCH).
template <typename R, int CX, int KL, int KCH>
__global__ void __launch_bounds__(CX * KL) k_acoustic_column_chunked(AcouArgs<R> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Layout& L = a.L;
  const int nz = L.nz;
  const size_t n1 = (size_t)(nz + 1) * CX;
  R* sA = reinterpret_cast<R*>(smem_raw);
  R* sB = sA + n1;
  R* sC = sB + n1;
  R* sD = sC + n1;
  R* sW = sD + n1;
  const int tx = threadIdx.x, lane = threadIdx.y;
  const int i = blockIdx.x * CX + tx, j = blockIdx.y;
  const bool active = i < L.nx;
  const R dtau = a.dtau;
  const R c1 = ((R)1 + a.p.acoustic_beta) * (R)0.5;
  const R c2 = ((R)1 - a.p.acoustic_beta) * (R)0.5;
  const int c2d = L.at2i(active ? i : 0, j);
  const R J = a.m.jac[c2d], hxc = a.m.hx[c2d], hyc = a.m.hy[c2d], mc = a.m.mapf[c2d];
  const R invJ = (R)1 / J;
  const R mcx = mc * a.co.inv_dx, mcy = mc * a.co.inv_dy;
  const bool terrain = hxc != (R)0 || hyc != (R)0;
  const int sx = 1, sy = L.px, pl = L.planei();
  const int c0 = L.ati(active ? i : 0, j, 0);
  const R* __restrict__ u = a.u_out;
  const R* __restrict__ v = a.v_out;
  const int ch = (nz + KL) / KL;
  const int klo = lane * ch;  // first level of the chunk; s = k - klo + 1
  R av[KCH + 2], sv[KCH + 2], P[KCH + 1], E[KCH + 1], th[KCH + 1], tt[KCH + 1], db[KCH + 1];
#define SQ(X, k) X[(k) * CX + tx]
  if (active) {
    // phase 1 on levels klo-1 .. klo+ch
#pragma unroll
    for (int s = 0; s < KCH + 2; ++s) {
      const int k = klo - 1 + s;
      R avk = 0, svk = 0;
      if (s <= ch + 1 && k >= 1 && k < nz) {
        const int c = c0 + k * pl, cm = c - pl;
        avk = a.co.aw[c];
        if (terrain) {
          R uw = (R)0.25 * (u[cm] + u[cm + sx] + u[c] + u[c + sx]);
          R vw = (R)0.25 * (v[cm] + v[cm + sy] + v[c] + v[c + sy]);
          svk = avk * (uw * hxc + vw * hyc) * a.co.fac_w[L.at1(k)];
        }
      }
      av[s] = avk;
      sv[s] = svk;
    }
    // phase 2 on levels klo-1 .. klo+ch-1
#pragma unroll
    for (int s = 0; s < KCH + 1; ++s) {
      const int k = klo - 1 + s;
      R pk = 0, ek = 0;
      if (s <= ch && k >= 0 && k < nz) {
        const int kk = L.at1(k);
        const int c = c0 + k * pl;
        R Kt = a.co.kt3[c];
        R Dh = (a.co.rtjx[c + sx] * u[c + sx] - a.co.rtjx[c] * u[c]) * mcx +
               (a.co.rtjy[c + sy] * v[c + sy] - a.co.rtjy[c] * v[c]) * mcy;
        R idz = a.co.inv_dzc[kk];
        R wk = a.w_in[c], wkp = a.w_in[c + pl];
        R tpi = a.tpi ? a.tpi[c] : (R)0;
        pk = a.pi_cur[c] + dtau * tpi -
             dtau * Kt * (Dh - (sv[s + 1] - sv[s]) * idz + c2 * (av[s + 1] * wkp - av[s] * wk) * idz);
        ek = dtau * Kt * c1 * idz;
      }
      P[s] = pk;
      E[s] = ek;
    }
    // phase 3 on the inner levels of the chunk, and phase 5's inputs
#pragma unroll
    for (int s = 1; s < KCH + 1; ++s) {
      const int k = klo - 1 + s;
      if (s <= ch && k < nz) {
        const int c = c0 + k * pl;
        th[s] = a.th_in[c];
        tt[s] = a.tth[c];
        db[s] = a.b.dthbdz[c];
      }
      if (s <= ch && k >= 1 && k < nz) {
        const int kk = L.at1(k);
        const int c = c0 + k * pl, cm = c - pl;
        const R iJdz = invJ * a.co.inv_dzw[kk];
        R thc = th[s], thm = a.th_in[cm];
        R thbw = a.b.thbw[c];
        R thvw = thbw + (R)0.5 * (thm + thc);
        if (a.p.moisture) thvw *= (R)1 + Phys<R>::eps61 * (R)0.5 * (a.qv[cm] + a.qv[c]);
        R G = dtau * Phys<R>::cp * thvw * c1 * iJdz;
        R Em = E[s - 1], Ek = E[s];
        SQ(sA, k) = -G * Em * av[s - 1];
        SQ(sB, k) = (R)1 + G * av[s] * (Ek + Em);
        SQ(sC, k) = -G * Ek * av[s + 1];
        R buoy = Phys<R>::grav * (R)0.5 * (thm + thc) / thbw;
        if (a.p.moisture) {
          R dqv = (R)0.5 * (a.qv[cm] + a.qv[c]) - (R)0.5 * (a.b.qvb[cm] + a.b.qvb[c]);
          R qcr = (R)0.5 * (a.qc[cm] + a.qc[c]) + (R)0.5 * (a.qr[cm] + a.qr[c]);
          buoy += Phys<R>::grav * (Phys<R>::eps61 * dqv - qcr);
        }
        R RHS = a.w_in[c] + dtau * (buoy + a.tw[c]) -
                dtau * Phys<R>::cp * thvw * c2 * (a.pi_cur[c] - a.pi_cur[cm]) * iJdz;
        SQ(sD, k) = RHS - G * (P[s] - P[s - 1]);
      }
    }
  }
  __syncthreads();
  // phase 4: the Thomas sweep of column_core
  if (active && lane == 0) {
    R cprev = 0, dprev = 0;
    R Ak = SQ(sA, 1), Bk = SQ(sB, 1), Ck = SQ(sC, 1), Dk = SQ(sD, 1);
    for (int k = 1; k < nz; ++k) {
      R An = 0, Bn = 1, Cn = 0, Dn = 0;
      if (k + 1 < nz) {
        An = SQ(sA, k + 1);
        Bn = SQ(sB, k + 1);
        Cn = SQ(sC, k + 1);
        Dn = SQ(sD, k + 1);
      }
      R r, ck, dk;
      if (k == 1) {
        r = (R)1 / Bk;
        ck = Ck * r;
        dk = Dk * r;
      } else {
        r = (R)1 / (Bk - Ak * cprev);
        ck = Ck * r;
        dk = (Dk - Ak * dprev) * r;
      }
      SQ(sC, k) = ck;
      SQ(sD, k) = dk;
      cprev = ck;
      dprev = dk;
      Ak = An, Bk = Bn, Ck = Cn, Dk = Dn;
    }
    SQ(sW, nz) = 0;
    R wabove = 0;
    for (int k = nz - 1; k >= 1; --k) {
      R wk = SQ(sD, k) - SQ(sC, k) * wabove;
      SQ(sW, k) = wk;
      wabove = wk;
    }
    R us = (R)0.5 * (u[c0] + u[c0 + sx]);
    R vs = (R)0.5 * (v[c0] + v[c0 + sy]);
    SQ(sW, 0) = us * hxc + vs * hyc;
  }
  __syncthreads();
  // phase 5 on the chunk's levels
  if (active)
#pragma unroll
    for (int s = 1; s < KCH + 1; ++s) {
      const int k = klo - 1 + s;
      if (s > ch || k > nz) continue;
      const int c = c0 + k * pl;
      if (k < nz) {
        R wn = SQ(sW, k), wn1 = SQ(sW, k + 1);
        a.pi_next[c] = P[s] - E[s] * (av[s + 1] * wn1 - av[s] * wn);
        R wc = (R)0.5 * (wn + wn1);
        a.th_out[c] = th[s] + dtau * (tt[s] - wc * db[s]);
        a.w_out[c] = wn;
      } else {
        a.w_out[c] = 0;
      }
    }
#undef SQ
}

// Column variant with a parallel tridiagonal solve (pcr_solve,
// acou_pcr.cuh).  Level lane p owns the KCH levels klo = p KCH .. klo + KCH
// - 1 (in registers); the system is padded with identity rows (x = 0) at
// level 0, the lid and above it, which leaves the solution unchanged (the
// rows beside them couple to them with zero coefficients: A at level 1 and C
// at level nz - 1 multiply aw = 0), so every lane has exactly KCH rows and
// every lane works, instead of one lane sweeping the whole column while the
// others wait.  Phases 1-3 and 5 are the chunked kernel's expressions; the
// solution differs from the serial Thomas sweep by rounding only (another
// elimination order), so this variant is not bit-identical to the other
// column kernels.
template <typename R, int CX, int KL, int KCH>
__global__ void __launch_bounds__(CX * KL, sizeof(R) == 4 ? 2 : 1) k_acoustic_column_pcr(AcouArgs<R> a) {
  static_assert(KCH >= 2, "every lane needs an interior row");
  extern __shared__ __align__(16) unsigned char smem_raw[];  // pcr_solve's work area
  const Layout& L = a.L;
  const int nz = L.nz;
  const int tx = threadIdx.x, lane = threadIdx.y;
  const int i = blockIdx.x * CX + tx, j = blockIdx.y;
  const bool active = i < L.nx;
  const R dtau = a.dtau;
  const R c1 = ((R)1 + a.p.acoustic_beta) * (R)0.5;
  const R c2 = ((R)1 - a.p.acoustic_beta) * (R)0.5;
  const int c2d = L.at2i(active ? i : 0, j);
  const R J = a.m.jac[c2d], hxc = a.m.hx[c2d], hyc = a.m.hy[c2d], mc = a.m.mapf[c2d];
  const R invJ = (R)1 / J;
  const R mcx = mc * a.co.inv_dx, mcy = mc * a.co.inv_dy;
  const bool terrain = hxc != (R)0 || hyc != (R)0;
  const int sx = 1, sy = L.px, pl = L.planei();
  const int c0 = L.ati(active ? i : 0, j, 0);
  const R* __restrict__ u = a.u_out;
  const R* __restrict__ v = a.v_out;
  const int klo = lane * KCH;
  R av[KCH + 2], sv[KCH + 2], P[KCH + 1], E[KCH + 1], th[KCH + 1], tt[KCH + 1], db[KCH + 1];
  R Ar[KCH + 1], Br[KCH + 1], Cr[KCH + 1], Dr[KCH + 1];
  R wsurf = 0;
#pragma unroll
  for (int q = 0; q < KCH + 1; ++q) Ar[q] = 0, Br[q] = 1, Cr[q] = 0, Dr[q] = 0;
  if (active) {
    // phase 1 on levels klo-1 .. klo+KCH
#pragma unroll
    for (int q = 0; q < KCH + 2; ++q) {
      const int k = klo - 1 + q;
      R avk = 0, svk = 0;
      if (k >= 1 && k < nz) {
        const int c = c0 + k * pl, cm = c - pl;
        avk = a.co.aw[c];
        if (terrain) {
          R uw = (R)0.25 * (u[cm] + u[cm + sx] + u[c] + u[c + sx]);
          R vw = (R)0.25 * (v[cm] + v[cm + sy] + v[c] + v[c + sy]);
          svk = avk * (uw * hxc + vw * hyc) * a.co.fac_w[L.at1(k)];
        }
      }
      av[q] = avk;
      sv[q] = svk;
    }
    // phase 2 on levels klo-1 .. klo+KCH-1
#pragma unroll
    for (int q = 0; q < KCH + 1; ++q) {
      const int k = klo - 1 + q;
      R pk = 0, ek = 0;
      if (k >= 0 && k < nz) {
        const int kk = L.at1(k);
        const int c = c0 + k * pl;
        R Kt = a.co.kt3[c];
        R Dh = (a.co.rtjx[c + sx] * u[c + sx] - a.co.rtjx[c] * u[c]) * mcx +
               (a.co.rtjy[c + sy] * v[c + sy] - a.co.rtjy[c] * v[c]) * mcy;
        R idz = a.co.inv_dzc[kk];
        R wk = a.w_in[c], wkp = a.w_in[c + pl];
        R tpi = a.tpi ? a.tpi[c] : (R)0;
        pk = a.pi_cur[c] + dtau * tpi -
             dtau * Kt * (Dh - (sv[q + 1] - sv[q]) * idz + c2 * (av[q + 1] * wkp - av[q] * wk) * idz);
        ek = dtau * Kt * c1 * idz;
      }
      P[q] = pk;
      E[q] = ek;
    }
    // phase 3: rows of the inner levels, and phase 5's inputs
#pragma unroll
    for (int q = 1; q < KCH + 1; ++q) {
      const int k = klo - 1 + q;
      th[q] = tt[q] = db[q] = 0;
      if (k < nz) {
        const int c = c0 + k * pl;
        th[q] = a.th_in[c];
        tt[q] = a.tth[c];
        db[q] = a.b.dthbdz[c];
      }
      if (k >= 1 && k < nz) {
        const int kk = L.at1(k);
        const int c = c0 + k * pl, cm = c - pl;
        const R iJdz = invJ * a.co.inv_dzw[kk];
        R thc = th[q], thm = a.th_in[cm];
        R thbw = a.b.thbw[c];
        R thvw = thbw + (R)0.5 * (thm + thc);
        if (a.p.moisture) thvw *= (R)1 + Phys<R>::eps61 * (R)0.5 * (a.qv[cm] + a.qv[c]);
        R G = dtau * Phys<R>::cp * thvw * c1 * iJdz;
        R Em = E[q - 1], Ek = E[q];
        Ar[q] = -G * Em * av[q - 1];
        Br[q] = (R)1 + G * av[q] * (Ek + Em);
        Cr[q] = -G * Ek * av[q + 1];
        R buoy = Phys<R>::grav * (R)0.5 * (thm + thc) / thbw;
        if (a.p.moisture) {
          R dqv = (R)0.5 * (a.qv[cm] + a.qv[c]) - (R)0.5 * (a.b.qvb[cm] + a.b.qvb[c]);
          R qcr = (R)0.5 * (a.qc[cm] + a.qc[c]) + (R)0.5 * (a.qr[cm] + a.qr[c]);
          buoy += Phys<R>::grav * (Phys<R>::eps61 * dqv - qcr);
        }
        R RHS = a.w_in[c] + dtau * (buoy + a.tw[c]) -
                dtau * Phys<R>::cp * thvw * c2 * (a.pi_cur[c] - a.pi_cur[cm]) * iJdz;
        Dr[q] = RHS - G * (P[q] - P[q - 1]);
      }
    }
    if (lane == 0) {  // diagnostic surface w from the new u, v
      R us = (R)0.5 * (u[c0] + u[c0 + sx]);
      R vs = (R)0.5 * (v[c0] + v[c0 + sy]);
      wsurf = us * hxc + vs * hyc;
    }
  }
  PcrLane<R, KCH> sol;
  pcr_solve<R, CX, KL, KCH>(Ar, Br, Cr, Dr, reinterpret_cast<R*>(smem_raw), tx, lane,
                            [] { __syncthreads(); }, sol);
  const R y = sol.y, yprev = sol.yprev, ynext = sol.ynext, gn = sol.gn, an = sol.an, bn = sol.bn;
  const R(&Gx)[KCH + 1] = sol.Gx;
  const R(&Ax)[KCH + 1] = sol.Ax;
  const R(&Bx)[KCH + 1] = sol.Bx;
  // ---- phase 5: pi', theta', w of the lane's levels
  if (active) {
    R wl[KCH + 2];  // w at the lane's levels and the level above them
#pragma unroll
    for (int q = 1; q < KCH; ++q) wl[q] = Gx[q] + Ax[q] * yprev + Bx[q] * y;
    wl[KCH] = y;
    wl[KCH + 1] = gn + an * y + bn * ynext;
    if (lane == 0) wl[1] = wsurf;  // level 0: the diagnostic surface w
#pragma unroll
    for (int q = 1; q < KCH + 1; ++q) {
      const int k = klo - 1 + q;
      if (k > nz) continue;
      const int c = c0 + k * pl;
      if (k == nz) {
        a.w_out[c] = 0;
        continue;
      }
      const R wn = wl[q], wn1 = k + 1 >= nz ? (R)0 : wl[q + 1];
      a.pi_next[c] = P[q] - E[q] * (av[q + 1] * wn1 - av[q] * wn);
      R wc = (R)0.5 * (wn + wn1);
      a.th_out[c] = th[q] + dtau * (tt[q] - wc * db[q]);
      a.w_out[c] = wn;
    }
  }
}

// The whole substep in one launch: a CTA first computes the u faces
// i0..i0+CX of its row and the v faces of rows j and j+1 of its columns with
// uv_body's arithmetic into shared tiles (storing the faces it owns: u faces
// of its columns and u(nx), v faces of row j and v(ny)), then solves its
// columns from the tiles.  A face beside the tile is computed by both CTAs
// that need it.  Every CTA reads theta' and pi' of neighbouring columns that
// other CTAs update in the same launch, so the integrator gives this kernel
// distinct theta'_in / theta'_out buffers (pi' and u, v already are).
template <typename R, int CX, int KL>
__global__ void __launch_bounds__(CX * KL) k_acoustic_fused(AcouArgs<R> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Layout& L = a.L;
  const int nz = L.nz;
  R* cols = reinterpret_cast<R*>(smem_raw);
  R* us = cols + (size_t)9 * (nz + 1) * CX;
  R* vs = us + (size_t)nz * (CX + 1);
  const int i0 = blockIdx.x * CX, j = blockIdx.y;
  const int tid = threadIdx.y * CX + threadIdx.x;
  const int nu = (CX + 1) * nz, nv = 2 * CX * nz;
  for (int e = tid; e < nu + nv; e += CX * KL) {
    if (e < nu) {
      const int f = e % (CX + 1), k = e / (CX + 1), i = i0 + f;
      if (i <= L.nx) {
        const R val = u_face(a, i, j, k);
        us[e] = val;
        if (f < CX || i == L.nx) a.u_out[L.ati(i, j, k)] = val;
      }
    } else {
      const int e2 = e - nu, col = e2 % CX, row = (e2 / CX) & 1, k = e2 / (2 * CX);
      const int i = i0 + col, jj = j + row;
      if (i < L.nx) {
        const R val = v_face(a, i, jj, k);
        vs[e2] = val;
        if (row == 0 || jj == L.ny) a.v_out[L.ati(i, jj, k)] = val;
      }
    }
  }
  __syncthreads();
  column_core<R, CX, KL>(a, blockIdx.x, j, cols, UvTile<R, CX>{us, vs, (int)threadIdx.x});
}
// the shared column arrays are reused by the next work item only after the
// barrier that opens it
template <typename R, int CX, int KL>
__global__ void __launch_bounds__(CX * KL) k_acoustic_column_batch(Batch<AcouArgs<R>> b) {
  for_each_work(b, [](const AcouArgs<R>& a, int x, int y, int) { column_body<R, CX, KL>(a, x, y); });
}

// --------------------------------------------- TMA-staged column variant
constexpr int kTmaKL = 32;

// shared-memory layout: the barrier, then each field's box (levels -1..nz,
// x fastest), then the nine column work arrays
template <typename R>
struct TmaColLayout {
  size_t field[TC_N];
  size_t work, total;
  __host__ __device__ TmaColLayout(int nz) {
    const int nzs = nz + 2;
    size_t o = 128;  // the mbarrier lives in the first 8 bytes
    for (int f = 0; f < TC_N; ++f) {
      int bx, by;
      tma_col_box(f, &bx, &by);
      field[f] = o;
      o += ((size_t)bx * by * nzs * sizeof(R) + 127) / 128 * 128;
    }
    work = o;
    total = o + (size_t)9 * (nz + 1) * kTmaCX * sizeof(R);
  }
};

template <typename R>
__global__ void __launch_bounds__(kTmaCX * kTmaKL)
    k_acoustic_column_tma(const __grid_constant__ TmaColParams<R> p) {
  extern __shared__ __align__(128) unsigned char smem_tma[];
  const AcouArgs<R>& a = p.a;
  const Layout& L = a.L;
  const int nz = L.nz, nzs = nz + 2;
  const int tx = threadIdx.x, lane_k = threadIdx.y;
  const int tid = tx + kTmaCX * lane_k;
  const int i0 = blockIdx.x * kTmaCX, i = i0 + tx, j = blockIdx.y;
  const bool active = i < L.nx;
  const bool moist = a.p.moisture != 0;
  const TmaColLayout<R> lay(nz);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_tma);
  auto fld = [&](int f) { return reinterpret_cast<R*>(smem_tma + lay.field[f]); };

  if (tid == 0) {
    tma::mbar_init(bar, 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t bytes = 0;
    for (int f = 0; f < TC_N; ++f) {
      if (f == TC_TPI && !p.has_tpi) continue;
      if (f >= TC_QV && !moist) continue;
      int bx, by;
      tma_col_box(f, &bx, &by);
      bytes += (uint32_t)((size_t)bx * by * nzs * sizeof(R));
    }
    tma::mbar_arrive_expect_tx(bar, bytes);
    const int x = i0 + kOX, y = j + kOY, z = kOZ - 1;
    for (int f = 0; f < TC_N; ++f) {
      if (f == TC_TPI && !p.has_tpi) continue;
      if (f >= TC_QV && !moist) continue;
      tma::load_3d(fld(f), &p.map[f], x, y, z, bar);
    }
  }
  // one thread polls the barrier (bounded) while the others sleep in the CTA
  // barrier; on a timeout every thread leaves after the copies drain
  bool ok = true;
  if (tid == 0) ok = tma::mbar_wait(bar, 0, 1u << 24);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicExch(p.err, 1u);
      tma::mbar_wait(bar, 0, 1u << 22);
    }
    return;
  }

  const R* sU = fld(TC_U);
  const R* sRX = fld(TC_RTJX);
  const R* sV = fld(TC_V);
  const R* sRY = fld(TC_RTJY);
#define UF(k, d) sU[((k) + 1) * (kTmaCX + 4) + tx + (d)]
#define RXF(k, d) sRX[((k) + 1) * (kTmaCX + 4) + tx + (d)]
#define VF(k, r) sV[(((k) + 1) * 2 + (r)) * kTmaCX + tx]
#define RYF(k, r) sRY[(((k) + 1) * 2 + (r)) * kTmaCX + tx]
#define CF(f, k) fld(f)[((k) + 1) * kTmaCX + tx]
  ColSmem<R, kTmaCX> S(reinterpret_cast<R*>(smem_tma + lay.work), nz + 1);
#define SM(X, k) S.X[(k) * kTmaCX + tx]
  const R dtau = a.dtau;
  const R c1 = ((R)1 + a.p.acoustic_beta) * (R)0.5;
  const R c2 = ((R)1 - a.p.acoustic_beta) * (R)0.5;
  const int c2d = L.at2i(active ? i : 0, j);
  const R J = a.m.jac[c2d], hxc = a.m.hx[c2d], hyc = a.m.hy[c2d], mc = a.m.mapf[c2d];
  const R invJ = (R)1 / J;
  const R mcx = mc * a.co.inv_dx, mcy = mc * a.co.inv_dy;
  const bool terrain = hxc != (R)0 || hyc != (R)0;

  // phase 1: Av and the terrain cross flux Sv (kernels.cu:552-568)
  if (active)
    for (int k = lane_k; k <= nz; k += kTmaKL) {
      R av = 0, sv = 0;
      if (k >= 1 && k < nz) {
        av = CF(TC_AW, k);
        if (terrain) {
          R uw = (R)0.25 * (UF(k - 1, 0) + UF(k - 1, 1) + UF(k, 0) + UF(k, 1));
          R vw = (R)0.25 * (VF(k - 1, 0) + VF(k - 1, 1) + VF(k, 0) + VF(k, 1));
          sv = av * (uw * hxc + vw * hyc) * a.co.fac_w[L.at1(k)];
        }
      }
      SM(Av, k) = av;
      SM(Sv, k) = sv;
    }
  __syncthreads();
  // phase 2: explicit pi' (kernels.cu:570-587)
  if (active)
    for (int k = lane_k; k < nz; k += kTmaKL) {
      R Kt = CF(TC_KT3, k);
      R Dh = (RXF(k, 1) * UF(k, 1) - RXF(k, 0) * UF(k, 0)) * mcx +
             (RYF(k, 1) * VF(k, 1) - RYF(k, 0) * VF(k, 0)) * mcy;
      R idz = a.co.inv_dzc[L.at1(k)];
      R wk = CF(TC_W, k), wkp = CF(TC_W, k + 1);
      R tpi = p.has_tpi ? CF(TC_TPI, k) : (R)0;
      SM(P, k) = CF(TC_PI, k) + dtau * tpi -
                 dtau * Kt *
                     (Dh - (SM(Sv, k + 1) - SM(Sv, k)) * idz +
                      c2 * (SM(Av, k + 1) * wkp - SM(Av, k) * wk) * idz);
      SM(E, k) = dtau * Kt * c1 * idz;
    }
  __syncthreads();
  // phase 3: tridiagonal rows (kernels.cu:589-611)
  if (active)
    for (int k = 1 + lane_k; k < nz; k += kTmaKL) {
      const R iJdz = invJ * a.co.inv_dzw[L.at1(k)];
      R thc = CF(TC_TH, k), thm = CF(TC_TH, k - 1);
      R thbw = CF(TC_THBW, k);
      R thvw = thbw + (R)0.5 * (thm + thc);
      if (moist) thvw *= (R)1 + Phys<R>::eps61 * (R)0.5 * (CF(TC_QV, k - 1) + CF(TC_QV, k));
      R G = dtau * Phys<R>::cp * thvw * c1 * iJdz;
      R Em = SM(E, k - 1), Ek = SM(E, k);
      SM(A, k) = -G * Em * SM(Av, k - 1);
      SM(B, k) = (R)1 + G * SM(Av, k) * (Ek + Em);
      SM(C, k) = -G * Ek * SM(Av, k + 1);
      R buoy = Phys<R>::grav * (R)0.5 * (thm + thc) / thbw;
      if (moist) {
        R dqv = (R)0.5 * (CF(TC_QV, k - 1) + CF(TC_QV, k)) -
                (R)0.5 * (CF(TC_QVB, k - 1) + CF(TC_QVB, k));
        R qcr = (R)0.5 * (CF(TC_QC, k - 1) + CF(TC_QC, k)) + (R)0.5 * (CF(TC_QR, k - 1) + CF(TC_QR, k));
        buoy += Phys<R>::grav * (Phys<R>::eps61 * dqv - qcr);
      }
      R RHS = CF(TC_W, k) + dtau * (buoy + CF(TC_TW, k)) -
              dtau * Phys<R>::cp * thvw * c2 * (CF(TC_PI, k) - CF(TC_PI, k - 1)) * iJdz;
      SM(D, k) = RHS - G * (SM(P, k) - SM(P, k - 1));
    }
  __syncthreads();
  // phase 4: Thomas sweep, one lane per column (kernels.cu:612-634)
  if (active && lane_k == 0) {
    R cprev = 0, dprev = 0;
    R Ak = SM(A, 1), Bk = SM(B, 1), Ck = SM(C, 1), Dk = SM(D, 1);
    for (int k = 1; k < nz; ++k) {
      R An = 0, Bn = 1, Cn = 0, Dn = 0;
      if (k + 1 < nz) {
        An = SM(A, k + 1);
        Bn = SM(B, k + 1);
        Cn = SM(C, k + 1);
        Dn = SM(D, k + 1);
      }
      R r, ck, dk;
      if (k == 1) {
        r = (R)1 / Bk;
        ck = Ck * r;
        dk = Dk * r;
      } else {
        r = (R)1 / (Bk - Ak * cprev);
        ck = Ck * r;
        dk = (Dk - Ak * dprev) * r;
      }
      SM(C, k) = ck;
      SM(D, k) = dk;
      cprev = ck;
      dprev = dk;
      Ak = An, Bk = Bn, Ck = Cn, Dk = Dn;
    }
    SM(Wn, nz) = 0;
    R wabove = 0;
    for (int k = nz - 1; k >= 1; --k) {
      R wk = SM(D, k) - SM(C, k) * wabove;
      SM(Wn, k) = wk;
      wabove = wk;
    }
    R us = (R)0.5 * (UF(0, 0) + UF(0, 1));
    R vs = (R)0.5 * (VF(0, 0) + VF(0, 1));
    SM(Wn, 0) = us * hxc + vs * hyc;
  }
  __syncthreads();
  // phase 5: pi', theta', w (kernels.cu:636-644)
  if (active) {
    const int c0 = L.ati(i, j, 0), pl = L.planei();
    for (int k = lane_k; k <= nz; k += kTmaKL) {
      const int c = c0 + k * pl;
      if (k < nz) {
        R wn = SM(Wn, k), wn1 = SM(Wn, k + 1);
        a.pi_next[c] = SM(P, k) - SM(E, k) * (SM(Av, k + 1) * wn1 - SM(Av, k) * wn);
        R wc = (R)0.5 * (wn + wn1);
        a.th_out[c] = CF(TC_TH, k) + dtau * (CF(TC_TTH, k) - wc * CF(TC_DTHB, k));
        a.w_out[c] = wn;
      } else {
        a.w_out[c] = 0;
      }
    }
  }
#undef UF
#undef RXF
#undef VF
#undef RYF
#undef CF
#undef SM
}

template <typename R>
size_t acoustic_column_tma_smem(int nz) {
  if (nz + 2 > 256) return 0;  // a box extent is at most 256 elements
  const size_t t = TmaColLayout<R>(nz).total;
  return t <= 227 * 1024 ? t : 0;
}

template <typename R>
int prepare_acoustic_column_tma(int nz) {
  const size_t sm = acoustic_column_tma_smem<R>(nz);
  if (!sm) return 2;
  return raise_smem_limit(k_acoustic_column_tma<R>, sm) == cudaSuccess
             ? 0
             : 1;
}

template <typename R>
int launch_acoustic_column_tma(const TmaColParams<R>& p, cudaStream_t st) {
  const size_t sm = acoustic_column_tma_smem<R>(p.a.L.nz);
  if (!sm) return 2;
  dim3 grd((p.a.L.nx + kTmaCX - 1) / kTmaCX, p.a.L.ny), blk(kTmaCX, kTmaKL);
  k_acoustic_column_tma<R><<<grd, blk, sm, st>>>(p);
  return 0;
}

// ------------------------------------------------------------ host launch
template <typename R>
void launch_acoustic_coef(const Layout& L, const DBase<R>& b, const DMetric<R>& m, R* scratch,
                          R* rtjx, R* rtjy, R* kt3, R* aw, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  dim3 grd((L.px + 31) / 32, (L.py + 3) / 4, (L.pz + 1) / 2);
  k_coef_centre<R><<<grd, blk, 0, st>>>(L, b, m, scratch, kt3, aw);
  k_coef_face<R><<<grd, blk, 0, st>>>(L, scratch, rtjx, rtjy);
}

template <typename R>
dim3 grid_uv(const Layout& L) {
  return dim3((L.nx + 1 + 31) / 32, (L.ny + 1 + 3) / 4, (L.nz + 1) / 2);
}

// the forward u, v kernel's grid: faces 0..nx x 0..ny in kUvBx x kUvBy x
// kUvBz blocks
template <typename R>
dim3 grid_uv_fwd(const Layout& L) {
  return dim3((L.nx + 1 + kUvBx - 1) / kUvBx, (L.ny + 1 + kUvBy - 1) / kUvBy, (L.nz + kUvBz - 1) / kUvBz);
}

template <typename R, int S>
static void launch_uv_shape(const AcouArgs<R>& a, cudaStream_t st) {
  constexpr int BX = kUvShapes[S][0], BY = kUvShapes[S][1], BZ = kUvShapes[S][2];
  const Layout& L = a.L;
  const dim3 g((L.nx + 1 + BX - 1) / BX, (L.ny + 1 + BY - 1) / BY, (L.nz + BZ - 1) / BZ), t(BX, BY, BZ);
  if (a.b.lvl) k_acoustic_uv<R, true, S><<<g, t, 0, st>>>(a);
  else k_acoustic_uv<R, false, S><<<g, t, 0, st>>>(a);
}

template <typename R>
void launch_acoustic_uv(const AcouArgs<R>& a, cudaStream_t st, int shape) {
  if (shape == 1) launch_uv_shape<R, 1>(a, st);
  else launch_uv_shape<R, 0>(a, st);
}

template <typename R>
void batch_uv(const Batch<AcouArgs<R>>& b, int nblocks, cudaStream_t st) {
  k_acoustic_uv_batch<R><<<nblocks, dim3(kUvBx, kUvBy, kUvBz), 0, st>>>(b);
}

template <typename R>
size_t column_smem(int nz, int cx) {
  return (size_t)9 * (nz + 1) * cx * sizeof(R);
}

template <typename R, int CX, int KL>
static cudaError_t column_attr(size_t sm) {
  cudaError_t e = raise_smem_limit(k_acoustic_column<R, CX, KL>, sm);
  if (e != cudaSuccess) return e;
  return raise_smem_limit(k_acoustic_column_batch<R, CX, KL>, sm);
}

cudaError_t raise_smem_limit(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> limits;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_pair(func, dev);
  auto it = limits.find(key);
  if (it != limits.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) limits[key] = bytes;
  return e;
}

// Tile shapes (columns x level lanes) the autotuner chooses from.
static const int kColumnShapes[][2] = {{32, 8}, {16, 16}, {8, 32}, {32, 4}, {16, 8}, {8, 16}};
constexpr int kNumColumnShapes = 6;

int acoustic_column_shapes() { return kNumColumnShapes; }

template <typename R>
static bool column_fits(int nz, int shape) {
  return column_smem<R>(nz, kColumnShapes[shape][0]) <= 200 * 1024;
}

template <typename R>
bool acoustic_column_fits(int nz, int shape) {
  return shape >= 0 && shape < kNumColumnShapes && column_fits<R>(nz, shape);
}

// Sets the dynamic shared-memory limit of every tile shape that fits, once,
// outside any stream capture.
template <typename R>
int prepare_acoustic_column(int nz) {
  bool any = false;
  for (int s = 0; s < kNumColumnShapes; ++s) {
    if (!column_fits<R>(nz, s)) continue;
    any = true;
    size_t sm = column_smem<R>(nz, kColumnShapes[s][0]);
    cudaError_t e;
    switch (s) {
      case 0: e = column_attr<R, 32, 8>(sm); break;
      case 1: e = column_attr<R, 16, 16>(sm); break;
      case 2: e = column_attr<R, 8, 32>(sm); break;
      case 3: e = column_attr<R, 32, 4>(sm); break;
      case 4: e = column_attr<R, 16, 8>(sm); break;
      default: e = column_attr<R, 8, 16>(sm); break;
    }
    if (e != cudaSuccess) return 1;
  }
  return any ? 0 : 2;
}

// shape: index into the tile shapes; out of range or too large for the
// column picks the first shape that fits.  Returns 0 ok, 2 column too deep.
template <typename R>
int launch_acoustic_column(const AcouArgs<R>& a, int shape, cudaStream_t st) {
  const int nz = a.L.nz;
  if (shape < 0 || shape >= kNumColumnShapes || !column_fits<R>(nz, shape)) {
    shape = -1;
    for (int s = 0; s < kNumColumnShapes && shape < 0; ++s)
      if (column_fits<R>(nz, s)) shape = s;
    if (shape < 0) return 2;
  }
  const int cx = kColumnShapes[shape][0], kl = kColumnShapes[shape][1];
  const size_t sm = column_smem<R>(nz, cx);
  const dim3 grd = grid_column<R>(a.L, shape), blk(cx, kl);
  switch (shape) {
    case 0: k_acoustic_column<R, 32, 8><<<grd, blk, sm, st>>>(a); break;
    case 1: k_acoustic_column<R, 16, 16><<<grd, blk, sm, st>>>(a); break;
    case 2: k_acoustic_column<R, 8, 32><<<grd, blk, sm, st>>>(a); break;
    case 3: k_acoustic_column<R, 32, 4><<<grd, blk, sm, st>>>(a); break;
    case 4: k_acoustic_column<R, 16, 8><<<grd, blk, sm, st>>>(a); break;
    default: k_acoustic_column<R, 8, 16><<<grd, blk, sm, st>>>(a); break;
  }
  return 0;
}

template <typename R>
dim3 grid_column(const Layout& L, int shape) {
  const int cx = kColumnShapes[shape][0];
  return dim3((L.nx + cx - 1) / cx, L.ny, 1);
}

// Batched columns: the shared arrays are sized for the deepest member (nz_max)
// and the tile shape must fit it (prepare_acoustic_column<R>(nz_max) done).
template <typename R>
int batch_column(const Batch<AcouArgs<R>>& b, int shape, int nz_max, int nblocks, cudaStream_t st) {
  if (shape < 0 || shape >= kNumColumnShapes || !column_fits<R>(nz_max, shape)) return 2;
  const int cx = kColumnShapes[shape][0], kl = kColumnShapes[shape][1];
  const size_t sm = column_smem<R>(nz_max, cx);
  const dim3 blk(cx, kl);
  switch (shape) {
    case 0: k_acoustic_column_batch<R, 32, 8><<<nblocks, blk, sm, st>>>(b); break;
    case 1: k_acoustic_column_batch<R, 16, 16><<<nblocks, blk, sm, st>>>(b); break;
    case 2: k_acoustic_column_batch<R, 8, 32><<<nblocks, blk, sm, st>>>(b); break;
    case 3: k_acoustic_column_batch<R, 32, 4><<<nblocks, blk, sm, st>>>(b); break;
    case 4: k_acoustic_column_batch<R, 16, 8><<<nblocks, blk, sm, st>>>(b); break;
    default: k_acoustic_column_batch<R, 8, 16><<<nblocks, blk, sm, st>>>(b); break;
  }
  return 0;
}

// Tile shapes of the fused substep kernel (indices into kColumnShapes)
static const int kFusedShapes[] = {0, 4, 1};
constexpr int kNumFusedShapes = 3;

int acoustic_fused_shapes() { return kNumFusedShapes; }

template <typename R>
size_t fused_smem(int nz, int cx) {
  return column_smem<R>(nz, cx) + ((size_t)nz * (cx + 1) + (size_t)2 * cx * nz) * sizeof(R);
}

template <typename R>
static bool fused_fits(int nz, int f) {
  return f >= 0 && f < kNumFusedShapes && fused_smem<R>(nz, kColumnShapes[kFusedShapes[f]][0]) <= 200 * 1024;
}

template <typename R>
bool acoustic_fused_fits(int nz, int f) {
  return fused_fits<R>(nz, f);
}

template <typename R>
int prepare_acoustic_fused(int nz) {
  for (int f = 0; f < kNumFusedShapes; ++f) {
    if (!fused_fits<R>(nz, f)) continue;
    const size_t sm = fused_smem<R>(nz, kColumnShapes[kFusedShapes[f]][0]);
    cudaError_t e;
    switch (kFusedShapes[f]) {
      case 0: e = raise_smem_limit(k_acoustic_fused<R, 32, 8>, sm); break;
      case 4: e = raise_smem_limit(k_acoustic_fused<R, 16, 8>, sm); break;
      default: e = raise_smem_limit(k_acoustic_fused<R, 16, 16>, sm); break;
    }
    if (e != cudaSuccess) return 1;
  }
  return 0;
}

// f: index into the fused tile shapes.  Returns 0 ok, 2 the column does not fit.
template <typename R>
int launch_acoustic_fused(const AcouArgs<R>& a, int f, cudaStream_t st) {
  const int nz = a.L.nz;
  if (!fused_fits<R>(nz, f)) return 2;
  const int shape = kFusedShapes[f];
  const int cx = kColumnShapes[shape][0], kl = kColumnShapes[shape][1];
  const size_t sm = fused_smem<R>(nz, cx);
  const dim3 grd((a.L.nx + cx - 1) / cx, a.L.ny, 1), blk(cx, kl);
  switch (shape) {
    case 0: k_acoustic_fused<R, 32, 8><<<grd, blk, sm, st>>>(a); break;
    case 4: k_acoustic_fused<R, 16, 8><<<grd, blk, sm, st>>>(a); break;
    default: k_acoustic_fused<R, 16, 16><<<grd, blk, sm, st>>>(a); break;
  }
  return 0;
}

// Shapes of the chunked column kernel: columns, level lanes, largest chunk
static const int kChunkShapes[][3] = {{32, 8, 8}, {16, 16, 4}, {32, 16, 4}};
constexpr int kNumChunkShapes = 3;

int acoustic_chunked_shapes() { return kNumChunkShapes; }

template <typename R>
size_t chunked_smem(int nz, int cx) {
  return (size_t)5 * (nz + 1) * cx * sizeof(R);
}

template <typename R>
bool acoustic_chunked_fits(int nz, int f) {
  return f >= 0 && f < kNumChunkShapes && nz + 1 <= kChunkShapes[f][1] * kChunkShapes[f][2] &&
         chunked_smem<R>(nz, kChunkShapes[f][0]) <= 48 * 1024;
}

// f: index into the chunked shapes.  Returns 0 ok, 2 the column does not fit.
template <typename R>
int launch_acoustic_column_chunked(const AcouArgs<R>& a, int f, cudaStream_t st) {
  const int nz = a.L.nz;
  if (!acoustic_chunked_fits<R>(nz, f)) return 2;
  const int cx = kChunkShapes[f][0], kl = kChunkShapes[f][1];
  const size_t sm = chunked_smem<R>(nz, cx);
  const dim3 grd((a.L.nx + cx - 1) / cx, a.L.ny, 1), blk(cx, kl);
  switch (f) {
    case 0: k_acoustic_column_chunked<R, 32, 8, 8><<<grd, blk, sm, st>>>(a); break;
    case 1: k_acoustic_column_chunked<R, 16, 16, 4><<<grd, blk, sm, st>>>(a); break;
    default: k_acoustic_column_chunked<R, 32, 16, 4><<<grd, blk, sm, st>>>(a); break;
  }
  return 0;
}

// Shapes of the parallel-solve column kernel: columns, level lanes, largest chunk
static const int kPcrShapes[][3] = {{32, 16, 3}, {16, 32, 3}, {32, 16, 4}};
constexpr int kNumPcrShapes = 3;

int acoustic_pcr_shapes() { return kNumPcrShapes; }

template <typename R>
size_t pcr_smem(int cx, int kl) {
  return (size_t)kPcrWork * cx * kl * sizeof(R);
}

template <typename R>
bool acoustic_pcr_fits(int nz, int f) {
  return f >= 0 && f < kNumPcrShapes && nz + 1 <= kPcrShapes[f][1] * kPcrShapes[f][2] &&
         pcr_smem<R>(kPcrShapes[f][0], kPcrShapes[f][1]) <= 48 * 1024;
}

// f: index into the parallel-solve shapes.  Returns 0 ok, 2 does not fit.
template <typename R>
int launch_acoustic_column_pcr(const AcouArgs<R>& a, int f, cudaStream_t st) {
  if (!acoustic_pcr_fits<R>(a.L.nz, f)) return 2;
  const int cx = kPcrShapes[f][0], kl = kPcrShapes[f][1];
  const size_t sm = pcr_smem<R>(cx, kl);
  const dim3 grd((a.L.nx + cx - 1) / cx, a.L.ny, 1), blk(cx, kl);
  switch (f) {
    case 0: k_acoustic_column_pcr<R, 32, 16, 3><<<grd, blk, sm, st>>>(a); break;
    case 1: k_acoustic_column_pcr<R, 16, 32, 3><<<grd, blk, sm, st>>>(a); break;
    default: k_acoustic_column_pcr<R, 32, 16, 4><<<grd, blk, sm, st>>>(a); break;
  }
  return 0;
}

// the plain column tile shape of fused shape f
int acoustic_fused_column_shape(int f) {
  return (f >= 0 && f < kNumFusedShapes) ? kFusedShapes[f] : 0;
}

template <typename R>
int occupancy_column(int shape, int nz_max) {
  if (shape < 0 || shape >= kNumColumnShapes || !column_fits<R>(nz_max, shape)) return 1;
  const int cx = kColumnShapes[shape][0], kl = kColumnShapes[shape][1];
  const size_t sm = column_smem<R>(nz_max, cx);
  int n = 0;
  cudaError_t e;
  switch (shape) {
    case 0: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_acoustic_column_batch<R, 32, 8>, cx * kl, sm); break;
    case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_acoustic_column_batch<R, 16, 16>, cx * kl, sm); break;
    case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_acoustic_column_batch<R, 8, 32>, cx * kl, sm); break;
    case 3: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_acoustic_column_batch<R, 32, 4>, cx * kl, sm); break;
    case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_acoustic_column_batch<R, 16, 8>, cx * kl, sm); break;
    default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_acoustic_column_batch<R, 8, 16>, cx * kl, sm); break;
  }
  return e == cudaSuccess && n > 0 ? n : 1;
}

template <typename R>
int prepare_acoustic_uv_pipe() {
  const size_t sm = UvpLayout<R>(true).total;
  if (sm > 227 * 1024) return 2;
  return raise_smem_limit(k_acoustic_uv_pipe<R>, sm) == cudaSuccess ? 0 : 1;
}

template <typename R>
int launch_acoustic_uv_pipe(const PipeUvParams<R>& p, cudaStream_t st) {
  const size_t sm = UvpLayout<R>(p.a.p.moisture != 0).total;
  if (sm > 227 * 1024) return 2;
  static std::mutex mu;
  static std::map<std::pair<int, size_t>, int> limit;  // (device, smem) -> resident CTAs
  int dev = 0, lim = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 2;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = limit.find(std::make_pair(dev, sm));
    if (it != limit.end()) {
      lim = it->second;
    } else {
      int sms = 0, occ = 0;
      if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_acoustic_uv_pipe<R>, kUvpThreads + 32,
                                                        sm) != cudaSuccess)
        return 2;
      lim = limit[std::make_pair(dev, sm)] = sms * occ;
    }
  }
  if (lim <= 0) return 2;
  const Layout& L = p.a.L;
  const int ntiles = ((L.nx + kUvpX - 1) / kUvpX) * ((L.ny + kUvpY - 1) / kUvpY) *
                     ((L.nz + kUvpZ - 1) / kUvpZ);
  k_acoustic_uv_pipe<R><<<ntiles < lim ? ntiles : lim, kUvpThreads + 32, sm, st>>>(p);
  return 0;
}

#define WFE_INST(R)                                                                            \
  template int prepare_acoustic_uv_pipe<R>();                                                  \
  template int launch_acoustic_uv_pipe<R>(const PipeUvParams<R>&, cudaStream_t);               \
  template size_t acoustic_column_tma_smem<R>(int);                                            \
  template int prepare_acoustic_column_tma<R>(int);                                            \
  template int launch_acoustic_column_tma<R>(const TmaColParams<R>&, cudaStream_t);            \
  template dim3 grid_uv<R>(const Layout&);                                                     \
  template dim3 grid_uv_fwd<R>(const Layout&);                                                 \
  template dim3 grid_column<R>(const Layout&, int);                                            \
  template void batch_uv<R>(const Batch<AcouArgs<R>>&, int, cudaStream_t);                     \
  template int batch_column<R>(const Batch<AcouArgs<R>>&, int, int, int, cudaStream_t);        \
  template int occupancy_column<R>(int, int);                                                  \
  template bool acoustic_column_fits<R>(int, int);                                             \
  template void launch_acoustic_coef<R>(const Layout&, const DBase<R>&, const DMetric<R>&, R*, \
                                        R*, R*, R*, R*, cudaStream_t);                         \
  template void launch_acoustic_uv<R>(const AcouArgs<R>&, cudaStream_t, int);                  \
  template int launch_acoustic_column<R>(const AcouArgs<R>&, int, cudaStream_t);               \
  template int prepare_acoustic_column<R>(int);                                                 \
  template bool acoustic_fused_fits<R>(int, int);                                              \
  template int prepare_acoustic_fused<R>(int);                                                 \
  template int launch_acoustic_fused<R>(const AcouArgs<R>&, int, cudaStream_t);                \
  template bool acoustic_chunked_fits<R>(int, int);                                            \
  template bool acoustic_pcr_fits<R>(int, int);                                                \
  template int launch_acoustic_column_pcr<R>(const AcouArgs<R>&, int, cudaStream_t);           \
  template int launch_acoustic_column_chunked<R>(const AcouArgs<R>&, int, cudaStream_t);
WFE_INST(float)
WFE_INST(double)
#undef WFE_INST

}  // namespace wfe
