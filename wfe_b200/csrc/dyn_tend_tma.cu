// TMA-staged scalar tendencies: theta' and the three moisture species
// (flux-form 5th-order advection, src/dynamics/kernels.cu:114-179 and
// 886-899; the scalar part of tend_body in dyn_tend.cu, same expressions).
//
// A CTA owns a tile of kTtX x kTtY x kTtZ cells.  The three mass-flux tiles
// and, field by field, the advected scalar's tile with its 3-cell halo arrive
// in shared memory by bulk tensor loads; the next field's load is issued before
// this field's arithmetic (two scalar buffers).  Each face flux of the tile is
// computed once into shared memory (the cell-per-thread kernel computes every
// interior face twice), then every cell combines its six faces.  Results are
// bit-identical to tend_body: each flux and each cell sum is the same
// expression on the same values.
//
// Not for positive-definite moisture (its limited fluxes need the outflow
// ratios of the upwind cells); the host offers this variant only without it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "core.cuh"
#include "dyn_common.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace wfe {
namespace {

// box extents: the scalar box starts 4 cells left of the tile (16-byte aligned
// x coordinate) and 3 cells below / in front of it
constexpr int kQbX = kTtX + 8, kQbY = kTtY + 6, kQbZ = kTtZ + 6;
constexpr int kMxX = kTtX + 4;  // x faces i0 .. i0 + kTtX (rows a multiple of 16 bytes)

template <typename R>
struct TendTmaLayout {
  size_t mfx, mfy, mfz, q[2], fx, fy, fz, total;
  __host__ __device__ TendTmaLayout() {
    auto al = [](size_t n) { return (n + 127) / 128 * 128; };
    size_t o = 128;  // three mbarriers
    mfx = o;
    o += al((size_t)kMxX * kTtY * kTtZ * sizeof(R));
    mfy = o;
    o += al((size_t)kTtX * (kTtY + 1) * kTtZ * sizeof(R));
    mfz = o;
    o += al((size_t)kTtX * kTtY * (kTtZ + 1) * sizeof(R));
    for (int b = 0; b < 2; ++b) {
      q[b] = o;
      o += al((size_t)kQbX * kQbY * kQbZ * sizeof(R));
    }
    fx = o;
    o += al((size_t)(kTtX + 1) * kTtY * kTtZ * sizeof(R));
    fy = o;
    o += al((size_t)kTtX * (kTtY + 1) * kTtZ * sizeof(R));
    fz = o;
    o += al((size_t)kTtX * kTtY * (kTtZ + 1) * sizeof(R));
    total = o;
  }
};


template <typename R>
__global__ void __launch_bounds__(kTtX * kTtY * 2) k_tend_scal_tma(const __grid_constant__ TendTmaParams<R> p) {
  extern __shared__ __align__(128) unsigned char smem_tt[];
  const TendArgs<R>& a = p.a;
  const Layout& L = a.L;
  const TendTmaLayout<R> lay;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_tt);  // [0], [1] scalars, [2] mass fluxes
  const int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
  const int tid = tx + kTtX * (ty + kTtY * tz);
  constexpr int kThreads = kTtX * kTtY * 2;
  const int i0 = blockIdx.x * kTtX, j0 = blockIdx.y * kTtY, k0 = blockIdx.z * kTtZ;
  const bool moist = a.p.moisture != 0;
  const int nf = moist ? 4 : 1;
  const uint32_t qbytes = (uint32_t)((size_t)kQbX * kQbY * kQbZ * sizeof(R));
  R* sq[2] = {reinterpret_cast<R*>(smem_tt + lay.q[0]), reinterpret_cast<R*>(smem_tt + lay.q[1])};
  const R* smx = reinterpret_cast<const R*>(smem_tt + lay.mfx);
  const R* smy = reinterpret_cast<const R*>(smem_tt + lay.mfy);
  const R* smz = reinterpret_cast<const R*>(smem_tt + lay.mfz);
  R* Fx = reinterpret_cast<R*>(smem_tt + lay.fx);
  R* Fy = reinterpret_cast<R*>(smem_tt + lay.fy);
  R* Fz = reinterpret_cast<R*>(smem_tt + lay.fz);

  if (tid == 0) {
    for (int b = 0; b < 3; ++b) tma::mbar_init(bar + b, 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  if (tid == 0) {
    const uint32_t mb = (uint32_t)(((size_t)kMxX * kTtY * kTtZ + (size_t)kTtX * (kTtY + 1) * kTtZ +
                                    (size_t)kTtX * kTtY * (kTtZ + 1)) *
                                   sizeof(R));
    tma::mbar_arrive_expect_tx(bar + 2, mb);
    tma::load_3d(smem_tt + lay.mfx, &p.mfx, i0 + kOX, j0 + kOY, k0 + kOZ, bar + 2);
    tma::load_3d(smem_tt + lay.mfy, &p.mfy, i0 + kOX, j0 + kOY, k0 + kOZ, bar + 2);
    tma::load_3d(smem_tt + lay.mfz, &p.mfz, i0 + kOX, j0 + kOY, k0 + kOZ, bar + 2);
    tma::mbar_arrive_expect_tx(bar + 0, qbytes);
    tma::load_3d(sq[0], &p.q[0], i0 + kOX - 4, j0 + kOY - 3, k0 + kOZ - 3, bar + 0);
  }
  bool ok = true;
  if (tid == 0) ok = tma::mbar_wait(bar + 2, 0, 1u << 24);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicExch(p.err, 1u);
      tma::mbar_wait(bar + 2, 0, 1u << 22);
      tma::mbar_wait(bar + 0, 0, 1u << 22);
    }
    return;
  }

  // the thread's two cells: (tx, ty, tz) and (tx, ty, tz + 2) of the tile
  const int i = i0 + tx, j = j0 + ty;
  const bool col = i < L.nx && j < L.ny;
  const bool bdy = a.lo[0] != nullptr;
  R rt[2], dv[2];
  size_t cc[2];
  bool act[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int kz = tz + 2 * h, k = k0 + kz;
    act[h] = col && k < L.nz;
    cc[h] = L.at(act[h] ? i : 0, act[h] ? j : 0, act[h] ? k : 0);
    rt[h] = 1;
    dv[h] = 0;
    if (act[h]) {
      const R* mx = smx + ((size_t)kz * kTtY + ty) * kMxX + tx;
      const R* my = smy + ((size_t)kz * (kTtY + 1) + ty) * kTtX + tx;
      const R* mz = smz + ((size_t)kz * kTtY + ty) * kTtX + tx;
      // divergence (dyn_tend.cu divergence: same order)
      dv[h] = (mx[1] - mx[0]) * a.co.inv_dx + (my[kTtX] - my[0]) * a.co.inv_dy +
              (mz[kTtY * kTtX] - mz[0]) * a.co.inv_dzc[L.at1(k)];
      rt[h] = a.b.rhob[cc[h]] * a.m.jac[L.at2(i, j)];
    }
  }

  const R* const qsrc[4] = {a.thp, a.qv, a.qc, a.qr};
  for (int n = 0; n < nf; ++n) {
    const int b = n & 1;
    if (tid == 0 && n + 1 < nf) {
      // buffer b ^ 1 was last read by field n - 1, which every thread has left
      tma::mbar_arrive_expect_tx(bar + (b ^ 1), qbytes);
      tma::load_3d(sq[b ^ 1], &p.q[n + 1], i0 + kOX - 4, j0 + kOY - 3, k0 + kOZ - 3, bar + (b ^ 1));
    }
    if (tid == 0) ok = tma::mbar_wait(bar + b, (uint32_t)((n >> 1) & 1), 1u << 24);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(p.err, 1u);
        tma::mbar_wait(bar + b, (uint32_t)((n >> 1) & 1), 1u << 22);
        if (n + 1 < nf) tma::mbar_wait(bar + (b ^ 1), (uint32_t)(((n + 1) >> 1) & 1), 1u << 22);
      }
      return;
    }
    const R* Q = sq[b];
    auto QB = [&](int x, int y, int z) -> R { return Q[((size_t)z * kQbY + y) * kQbX + x]; };
    // face fluxes of the tile, each once (face_sc's expression)
    for (int f = tid; f < (kTtX + 1) * kTtY * kTtZ; f += kThreads) {
      const int ii = f % (kTtX + 1), r = f / (kTtX + 1), jj = r % kTtY, kz = r / kTtY;
      const R fv = smx[((size_t)kz * kTtY + jj) * kMxX + ii];
      const int x = ii + 1, y = jj + 3, z = kz + 3;
      Fx[f] = mul_rn(fv, face5(QB(x, y, z), QB(x + 1, y, z), QB(x + 2, y, z), QB(x + 3, y, z), QB(x + 4, y, z),
                         QB(x + 5, y, z), fv));
    }
    for (int f = tid; f < kTtX * (kTtY + 1) * kTtZ; f += kThreads) {
      const int ii = f % kTtX, r = f / kTtX, jj = r % (kTtY + 1), kz = r / (kTtY + 1);
      const R fv = smy[((size_t)kz * (kTtY + 1) + jj) * kTtX + ii];
      const int x = ii + 4, y = jj, z = kz + 3;
      Fy[f] = mul_rn(fv, face5(QB(x, y, z), QB(x, y + 1, z), QB(x, y + 2, z), QB(x, y + 3, z), QB(x, y + 4, z),
                         QB(x, y + 5, z), fv));
    }
    for (int f = tid; f < kTtX * kTtY * (kTtZ + 1); f += kThreads) {
      const int ii = f % kTtX, r = f / kTtX, jj = r % kTtY, kz = r / kTtY;
      const R fv = smz[((size_t)kz * kTtY + jj) * kTtX + ii];
      const int x = ii + 4, y = jj + 3, z = kz;
      Fz[f] = mul_rn(fv, face5(QB(x, y, z), QB(x, y, z + 1), QB(x, y, z + 2), QB(x, y, z + 3), QB(x, y, z + 4),
                         QB(x, y, z + 5), fv));
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!act[h]) continue;
      const int kz = tz + 2 * h, k = k0 + kz, kk = L.at1(k);
      const size_t c = cc[h];
      const R FxL = Fx[((size_t)kz * kTtY + ty) * (kTtX + 1) + tx];
      const R FxR = Fx[((size_t)kz * kTtY + ty) * (kTtX + 1) + tx + 1];
      const R FyL = Fy[((size_t)kz * (kTtY + 1) + ty) * kTtX + tx];
      const R FyR = Fy[((size_t)kz * (kTtY + 1) + ty + 1) * kTtX + tx];
      const R FzB = Fz[((size_t)kz * kTtY + ty) * kTtX + tx];
      const R FzT = Fz[((size_t)(kz + 1) * kTtY + ty) * kTtX + tx];
      const R q0 = QB(tx + 4, ty + 3, kz + 3);
      R fdiv = (FxR - FxL) * a.co.inv_dx + (FyR - FyL) * a.co.inv_dy + (FzT - FzB) * a.co.inv_dzc[kk];
      R t = (-fdiv + q0 * dv[h]) / rt[h];
      if (n == 0) {
        // theta' (tend_body): sponge, diffusion, Davies; pi' relaxation
        t = t - a.co.spg_c[kk] * q0;
        if (a.p.diff_K > (R)0) {
          const R dzl = a.m.dzeta_c[kk] * a.m.jac[L.at2(i, j)];
          const int x = tx + 4, y = ty + 3, z = kz + 3;
          const R lap = (QB(x + 1, y, z) - 2 * q0 + QB(x - 1, y, z)) / (a.dx * a.dx) +
                        (QB(x, y + 1, z) - 2 * q0 + QB(x, y - 1, z)) / (a.dy * a.dy) +
                        (QB(x, y, z + 1) - 2 * q0 + QB(x, y, z - 1)) / (dzl * dzl);
          t += a.p.diff_K * lap;
        }
        if (bdy) t += davies(a, 2, a.thp, i, j, k);
        a.tth[c] = t;
        if (a.tpi) a.tpi[c] = bdy ? davies(a, 3, a.pip, i, j, k) : (R)0;
      } else {
        // moisture species and its stage value (kernels.cu:268-273)
        if (n == 1 && bdy) t += davies(a, 4, qsrc[1], i, j, k);
        R* qo = n == 1 ? a.qo_v : (n == 2 ? a.qo_c : a.qo_r);
        const R* qn = n == 1 ? a.qn_v : (n == 2 ? a.qn_c : a.qn_r);
        R* tq = n == 1 ? a.tqv : (n == 2 ? a.tqc : a.tqr);
        if (qo) qo[c] = qn[c] + a.dt_stage * t;
        else tq[c] = t;
      }
    }
    __syncthreads();  // the flux arrays and buffer b are free again
  }
}

}  // namespace

template <typename R>
size_t tend_scal_tma_smem() {
  return TendTmaLayout<R>().total;
}

template <typename R>
int prepare_tend_scal_tma() {
  return raise_smem_limit(k_tend_scal_tma<R>, tend_scal_tma_smem<R>()) == cudaSuccess
             ? 0
             : 1;
}

template <typename R>
void launch_tend_scal_tma(const TendTmaParams<R>& p, cudaStream_t st) {
  const Layout& L = p.a.L;
  dim3 grd((L.nx + kTtX - 1) / kTtX, (L.ny + kTtY - 1) / kTtY, (L.nz + kTtZ - 1) / kTtZ);
  k_tend_scal_tma<R><<<grd, dim3(kTtX, kTtY, 2), tend_scal_tma_smem<R>(), st>>>(p);
}

#define WFE_INST(R)                                 \
  template size_t tend_scal_tma_smem<R>();          \
  template int prepare_tend_scal_tma<R>();          \
  template void launch_tend_scal_tma<R>(const TendTmaParams<R>&, cudaStream_t);
WFE_INST(float)
WFE_INST(double)
#undef WFE_INST

}  // namespace wfe
