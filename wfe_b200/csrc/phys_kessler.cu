// Kessler warm rain with the mixed-phase blend (src/physics/kessler.cu:22-149),
// the |f| watchdog reduction (src/dynamics/kernels.cu:278-289) and an FP64
// dry-air mass diagnostic, on the B200.
//
// The reference runs one thread per column with four 320-deep local arrays
// (a 5 KB stack) and walks every level serially.  Here a CTA owns CX columns
// with the column arrays in shared memory: the fall speeds, the flux
// divergence of each sedimentation subcycle and the per-level conversions run
// in parallel over the levels; only the rain accumulation is serial.  Every
// value is computed with the reference's expressions, so subcycle counts and
// branch decisions are the same.
#include <cuda_runtime.h>

#include "core.cuh"
#include "kernels.cuh"
#include "phys_common.cuh"

namespace wfe {

// HB: the base state from its level tables (DBase::lvl)
template <typename R, int CX, bool HB = false>
__device__ __forceinline__ void kessler_body(const KesArgs<R>& a, int bx, int by) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Layout& L = a.L;
  const int nz = L.nz;
  const int tx = threadIdx.x, lane = threadIdx.y, KL = blockDim.y;
  const int i = bx * CX + tx, j = by;
  const bool active = i < L.nx;
  R* qrl = reinterpret_cast<R*>(smem_raw);
  R* rhol = qrl + (size_t)nz * CX;
  R* dzl = rhol + (size_t)nz * CX;
  R* vr = dzl + (size_t)nz * CX;
  R* F = vr + (size_t)nz * CX;                 // (nz + 1) * CX
  R* red = F + (size_t)(nz + 1) * CX;          // KL * CX * 2 partial max/min
  __shared__ int nsub_s[CX];
  __shared__ R dts_s[CX];
#define S(X, k) X[(size_t)(k) * CX + tx]
  // base state at level k of this column (c its cell index)
  auto rhob = [&](int c, int k) { return HB ? a.b.lvl[BL_RHOB * L.pz + L.at1(k)] : a.b.rhob[c]; };
  auto thb = [&](int c, int k) { return HB ? a.b.lvl[BL_THB * L.pz + L.at1(k)] : a.b.thb[c]; };
  auto pib = [&](int c, int k) { return HB ? a.b.lvl[BL_PIB * L.pz + L.at1(k)] : a.b.pib[c]; };
  const R J = active ? a.m.jac[L.at2i(i, j)] : (R)1;
  const R rho_sfc = active ? rhob(L.ati(i, j, 0), 0) : (R)1;

  // 1) column set-up and the first fall speeds (kessler.cu:199-214)
  R vmax = 0, dmin = (R)1e30;
  if (active)
    for (int k = lane; k < nz; k += KL) {
      const int c = L.ati(i, j, k);
      R q = a.qr[c];
      R qk = q > (R)0 ? q : (R)0;
      R rh = rhob(c, k);
      R dz = a.m.dzeta_c[L.at1(k)] * J;
      R T = (thb(c, k) + a.thp[c]) * (pib(c, k) + a.pip[c]);
      R vk = fall_speed(rh * qk, rho_sfc, rh, T);
      S(qrl, k) = qk;
      S(rhol, k) = rh;
      S(dzl, k) = dz;
      S(vr, k) = vk;
      if (vk > vmax) vmax = vk;
      if (dz < dmin) dmin = dz;
    }
  red[(size_t)lane * CX + tx] = vmax;
  red[(size_t)(KL + lane) * CX + tx] = dmin;
  __syncthreads();
  if (lane == 0) {
    R vm = 0, dm = (R)1e30;
    for (int l = 0; l < KL; ++l) {
      R x = red[(size_t)l * CX + tx], y = red[(size_t)(KL + l) * CX + tx];
      if (x > vm) vm = x;
      if (y < dm) dm = y;
    }
    int ns = active ? 1 + (int)(vm * a.dt / ((R)0.8 * dm)) : 0;
    nsub_s[tx] = ns;
    dts_s[tx] = active ? a.dt / (R)ns : (R)0;
  }
  __syncthreads();
  int nsub_max = 0;
  for (int c = 0; c < CX; ++c) nsub_max = max(nsub_max, nsub_s[c]);
  const int nsub = nsub_s[tx];
  const R dts = dts_s[tx];

  // 2) upwind sedimentation subcycles (kessler.cu:215-236)
  R acc = 0;
  for (int s = 0; s < nsub_max; ++s) {
    const bool on = active && s < nsub;
    if (on)
      for (int k = lane; k <= nz; k += KL) S(F, k) = (k < nz) ? S(rhol, k) * S(qrl, k) * S(vr, k) : (R)0;
    __syncthreads();
    if (on) {
      if (lane == 0) acc += dts * S(F, 0);
      for (int k = lane; k < nz; k += KL)
        S(qrl, k) += dts * (S(F, k + 1) - S(F, k)) / (S(rhol, k) * S(dzl, k));
    }
    __syncthreads();
    if (on && s + 1 < nsub)
      for (int k = lane; k < nz; k += KL) {
        const int c = L.ati(i, j, k);
        R q = S(qrl, k);
        R rq = S(rhol, k) * (q > (R)0 ? q : (R)0);
        R T = (thb(c, k) + a.thp[c]) * (pib(c, k) + a.pip[c]);
        S(vr, k) = fall_speed(rq, rho_sfc, S(rhol, k), T);
      }
    __syncthreads();
  }
  if (active && lane == 0) a.rain[L.at2i(i, j)] += acc;

  // 3) conversions, evaporation and mixed-phase saturation adjustment,
  //    independent per level (kessler.cu:239-297; phys_common.cuh)
  if (active)
    for (int k = lane; k < nz; k += KL) {
      const int c = L.ati(i, j, k);
      R thp = a.thp[c], qv = a.qv[c], qc = a.qc[c], qr = S(qrl, k);
      const R pip = a.pip[c];
      kessler_convert<R, R>(thp, qv, qc, qr, pip, S(rhol, k), thb(c, k), pib(c, k), a.dt);
      a.thp[c] = thp;
      a.qv[c] = qv;
      a.qc[c] = qc;
      a.qr[c] = qr;
    }
#undef S
}

template <typename R, int CX, bool HB>
__global__ void k_kessler(KesArgs<R> a) {
  kessler_body<R, CX, HB>(a, blockIdx.x, blockIdx.y);
}
template <typename R, int CX>
__global__ void k_kessler_batch(Batch<KesArgs<R>> b) {
  for_each_work(b, [](const KesArgs<R>& a, int x, int y, int) { kessler_body<R, CX>(a, x, y); });
}

template <typename R>
static size_t kessler_smem(int nz, int cx, int kl) {
  return ((size_t)4 * nz + (nz + 1) + 2 * kl) * cx * sizeof(R);
}

template <typename R>
static int kessler_cx(int nz) {
  const size_t lim = 200 * 1024;
  if (kessler_smem<R>(nz, 32, 8) <= lim) return 32;
  if (kessler_smem<R>(nz, 8, 32) <= lim) return 8;
  return 0;
}

// Sets the dynamic shared-memory limit once, outside any stream capture.
template <typename R>
int prepare_kessler(int nz) {
  int cx = kessler_cx<R>(nz);
  cudaError_t e;
  if (cx == 32) {
    const size_t sm = kessler_smem<R>(nz, 32, 8);
    e = raise_smem_limit(k_kessler<R, 32, false>, sm);
    if (e == cudaSuccess) e = raise_smem_limit(k_kessler<R, 32, true>, sm);
    if (e == cudaSuccess) e = raise_smem_limit(k_kessler_batch<R, 32>, sm);
  } else if (cx == 8) {
    const size_t sm = kessler_smem<R>(nz, 8, 32);
    e = raise_smem_limit(k_kessler<R, 8, false>, sm);
    if (e == cudaSuccess) e = raise_smem_limit(k_kessler<R, 8, true>, sm);
    if (e == cudaSuccess) e = raise_smem_limit(k_kessler_batch<R, 8>, sm);
  } else {
    return 2;
  }
  return e == cudaSuccess ? 0 : 1;
}

// Batched columns use the tile of the deepest member (nz_max); the shared
// arrays are sized for it (prepare_kessler<R>(nz_max) done).
template <typename R>
dim3 grid_kessler(const Layout& L, int nz_max) {
  const int cx = kessler_cx<R>(nz_max);
  return cx ? dim3((L.nx + cx - 1) / cx, L.ny, 1) : dim3(0, 0, 0);
}

template <typename R>
int batch_kessler(const Batch<KesArgs<R>>& b, int nz_max, int nblocks, cudaStream_t st) {
  const int cx = kessler_cx<R>(nz_max);
  if (cx == 32)
    k_kessler_batch<R, 32><<<nblocks, dim3(32, 8), kessler_smem<R>(nz_max, 32, 8), st>>>(b);
  else if (cx == 8)
    k_kessler_batch<R, 8><<<nblocks, dim3(8, 32), kessler_smem<R>(nz_max, 8, 32), st>>>(b);
  else
    return 2;
  return 0;
}

template <typename R>
int occupancy_kessler(int nz_max) {
  const int cx = kessler_cx<R>(nz_max);
  int n = 0;
  cudaError_t e = cudaErrorInvalidValue;
  if (cx == 32)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_kessler_batch<R, 32>, 256,
                                                      kessler_smem<R>(nz_max, 32, 8));
  else if (cx == 8)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_kessler_batch<R, 8>, 256,
                                                      kessler_smem<R>(nz_max, 8, 32));
  return e == cudaSuccess && n > 0 ? n : 1;
}

template <typename R>
int launch_kessler(const KesArgs<R>& a, cudaStream_t st) {
  const int nz = a.L.nz;
  const int cx = kessler_cx<R>(nz);
  const bool hb = a.b.lvl != nullptr;
  if (cx == 32) {
    const dim3 g((a.L.nx + 31) / 32, a.L.ny), t(32, 8);
    if (hb) k_kessler<R, 32, true><<<g, t, kessler_smem<R>(nz, 32, 8), st>>>(a);
    else k_kessler<R, 32, false><<<g, t, kessler_smem<R>(nz, 32, 8), st>>>(a);
  } else if (cx == 8) {
    const dim3 g((a.L.nx + 7) / 8, a.L.ny), t(8, 32);
    if (hb) k_kessler<R, 8, true><<<g, t, kessler_smem<R>(nz, 8, 32), st>>>(a);
    else k_kessler<R, 8, false><<<g, t, kessler_smem<R>(nz, 8, 32), st>>>(a);
  } else {
    return 2;
  }
  return 0;
}

// ------------------------------------------------------------- watchdog
// max |f| over the points the reference defines (interior cells, faces up to
// nx / ny, w levels up to nz); as float bits so that NaN ranks above every
// finite value (kernels.cu:275-289).
template <typename R>
__global__ void __launch_bounds__(256) k_absmax(const R* __restrict__ f, size_t n, unsigned int* result) {
  // |f| as float bits: the unsigned order of non-negative floats, NaN above
  // every finite value; one atomic per block (the blocks' atomics on one
  // address serialise in L2)
  __shared__ unsigned int warp_best[8];
  unsigned int best = 0;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (size_t)gridDim.x * blockDim.x) {
    float v = fabsf((float)f[idx]);
    unsigned int b = __float_as_uint(v);
    best = b > best ? b : best;
  }
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) warp_best[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x < 32) {
    best = threadIdx.x < (blockDim.x >> 5) ? warp_best[threadIdx.x] : 0u;
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (threadIdx.x == 0) atomicMax(result, best);
  }
}

// The watchdog's pipelined form: the blocks' maxima meet in acc[0]; the last
// block to finish (counted in acc[1]) writes the result straight into mapped
// page-locked host memory and resets acc for the next call, so one launch is
// all a step's watchdog adds to the stream (no memset, no copy).
template <typename R>
__global__ void __launch_bounds__(256) k_absmax_to_host(const R* __restrict__ f, size_t n, unsigned int* acc,
                                                        unsigned int* host_out) {
  __shared__ unsigned int warp_best[8];
  unsigned int best = 0;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (size_t)gridDim.x * blockDim.x) {
    float v = fabsf((float)f[idx]);
    unsigned int b = __float_as_uint(v);
    best = b > best ? b : best;
  }
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) warp_best[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x < 32) {
    best = threadIdx.x < (blockDim.x >> 5) ? warp_best[threadIdx.x] : 0u;
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (threadIdx.x == 0) {
      atomicMax(acc, best);
      __threadfence();
      if (atomicAdd(acc + 1, 1u) == gridDim.x - 1) {
        const unsigned int v = atomicExch(acc, 0u);
        acc[1] = 0;
        *reinterpret_cast<volatile unsigned int*>(host_out) = v;
        __threadfence_system();
      }
    }
  }
}

template <typename R>
void launch_absmax_to_host(const R* f, size_t n, unsigned int* acc, unsigned int* host_out,
                           cudaStream_t st) {
  int grd = (int)((n + 255) / 256);
  if (grd > 148 * 2) grd = 148 * 2;
  k_absmax_to_host<R><<<grd, 256, 0, st>>>(f, n, acc, host_out);
}

template <typename R>
void launch_absmax(const R* f, size_t n, unsigned int* result, cudaStream_t st) {
  int grd = (int)((n + 255) / 256);
  if (grd > 148 * 2) grd = 148 * 2;
  k_absmax<R><<<grd, 256, 0, st>>>(f, n, result);
}

// ---------------------------------------------------------- dry-air mass
// sum over interior cells of rho / (1 + qv + qc + qr) * J * dzeta * dx * dy,
// rho = p00 pi^(cv/Rd) / (Rd theta (1 + 0.61 qv)), accumulated in FP64 with a
// fixed reduction order (one CTA per level, then the levels in order) so the
// result is bit-reproducible run to run.
template <typename R>
__global__ void k_dry_mass_plane(Layout L, DBase<R> b, DMetric<R> m, const R* pip, const R* thp,
                                 const R* qv, const R* qc, const R* qr, int moist,
                                 double* plane_sums) {
  __shared__ double part[256];
  const int k = blockIdx.x;
  double s = 0.0;
  const int n2 = L.nx * L.ny;
  for (int q = threadIdx.x; q < n2; q += blockDim.x) {
    int i = q % L.nx, j = q / L.nx;
    size_t c = L.at(i, j, k);
    double pi = (double)b.pib[c] + (double)pip[c];
    double th = (double)b.thb[c] + (double)thp[c];
    double v = moist ? (double)qv[c] : 0.0;
    double qt = moist ? v + (double)qc[c] + (double)qr[c] : 0.0;
    double rho = 1.0e5 * pow(pi, (1004.5 - 287.04) / 287.04) / (287.04 * th * (1.0 + 0.61 * v));
    s += rho / (1.0 + qt) * (double)m.jac[L.at2(i, j)];
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) plane_sums[k] = part[0] * (double)m.dzeta_c[L.at1(k)];
}

__global__ void k_dry_mass_total(const double* plane_sums, int nz, double area, double* result) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double t = 0.0;
  for (int k = 0; k < nz; ++k) t += plane_sums[k];
  *result = t * area;
}

template <typename R>
void launch_dry_mass(const Layout& L, const DBase<R>& b, const DMetric<R>& m, const R* pip,
                     const R* thp, const R* qv, const R* qc, const R* qr, int moist, R dx, R dy,
                     double* plane_sums, double* result, cudaStream_t st) {
  k_dry_mass_plane<R><<<L.nz, 256, 0, st>>>(L, b, m, pip, thp, qv, qc, qr, moist, plane_sums);
  k_dry_mass_total<<<1, 32, 0, st>>>(plane_sums, L.nz, (double)dx * (double)dy, result);
}

#define WFE_INST(R)                                                                           \
  template int launch_kessler<R>(const KesArgs<R>&, cudaStream_t);                            \
  template int prepare_kessler<R>(int);                                                        \
  template dim3 grid_kessler<R>(const Layout&, int);                                           \
  template int batch_kessler<R>(const Batch<KesArgs<R>>&, int, int, cudaStream_t);             \
  template int occupancy_kessler<R>(int);                            \
  template void launch_absmax<R>(const R*, size_t, unsigned int*, cudaStream_t);              \
  template void launch_absmax_to_host<R>(const R*, size_t, unsigned int*, unsigned int*, cudaStream_t); \
  template void launch_dry_mass<R>(const Layout&, const DBase<R>&, const DMetric<R>&, const R*, \
                                   const R*, const R*, const R*, const R*, int, R, R, double*, \
                                   double*, cudaStream_t);
WFE_INST(float)
WFE_INST(double)
#undef WFE_INST

}  // namespace wfe
