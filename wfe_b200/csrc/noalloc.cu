// Dry-air mass of caller-owned device fields without any device allocation.
//
// Some callers cannot call cudaMalloc: a diagnostics hook running inside
// another framework's CUDA stream capture (allocation is illegal while a
// stream is being captured), or a serving process whose device memory is owned
// by a fixed-budget pool allocator that forbids foreign allocations.  For them,
// wfe_dry_mass_noalloc computes what wfe_dry_mass computes, but its per-level
// partial sums live in a file-scope __device__ array of at most
// WFE_NOALLOC_MAX_LEVELS doubles instead of a buffer the library allocates.
// Every GPU that loads this library holds the array (8 KB) until exit.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "wfe_b200.h"

namespace wfe {
void set_thread_error(const std::string& m);  // message for wfe_last_error(NULL)
}

namespace {

// Per-level partial sums shared by every call on a device; each call
// overwrites the first nz entries before reading them.
static __device__ __align__(256) double g_noalloc_planes[WFE_NOALLOC_MAX_LEVELS];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_planes_addr[kMaxDevices] = {};  // device address of the array, per device

// Same arithmetic and reduction order as the library's dry-mass diagnostic,
// on the reference padded layout (NX = nx + 6, NY = ny + 6, ng = 3).
__global__ void k_dry_mass_plane_ref(int nx, int ny, int NX, int NY, const double* pib,
                                     const double* thb, const double* pip, const double* thp,
                                     const double* qv, const double* qc, const double* qr,
                                     const double* jac, const double* dzeta_c, double* planes) {
  __shared__ double part[256];
  const int k = blockIdx.x;
  double s = 0.0;
  const int n2 = nx * ny;
  for (int q = threadIdx.x; q < n2; q += blockDim.x) {
    int i = q % nx, j = q / nx;
    size_t c = ((size_t)(k + 3) * NY + (j + 3)) * NX + (i + 3);
    double pi = pib[c] + pip[c];
    double th = thb[c] + thp[c];
    double v = qv ? qv[c] : 0.0;
    double qt = qv ? v + (qc ? qc[c] : 0.0) + (qr ? qr[c] : 0.0) : 0.0;
    double rho = 1.0e5 * pow(pi, (1004.5 - 287.04) / 287.04) / (287.04 * th * (1.0 + 0.61 * v));
    s += rho / (1.0 + qt) * jac[(size_t)(j + 3) * NX + (i + 3)];
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) planes[k] = part[0] * dzeta_c[k + 3];
}

__global__ void k_dry_mass_total_ref(const double* planes, int nz, double area, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double t = 0.0;
  for (int k = 0; k < nz; ++k) t += planes[k];
  *out = t * area;
}

// Resolves the array's device address once per device, with that device
// current (the first call on a device does this).
int planes_address(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    wfe::set_thread_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return WFE_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    wfe::set_thread_error("device index out of range");
    return WFE_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_planes_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_planes);
    if (e != cudaSuccess) {
      wfe::set_thread_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return WFE_ERR_CUDA;
    }
    g_planes_addr[dev] = static_cast<double*>(p);
  }
  *out = g_planes_addr[dev];
  return WFE_OK;
}

}  // namespace

extern "C" int wfe_dry_mass_noalloc(int nx, int ny, int nz, double dx, double dy,
                                    const double* pib, const double* thb, const double* pip,
                                    const double* thp, const double* qv, const double* qc,
                                    const double* qr, const double* jac, const double* dzeta_c,
                                    double* out, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !pib || !thb || !pip || !thp || !jac || !dzeta_c || !out) {
    wfe::set_thread_error("wfe_dry_mass_noalloc: bad argument");
    return WFE_ERR_ARG;
  }
  if (nz > WFE_NOALLOC_MAX_LEVELS) {
    wfe::set_thread_error("wfe_dry_mass_noalloc: nz = " + std::to_string(nz) +
                    " exceeds the static scratch of " + std::to_string(WFE_NOALLOC_MAX_LEVELS) +
                    " levels");
    return WFE_ERR_ARG;
  }
  double* planes = nullptr;
  int rc = planes_address(&planes);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_dry_mass_plane_ref<<<nz, 256, 0, st>>>(nx, ny, nx + 6, ny + 6, pib, thb, pip, thp, qv, qc, qr,
                                           jac, dzeta_c, planes);
  k_dry_mass_total_ref<<<1, 32, 0, st>>>(planes, nz, dx * dy, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    wfe::set_thread_error(std::string("wfe_dry_mass_noalloc launch: ") + cudaGetErrorString(e));
    return WFE_ERR_CUDA;
  }
  return WFE_OK;
}
