// Dry-air mass of caller-owned device fields without any device allocation.
//
// Some callers cannot call cudaMalloc: a diagnostics hook running inside
// another framework's CUDA stream capture (allocation is illegal while a
// stream is being captured), or a serving process whose device memory is owned
// by a fixed-budget pool allocator that forbids foreign allocations.  For them,
// wfe_dry_mass_noalloc computes what wfe_dry_mass computes, but its per-level
// partial sums live in a file-scope __device__ array of at most
// WFE_NOALLOC_MAX_LEVELS doubles instead of a buffer the library allocates.
// Every GPU that loads this library holds the array (8 KB) until exit; each
// CUDA context on a device has its own copy (the address is looked up once
// per context, on the first call made in it).
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

// The array's device address belongs to the CUDA context the module was
// loaded into, so it is cached per context, not per device ordinal: a
// context created later on the same device (after cudaDeviceReset, or a
// caller-made driver context) gets its own lookup.
constexpr int kMaxContexts = 64;
std::mutex g_mu;
void* g_ctx[kMaxContexts] = {};
double* g_planes_addr[kMaxContexts] = {};
int g_nctx = 0;

using CtxGetCurrent = int (*)(void**);  // cuCtxGetCurrent(CUcontext*), CUresult as int

// The context current on this thread, through the driver entry point the
// runtime hands out (no link against libcuda needed).
int current_context(void** ctx) {
  static CtxGetCurrent fn = nullptr;
  static std::once_flag once;
  static cudaError_t init = cudaSuccess;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    init = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
    if (init == cudaSuccess && q != cudaDriverEntryPointSuccess) init = cudaErrorSymbolNotFound;
    fn = reinterpret_cast<CtxGetCurrent>(f);
  });
  if (init != cudaSuccess || !fn) {
    wfe::set_thread_error(std::string("cuCtxGetCurrent entry point: ") + cudaGetErrorString(init));
    return WFE_ERR_CUDA;
  }
  *ctx = nullptr;
  if (fn(ctx) != 0) {
    wfe::set_thread_error("cuCtxGetCurrent failed");
    return WFE_ERR_CUDA;
  }
  return WFE_OK;
}

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

// Resolves the array's device address once per context, with the caller's
// device current (the first call in a context does this; with no context
// current yet, the device's primary context is made current first).
int planes_address(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    wfe::set_thread_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return WFE_ERR_CUDA;
  }
  void* ctx = nullptr;
  int rc = current_context(&ctx);
  if (rc) return rc;
  if (!ctx) {
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) {
      wfe::set_thread_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
      return WFE_ERR_CUDA;
    }
    if ((rc = current_context(&ctx))) return rc;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  for (int q = 0; q < g_nctx; ++q)
    if (g_ctx[q] == ctx) {
      *out = g_planes_addr[q];
      return WFE_OK;
    }
  if (g_nctx == kMaxContexts) {
    wfe::set_thread_error("wfe_dry_mass_noalloc: more than 64 CUDA contexts");
    return WFE_ERR_CUDA;
  }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_planes);
  if (e != cudaSuccess) {
    wfe::set_thread_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return WFE_ERR_CUDA;
  }
  g_ctx[g_nctx] = ctx;
  g_planes_addr[g_nctx] = static_cast<double*>(p);
  ++g_nctx;
  *out = static_cast<double*>(p);
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
