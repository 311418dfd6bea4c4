// On-device repack of state fields into the Writer's interior layout
// (src/io/writer.cpp:89-107: float32 blocks nzl x ny x nx, i fastest), so that
// a snapshot crosses the host link as one contiguous copy per field with no
// host-side repack.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace wfe {
namespace {

template <typename R, typename T>
__global__ void k_pack_interior(const R* __restrict__ src, Layout L, int nzl, T* __restrict__ dst) {
  const size_t n = (size_t)nzl * L.ny * L.nx;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % L.nx);
    const int j = (int)((q / L.nx) % L.ny);
    const int k = (int)(q / ((size_t)L.nx * L.ny));
    dst[q] = (T)src[L.at(i, j, k)];
  }
}

template <typename R, typename T>
__global__ void k_pack_interior2d(const R* __restrict__ src, Layout L, T* __restrict__ dst) {
  const size_t n = (size_t)L.ny * L.nx;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % L.nx);
    const int j = (int)(q / L.nx);
    dst[q] = (T)src[L.at2(i, j)];
  }
}

// the inverse: a contiguous interior block (float32 or float64) into the
// interior points of a field; ghosts and padding keep their values
template <typename R, typename T>
__global__ void k_unpack_interior(const T* __restrict__ src, Layout L, int nzl, R* __restrict__ dst) {
  const size_t n = (size_t)nzl * L.ny * L.nx;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % L.nx);
    const int j = (int)((q / L.nx) % L.ny);
    const int k = (int)(q / ((size_t)L.nx * L.ny));
    dst[L.at(i, j, k)] = (R)src[q];
  }
}

int grid_for(size_t n) {
  size_t g = (n + 255) / 256;
  return (int)(g > 148 * 16 ? 148 * 16 : (g ? g : 1));
}

}  // namespace

template <typename R>
void launch_pack_interior(const R* src, const Layout& L, int nzl, void* dst, bool f32,
                          cudaStream_t st) {
  const size_t n = (size_t)nzl * L.ny * L.nx;
  if (f32) k_pack_interior<R, float><<<grid_for(n), 256, 0, st>>>(src, L, nzl, (float*)dst);
  else k_pack_interior<R, double><<<grid_for(n), 256, 0, st>>>(src, L, nzl, (double*)dst);
}

template <typename R>
void launch_pack_interior2d(const R* src, const Layout& L, void* dst, bool f32, cudaStream_t st) {
  const size_t n = (size_t)L.ny * L.nx;
  if (f32) k_pack_interior2d<R, float><<<grid_for(n), 256, 0, st>>>(src, L, (float*)dst);
  else k_pack_interior2d<R, double><<<grid_for(n), 256, 0, st>>>(src, L, (double*)dst);
}

template <typename R>
void launch_unpack_interior(const void* src, const Layout& L, int nzl, R* dst, bool f32,
                            cudaStream_t st) {
  const size_t n = (size_t)nzl * L.ny * L.nx;
  if (f32) k_unpack_interior<R, float><<<grid_for(n), 256, 0, st>>>((const float*)src, L, nzl, dst);
  else k_unpack_interior<R, double><<<grid_for(n), 256, 0, st>>>((const double*)src, L, nzl, dst);
}

template void launch_unpack_interior<float>(const void*, const Layout&, int, float*, bool, cudaStream_t);
template void launch_unpack_interior<double>(const void*, const Layout&, int, double*, bool, cudaStream_t);
template void launch_pack_interior<float>(const float*, const Layout&, int, void*, bool, cudaStream_t);
template void launch_pack_interior<double>(const double*, const Layout&, int, void*, bool, cudaStream_t);
template void launch_pack_interior2d<float>(const float*, const Layout&, void*, bool, cudaStream_t);
template void launch_pack_interior2d<double>(const double*, const Layout&, void*, bool, cudaStream_t);

}  // namespace wfe
