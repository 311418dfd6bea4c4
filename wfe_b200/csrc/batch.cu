// Dispatch of batched launches by kernel kind: argument-block sizes, the
// sub-launches of a kind, each member's grid and the batched launch itself.
// The kernels, their bodies and their single-case launches live in
// dyn_tend.cu, dyn_acou.cu, phys_kessler.cu and phys_sfc.cu.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace wfe {

template <typename R>
size_t kind_args_size(int kind) {
  switch (kind) {
    case K_FILL: return sizeof(FillArgs<R>);
    case K_FLUX: return sizeof(FluxArgs<R>);
    case K_PD: return sizeof(PdArgs<R>);
    case K_TEND: return sizeof(TendArgs<R>);
    case K_UV:
    case K_COL: return sizeof(AcouArgs<R>);
    case K_KES: return sizeof(KesArgs<R>);
    case K_SFC: return sizeof(SfcArgs<R>);
    case K_CLOCK: return sizeof(ClockArgs);
    default: return 0;
  }
}

template <typename R>
int kind_subs(int kind, int variant) {
  if (kind == K_TEND) return variant == 1 ? 2 : 1;
  if (kind == K_SFC) return 2;
  return 1;
}

template <typename R>
dim3 kind_grid(int kind, int variant, int sub, const void* args, int nz_max) {
  switch (kind) {
    case K_FILL: return grid_fill<R>(*static_cast<const FillArgs<R>*>(args));
    case K_FLUX: return grid_flux<R>(*static_cast<const FluxArgs<R>*>(args));
    case K_PD: return grid_pd<R>(static_cast<const PdArgs<R>*>(args)->t.L);
    case K_TEND: return grid_tend<R>(static_cast<const TendArgs<R>*>(args)->L);
    case K_UV: return grid_uv_fwd<R>(static_cast<const AcouArgs<R>*>(args)->L);
    case K_COL: return grid_column<R>(static_cast<const AcouArgs<R>*>(args)->L, variant);
    case K_KES: return grid_kessler<R>(static_cast<const KesArgs<R>*>(args)->L, nz_max);
    case K_SFC: return grid_sfc<R>(static_cast<const SfcArgs<R>*>(args)->L, sub, nz_max);
    case K_CLOCK: return grid_clock();
    default: return dim3(0, 0, 0);
  }
}

template <typename R>
int kind_occupancy(int kind, int variant, int sub, int nz_max) {
  switch (kind) {
    case K_TEND: return occupancy_tend<R>(variant, sub);
    case K_COL: return occupancy_column<R>(variant, nz_max);
    case K_KES: return occupancy_kessler<R>(nz_max);
    case K_SFC: return 4;     // 128-thread column kernels with shared columns
    case K_CLOCK: return 16;  // one warp
    default: return 6;        // 256-thread stencil kernels without shared arrays
  }
}

template <typename R>
int launch_kind_batch(int kind, int variant, int sub, const void* d_args, const int4* d_work,
                      int nwork, int nblocks, int nz_max, cudaStream_t st) {
  if (nwork <= 0) return 0;
  if (nblocks <= 0 || nblocks > nwork) nblocks = nwork;
  switch (kind) {
    case K_FILL:
      batch_fill<R>(Batch<FillArgs<R>>{static_cast<const FillArgs<R>*>(d_args), d_work, nwork},
                    nblocks, st);
      return 0;
    case K_FLUX:
      batch_flux<R>(Batch<FluxArgs<R>>{static_cast<const FluxArgs<R>*>(d_args), d_work, nwork},
                    nblocks, st);
      return 0;
    case K_PD:
      batch_pd<R>(Batch<PdArgs<R>>{static_cast<const PdArgs<R>*>(d_args), d_work, nwork}, nblocks,
                  st);
      return 0;
    case K_TEND:
      batch_tend<R>(Batch<TendArgs<R>>{static_cast<const TendArgs<R>*>(d_args), d_work, nwork},
                    variant, sub, nblocks, st);
      return 0;
    case K_UV:
      batch_uv<R>(Batch<AcouArgs<R>>{static_cast<const AcouArgs<R>*>(d_args), d_work, nwork},
                  nblocks, st);
      return 0;
    case K_COL:
      return batch_column<R>(
          Batch<AcouArgs<R>>{static_cast<const AcouArgs<R>*>(d_args), d_work, nwork}, variant,
          nz_max, nblocks, st);
    case K_KES:
      return batch_kessler<R>(
          Batch<KesArgs<R>>{static_cast<const KesArgs<R>*>(d_args), d_work, nwork}, nz_max,
          nblocks, st);
    case K_SFC:
      batch_sfc<R>(Batch<SfcArgs<R>>{static_cast<const SfcArgs<R>*>(d_args), d_work, nwork}, sub,
                   nblocks, nz_max, st);
      return 0;
    case K_CLOCK:
      batch_clock(Batch<ClockArgs>{static_cast<const ClockArgs*>(d_args), d_work, nwork}, nblocks,
                  st);
      return 0;
    default: return 1;
  }
}

#define WFE_INST(R)                                                                     \
  template size_t kind_args_size<R>(int);                                               \
  template int kind_subs<R>(int, int);                                                  \
  template dim3 kind_grid<R>(int, int, int, const void*, int);                          \
  template int kind_occupancy<R>(int, int, int, int);                                   \
  template int launch_kind_batch<R>(int, int, int, const void*, const int4*, int, int, int, \
                                    cudaStream_t);
WFE_INST(float)
WFE_INST(double)
#undef WFE_INST

}  // namespace wfe
