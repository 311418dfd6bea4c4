// Argument blocks and launch entry points of the wfe_b200 device kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "core.cuh"

namespace wfe {

// Up to 8 fields whose ghost rings one launch fills (kind: 0 cell scalar,
// 1 u, 2 v, 3 w).
template <typename R>
struct GhostJob {
  R* f[8];
  int kind[8];
  int n;
};

template <typename R>
struct TendArgs {
  Layout L;
  DBase<R> b;
  DMetric<R> m;
  DParams<R> p;
  DCoef<R> co;  // per-level reciprocals and Rayleigh coefficients
  R dx, dy, dt;                                   // grid spacing, large step
  const R *u, *v, *w, *thp, *pip, *qv, *qc, *qr;  // stage estimate, ghosts filled
  const R *mfx, *mfy, *mfz;                       // mass fluxes on the ring
  const R *ratio_v, *ratio_c, *ratio_r;           // PD outflow ratios or null
  R *tu, *tv, *tw, *tth, *tpi;                    // tpi may be null
  R *tqv, *tqc, *tqr;                             // used when qo_* are null
  const R *qn_v, *qn_c, *qn_r;                    // time-n moisture
  R *qo_v, *qo_c, *qo_r;                          // stage moisture q_n + dt_stage*tq
  R dt_stage;
  const R* lo[5];                                 // Davies targets, lo[0] null if off
  const R* hi[5];
  const R* wgt;
  const double* clock;  // device clock: t (step start), t_lo, t_hi of the targets
};

// Device clock read by time-dependent terms (Davies time interpolation,
// surface solar geometry) so that captured step graphs stay valid:
// [0] t at the start of the step, [1] t_lo, [2] t_hi, [3] dt.
enum { CLK_T = 0, CLK_TLO = 1, CLK_THI = 2, CLK_DT = 3, CLK_N = 4 };

template <typename R>
struct AcouArgs {
  Layout L;
  DBase<R> b;
  DMetric<R> m;
  DCoef<R> co;
  DParams<R> p;
  R dx, dy, dtau;
  const R *u_in, *v_in;
  R *u_out, *v_out;
  const R* w_in;
  R* w_out;
  const R *pi_prev, *pi_cur;
  R* pi_next;
  const R* th_in;
  R* th_out;
  const R *n_pip, *n_thp;          // time-n pi', theta' (ghost values)
  const R *qv, *qc, *qr;           // time-n moisture, stage constant
  const R *tu, *tv, *tw, *tth, *tpi;  // tpi may be null (no slow pi' tendency)
};

template <typename R>
struct KesArgs {
  Layout L;
  DBase<R> b;
  DMetric<R> m;
  R dt;
  R *thp, *qv, *qc, *qr, *rain;
  const R* pip;
};

// Surface layer, PBL, soil and radiation columns (src/physics/surface.cu).
template <typename R>
struct SfcArgs {
  Layout L;
  DBase<R> b;
  DMetric<R> m;
  R dt;
  double start_hour;
  int doy, nonlocal;
  const double* clock;  // utc from clock[CLK_T] + clock[CLK_DT]
  R *thp, *qv, *u, *v;
  const R *pip, *qc;
  R *tsk, *km, *cdv, *pblh, *t2m, *u10, *soilt;
  const R *tdeep, *land, *lat, *lon, *soilw;
  R* scratch;  // sfc_scratch_count(L) elements of column work arrays
};

// Argument blocks of the kernels whose single launches take loose arguments.
template <typename R>
struct FillArgs {
  Layout L;
  GhostJob<R> job;
  int open_x, open_y;
};
template <typename R>
struct FluxArgs {
  Layout L;
  DBase<R> b;
  DMetric<R> m;
  const R *u, *v, *w;
  R *mfx, *mfy, *mfz;
};
template <typename R>
struct PdArgs {
  TendArgs<R> t;
  R *rv, *rc, *rr;
};
struct ClockArgs {
  double* clk;
  double t, t_lo, t_hi, dt;
  int advance;
};

// ------------------------------------------------------------------ batches
// A batched launch runs one kernel over the blocks of several members (cases
// of possibly different sizes advancing together): work[w] = (member, bx, by,
// bz) names block w's member and its block coordinates in that member's own
// grid.  Blocks walk the list with stride gridDim.x (a persistent grid when
// the launch has fewer blocks than items).
template <typename A>
struct Batch {
  const A* args;     // device array, one argument block per member
  const int4* work;  // device work list
  int nwork;
};

// Walks a batch's work list: for item w the block stages member work[w].x's
// argument block in shared memory and runs body(args, bx, by, bz) with the
// item's block coordinates.
template <typename A, typename F>
__device__ __forceinline__ void for_each_work(const Batch<A>& b, F&& body) {
  static_assert(sizeof(A) % 4 == 0, "argument blocks are staged as 32-bit words");

  __shared__ __align__(16) int raw[sizeof(A) / 4];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nth = blockDim.x * blockDim.y * blockDim.z;
  for (int w = blockIdx.x; w < b.nwork; w += gridDim.x) {
    const int4 it = b.work[w];
    __syncthreads();  // every thread is done with the previous item's arguments
    const int* src = reinterpret_cast<const int*>(b.args + it.x);
    for (int q = tid; q < (int)(sizeof(A) / 4); q += nth) raw[q] = src[q];
    __syncthreads();
    body(*reinterpret_cast<const A*>(raw), it.y, it.z, it.w);
  }
}

// Kernel kinds of one RK3 step as recorded for batched replay.  variant is the
// tuned launch variant (tendencies: 0 fused / 1 split; acoustic column: tile
// shape); one kind may launch several kernels ("subs") over separate grids.
enum Kind { K_FILL = 0, K_FLUX, K_PD, K_TEND, K_UV, K_COL, K_KES, K_SFC, K_CLOCK, K_NKIND };

template <typename R>
size_t kind_args_size(int kind);
template <typename R>
int kind_subs(int kind, int variant);
// grid of sub-launch `sub` of one member (args: that member's argument block)
template <typename R>
dim3 kind_grid(int kind, int variant, int sub, const void* args, int nz_max);
// resident blocks per SM of the batched kernel of sub-launch `sub`
template <typename R>
int kind_occupancy(int kind, int variant, int sub, int nz_max);
// one batched launch of sub-launch `sub`; d_args holds one argument block of
// the kind per member; nz_max sizes the shared memory of the column kernels
template <typename R>
int launch_kind_batch(int kind, int variant, int sub, const void* d_args, const int4* d_work,
                      int nwork, int nblocks, int nz_max, cudaStream_t st);

// Per-file batched launchers and grids behind the dispatch above.
template <typename R>
dim3 grid_fill(const FillArgs<R>& a);
template <typename R>
dim3 grid_flux(const FluxArgs<R>& a);
template <typename R>
dim3 grid_cells(const Layout& L);  // cells in 32 x 4 x 2 blocks
template <typename R>
dim3 grid_tend(const Layout& L);  // the tendency kernels' blocks
template <typename R>
dim3 grid_pd(const Layout& L);  // positive-definite outflow ratios
dim3 grid_clock();
template <typename R>
void batch_fill(const Batch<FillArgs<R>>& b, int nblocks, cudaStream_t st);
template <typename R>
void batch_flux(const Batch<FluxArgs<R>>& b, int nblocks, cudaStream_t st);
template <typename R>
void batch_pd(const Batch<PdArgs<R>>& b, int nblocks, cudaStream_t st);
template <typename R>
void batch_tend(const Batch<TendArgs<R>>& b, int variant, int sub, int nblocks, cudaStream_t st);
void batch_clock(const Batch<ClockArgs>& b, int nblocks, cudaStream_t st);
template <typename R>
int occupancy_tend(int variant, int sub);
template <typename R>
dim3 grid_uv(const Layout& L);  // faces 0..nx x 0..ny in 32 x 4 x 2 blocks (linearised u, v)
template <typename R>
dim3 grid_uv_fwd(const Layout& L);  // the forward u, v kernel's blocks
template <typename R>
dim3 grid_column(const Layout& L, int shape);
template <typename R>
void batch_uv(const Batch<AcouArgs<R>>& b, int nblocks, cudaStream_t st);
template <typename R>
int batch_column(const Batch<AcouArgs<R>>& b, int shape, int nz_max, int nblocks, cudaStream_t st);
template <typename R>
int occupancy_column(int shape, int nz_max);
template <typename R>
dim3 grid_kessler(const Layout& L, int nz_max);
template <typename R>
int batch_kessler(const Batch<KesArgs<R>>& b, int nz_max, int nblocks, cudaStream_t st);
template <typename R>
int occupancy_kessler(int nz_max);
template <typename R>
dim3 grid_sfc(const Layout& L, int sub, int nz_max);
template <typename R>
void batch_sfc(const Batch<SfcArgs<R>>& b, int sub, int nblocks, int nz_max, cudaStream_t st);
// sets the shared-memory limits of the level-parallel surface kernels
template <typename R>
int prepare_sfc(int nz);
// whether a column of nz levels needs the scratch buffer (sfc_scratch_count)
template <typename R>
bool sfc_needs_scratch(int nz);

// Tangent-linear (tl_) and adjoint (ad_) launches of the dynamics (lin.cu)
// and of the Kessler column (lin_kessler.cu): a is the forward argument block
// of the linearised launch, d the same block over the tangent or adjoint
// buffers.  The TL of the ghost fill and of the mass fluxes is the forward
// launch on d.  The column launches return 2 when nz exceeds
// lin_max_levels().
template <typename R>
void ad_fill(const FillArgs<R>& d, cudaStream_t st);
template <typename R>
void ad_flux(const FluxArgs<R>& d, cudaStream_t st);
template <typename R>
void tl_tend(const TendArgs<R>& a, const TendArgs<R>& d, cudaStream_t st);
template <typename R>
void ad_tend(const TendArgs<R>& a, const TendArgs<R>& d, cudaStream_t st);
template <typename R>
void tl_uv(const AcouArgs<R>& a, const AcouArgs<R>& d, cudaStream_t st);
// scratch cell fields of the gather-form adjoints (six, n3 each)
template <typename R>
struct LinScratch {
  R* f[6];
};
template <typename R>
void ad_uv(const AcouArgs<R>& a, const AcouArgs<R>& d, const LinScratch<R>& scr, cudaStream_t st);
template <typename R>
// with_forward: the launch also writes the forward column's outputs (the
// values the forward launch would write, bit for bit)
int tl_column(const AcouArgs<R>& a, const AcouArgs<R>& d, bool with_forward, cudaStream_t st);
template <typename R>
int ad_column(const AcouArgs<R>& a, const AcouArgs<R>& d, const LinScratch<R>& scr, cudaStream_t st);
// the same adjoint from the forward launch's outputs still in place (w_out,
// pi_next) with a.w_in / a.th_in pointing at the launch's inputs
template <typename R>
int ad_column_stored(const AcouArgs<R>& a, const AcouArgs<R>& d, const LinScratch<R>& scr, cudaStream_t st);
template <typename R>
void tl_kessler(const KesArgs<R>& a, const KesArgs<R>& d, cudaStream_t st);
template <typename R>
void ad_kessler(const KesArgs<R>& a, const KesArgs<R>& d, cudaStream_t st);
int lin_max_levels();
// shared-memory limits of the linearised column kernels for nz levels (once,
// outside any stream capture); 2 when nz exceeds lin_max_levels()
template <typename R>
int lin_prepare(int nz);
template <typename R>
int lin_kessler_prepare(int nz);
// copy `count` whole fields of n elements each (src[f] -> dst[f]) in one
// launch; 16-byte aligned pointers and n * sizeof(R) a multiple of 16, else
// nothing is launched and 1 is returned
constexpr int kCopyMax = 8;
template <typename R>
struct CopyJob {
  const R* src[kCopyMax];
  R* dst[kCopyMax];
  int count;
};
template <typename R>
int copy_fields(const CopyJob<R>& job, size_t n, cudaStream_t st);
// zero a cell field outside the interior cells (the pi' ghost ring, which no
// launch of a step reads or writes)
template <typename R>
void zero_ring(R* f, const Layout& L, cudaStream_t st);

template <typename R>
int launch_sfc(const SfcArgs<R>& a, cudaStream_t st);
template <typename R>
size_t sfc_scratch_count(const Layout& L);
void launch_clock(double* clock, double t, double t_lo, double t_hi, double dt, int advance,
                  cudaStream_t st);
template <typename R>
void launch_axpy(const R* x, const R* y, R a, R* out, size_t n, cudaStream_t st);

template <typename R>
void launch_fill_ghosts(const Layout& L, const GhostJob<R>& job, int open_x, int open_y,
                        cudaStream_t st);
template <typename R>
void launch_mass_flux(const Layout& L, const DBase<R>& b, const DMetric<R>& m, const R* u,
                      const R* v, const R* w, R* mfx, R* mfy, R* mfz, cudaStream_t st);
template <typename R>
void launch_pd_ratio(const TendArgs<R>& a, R* rv, R* rc, R* rr, cudaStream_t st);
// variant 0: one fused launch; 1: momentum and scalar launches
// variant: 0 fused, 1 momentum + scalar launches, 3 momentum only (the
// scalars then come from launch_tend_scal_tma)
template <typename R>
void launch_tendencies(const TendArgs<R>& a, int variant, cudaStream_t st);
// TMA-staged scalar tendencies (dyn_tend_tma.cu): a CTA per tile of
// kTtX x kTtY x kTtZ cells; tensor maps over the pitched fields with boxes
// mfx (kTtX + 4) x kTtY x kTtZ, mfy kTtX x (kTtY + 1) x kTtZ, mfz
// kTtX x kTtY x (kTtZ + 1), scalars (kTtX + 8) x (kTtY + 6) x (kTtZ + 6) for
// theta', qv, qc, qr (q[1..3] only with moisture).  No positive-definite
// moisture.
constexpr int kTtX = 32, kTtY = 4, kTtZ = 4;
template <typename R>
struct TendTmaParams {
  TendArgs<R> a;
  unsigned* err;  // set to 1 when a tile's loads did not arrive in time
  CUtensorMap mfx, mfy, mfz, q[4];
};
template <typename R>
size_t tend_scal_tma_smem();
template <typename R>
int prepare_tend_scal_tma();
template <typename R>
void launch_tend_scal_tma(const TendTmaParams<R>& p, cudaStream_t st);

template <typename R>
void launch_acoustic_coef(const Layout& L, const DBase<R>& b, const DMetric<R>& m, R* scratch,
                          R* rtjx, R* rtjy, R* kt3, R* aw, cudaStream_t st);
template <typename R>
// shape 0: 16 x 16 x 1 face tiles, 1: 32 x 2 x 4 (grids of few rows); the
// same values either way
void launch_acoustic_uv(const AcouArgs<R>& a, cudaStream_t st, int shape = 0);
// TMA variant of the column kernel (dyn_acou.cu): a CTA owns kTmaCX columns of
// one row; every input column block (levels -1..nz) arrives in shared memory
// by one bulk tensor load per field, then the five phases run from shared
// memory.  Tensor maps, one per input field, in this order:
enum {
  TC_U = 0, TC_RTJX, TC_V, TC_RTJY,  // faces: u, rtjx (x faces i0..), v, rtjy (rows j, j+1)
  TC_W, TC_PI, TC_TH, TC_TW, TC_TTH, TC_TPI, TC_AW, TC_KT3, TC_THBW, TC_DTHB,
  TC_QV, TC_QC, TC_QR, TC_QVB, TC_N
};
constexpr int kTmaCX = 16;
// box (x, y) extents of map f; the z extent is nz + 2 (levels -1 .. nz)
WFE_HD void tma_col_box(int f, int* bx, int* by) {
  *bx = (f == TC_U || f == TC_RTJX) ? kTmaCX + 4 : kTmaCX;
  *by = (f == TC_V || f == TC_RTJY) ? 2 : 1;
}
template <typename R>
struct TmaColParams {
  AcouArgs<R> a;
  unsigned* err;   // set to 1 when a tile's loads did not arrive in time
  int has_tpi;     // TC_TPI map valid
  CUtensorMap map[TC_N];
};
// Persistent, pipelined column kernel (dyn_acou_pipe.cu): one producer warp
// streams each tile's input boxes (the TC_* fields above, levels 0..nz-1 and
// w 0..nz) into a ring of shared-memory stages by bulk tensor loads while the
// consumer warps run the column phases of the tile before; the same
// expressions as the chunked kernel, bit for bit.  Maps are encoded with the
// boxes of acoustic_pipe_box for the chosen shape.
// The column inputs that depend on the level alone when the base state and
// the metric are horizontally uniform (flat ground, one map factor): the
// pipelined column kernels then read them from per-level tables, in this
// order, instead of streaming a box of each per tile.
enum { PF_RTJX = 0, PF_RTJY, PF_AW, PF_KT3, PF_THBW, PF_DTHB, PF_QVB, PF_N };
WFE_HD int pipe_prof_slot(int f) {
  switch (f) {
    case TC_RTJX: return PF_RTJX;
    case TC_RTJY: return PF_RTJY;
    case TC_AW: return PF_AW;
    case TC_KT3: return PF_KT3;
    case TC_THBW: return PF_THBW;
    case TC_DTHB: return PF_DTHB;
    case TC_QVB: return PF_QVB;
    default: return -1;
  }
}
template <typename R>
struct PipeColParams {
  AcouArgs<R> a;
  unsigned* err;   // set to 1 when a stage wait gave up
  int has_tpi;     // TC_TPI map valid
  const R* prof;   // PF_N tables of nz + 1 levels, or null (boxes for all)
  CUtensorMap map[TC_N];
};
int acoustic_pipe_shapes();
// box extents of field f (TC_*) for pipe shape `shape` and nz levels
void acoustic_pipe_box(int shape, int f, int nz, int* bx, int* by, int* bz);
// 0 when the shape's stages do not fit in shared memory
template <typename R>
size_t acoustic_pipe_smem(int shape, int nz, bool moist, bool tpi, bool prof = false);
// raises every shape's shared-memory limit to the largest layout it may use
template <typename R>
int prepare_acoustic_pipe(int nz);
// Returns 0 ok, 2 does not fit
template <typename R>
int launch_acoustic_column_pipe(const PipeColParams<R>& p, int shape, cudaStream_t st);
// The same pipeline feeding the parallel-solve column (level lanes own
// consecutive rows in registers, cyclic reduction across the lanes: equal to
// the Thomas kernels to rounding); its own shapes, boxes and layouts, the
// same params (maps encoded with acoustic_pipe_pcr_box).  prepare_acoustic_pipe
// raises these kernels' limits too.
int acoustic_pipe_pcr_shapes();
void acoustic_pipe_pcr_box(int shape, int f, int nz, int* bx, int* by, int* bz);
template <typename R>
size_t acoustic_pipe_pcr_smem(int shape, int nz, bool moist, bool tpi, bool prof = false);
template <typename R>
int launch_acoustic_column_pipe_pcr(const PipeColParams<R>& p, int shape, cudaStream_t st);
// Persistent, pipelined forward u, v kernel (dyn_acou_pipe.cu): tiles of
// kUvpX x kUvpY x kUvpZ faces; a producer warp streams each tile's boxes (the
// cell fields with a one-cell halo toward -x, -y and +-z, the face fields
// without) into a ring of shared-memory stages; interior faces are computed
// from shared memory with the u, v kernel's expressions (bit-identical),
// the lateral edge faces (radiation or periodic) by its global-memory path.
enum { UV_PI = 0, UV_PIP, UV_TH, UV_THB, UV_QV, UV_U, UV_TU, UV_V, UV_TV, UV_N };
constexpr int kUvpX = 32, kUvpY = 4, kUvpZ = 4;
// box extents of map f
WFE_HD void uv_pipe_box(int f, int* bx, int* by, int* bz) {
  const bool halo = f <= UV_QV;
  *bx = halo ? kUvpX + 4 : kUvpX;
  *by = halo ? kUvpY + 1 : kUvpY;
  *bz = halo ? kUvpZ + 2 : kUvpZ;
}
template <typename R>
struct PipeUvParams {
  AcouArgs<R> a;
  unsigned* err;
  CUtensorMap map[UV_N];
};
template <typename R>
int prepare_acoustic_uv_pipe();
// Returns 0 ok, 2 not usable
template <typename R>
int launch_acoustic_uv_pipe(const PipeUvParams<R>& p, cudaStream_t st);
// shared memory of the TMA column kernel for nz levels (0: does not fit)
template <typename R>
size_t acoustic_column_tma_smem(int nz);
template <typename R>
int prepare_acoustic_column_tma(int nz);
template <typename R>
int launch_acoustic_column_tma(const TmaColParams<R>& p, cudaStream_t st);

// shape: tile-shape index (columns x level lanes) in [0, acoustic_column_shapes());
// one that does not fit the column depth falls back to the first that does
template <typename R>
int launch_acoustic_column(const AcouArgs<R>& a, int shape, cudaStream_t st);
int acoustic_column_shapes();
// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) that never lowers the
// limit an earlier call set for the same kernel on the current device: cases
// of different depths in one process share the kernels, and a shallower
// case's set-up must not cut the limit a deeper case relies on
cudaError_t raise_smem_limit(const void* func, size_t bytes);
template <typename K>
cudaError_t raise_smem_limit(K* func, size_t bytes) {
  return raise_smem_limit(reinterpret_cast<const void*>(func), bytes);
}
// The fused substep kernel (u, v faces of the tile, then its columns), in
// acoustic_fused_shapes() tile shapes; theta'_in and theta'_out must be
// distinct buffers (pi', u and v always are).  Returns 0 ok, 2 too deep.
template <typename R>
int launch_acoustic_fused(const AcouArgs<R>& a, int f, cudaStream_t st);
int acoustic_fused_shapes();
int acoustic_fused_column_shape(int f);
template <typename R>
bool acoustic_fused_fits(int nz, int f);
template <typename R>
int prepare_acoustic_fused(int nz);
// The column kernel with contiguous level chunks per lane (fewer barriers),
// acoustic_chunked_shapes() shapes; same values as launch_acoustic_column.
template <typename R>
int launch_acoustic_column_chunked(const AcouArgs<R>& a, int f, cudaStream_t st);
int acoustic_chunked_shapes();
template <typename R>
bool acoustic_chunked_fits(int nz, int f);
// The column kernel with a parallel (partitioned + cyclic-reduction)
// tridiagonal solve, acoustic_pcr_shapes() shapes; the same rows as the
// other column kernels, the solution equal to theirs up to rounding.
template <typename R>
int launch_acoustic_column_pcr(const AcouArgs<R>& a, int f, cudaStream_t st);
int acoustic_pcr_shapes();
template <typename R>
bool acoustic_pcr_fits(int nz, int f);
// whether tile shape `shape` holds a column of nz levels in shared memory
template <typename R>
bool acoustic_column_fits(int nz, int shape);
template <typename R>
int prepare_acoustic_column(int nz);
template <typename R>
int prepare_kessler(int nz);

template <typename R>
int launch_kessler(const KesArgs<R>& a, cudaStream_t st);
// interior of a 3D field (nzl levels) or of a 2D field into a contiguous
// float32 (f32) or float64 device buffer in the Writer's layout (io.cu)
template <typename R>
void launch_pack_interior(const R* src, const Layout& L, int nzl, void* dst, bool f32,
                          cudaStream_t st);
template <typename R>
void launch_pack_interior2d(const R* src, const Layout& L, void* dst, bool f32, cudaStream_t st);
// a contiguous float32 (f32) or float64 interior block into a field's
// interior points (io.cu)
template <typename R>
void launch_unpack_interior(const void* src, const Layout& L, int nzl, R* dst, bool f32,
                            cudaStream_t st);
template <typename R>
void launch_absmax(const R* f, size_t n, unsigned int* result, cudaStream_t st);
// max |f| as float bits into mapped host memory; acc: two device words, zero
// before the first call and left zero by every call (phys_kessler.cu)
template <typename R>
void launch_absmax_to_host(const R* f, size_t n, unsigned int* acc, unsigned int* host_out,
                           cudaStream_t st);
template <typename R>
void launch_dry_mass(const Layout& L, const DBase<R>& b, const DMetric<R>& m, const R* pip,
                     const R* thp, const R* qv, const R* qc, const R* qr, int moist, R dx, R dy,
                     double* plane_sums, double* result, cudaStream_t st);

}  // namespace wfe
