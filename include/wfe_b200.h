/* wfe_b200 -- B200-native (sm_100a) implementation of the WFE per-step
 * dynamical core and column physics, behind a plain C ABI.
 *
 * The reference (Xassemblianist/WFE) has no plugin or FFI layer: its operator
 * API is the C++ free-function surface of src/dynamics/kernels.hpp:14-71,
 * src/physics/kessler.hpp:17-18 and src/physics/surface.hpp:20-44,
 * orchestrated by Integrator (src/dynamics/integrator.hpp:18-42) and set up by
 * src/main.cpp:245-383.  Each entry point below names the reference interface
 * it replaces.  All functions return WFE_OK (0) or an error code; the library
 * never exits the process (the reference prints and calls exit(1):
 * src/core/cuda_check.hpp:7-39).  wfe_last_error() returns the message of the
 * last failure on a context (or of the last failed creation for NULL).
 *
 * Layouts at the boundary are the reference's: WFE_LAYOUT_PADDED is the
 * GDims buffer (NX = nx+6, NY = ny+6, NZ = nz+7, ng = 3, i fastest;
 * src/core/grid.hpp:22-36); WFE_LAYOUT_INTERIOR is the Writer's interior
 * float layout (nz, or nz+1 for w, x ny x nx; src/io/writer.cpp:89-107).
 * Internally the fields are pitched for the B200; no device memory or torch
 * types cross this boundary.
 */
#ifndef WFE_B200_H
#define WFE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct wfe_ctx wfe_ctx;

enum {
  WFE_OK = 0,
  WFE_ERR_ARG = 1,     /* bad argument */
  WFE_ERR_CUDA = 2,    /* CUDA failure or no device (there is no CPU fallback) */
  WFE_ERR_CONFIG = 3,  /* case configuration error (reference: exit 1) */
  WFE_ERR_IO = 4,      /* input / boundary file error (reference: exit 1) */
  WFE_ERR_NAN = 5,     /* non-finite state (reference main: exit 2) */
  WFE_ERR_WABORT = 6   /* |w| above w_abort (reference main: exit 3) */
};
enum { WFE_F32 = 0, WFE_F64 = 1 };
enum { WFE_U = 0, WFE_V, WFE_W, WFE_THP, WFE_PIP, WFE_QV, WFE_QC, WFE_QR };
/* WFE_ROLE_LIN: the tangent-linear / adjoint field of the state (wfe_lin_enable) */
enum { WFE_ROLE_STATE = 0, WFE_ROLE_TEND = 1, WFE_ROLE_WORK = 2, WFE_ROLE_PIPREV = 3,
       WFE_ROLE_LIN = 4 };
enum { WFE_LAYOUT_PADDED = 0, WFE_LAYOUT_INTERIOR = 1 };
enum { WFE_DTYPE_F64 = 0, WFE_DTYPE_F32 = 1 };
enum { WFE_2D_RAIN = 0, WFE_2D_TSK = 1, WFE_2D_PBLH = 2, WFE_2D_T2M = 3, WFE_2D_U10 = 4 };

/* ------------------------------------------------------------- set-up */

/* Reads a case .ini plus "key=value" overrides and builds everything
 * src/main.cpp:248-383 builds before its time loop: grid, DynParams, Gal-Chen
 * metric (Metric::build, src/core/metric.cpp:12-168), base state
 * (BaseState::build, src/core/base_state.cpp:21-193), the initial state
 * (idealised or file mode), the boundary manager and the surface physics,
 * then uploads it to `device` (Integrator::init, integrator.cpp:43-69).
 * precision: WFE_F32 or WFE_F64 (the reference's WFE_DOUBLE build).
 * device < 0 builds the host set-up only (no GPU needed; the get_* calls
 * work, every device call returns WFE_ERR_CUDA). */
int wfe_case_create(const char* ini_path, const char* const* overrides, int n_overrides,
                    int precision, int device, wfe_ctx** out);
/* Same, from the text of a case file instead of a path. */
int wfe_case_create_text(const char* ini_text, const char* const* overrides, int n_overrides,
                         int precision, int device, wfe_ctx** out);
int wfe_ctx_destroy(wfe_ctx* ctx);
const char* wfe_last_error(const wfe_ctx* ctx);

/* dims: nx ny nz ng NX NY NZ; spacing: dx dy dz dt t_end zt */
int wfe_get_dims(const wfe_ctx* ctx, int dims[7]);
int wfe_get_spacing(const wfe_ctx* ctx, double out[6]);
/* flags: moisture microphysics pd_moist bc_x_open bc_y_open w_damping
 *        file_mode physics_on boundary_on acoustic_ns */
int wfe_get_flags(const wfe_ctx* ctx, int flags[10]);

/* Host copies of the set-up arrays (reference padded layout, FP64):
 * metric: 0..3 zeta_w zeta_c dzeta_c dzeta_w [NZ], 4..11 h hx hy hx_u hy_v
 * jac fcor mapf [NX*NY] (DevMetric, src/core/metric.hpp:16-30);
 * base: 0..8 thb pib rhob dthbdz thbw rhobw thvb thvbw qvb [NX*NY*NZ], 9 ub
 * [NZ] (DevProf, src/core/base_state.hpp:16-27).  These never touch the GPU. */
int wfe_get_metric(const wfe_ctx* ctx, int which, double* out);
int wfe_get_base(const wfe_ctx* ctx, int which, double* out);

/* --------------------------------------------------------- field I/O */

/* Field3D::upload / download (src/core/field3d.hpp:38-43) of one prognostic
 * field of a role: WFE_ROLE_STATE is Integrator::state() (time n),
 * WFE_ROLE_TEND the slow tendencies (u v w thp pip qv qc qr), WFE_ROLE_WORK
 * the acoustic work state, WFE_ROLE_PIPREV the pi' of the previous acoustic
 * substep (field ignored).  dtype: WFE_DTYPE_F64 / F32 of the host buffer. */
int wfe_field_upload(wfe_ctx* ctx, int role, int field, const void* host, int dtype, int layout);
int wfe_field_download(wfe_ctx* ctx, int role, int field, void* host, int dtype, int layout);
/* 2D fields (Integrator::rain, SfcPBL::tsk/pblh/t2m/u10) as padded NX*NY or
 * interior ny*nx */
int wfe_field2d_download(wfe_ctx* ctx, int which, void* host, int dtype, int layout);

/* The driver settings src/main.cpp reads besides the case (main.cpp:262-275,
 * 418-420): out_interval, diag_interval and w_abort [s, s, m/s] into
 * out[3]; out_dir into a caller buffer of out_dir_len bytes (truncated,
 * always terminated). */
int wfe_get_run_config(const wfe_ctx* ctx, double out[3], char* out_dir, int out_dir_len);

/* ----------------------------------------------------------- stepping */

/* Integrator::step(dt, t) (src/dynamics/integrator.cpp:71-111): one
 * Wicker-Skamarock RK3 large step with split-explicit acoustic substeps, then
 * Kessler and the surface physics; boundary relaxation targets are switched
 * as BdyManager::update (src/dynamics/boundary.cpp:83-89) does. */
int wfe_step(wfe_ctx* ctx, double dt, double t);
/* nsteps such steps from t0, replayed from captured CUDA graphs (the device
 * clock advances inside the graph); asynchronous until wfe_sync. */
int wfe_run(wfe_ctx* ctx, int nsteps, double dt, double t0);
int wfe_sync(wfe_ctx* ctx);
/* field_absmax (src/dynamics/kernels.cu:967-979): max |f| of a state field,
 * NaN reported as a value above every finite one. */
int wfe_absmax(wfe_ctx* ctx, int field, float* out);
/* The same value without stopping the stream (no counterpart in the
 * reference): wfe_absmax_begin enqueues the reduction and its copy into
 * page-locked slot `slot` (0 or 1) behind the work already queued;
 * wfe_absmax_end waits for that slot and returns the value.  A driver loop
 * can enqueue step s + 1 before reading step s's |w|, so the GPU never waits
 * for the host; its watchdog then trips one step later. */
int wfe_absmax_begin(wfe_ctx* ctx, int field, int slot);
int wfe_absmax_end(wfe_ctx* ctx, int slot, float* out);
/* FP64 dry-air mass of the state [kg] (no reference counterpart). */
int wfe_dry_mass(wfe_ctx* ctx, double* out);
/* launches of the package's own kernels per large step in the last
 * wfe_step / wfe_run */
long wfe_launches_per_step(const wfe_ctx* ctx);
/* The kernel variants the case runs (no reference counterpart): out[0] the
 * tendency variant, out[1] the acoustic column variant, out[2] the forward
 * u, v variant (all -1 before the first wfe_step / wfe_run tunes them), and
 * out[3] a bit set of the per-level tables in use where the set-up is
 * horizontally uniform: 1 the column coefficients (read by the pipelined
 * column kernels, variants 13-15 and 19-22), 2 the base state (read by the
 * mass-flux, Kessler and u, v kernels). */
int wfe_case_variants(const wfe_ctx* ctx, int out[4]);

/* nsteps graph-replayed steps timed with CUDA events recorded on the
 * library's own stream; *ms = elapsed device time (no reference counterpart;
 * the reference times sections with host clocks under WFE_PROF,
 * src/dynamics/integrator.cpp:18-40). */
int wfe_time_run(wfe_ctx* ctx, int nsteps, double dt, double t0, double* ms);
/* One step captured as a CUDA graph with an event node before and after
 * every kernel launch, replayed once; per kernel name (comma-separated in
 * names_csv) the summed device time and launch count.  Advances the state
 * like wfe_step. */
int wfe_kernel_times(wfe_ctx* ctx, double dt, double t, int cap, double* total_ms, int* counts,
                     char* names_csv, int names_len, int* n_out);

/* Asynchronous snapshot (no reference counterpart; replaces the Writer's
 * blocking cudaMemcpy of a padded field and its host repack,
 * src/io/writer.cpp:89-107).  Each requested field -- WFE_U..WFE_QR, or
 * WFE_SNAP_2D + WFE_2D_* -- is packed on the device into the interior layout
 * (float32 for WFE_DTYPE_F32, else float64) on the library's stream, in order
 * with the steps already issued, then copied into host[q] on a separate copy
 * stream, so steps issued afterwards overlap the transfer.  The host buffers
 * (interior_count elements each) are complete after wfe_snapshot_wait; a new
 * wfe_snapshot_begin waits for the previous one first.  For the copies to be
 * asynchronous the buffers must be page-locked: wfe_host_alloc. */
enum { WFE_SNAP_2D = 100 };
int wfe_snapshot_begin(wfe_ctx* ctx, int n, const int* fields, void* const* host, int dtype);
int wfe_snapshot_wait(wfe_ctx* ctx);
void* wfe_host_alloc(size_t bytes); /* page-locked host memory, NULL on failure */
int wfe_host_free(void* p);

/* ------------------------------------------------- operator-level API */
/* apply_bcs (src/dynamics/kernels.cu:805-835) on the state */
int wfe_op_apply_bcs(wfe_ctx* ctx);
/* compute_mass_fluxes + compute_divergence + compute_tendencies (+ bdy_relax
 * when a boundary is set, at time t: BdyManager::tfrac) (kernels.cu:837-913,
 * 981-995): state -> tend */
int wfe_op_tendencies(wfe_ctx* ctx, double dt, double t);
/* nsub x acoustic_substep (kernels.cu:929-965) starting from a copy of the
 * state (as Integrator::step does at a stage): result in WFE_ROLE_WORK */
int wfe_op_acoustic(wfe_ctx* ctx, double dtau, int nsub);
/* update_moisture_stage (kernels.cu:997-1005): work.q = state.q + dt tend.q */
int wfe_op_moisture_stage(wfe_ctx* ctx, double dt);
/* kessler_step (src/physics/kessler.cu:143-149) on the state */
int wfe_op_kessler(wfe_ctx* ctx, double dt);
/* SfcPBL::step (src/physics/surface.cu:499-514) on the state, t = end of step */
int wfe_op_sfc(wfe_ctx* ctx, double dt, double t);

/* BdyManager with caller-supplied targets (u v thp pip qv, padded layout,
 * FP64) and weights (padded NX*NY): lo/hi valid at t_lo/t_hi. */
int wfe_set_boundary(wfe_ctx* ctx, const double* const lo[5], const double* const hi[5],
                     const double* wgt, double t_lo, double t_hi);
/* BdyManager::init's relaxation weights (src/dynamics/boundary.cpp:24-39),
 * padded NX*NY FP64 into `out`: cos^2 ramp over `width` rows next to the
 * open edges with 1/tau at the edge, and 1/nudge_tau (0: none) everywhere
 * as the interior analysis-nudging floor.  Host only: works on a context
 * created without a device. */
int wfe_bdy_weights(const wfe_ctx* ctx, int width, double tau, double nudge_tau, double* out);
/* No counterpart in the reference: switches the relaxation of
 * wfe_set_boundary off again (the next step has no Davies / nudging term),
 * e.g. to run the tangent-linear and adjoint runs of the next analysis
 * cycle after a nudged forecast. */
int wfe_clear_boundary(wfe_ctx* ctx);
/* SfcPBL::init (surface.cu:440-482) from interior ny*nx FP64 arrays. */
int wfe_set_physics(wfe_ctx* ctx, const double* tsk, const double* land, const double* lat,
                    const double* lon, const double* soilw, double start_hour_utc, int doy,
                    int nonlocal);

/* ------------------------------------- tangent-linear and adjoint runs */
/* No counterpart in the reference.  Linearisation of the model step (5th-
 * order advection of momentum, theta' and the moisture species with the
 * Gal-Chen metric, Rayleigh sponge, constant-K diffusion, Coriolis, the
 * split-explicit acoustic step with its implicit w - pi' columns and moist
 * buoyancy, open and periodic lateral boundaries, the Kessler column with the
 * mixed-phase blend) about the forward trajectory; cases with the
 * positive-definite moisture limiter, Davies relaxation, surface physics or
 * w damping are refused.  wfe_lin_enable gives the context a linearised field for every
 * prognostic (WFE_ROLE_LIN in wfe_field_upload / wfe_field_download), all
 * zero.  wfe_tl_run advances the state x0 -> xN and the linearised field
 * dx0 -> dxN = M dx0 (M: the Jacobian of the N steps at x0).  wfe_ad_run
 * advances the state x0 -> xN with checkpoints of the state every
 * `checkpoint_every` steps, then sweeps back, recomputing between
 * checkpoints: the linearised field holds dJ/dxN on entry and M^T dJ/dxN =
 * dJ/dx0 on exit. */
int wfe_lin_enable(wfe_ctx* ctx);
int wfe_lin_zero(wfe_ctx* ctx);
int wfe_tl_run(wfe_ctx* ctx, int nsteps, double dt, double t0);
/* checkpoint_every <= 0: the longest interval whose undo log (every buffer
 * each launch of a step overwrites) fits in 80 % of the free device memory;
 * when the whole run fits, nothing is recomputed. */
int wfe_ad_run(wfe_ctx* ctx, int nsteps, double dt, double t0, int checkpoint_every);

/* --------------------------------------------------- batched ensembles */
/* No counterpart in the reference, whose ensemble driver runs one process per
 * member (tools/run_ensemble.py:61-64).  An ensemble advances member contexts
 * of possibly different grid sizes together: every kernel of the RK3 step is
 * one batched launch over a member x tile work list, and the whole step with
 * its acoustic substeps is captured in one CUDA graph per rotation phase.
 * Members are contexts created with a device (same device, same precision,
 * same moisture / microphysics / positive-definite / boundary / surface /
 * acoustic_ns settings, same step count so far); they stay owned by the
 * caller, must outlive the ensemble, and keep serving field transfers,
 * wfe_absmax, wfe_dry_mass and so on.  Errors are reported through
 * wfe_last_error(NULL). */
typedef struct wfe_ens wfe_ens;
int wfe_ensemble_create(wfe_ctx* const* members, int n, wfe_ens** out);
int wfe_ensemble_destroy(wfe_ens* ens);
/* nsteps steps of every member from t0 with a common dt; boundary files of
 * file-mode members are switched between graph replays as wfe_run does;
 * asynchronous until wfe_ensemble_sync (member transfers wait for it too). */
int wfe_ensemble_run(wfe_ens* ens, int nsteps, double dt, double t0);
/* one step with direct batched launches (no graph) */
int wfe_ensemble_step(wfe_ens* ens, double dt, double t);
int wfe_ensemble_sync(wfe_ens* ens);
/* nsteps graph-replayed steps timed with CUDA events on the ensemble's stream */
int wfe_ensemble_time_run(wfe_ens* ens, int nsteps, double dt, double t0, double* ms);
/* launches per step; tuned variants: tendencies split, acoustic column tile
 * shape, and the mode (0 batched launches, one block per work item; 1
 * batched on a persistent grid; 2 every member's own graph on its own
 * stream, the members running concurrently; 3 every member's own graphs,
 * one member after another).  The first run of 19 or more steps times the
 * batched, concurrent and one-after-another modes on real steps (after three
 * warm-up steps of each: two timed steps batched, then four concurrent and
 * four one after another, in the order concurrent, sequential, sequential,
 * concurrent so that a drift of the step cost weighs on both) and keeps the
 * fastest: all give the same values, bit for bit.  WFE_ENSEMBLE_MODE =
 * batched | members | sequential forces one. */
long wfe_ensemble_launches_per_step(const wfe_ens* ens);
int wfe_ensemble_variants(const wfe_ens* ens, int out[3]);

/* ------------------------------------------- allocation-free variant */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory -- a diagnostics hook running inside another framework's CUDA stream
 * capture, where cudaMalloc is illegal, or a process whose device memory
 * belongs to a fixed-budget pool allocator -- this computes the dry-air mass
 * wfe_dry_mass reports, from device fields the caller owns, and allocates
 * nothing: its per-level partial sums live in a file-scope __device__ array of
 * WFE_NOALLOC_MAX_LEVELS doubles (8 KB, held by every GPU that loads the
 * library until exit).  Inputs are FP64 device arrays in the reference padded
 * layout (3D: (nx+6)*(ny+6)*(nz+7); jac: (nx+6)*(ny+6); dzeta_c: nz+7); qv, qc,
 * qr may be NULL for a dry state; out is a device double.  The call is
 * asynchronous on `stream` (a cudaStream_t, NULL for the legacy stream).
 * nz > WFE_NOALLOC_MAX_LEVELS is rejected with WFE_ERR_ARG and a message in
 * wfe_last_error(NULL).  The first call in a CUDA context (normally the
 * device's primary context) looks up the array's device address in that
 * context, with the caller's device current; make it before any stream
 * capture.  All calls in a context share the array: calls that overlap on the
 * GPU (different streams, or other host threads) race and must be serialised
 * by the caller. */
#define WFE_NOALLOC_MAX_LEVELS 1024
int wfe_dry_mass_noalloc(int nx, int ny, int nz, double dx, double dy, const double* pib,
                         const double* thb, const double* pip, const double* thp, const double* qv,
                         const double* qc, const double* qr, const double* jac,
                         const double* dzeta_c, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
