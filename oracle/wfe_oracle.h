/* CPU FP64 oracle for WFE's per-step hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain restatement of the reference algorithm (Xassemblianist/WFE) on the
 * reference's own padded C-grid layout, used by tests/ as the checker, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product
 * (wfe_b200/) never links or calls it.
 *
 * Parity: pinned against golden vectors produced by the reference's own FP64
 * build (tests/golden/, generated by tests/golden/make_golden.py from
 * oracle/_ref/, which oracle/Makefile compiles from the reference sources).
 *
 * Layout: every 3D array has NX*NY*NZ doubles, NX = nx+2ng, NY = ny+2ng,
 * NZ = nz+1+2ng, ng = 3, i fastest: ((k+ng)*NY + (j+ng))*NX + (i+ng)
 * (src/core/grid.hpp:22-36).  2D arrays are NX*NY, 1D vertical arrays NZ.
 */
#ifndef WFE_ORACLE_H
#define WFE_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, nz, ng, NX, NY, NZ;
  double dx, dy, dz;
} orc_grid;

/* src/dynamics/params.hpp:8-25 */
typedef struct {
  double diff_K, coriolis_f;
  int coriolis_use_ub;
  double rayleigh_zd, rayleigh_alpha;
  int acoustic_ns;
  double acoustic_beta, acoustic_smdiv;
  int bc_x_open, bc_y_open;
  double cstar;
  int moisture, microphysics, pd_moist, w_damping;
  double w_abort;
} orc_params;

/* src/core/metric.hpp:16-30 */
typedef struct {
  double *zeta_w, *zeta_c, *dzeta_c, *dzeta_w;
  double *h, *hx, *hy, *hx_u, *hy_v, *jac, *fcor, *mapf;
  double zt;
} orc_metric;

/* src/core/base_state.hpp:16-27 */
typedef struct {
  double *thb, *pib, *rhob, *dthbdz, *thbw, *rhobw, *thvb, *thvbw, *qvb;
  double *ub;
} orc_base;

typedef struct {
  double *u, *v, *w, *thp, *pip, *qv, *qc, *qr;
} orc_state;

/* metric options (src/core/metric.cpp:24-145) */
typedef struct {
  int stretch;              /* 0 none, 1 geometric */
  double dz0, dz_ratio, dz_max;
  int terrain;              /* 0 none, 1 schaer, 2 gauss, 3 file */
  double h0, a, lam, xc, yc, ya;
  double coriolis_f;
  const double *h_file, *fcor_file, *mapf_file; /* interior ny*nx, or NULL */
} orc_metric_cfg;

/* base-state options (src/core/base_state.cpp:25-192) */
typedef struct {
  int profile;              /* 0 isentropic, 1 constant_N, 2 wk82, 3 file */
  double theta0, bv_N;
  int wind_profile;         /* 0 const, 1 tanh, 2 linear (extension) */
  double wind_u, wind_us, wind_zs, wind_offset;
  int np_prof;              /* file profile tables */
  const double *prof_z, *prof_th, *prof_qv, *prof_u;
} orc_base_cfg;

/* ---------------------------------------------------------------- set-up
 * orc_metric_build / orc_base_build fill arrays the caller allocated
 * (NZ doubles for vertical arrays, NX*NY for 2D, NX*NY*NZ for 3D). */
void orc_grid_make(orc_grid* g, int nx, int ny, int nz, double dx, double dy, double dz);
size_t orc_npts(const orc_grid* g);
void orc_metric_build(const orc_grid* g, const orc_metric_cfg* c, orc_metric* m);
/* returns has_moisture */
int orc_base_build(const orc_grid* g, const orc_base_cfg* c, const orc_metric* m, orc_base* b);

/* initial conditions (src/main.cpp:28-195) */
void orc_ic_bubble(const orc_grid* g, const orc_metric* m, double dth, double xc, double yc,
                   double zc, double xr, double yr, double zr, double* thp);
void orc_ic_wind(const orc_grid* g, const orc_base* b, double* u);
void orc_ic_moisture(const orc_grid* g, const orc_base* b, double* qv);
void orc_ic_from_input(const orc_grid* g, const orc_base* b, const double* in_u,
                       const double* in_v, const double* in_th, const double* in_pi,
                       const double* in_qv, orc_state* s);
void orc_ic_perturb(const orc_grid* g, double amp, unsigned seed, double* thp);
/* Lambert conformal map factor at the interior points (src/main.cpp:326-340) */
void orc_lambert_mapf(int n, const double* lat, double lat1, double lat2, double* mapf);

/* ------------------------------------------------------------- operators */
void orc_apply_bcs(const orc_grid* g, const orc_params* p, orc_state* s);
void orc_bc_field(const orc_grid* g, const orc_params* p, double* f, int kind);
void orc_mass_fluxes(const orc_grid* g, const orc_base* b, const orc_metric* m,
                     const orc_state* s, double* mfx, double* mfy, double* mfz);
void orc_divergence(const orc_grid* g, const orc_metric* m, const double* mfx,
                    const double* mfy, const double* mfz, double* div);
/* pd scratch: 4 arrays of npts (fx, fy, fz, ratio), or NULL */
void orc_tendencies(const orc_grid* g, const orc_base* b, const orc_metric* m,
                    const orc_params* p, double dt, const orc_state* s, const double* mfx,
                    const double* mfy, const double* mfz, const double* div, orc_state* tend,
                    double* const* pd);
void orc_bdy_relax(const orc_grid* g, const orc_state* s, double* const* lo,
                   double* const* hi, double tf, const double* wgt, orc_state* tend);
void orc_acoustic_coef(const orc_grid* g, const orc_base* b, const orc_metric* m,
                       double* rtjx, double* rtjy, double* kt3, double* aw);
void orc_acoustic_substep(const orc_grid* g, const orc_base* b, const orc_metric* m,
                          const orc_params* p, double dtau, orc_state* s,
                          const orc_state* tend, double* piprev, const double* rtjx,
                          const double* rtjy, const double* kt3, const double* aw);
void orc_moisture_stage(const orc_grid* g, const orc_state* s0, const orc_state* tend,
                        double dt, orc_state* out);
void orc_kessler(const orc_grid* g, const orc_base* b, const orc_metric* m, double dt,
                 orc_state* s, double* rain);
float orc_absmax(const double* f, size_t n);
/* dry-air mass  sum rho_d J dx dy dzeta over the interior, with rho_d from the
 * full Exner pressure and virtual temperature (diagnostic; FP64) */
double orc_dry_mass(const orc_grid* g, const orc_base* b, const orc_metric* m,
                    const orc_state* s);

/* --------------------------------------------- surface layer / PBL / soil */
typedef struct {
  double *km, *tsk, *tdeep, *land, *lat, *lon, *soilw, *cdv, *pblh, *t2m, *u10, *soilt;
  double start_hour;
  int doy, nonlocal;
} orc_sfc;
/* allocate and fill from interior 2D inputs (src/physics/surface.cu:440-482) */
void orc_sfc_init(const orc_grid* g, orc_sfc* s, const double* tsk, const double* land,
                  const double* lat, const double* lon, const double* soilw,
                  double start_hour, int doy, int nonlocal);
void orc_sfc_free(orc_sfc* s);
void orc_sfc_step(const orc_grid* g, const orc_base* b, const orc_metric* m, orc_sfc* sf,
                  double dt, double t, orc_state* st);

/* Davies weights (src/dynamics/boundary.cpp:24-42) */
void orc_bdy_weights(const orc_grid* g, const orc_params* p, int bdy_width, double bdy_tau,
                     double nudge_tau, double* wgt);

/* ------------------------------------------------------------ integrator */
typedef struct orc_integ orc_integ;
orc_integ* orc_integ_create(const orc_grid* g, const orc_base* b, const orc_metric* m,
                            const orc_params* p);
void orc_integ_free(orc_integ* it);
orc_state* orc_integ_state(orc_integ* it);
double* orc_integ_rain(orc_integ* it);
/* boundary targets (5 fields each: u, v, thp, pip, qv) held by the caller;
 * tf(t) = clamp((t - t_lo) / (t_hi - t_lo), 0, 1) as BdyManager::tfrac */
void orc_integ_set_bdy(orc_integ* it, double* const* lo, double* const* hi, const double* wgt,
                       double t_lo, double t_hi);
void orc_integ_set_sfc(orc_integ* it, orc_sfc* sf);
void orc_integ_step(orc_integ* it, double dt, double t);

#ifdef __cplusplus
}
#endif
#endif
