/* CPU FP64 oracle for WFE's per-step hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Restates the reference algorithm (Xassemblianist/WFE) loop by loop on the
 * reference's padded layout, keeping the reference's in-place updates, ghost
 * fill order and ghost staleness (which the results depend on).  Citations are
 * path:line in the reference project.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load this library; the product never
 * does.  Parity of this oracle is pinned against golden vectors from the
 * reference's own FP64 build (tests/golden/).
 *
 * Written in a C subset of C++ so that the ensemble perturbation can use the
 * same standard-library generator (std::mt19937 + std::normal_distribution)
 * the reference calls (src/main.cpp:105-144).
 */
#include "wfe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <random>

/* ------------------------------------------------------------- constants */
/* src/core/constants.hpp:7-17 */
static const double GRAV = 9.81, CP = 1004.5, RD = 287.04, CV = 1004.5 - 287.04;
static const double P00 = 1.0e5, LV = 2.5e6, LF = 3.34e5, LS = 2.5e6 + 3.34e5;
static const double RV = 461.5, EPS61 = 0.61, TFRZ = 273.15;

#define I3(g, i, j, k) \
  ((((size_t)((k) + (g)->ng)) * (size_t)(g)->NY + (size_t)((j) + (g)->ng)) * (size_t)(g)->NX + (size_t)((i) + (g)->ng))
#define I2(g, i, j) ((size_t)((j) + (g)->ng) * (size_t)(g)->NX + (size_t)((i) + (g)->ng))

static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }
static double dmin(double a, double b) { return a < b ? a : b; }
static double dmax(double a, double b) { return a > b ? a : b; }

/* src/core/thermo.hpp:11-26 (device variant, clamped denominator) */
static double qsat_water(double p, double T) {
  double es = 610.78 * exp(17.269 * (T - 273.16) / (T - 35.86));
  double den = p - es;
  if (den < 1.0) den = 1.0;
  return 0.622 * es / den;
}
static double qsat_icep(double p, double T) {
  double es = 610.78 * exp(21.875 * (T - 273.16) / (T - 7.66));
  double den = p - es;
  if (den < 1.0) den = 1.0;
  return 0.622 * es / den;
}

/* ------------------------------------------------------------------ grid */
void orc_grid_make(orc_grid* g, int nx, int ny, int nz, double dx, double dy, double dz) {
  /* src/core/grid.hpp:34-36 */
  g->nx = nx; g->ny = ny; g->nz = nz; g->ng = 3;
  g->NX = nx + 6; g->NY = ny + 6; g->NZ = nz + 1 + 6;
  g->dx = dx; g->dy = dy; g->dz = dz;
}
size_t orc_npts(const orc_grid* g) { return (size_t)g->NX * g->NY * g->NZ; }

/* ---------------------------------------------------------------- metric */
static double terrain_height(const orc_metric_cfg* c, double x, double y) {
  /* src/core/metric.cpp:72-84 */
  const double pi = 3.14159265358979323846;
  if (c->terrain == 1) {
    double xr = x - c->xc;
    double env = exp(-(xr / c->a) * (xr / c->a));
    double cs = cos(pi * xr / c->lam);
    return c->h0 * env * cs * cs;
  }
  if (c->terrain == 2) {
    double xr = (x - c->xc) / c->a, yr = (y - c->yc) / c->ya;
    return c->h0 * exp(-xr * xr - yr * yr);
  }
  return 0.0;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

void orc_metric_build(const orc_grid* g, const orc_metric_cfg* c, orc_metric* m) {
  const int NZ = g->NZ, nz = g->nz, ng = g->ng;

  /* w-level heights: uniform or geometric stretch (metric.cpp:24-38) */
  double* zw = dalloc(nz + 1);
  if (c->stretch) {
    double d = c->dz0;
    for (int k = 1; k <= nz; ++k) {
      zw[k] = zw[k - 1] + d;
      d = dmin(d * c->dz_ratio, c->dz_max);
    }
  } else {
    for (int k = 0; k <= nz; ++k) zw[k] = (double)k * g->dz;
  }
  m->zt = zw[nz];
  /* linear extension into the ghosts (metric.cpp:41-56) */
  for (int kk = 0; kk < NZ; ++kk) {
    int k = kk - ng;
    double a, b;
    for (int s = 0; s < 2; ++s) {
      int q = k + s;
      double z;
      if (q < 0) z = zw[0] + (double)q * (zw[1] - zw[0]);
      else if (q > nz) z = zw[nz] + (double)(q - nz) * (zw[nz] - zw[nz - 1]);
      else z = zw[q];
      if (s == 0) a = z; else b = z;
    }
    m->zeta_w[kk] = a;
    m->zeta_c[kk] = 0.5 * (a + b);
  }
  for (int kk = 0; kk < NZ - 1; ++kk) m->dzeta_c[kk] = m->zeta_w[kk + 1] - m->zeta_w[kk];
  m->dzeta_c[NZ - 1] = m->dzeta_c[NZ - 2];
  for (int kk = 1; kk < NZ; ++kk) m->dzeta_w[kk] = m->zeta_c[kk] - m->zeta_c[kk - 1];
  m->dzeta_w[0] = m->dzeta_w[1];
  free(zw);

  const double zt = m->zt;
  if (c->terrain == 3) {
    /* interior copy with edge clamping, numerical slopes (metric.cpp:87-110) */
    for (int j = -ng; j < g->ny + ng; ++j)
      for (int i = -ng; i < g->nx + ng; ++i)
        m->h[I2(g, i, j)] = c->h_file[(size_t)clampi(j, 0, g->ny - 1) * g->nx + clampi(i, 0, g->nx - 1)];
    for (int j = -ng; j < g->ny + ng; ++j)
      for (int i = -ng; i < g->nx + ng; ++i) {
        size_t q = I2(g, i, j);
        m->jac[q] = (zt - m->h[q]) / zt;
        int im = i > -ng ? i - 1 : i, ip = i < g->nx + ng - 1 ? i + 1 : i;
        int jm = j > -ng ? j - 1 : j, jp = j < g->ny + ng - 1 ? j + 1 : j;
        m->hx[q] = (m->h[I2(g, ip, j)] - m->h[I2(g, im, j)]) / ((double)(ip - im) * g->dx);
        m->hy[q] = (m->h[I2(g, i, jp)] - m->h[I2(g, i, jm)]) / ((double)(jp - jm) * g->dy);
        m->hx_u[q] = (i == im) ? 0.0 : (m->h[q] - m->h[I2(g, im, j)]) / g->dx;
        m->hy_v[q] = (j == jm) ? 0.0 : (m->h[q] - m->h[I2(g, i, jm)]) / g->dy;
      }
  } else {
    /* analytic terrain at every padded column (metric.cpp:111-123) */
    for (int j = -ng; j < g->ny + ng; ++j)
      for (int i = -ng; i < g->nx + ng; ++i) {
        double x = ((double)i + 0.5) * g->dx, y = ((double)j + 0.5) * g->dy;
        size_t q = I2(g, i, j);
        m->h[q] = terrain_height(c, x, y);
        m->jac[q] = (zt - m->h[q]) / zt;
        m->hx[q] = (terrain_height(c, x + g->dx, y) - terrain_height(c, x - g->dx, y)) / (2.0 * g->dx);
        m->hy[q] = (terrain_height(c, x, y + g->dy) - terrain_height(c, x, y - g->dy)) / (2.0 * g->dy);
        m->hx_u[q] = (terrain_height(c, x, y) - terrain_height(c, x - g->dx, y)) / g->dx;
        m->hy_v[q] = (terrain_height(c, x, y) - terrain_height(c, x, y - g->dy)) / g->dy;
      }
  }
  /* Coriolis and map factor (metric.cpp:125-145) */
  for (int j = -ng; j < g->ny + ng; ++j)
    for (int i = -ng; i < g->nx + ng; ++i) {
      size_t q = I2(g, i, j);
      size_t src = (size_t)clampi(j, 0, g->ny - 1) * g->nx + clampi(i, 0, g->nx - 1);
      m->fcor[q] = c->fcor_file ? c->fcor_file[src] : c->coriolis_f;
      m->mapf[q] = c->mapf_file ? c->mapf_file[src] : 1.0;
    }
}

/* ------------------------------------------------------------ base state */
typedef struct {
  const orc_base_cfg* c;
} theta_ctx;

static double table_lookup(const orc_base_cfg* c, const double* tab, double z) {
  /* base_state.cpp:104-113 */
  double dzt = c->prof_z[1] - c->prof_z[0];
  double s = (z - c->prof_z[0]) / dzt;
  int it = (int)s;
  if (it < 0) it = 0;
  if (it > c->np_prof - 2) it = c->np_prof - 2;
  double f = s - it;
  return tab[it] * (1 - f) + tab[it + 1] * f;
}

static const double WK_ZTR = 12000.0, WK_THTR = 343.0, WK_TTR = 213.0, WK_QVMAX = 0.014;

static double theta_at(const orc_base_cfg* c, double z) {
  /* base_state.cpp:118-126 */
  if (c->profile == 3) return table_lookup(c, c->prof_th, z);
  if (c->profile == 2) {
    if (z <= WK_ZTR) return 300.0 + (WK_THTR - 300.0) * pow(z / WK_ZTR, 1.25);
    return WK_THTR * exp(GRAV * (z - WK_ZTR) / (CP * WK_TTR));
  }
  if (c->profile == 1) return c->theta0 * exp(c->bv_N * c->bv_N * z / GRAV);
  return c->theta0;
}

static double relhum_at(double z) {
  if (z <= WK_ZTR) return 1.0 - 0.75 * pow(z / WK_ZTR, 1.25);
  return 0.25;
}

static double qsat_host(double p, double T) { /* base_state.cpp:78-81 (no clamp) */
  double es = 610.78 * exp(17.269 * (T - 273.16) / (T - 35.86));
  return 0.622 * es / (p - es);
}

static void integrate_exner(double* pit, const double* thv, int n, int i0) {
  /* hydrostatic Exner integration on the 1 m table (base_state.cpp:143-153) */
  pit[i0] = 1.0;
  for (int it = i0 + 1; it < n; ++it) pit[it] = pit[it - 1] - GRAV * 1.0 / (CP * (0.5 * (thv[it - 1] + thv[it])));
  for (int it = i0 - 1; it >= 0; --it) pit[it] = pit[it + 1] + GRAV * 1.0 / (CP * (0.5 * (thv[it] + thv[it + 1])));
}

static double tab_interp(const double* tab, int n, double zmin, double z) {
  /* base_state.cpp:180-187 */
  double s = (z - zmin) / 1.0;
  int it = (int)s;
  if (it < 0) it = 0;
  if (it > n - 2) it = n - 2;
  double f = s - it;
  return tab[it] * (1 - f) + tab[it + 1] * f;
}

static double density(double pi, double thv) { /* base_state.cpp:188-191 */
  return P00 * pow(pi, CV / RD) / (RD * thv);
}

int orc_base_build(const orc_grid* g, const orc_base_cfg* c, const orc_metric* m, orc_base* b) {
  const int wk82 = c->profile == 2, file = c->profile == 3;
  const int moist = wk82 || file;

  /* 1 m table spanning the ghosts (base_state.cpp:133-141) */
  double zmin = -(double)(g->ng + 1) * g->dz * 4 - 100.0;
  double zmax = m->zt + (double)(g->ng + 1) * g->dz * 4 + 100.0;
  int ntab = (int)((zmax - zmin) / 1.0) + 2;
  int i0 = (int)(-zmin / 1.0);
  double* pit = dalloc(ntab);
  double* qvt = dalloc(ntab);
  double* thvt = dalloc(ntab);
  for (int it = 0; it < ntab; ++it) thvt[it] = theta_at(c, zmin + it * 1.0);
  integrate_exner(pit, thvt, ntab, i0);
  if (wk82) {
    /* moist theta_v - Exner iteration (base_state.cpp:156-170) */
    for (int iter = 0; iter < 5; ++iter) {
      for (int it = 0; it < ntab; ++it) {
        double z = zmin + it * 1.0;
        double th = theta_at(c, z), pi = pit[it];
        double T = th * pi;
        double p = P00 * pow(pi, CP / RD);
        double qv = dmin(relhum_at(z) * qsat_host(p, T), WK_QVMAX);
        if (z < 0) qv = qvt[it > 0 ? it : 0];
        qvt[it] = qv;
        thvt[it] = th * (1.0 + EPS61 * qv);
      }
      integrate_exner(pit, thvt, ntab, i0);
    }
  } else if (file) {
    for (int it = 0; it < ntab; ++it) {
      double z = zmin + it * 1.0;
      qvt[it] = dmax(0.0, table_lookup(c, c->prof_qv, z));
      thvt[it] = theta_at(c, z) * (1.0 + EPS61 * qvt[it]);
    }
    integrate_exner(pit, thvt, ntab, i0);
  }

  /* every padded point, at its physical height (base_state.cpp:197-218) */
  for (int k = -g->ng; k < g->nz + 1 + g->ng; ++k)
    for (int j = -g->ng; j < g->ny + g->ng; ++j)
      for (int i = -g->ng; i < g->nx + g->ng; ++i) {
        size_t q = I3(g, i, j, k);
        double hh = m->h[I2(g, i, j)];
        double zc = hh + m->zeta_c[k + g->ng] * (m->zt - hh) / m->zt;
        double zw = hh + m->zeta_w[k + g->ng] * (m->zt - hh) / m->zt;
        double thc = theta_at(c, zc), thw = theta_at(c, zw);
        double qvc = moist ? tab_interp(qvt, ntab, zmin, zc) : 0.0;
        double qvw = moist ? tab_interp(qvt, ntab, zmin, zw) : 0.0;
        double thvc = thc * (1.0 + EPS61 * qvc), thvw = thw * (1.0 + EPS61 * qvw);
        double pic = tab_interp(pit, ntab, zmin, zc), piw = tab_interp(pit, ntab, zmin, zw);
        b->thb[q] = thc;
        b->pib[q] = pic;
        b->rhob[q] = density(pic, thvc);
        b->dthbdz[q] = (theta_at(c, zc + 1.0) - theta_at(c, zc - 1.0)) / 2.0;
        b->thbw[q] = thw;
        b->rhobw[q] = density(piw, thvw);
        b->thvb[q] = thvc;
        b->thvbw[q] = thvw;
        b->qvb[q] = qvc;
      }
  free(pit); free(qvt); free(thvt);

  /* base wind (base_state.cpp:234-252); linear shear is an extension */
  for (int kk = 0; kk < g->NZ; ++kk) {
    double z = m->zeta_c[kk];
    if (z < 0) z = 0;
    if (c->wind_profile == 1) b->ub[kk] = c->wind_us * tanh(z / c->wind_zs) + c->wind_offset;
    else if (c->wind_profile == 2) b->ub[kk] = c->wind_us * dmin(z / c->wind_zs, 1.0) + c->wind_offset;
    else if (file && c->prof_u) b->ub[kk] = table_lookup(c, c->prof_u, z);
    else b->ub[kk] = c->wind_u;
  }
  return moist;
}

/* -------------------------------------------------- initial conditions */
void orc_ic_bubble(const orc_grid* g, const orc_metric* m, double dth, double xc, double yc,
                   double zc, double xr, double yr, double zr, double* thp) {
  /* src/main.cpp:28-54 */
  if (dth == 0.0) return;
  const double pi = 3.14159265358979323846;
  memset(thp, 0, orc_npts(g) * sizeof(double));
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        double x = ((double)i + 0.5) * g->dx, y = ((double)j + 0.5) * g->dy;
        double hh = m->h[I2(g, i, j)];
        double z = hh + m->zeta_c[k + g->ng] * (m->zt - hh) / m->zt;
        double rx = (x - xc) / xr, ry = (y - yc) / yr, rz = (z - zc) / zr;
        double r = sqrt(rx * rx + ry * ry + rz * rz);
        if (r < 1.0) {
          double cs = cos(pi * r / 2);
          thp[I3(g, i, j, k)] = dth * cs * cs;
        }
      }
}

void orc_ic_wind(const orc_grid* g, const orc_base* b, double* u) {
  /* src/main.cpp:186-195: u faces 0..nx */
  memset(u, 0, orc_npts(g) * sizeof(double));
  for (int k = 0; k < g->nz; ++k) {
    double ub = b->ub[k + g->ng];
    if (ub == 0.0) continue;
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i <= g->nx; ++i) u[I3(g, i, j, k)] = ub;
  }
}

void orc_ic_moisture(const orc_grid* g, const orc_base* b, double* qv) {
  /* src/main.cpp:147-154 */
  memset(qv, 0, orc_npts(g) * sizeof(double));
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) qv[I3(g, i, j, k)] = b->qvb[I3(g, i, j, k)];
}

void orc_ic_from_input(const orc_grid* g, const orc_base* b, const double* in_u,
                       const double* in_v, const double* in_th, const double* in_pi,
                       const double* in_qv, orc_state* s) {
  /* src/main.cpp:58-100: centres -> faces, full -> perturbation */
  const size_t n = orc_npts(g);
#define SRC(a, i, j, k) (a)[((size_t)(k) * g->ny + (j)) * g->nx + (i)]
  memset(s->u, 0, n * sizeof(double));
  memset(s->v, 0, n * sizeof(double));
  memset(s->thp, 0, n * sizeof(double));
  memset(s->pip, 0, n * sizeof(double));
  memset(s->qv, 0, n * sizeof(double));
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j) {
      for (int i = 0; i <= g->nx; ++i) {
        int il = i > 0 ? i - 1 : 0, ir = i < g->nx ? i : g->nx - 1;
        s->u[I3(g, i, j, k)] = 0.5 * (SRC(in_u, il, j, k) + SRC(in_u, ir, j, k));
      }
      for (int i = 0; i < g->nx; ++i) {
        int jl = j > 0 ? j - 1 : 0;
        size_t q = I3(g, i, j, k);
        s->v[q] = 0.5 * (SRC(in_v, i, jl, k) + SRC(in_v, i, j, k));
        s->thp[q] = SRC(in_th, i, j, k) - b->thb[q];
        s->pip[q] = SRC(in_pi, i, j, k) - b->pib[q];
        s->qv[q] = SRC(in_qv, i, j, k);
      }
    }
#undef SRC
}

void orc_ic_perturb(const orc_grid* g, double amp, unsigned seed, double* thp) {
  /* src/main.cpp:105-144: seeded normal noise, 6 box-smoothing passes, RMS scaling */
  if (amp <= 0.0) return;
  const size_t n = orc_npts(g);
  double* p = dalloc(n);
  double* tmp = dalloc(n);
  std::mt19937 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) p[I3(g, i, j, k)] = (double)nd(rng);
  for (int pass = 0; pass < 6; ++pass) {
    memcpy(tmp, p, n * sizeof(double));
    for (int k = 1; k < g->nz - 1; ++k)
      for (int j = 1; j < g->ny - 1; ++j)
        for (int i = 1; i < g->nx - 1; ++i) {
          double s6 = tmp[I3(g, i - 1, j, k)] + tmp[I3(g, i + 1, j, k)] + tmp[I3(g, i, j - 1, k)] +
                      tmp[I3(g, i, j + 1, k)] + tmp[I3(g, i, j, k - 1)] + tmp[I3(g, i, j, k + 1)];
          p[I3(g, i, j, k)] = 0.5 * tmp[I3(g, i, j, k)] + s6 / 12.0;
        }
  }
  double ss = 0;
  size_t cnt = 0;
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        double v = p[I3(g, i, j, k)];
        ss += v * v;
        ++cnt;
      }
  double rms = sqrt(ss / (double)cnt);
  if (rms >= 1e-9) {
    double sc = amp / rms;
    for (int k = 0; k < g->nz; ++k)
      for (int j = 0; j < g->ny; ++j)
        for (int i = 0; i < g->nx; ++i) thp[I3(g, i, j, k)] += sc * p[I3(g, i, j, k)];
  }
  free(p);
  free(tmp);
}

void orc_lambert_mapf(int n, const double* lat, double lat1, double lat2, double* mapf) {
  /* src/main.cpp:326-340 */
  double phi1 = lat1 * 0.01745329252, phi2 = lat2 * 0.01745329252;
  const double PI4 = 0.78539816339;
  double cn = (fabs(phi1 - phi2) < 1e-6)
                  ? sin(phi1)
                  : log(cos(phi1) / cos(phi2)) / log(tan(PI4 + phi2 / 2) / tan(PI4 + phi1 / 2));
  double A = cos(phi1) * pow(tan(PI4 + phi1 / 2), cn);
  for (int q = 0; q < n; ++q) {
    double phi = lat[q] * 0.01745329252;
    mapf[q] = A / (pow(tan(PI4 + phi / 2), cn) * cos(phi));
  }
}

/* ---------------------------------------------------- boundary conditions */
/* src/dynamics/kernels.cu:695-770; fill order z, then x, then y */
static void bc_z_zerograd(const orc_grid* g, double* f) {
  const size_t plane = (size_t)g->NX * g->NY;
  for (size_t col = 0; col < plane; ++col) {
    double bot = f[col + plane * (size_t)g->ng];
    double top = f[col + plane * (size_t)(g->nz - 1 + g->ng)];
    for (int m = 1; m <= g->ng; ++m) f[col + plane * (size_t)(g->ng - m)] = bot;
    for (int m = 1; m <= g->ng + 1; ++m) f[col + plane * (size_t)(g->nz - 1 + g->ng + m)] = top;
  }
}

static void bc_z_w(const orc_grid* g, double* f) {
  const size_t plane = (size_t)g->NX * g->NY;
  for (size_t col = 0; col < plane; ++col) {
#define AT(k) f[col + plane * (size_t)((k) + g->ng)]
    AT(g->nz) = 0.0;
    double w0 = AT(0);
    for (int m = 1; m <= g->ng; ++m) {
      AT(-m) = 2 * w0 - AT(m);
      AT(g->nz + m) = -AT(g->nz - m);
    }
#undef AT
  }
}

/* ilast = last valid index of the field in x.  The reference's zero-gradient
 * fill for u (ilast = nx) also stores one element past the row end (racing
 * with the next row's own left ghost); only in-row stores are made here. */
static void bc_x(const orc_grid* g, int open, double* f, int ilast) {
  for (int kr = 0; kr < g->NZ; ++kr)
    for (int jr = 0; jr < g->NY; ++jr) {
      double* row = f + ((size_t)kr * g->NY + jr) * g->NX;
      if (open) {
        double left = row[g->ng], right = row[g->ng + ilast];
        for (int m = 0; m < g->ng; ++m) {
          row[g->ng - 1 - m] = left;
          int ir = g->ng + ilast + 1 + m;
          if (ir < g->NX) row[ir] = right;
        }
      } else {
        for (int m = 0; m < g->ng; ++m) {
          row[g->ng + g->nx + m] = row[g->ng + m];
          row[g->ng - 1 - m] = row[g->ng + g->nx - 1 - m];
        }
      }
    }
}

static void bc_y(const orc_grid* g, int open, double* f, int jlast) {
  for (int kr = 0; kr < g->NZ; ++kr) {
    double* pl = f + (size_t)kr * g->NY * g->NX;
    for (int ir = 0; ir < g->NX; ++ir) {
      if (open) {
        double lo = pl[(size_t)g->ng * g->NX + ir], hi = pl[(size_t)(g->ng + jlast) * g->NX + ir];
        for (int m = 0; m < g->ng; ++m) {
          pl[(size_t)(g->ng - 1 - m) * g->NX + ir] = lo;
          int jr = g->ng + jlast + 1 + m;
          if (jr < g->NY) pl[(size_t)jr * g->NX + ir] = hi;
        }
      } else {
        for (int m = 0; m < g->ng; ++m) {
          pl[(size_t)(g->ng + g->ny + m) * g->NX + ir] = pl[(size_t)(g->ng + m) * g->NX + ir];
          pl[(size_t)(g->ng - 1 - m) * g->NX + ir] = pl[(size_t)(g->ng + g->ny - 1 - m) * g->NX + ir];
        }
      }
    }
  }
}

/* kind: 0 cell scalar, 1 u, 2 v, 3 w */
void orc_bc_field(const orc_grid* g, const orc_params* p, double* f, int kind) {
  if (kind == 3) bc_z_w(g, f); else bc_z_zerograd(g, f);
  bc_x(g, p->bc_x_open, f, kind == 1 ? g->nx : g->nx - 1);
  bc_y(g, p->bc_y_open, f, kind == 2 ? g->ny : g->ny - 1);
}

void orc_apply_bcs(const orc_grid* g, const orc_params* p, orc_state* s) {
  /* src/dynamics/kernels.cu:805-835 */
  orc_bc_field(g, p, s->u, 1);
  orc_bc_field(g, p, s->v, 2);
  orc_bc_field(g, p, s->w, 3);
  orc_bc_field(g, p, s->thp, 0);
  orc_bc_field(g, p, s->pip, 0);
  if (p->moisture) {
    orc_bc_field(g, p, s->qv, 0);
    orc_bc_field(g, p, s->qc, 0);
    orc_bc_field(g, p, s->qr, 0);
  }
}

/* ------------------------------------------------------ dynamics helpers */
/* Rayleigh damping coefficient (src/dynamics/kernels.cu:42-48) */
static double sponge(double zeta, double zt, const orc_params* p) {
  if (p->rayleigh_zd < 0.0) return 0.0;
  if (zeta <= p->rayleigh_zd || zt <= p->rayleigh_zd) return 0.0;
  const double halfpi = 1.5707963267948966;
  double s = sin(halfpi * (zeta - p->rayleigh_zd) / (zt - p->rayleigh_zd));
  return p->rayleigh_alpha * s * s;
}

/* 5th-order upwind face value between q0 (below) and q1 (above)
 * (src/dynamics/kernels.cu:51-57) */
static double face5(double qm2, double qm1, double q0, double q1, double q2, double q3,
                    double vel) {
  const double c = 1.0 / 60.0;
  double cen = c * (37.0 * (q0 + q1) - 8.0 * (qm1 + q2) + (qm2 + q3));
  double upw = c * ((q3 - qm2) - 5.0 * (q2 - qm1) + 10.0 * (q1 - q0));
  return (vel >= 0.0) ? (cen - upw) : (cen + upw);
}

/* flux-form advection of a cell-centred scalar (kernels.cu:114-179):
 * returns (-div(F) + q div(MF)) / (rho J) */
static double scalar_adv(const orc_grid* g, const orc_base* b, const orc_metric* m,
                         const double* q, const double* mfx, const double* mfy,
                         const double* mfz, const double* div, int i, int j, int k) {
#define Q(ii, jj, kz) q[I3(g, ii, jj, kz)]
  int kk = k + g->ng;
  double fxL = mfx[I3(g, i, j, k)], fxR = mfx[I3(g, i + 1, j, k)];
  double fyL = mfy[I3(g, i, j, k)], fyR = mfy[I3(g, i, j + 1, k)];
  double fzB = mfz[I3(g, i, j, k)], fzT = mfz[I3(g, i, j, k + 1)];
  double FxL = fxL * face5(Q(i - 3, j, k), Q(i - 2, j, k), Q(i - 1, j, k), Q(i, j, k), Q(i + 1, j, k), Q(i + 2, j, k), fxL);
  double FxR = fxR * face5(Q(i - 2, j, k), Q(i - 1, j, k), Q(i, j, k), Q(i + 1, j, k), Q(i + 2, j, k), Q(i + 3, j, k), fxR);
  double FyL = fyL * face5(Q(i, j - 3, k), Q(i, j - 2, k), Q(i, j - 1, k), Q(i, j, k), Q(i, j + 1, k), Q(i, j + 2, k), fyL);
  double FyR = fyR * face5(Q(i, j - 2, k), Q(i, j - 1, k), Q(i, j, k), Q(i, j + 1, k), Q(i, j + 2, k), Q(i, j + 3, k), fyR);
  double FzB = fzB * face5(Q(i, j, k - 3), Q(i, j, k - 2), Q(i, j, k - 1), Q(i, j, k), Q(i, j, k + 1), Q(i, j, k + 2), fzB);
  double FzT = fzT * face5(Q(i, j, k - 2), Q(i, j, k - 1), Q(i, j, k), Q(i, j, k + 1), Q(i, j, k + 2), Q(i, j, k + 3), fzT);
  double fdiv = (FxR - FxL) / g->dx + (FyR - FyL) / g->dy + (FzT - FzB) / m->dzeta_c[kk];
  double rt = b->rhob[I3(g, i, j, k)] * m->jac[I2(g, i, j)];
  return (-fdiv + Q(i, j, k) * div[I3(g, i, j, k)]) / rt;
#undef Q
}

/* ------------------------------------------------ mass fluxes, divergence */
void orc_mass_fluxes(const orc_grid* g, const orc_base* b, const orc_metric* m,
                     const orc_state* s, double* mfx, double* mfy, double* mfz) {
  /* horizontal fluxes on the ring -2..n+2 (kernels.cu:68-81) */
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g->nz; ++k)
    for (int j = -2; j <= g->ny + 2; ++j)
      for (int i = -2; i <= g->nx + 2; ++i) {
        size_t c = I3(g, i, j, k);
        double rjx = 0.5 * (b->rhob[I3(g, i - 1, j, k)] * m->jac[I2(g, i - 1, j)] + b->rhob[c] * m->jac[I2(g, i, j)]);
        mfx[c] = rjx * s->u[c];
        double rjy = 0.5 * (b->rhob[I3(g, i, j - 1, k)] * m->jac[I2(g, i, j - 1)] + b->rhob[c] * m->jac[I2(g, i, j)]);
        mfy[c] = rjy * s->v[c];
      }
  /* contravariant vertical flux rho^w J Omega at inner w levels (kernels.cu:83-97);
   * levels 0 and nz keep Omega = 0 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k < g->nz; ++k)
    for (int j = -2; j <= g->ny + 1; ++j)
      for (int i = -2; i <= g->nx + 1; ++i) {
        int kk = k + g->ng;
        size_t c = I3(g, i, j, k);
        double fac = 1.0 - m->zeta_w[kk] / m->zt;
        double uw = 0.25 * (s->u[I3(g, i, j, k - 1)] + s->u[I3(g, i + 1, j, k - 1)] + s->u[I3(g, i, j, k)] + s->u[I3(g, i + 1, j, k)]);
        double vw = 0.25 * (s->v[I3(g, i, j, k - 1)] + s->v[I3(g, i, j + 1, k - 1)] + s->v[I3(g, i, j, k)] + s->v[I3(g, i, j + 1, k)]);
        double cross = (uw * m->hx[I2(g, i, j)] + vw * m->hy[I2(g, i, j)]) * fac;
        mfz[c] = b->rhobw[c] * (s->w[c] - cross);
      }
}

void orc_divergence(const orc_grid* g, const orc_metric* m, const double* mfx,
                    const double* mfy, const double* mfz, double* div) {
  /* kernels.cu:99-110 */
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g->nz; ++k)
    for (int j = -1; j <= g->ny; ++j)
      for (int i = -1; i <= g->nx; ++i) {
        int kk = k + g->ng;
        div[I3(g, i, j, k)] = (mfx[I3(g, i + 1, j, k)] - mfx[I3(g, i, j, k)]) / g->dx +
                              (mfy[I3(g, i, j + 1, k)] - mfy[I3(g, i, j, k)]) / g->dy +
                              (mfz[I3(g, i, j, k + 1)] - mfz[I3(g, i, j, k)]) / m->dzeta_c[kk];
      }
}

/* ---------------------------------------------- positive-definite moisture */
/* Skamarock flux renormalisation, fluxes stored on the left/lower face
 * (kernels.cu:187-264, 855-869) */
static void advect_pd(const orc_grid* g, const orc_base* b, const orc_metric* m,
                      const orc_params* p, double dt, const double* q, const double* mfx,
                      const double* mfy, const double* mfz, const double* div, double* Fx,
                      double* Fy, double* Fz, double* ratio, double* tend) {
#define Q(ii, jj, kz) q[I3(g, ii, jj, kz)]
#pragma omp parallel for schedule(static)
  for (int k = 0; k <= g->nz; ++k)
    for (int j = 0; j <= g->ny; ++j)
      for (int i = 0; i <= g->nx; ++i) {
        size_t c = I3(g, i, j, k);
        if (j < g->ny && k < g->nz) {
          double f = mfx[c];
          Fx[c] = f * face5(Q(i - 3, j, k), Q(i - 2, j, k), Q(i - 1, j, k), Q(i, j, k), Q(i + 1, j, k), Q(i + 2, j, k), f);
        }
        if (i < g->nx && k < g->nz) {
          double f = mfy[c];
          Fy[c] = f * face5(Q(i, j - 3, k), Q(i, j - 2, k), Q(i, j - 1, k), Q(i, j, k), Q(i, j + 1, k), Q(i, j + 2, k), f);
        }
        if (i < g->nx && j < g->ny) {
          double f = mfz[c];
          Fz[c] = f * face5(Q(i, j, k - 3), Q(i, j, k - 2), Q(i, j, k - 1), Q(i, j, k), Q(i, j, k + 1), Q(i, j, k + 2), f);
        }
      }
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        double dzc = m->dzeta_c[k + g->ng];
        double out = dmax(0.0, Fx[I3(g, i + 1, j, k)]) / g->dx + dmax(0.0, -Fx[I3(g, i, j, k)]) / g->dx +
                     dmax(0.0, Fy[I3(g, i, j + 1, k)]) / g->dy + dmax(0.0, -Fy[I3(g, i, j, k)]) / g->dy +
                     dmax(0.0, Fz[I3(g, i, j, k + 1)]) / dzc + dmax(0.0, -Fz[I3(g, i, j, k)]) / dzc;
        double avail = b->rhob[I3(g, i, j, k)] * m->jac[I2(g, i, j)] * dmax(0.0, Q(i, j, k));
        double r = (dt * out > 1e-20) ? avail / (dt * out) : 1.0;
        ratio[I3(g, i, j, k)] = dmin(1.0, r);
      }
  /* ratio ghosts: lateral only (kernels.cu:865-866) */
  bc_x(g, p->bc_x_open, ratio, g->nx - 1);
  bc_y(g, p->bc_y_open, ratio, g->ny - 1);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        int kk = k + g->ng;
        double fxl = Fx[I3(g, i, j, k)], fxr = Fx[I3(g, i + 1, j, k)];
        double fyl = Fy[I3(g, i, j, k)], fyr = Fy[I3(g, i, j + 1, k)];
        double fzl = Fz[I3(g, i, j, k)], fzr = Fz[I3(g, i, j, k + 1)];
        double sxl = fxl * ratio[I3(g, fxl >= 0.0 ? i - 1 : i, j, k)];
        double sxr = fxr * ratio[I3(g, fxr >= 0.0 ? i : i + 1, j, k)];
        double syl = fyl * ratio[I3(g, i, fyl >= 0.0 ? j - 1 : j, k)];
        double syr = fyr * ratio[I3(g, i, fyr >= 0.0 ? j : j + 1, k)];
        double szl = fzl * ratio[I3(g, i, j, fzl >= 0.0 ? k - 1 : k)];
        double szr = fzr * ratio[I3(g, i, j, fzr >= 0.0 ? k : k + 1)];
        double fdiv = (sxr - sxl) / g->dx + (syr - syl) / g->dy + (szr - szl) / m->dzeta_c[kk];
        double rt = b->rhob[I3(g, i, j, k)] * m->jac[I2(g, i, j)];
        tend[I3(g, i, j, k)] = (-fdiv + Q(i, j, k) * div[I3(g, i, j, k)]) / rt;
      }
#undef Q
}

/* constant-K Laplacian added to a tendency (kernels.cu:430-443) */
static void add_diffusion(const orc_grid* g, const orc_metric* m, double K, const double* f,
                          double* tend, int kmin, int kend, int on_w) {
#pragma omp parallel for schedule(static)
  for (int k = kmin; k < kend; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        int kk = k + g->ng;
        double dzl = (on_w ? m->dzeta_w[kk] : m->dzeta_c[kk]) * m->jac[I2(g, i, j)];
        double c = f[I3(g, i, j, k)];
        double lap = (f[I3(g, i + 1, j, k)] - 2 * c + f[I3(g, i - 1, j, k)]) / (g->dx * g->dx) +
                     (f[I3(g, i, j + 1, k)] - 2 * c + f[I3(g, i, j - 1, k)]) / (g->dy * g->dy) +
                     (f[I3(g, i, j, k + 1)] - 2 * c + f[I3(g, i, j, k - 1)]) / (dzl * dzl);
        tend[I3(g, i, j, k)] += K * lap;
      }
}

/* --------------------------------------------------------- slow tendencies */
void orc_tendencies(const orc_grid* g, const orc_base* b, const orc_metric* m,
                    const orc_params* p, double dt, const orc_state* s, const double* mfx,
                    const double* mfy, const double* mfz, const double* div, orc_state* tend,
                    double* const* pd) {
  const double zt = m->zt;
#define MX(ii, jj, kz) mfx[I3(g, ii, jj, kz)]
#define MY(ii, jj, kz) mfy[I3(g, ii, jj, kz)]
#define MZ(ii, jj, kz) mfz[I3(g, ii, jj, kz)]
#define DV(ii, jj, kz) div[I3(g, ii, jj, kz)]
#define RJ(ii, jj, kz) (b->rhob[I3(g, ii, jj, kz)] * m->jac[I2(g, ii, jj)])
  /* u on x faces (kernels.cu:308-346) */
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        int kk = k + g->ng;
#define U(ii, jj, kz) s->u[I3(g, ii, jj, kz)]
        double fcL = 0.5 * (MX(i - 1, j, k) + MX(i, j, k)), fcR = 0.5 * (MX(i, j, k) + MX(i + 1, j, k));
        double FxL = fcL * face5(U(i - 3, j, k), U(i - 2, j, k), U(i - 1, j, k), U(i, j, k), U(i + 1, j, k), U(i + 2, j, k), fcL);
        double FxR = fcR * face5(U(i - 2, j, k), U(i - 1, j, k), U(i, j, k), U(i + 1, j, k), U(i + 2, j, k), U(i + 3, j, k), fcR);
        double fyB = 0.5 * (MY(i - 1, j, k) + MY(i, j, k)), fyT = 0.5 * (MY(i - 1, j + 1, k) + MY(i, j + 1, k));
        double FyB = fyB * face5(U(i, j - 3, k), U(i, j - 2, k), U(i, j - 1, k), U(i, j, k), U(i, j + 1, k), U(i, j + 2, k), fyB);
        double FyT = fyT * face5(U(i, j - 2, k), U(i, j - 1, k), U(i, j, k), U(i, j + 1, k), U(i, j + 2, k), U(i, j + 3, k), fyT);
        double fzB = 0.5 * (MZ(i - 1, j, k) + MZ(i, j, k)), fzT = 0.5 * (MZ(i - 1, j, k + 1) + MZ(i, j, k + 1));
        double FzB = fzB * face5(U(i, j, k - 3), U(i, j, k - 2), U(i, j, k - 1), U(i, j, k), U(i, j, k + 1), U(i, j, k + 2), fzB);
        double FzT = fzT * face5(U(i, j, k - 2), U(i, j, k - 1), U(i, j, k), U(i, j, k + 1), U(i, j, k + 2), U(i, j, k + 3), fzT);
        double fdiv = (FxR - FxL) / g->dx + (FyT - FyB) / g->dy + (FzT - FzB) / m->dzeta_c[kk];
        double dv = 0.5 * (DV(i - 1, j, k) + DV(i, j, k));
        double ru = 0.5 * (RJ(i - 1, j, k) + RJ(i, j, k));
        double vavg = 0.25 * (s->v[I3(g, i - 1, j, k)] + s->v[I3(g, i - 1, j + 1, k)] + s->v[I3(g, i, j, k)] + s->v[I3(g, i, j + 1, k)]);
        double fc = 0.5 * (m->fcor[I2(g, i - 1, j)] + m->fcor[I2(g, i, j)]);
        double relax = -sponge(m->zeta_c[kk], zt, p) * (U(i, j, k) - b->ub[kk]);
        tend->u[I3(g, i, j, k)] = (-fdiv + U(i, j, k) * dv) / ru + fc * vavg + relax;
#undef U
      }
  /* v on y faces (kernels.cu:348-385) */
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        int kk = k + g->ng;
#define V(ii, jj, kz) s->v[I3(g, ii, jj, kz)]
        double fcB = 0.5 * (MY(i, j - 1, k) + MY(i, j, k)), fcT = 0.5 * (MY(i, j, k) + MY(i, j + 1, k));
        double FyB = fcB * face5(V(i, j - 3, k), V(i, j - 2, k), V(i, j - 1, k), V(i, j, k), V(i, j + 1, k), V(i, j + 2, k), fcB);
        double FyT = fcT * face5(V(i, j - 2, k), V(i, j - 1, k), V(i, j, k), V(i, j + 1, k), V(i, j + 2, k), V(i, j + 3, k), fcT);
        double fxL = 0.5 * (MX(i, j - 1, k) + MX(i, j, k)), fxR = 0.5 * (MX(i + 1, j - 1, k) + MX(i + 1, j, k));
        double FxL = fxL * face5(V(i - 3, j, k), V(i - 2, j, k), V(i - 1, j, k), V(i, j, k), V(i + 1, j, k), V(i + 2, j, k), fxL);
        double FxR = fxR * face5(V(i - 2, j, k), V(i - 1, j, k), V(i, j, k), V(i + 1, j, k), V(i + 2, j, k), V(i + 3, j, k), fxR);
        double fzB = 0.5 * (MZ(i, j - 1, k) + MZ(i, j, k)), fzT = 0.5 * (MZ(i, j - 1, k + 1) + MZ(i, j, k + 1));
        double FzB = fzB * face5(V(i, j, k - 3), V(i, j, k - 2), V(i, j, k - 1), V(i, j, k), V(i, j, k + 1), V(i, j, k + 2), fzB);
        double FzT = fzT * face5(V(i, j, k - 2), V(i, j, k - 1), V(i, j, k), V(i, j, k + 1), V(i, j, k + 2), V(i, j, k + 3), fzT);
        double fdiv = (FxR - FxL) / g->dx + (FyT - FyB) / g->dy + (FzT - FzB) / m->dzeta_c[kk];
        double dv = 0.5 * (DV(i, j - 1, k) + DV(i, j, k));
        double rv = 0.5 * (RJ(i, j - 1, k) + RJ(i, j, k));
        double uavg = 0.25 * (s->u[I3(g, i, j - 1, k)] + s->u[I3(g, i + 1, j - 1, k)] + s->u[I3(g, i, j, k)] + s->u[I3(g, i + 1, j, k)]);
        double fc = 0.5 * (m->fcor[I2(g, i, j - 1)] + m->fcor[I2(g, i, j)]);
        double uref = p->coriolis_use_ub ? b->ub[kk] : 0.0;
        double relax = -sponge(m->zeta_c[kk], zt, p) * V(i, j, k);
        tend->v[I3(g, i, j, k)] = (-fdiv + V(i, j, k) * dv) / rv - fc * (uavg - uref) + relax;
#undef V
      }
  /* w on inner w levels (kernels.cu:387-425) */
#pragma omp parallel for schedule(static)
  for (int k = 1; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        int kk = k + g->ng;
#define W(ii, jj, kz) s->w[I3(g, ii, jj, kz)]
        double fxL = 0.5 * (MX(i, j, k - 1) + MX(i, j, k)), fxR = 0.5 * (MX(i + 1, j, k - 1) + MX(i + 1, j, k));
        double FxL = fxL * face5(W(i - 3, j, k), W(i - 2, j, k), W(i - 1, j, k), W(i, j, k), W(i + 1, j, k), W(i + 2, j, k), fxL);
        double FxR = fxR * face5(W(i - 2, j, k), W(i - 1, j, k), W(i, j, k), W(i + 1, j, k), W(i + 2, j, k), W(i + 3, j, k), fxR);
        double fyB = 0.5 * (MY(i, j, k - 1) + MY(i, j, k)), fyT = 0.5 * (MY(i, j + 1, k - 1) + MY(i, j + 1, k));
        double FyB = fyB * face5(W(i, j - 3, k), W(i, j - 2, k), W(i, j - 1, k), W(i, j, k), W(i, j + 1, k), W(i, j + 2, k), fyB);
        double FyT = fyT * face5(W(i, j - 2, k), W(i, j - 1, k), W(i, j, k), W(i, j + 1, k), W(i, j + 2, k), W(i, j + 3, k), fyT);
        double fzB = 0.5 * (MZ(i, j, k - 1) + MZ(i, j, k)), fzT = 0.5 * (MZ(i, j, k) + MZ(i, j, k + 1));
        double FzB = fzB * face5(W(i, j, k - 3), W(i, j, k - 2), W(i, j, k - 1), W(i, j, k), W(i, j, k + 1), W(i, j, k + 2), fzB);
        double FzT = fzT * face5(W(i, j, k - 2), W(i, j, k - 1), W(i, j, k), W(i, j, k + 1), W(i, j, k + 2), W(i, j, k + 3), fzT);
        double fdiv = (FxR - FxL) / g->dx + (FyT - FyB) / g->dy + (FzT - FzB) / m->dzeta_w[kk];
        double dv = 0.5 * (DV(i, j, k - 1) + DV(i, j, k));
        double rw = b->rhobw[I3(g, i, j, k)] * m->jac[I2(g, i, j)];
        double relax = -sponge(m->zeta_w[kk], zt, p) * W(i, j, k);
        double wk = W(i, j, k);
        if (p->w_damping) {
          double cr = fabs(wk) * dt / (m->dzeta_w[kk] * m->jac[I2(g, i, j)]);
          if (cr > 1.0) relax -= 0.3 * (cr - 1.0) * wk / dt;
        }
        tend->w[I3(g, i, j, k)] = (-fdiv + wk * dv) / rw + relax;
#undef W
      }
  /* theta' (kernels.cu:114-146) */
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        int kk = k + g->ng;
        tend->thp[I3(g, i, j, k)] = scalar_adv(g, b, m, s->thp, mfx, mfy, mfz, div, i, j, k) -
                                    sponge(m->zeta_c[kk], zt, p) * s->thp[I3(g, i, j, k)];
      }
  /* moisture (kernels.cu:886-899) */
  if (p->moisture) {
    const double* qs[3] = {s->qv, s->qc, s->qr};
    double* ts[3] = {tend->qv, tend->qc, tend->qr};
    for (int sp = 0; sp < 3; ++sp) {
      if (p->pd_moist && pd) {
        advect_pd(g, b, m, p, dt, qs[sp], mfx, mfy, mfz, div, pd[0], pd[1], pd[2], pd[3], ts[sp]);
      } else {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < g->nz; ++k)
          for (int j = 0; j < g->ny; ++j)
            for (int i = 0; i < g->nx; ++i)
              ts[sp][I3(g, i, j, k)] = scalar_adv(g, b, m, qs[sp], mfx, mfy, mfz, div, i, j, k);
      }
    }
  }
  memset(tend->pip, 0, orc_npts(g) * sizeof(double));
  if (p->diff_K > 0.0) {
    add_diffusion(g, m, p->diff_K, s->u, tend->u, 0, g->nz, 0);
    add_diffusion(g, m, p->diff_K, s->v, tend->v, 0, g->nz, 0);
    add_diffusion(g, m, p->diff_K, s->w, tend->w, 1, g->nz, 1);
    add_diffusion(g, m, p->diff_K, s->thp, tend->thp, 0, g->nz, 0);
  }
#undef MX
#undef MY
#undef MZ
#undef DV
#undef RJ
}

/* -------------------------------------------------------- Davies relaxation */
static void relax_one(const orc_grid* g, int imax, int jmax, const double* f, const double* lo,
                      const double* hi, double tf, const double* wgt, double* tend) {
  /* kernels.cu:292-304 */
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < jmax; ++j)
      for (int i = 0; i < imax; ++i) {
        int iw = i < g->nx ? i : g->nx - 1, jw = j < g->ny ? j : g->ny - 1;
        double w = wgt[I2(g, iw, jw)];
        if (w <= 0.0) continue;
        size_t c = I3(g, i, j, k);
        tend[c] += w * ((1.0 - tf) * lo[c] + tf * hi[c] - f[c]);
      }
}

void orc_bdy_relax(const orc_grid* g, const orc_state* s, double* const* lo,
                   double* const* hi, double tf, const double* wgt, orc_state* tend) {
  /* kernels.cu:981-995 */
  relax_one(g, g->nx + 1, g->ny, s->u, lo[0], hi[0], tf, wgt, tend->u);
  relax_one(g, g->nx, g->ny + 1, s->v, lo[1], hi[1], tf, wgt, tend->v);
  relax_one(g, g->nx, g->ny, s->thp, lo[2], hi[2], tf, wgt, tend->thp);
  relax_one(g, g->nx, g->ny, s->pip, lo[3], hi[3], tf, wgt, tend->pip);
  relax_one(g, g->nx, g->ny, s->qv, lo[4], hi[4], tf, wgt, tend->qv);
}

void orc_bdy_weights(const orc_grid* g, const orc_params* p, int bdy_width, double bdy_tau,
                     double nudge_tau, double* wgt) {
  /* src/dynamics/boundary.cpp:24-42 */
  double inner = (nudge_tau > 0.0) ? 1.0 / nudge_tau : 0.0;
  const double pi_half = 1.5707963267948966;
  memset(wgt, 0, (size_t)g->NX * g->NY * sizeof(double));
  for (int j = 0; j < g->ny; ++j)
    for (int i = 0; i < g->nx; ++i) {
      double wij = inner;
      int dist = 1 << 20;
      if (p->bc_x_open) { int d = i < g->nx - 1 - i ? i : g->nx - 1 - i; if (d < dist) dist = d; }
      if (p->bc_y_open) { int d = j < g->ny - 1 - j ? j : g->ny - 1 - j; if (d < dist) dist = d; }
      if (dist < bdy_width) {
        double s = cos(pi_half * (double)dist / (double)bdy_width);
        wij = dmax(wij, s * s / bdy_tau);
      }
      wgt[I2(g, i, j)] = wij;
    }
}

/* ------------------------------------------------------- acoustic substeps */
void orc_acoustic_coef(const orc_grid* g, const orc_base* b, const orc_metric* m,
                       double* rtjx, double* rtjy, double* kt3, double* aw) {
  /* kernels.cu:452-474 over the whole padded grid */
  const size_t n = orc_npts(g);
  double* rtjc = dalloc(n);
  for (int kr = 0; kr < g->NZ; ++kr)
    for (int jr = 0; jr < g->NY; ++jr)
      for (int ir = 0; ir < g->NX; ++ir) {
        size_t c = ((size_t)kr * g->NY + jr) * g->NX + ir, c2 = (size_t)jr * g->NX + ir;
        double J = m->jac[c2];
        rtjc[c] = b->rhob[c] * b->thvb[c] * J;
        kt3[c] = RD * b->pib[c] / (CV * b->rhob[c] * b->thvb[c] * J);
        aw[c] = b->rhobw[c] * b->thvbw[c];
      }
  for (int kr = 0; kr < g->NZ; ++kr)
    for (int jr = 0; jr < g->NY; ++jr)
      for (int ir = 0; ir < g->NX; ++ir) {
        size_t c = ((size_t)kr * g->NY + jr) * g->NX + ir;
        rtjx[c] = (ir > 0) ? 0.5 * (rtjc[c - 1] + rtjc[c]) : rtjc[c];
        rtjy[c] = (jr > 0) ? 0.5 * (rtjc[c - g->NX] + rtjc[c]) : rtjc[c];
      }
  free(rtjc);
}

void orc_acoustic_substep(const orc_grid* g, const orc_base* b, const orc_metric* m,
                          const orc_params* p, double dtau, orc_state* s,
                          const orc_state* tend, double* piprev, const double* rtjx,
                          const double* rtjy, const double* kt3, const double* aw) {
  const double zt = m->zt;
  double* u = s->u;
  double* v = s->v;
  const double* pip = s->pip;
  /* forward u, v: full-theta_v PGF with divergence damping pi* and the
   * explicit terrain cross term (kernels.cu:480-527) */
#define PS(ii, jj, kz) (pip[I3(g, ii, jj, kz)] + p->acoustic_smdiv * (pip[I3(g, ii, jj, kz)] - piprev[I3(g, ii, jj, kz)]))
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        const int kk = k + g->ng;
#define THV(ii, jj) ((b->thb[I3(g, ii, jj, k)] + s->thp[I3(g, ii, jj, k)]) * (p->moisture ? 1.0 + EPS61 * s->qv[I3(g, ii, jj, k)] : 1.0))
        double ps0 = PS(i, j, k);
        double dzc2 = m->zeta_c[kk + 1] - m->zeta_c[kk - 1];
        if (!(p->bc_x_open && i == 0)) {
          double thbu = 0.5 * (THV(i - 1, j) + THV(i, j));
          double mu = 0.5 * (m->mapf[I2(g, i - 1, j)] + m->mapf[I2(g, i, j)]);
          double grad = (ps0 - PS(i - 1, j, k)) / g->dx;
          double zxu = m->hx_u[I2(g, i, j)] * (1.0 - m->zeta_c[kk] / zt);
          if (zxu != 0.0) {
            double ju = 0.5 * (m->jac[I2(g, i - 1, j)] + m->jac[I2(g, i, j)]);
            double dpdz = 0.5 * ((PS(i - 1, j, k + 1) - PS(i - 1, j, k - 1)) + (PS(i, j, k + 1) - PS(i, j, k - 1))) / dzc2;
            grad -= zxu / ju * dpdz;
          }
          u[I3(g, i, j, k)] += dtau * (-CP * thbu * mu * grad + tend->u[I3(g, i, j, k)]);
        }
        if (!(p->bc_y_open && j == 0)) {
          double thbv = 0.5 * (THV(i, j - 1) + THV(i, j));
          double mv = 0.5 * (m->mapf[I2(g, i, j - 1)] + m->mapf[I2(g, i, j)]);
          double grad = (ps0 - PS(i, j - 1, k)) / g->dy;
          double zyv = m->hy_v[I2(g, i, j)] * (1.0 - m->zeta_c[kk] / zt);
          if (zyv != 0.0) {
            double jv = 0.5 * (m->jac[I2(g, i, j - 1)] + m->jac[I2(g, i, j)]);
            double dpdz = 0.5 * ((PS(i, j - 1, k + 1) - PS(i, j - 1, k - 1)) + (PS(i, j, k + 1) - PS(i, j, k - 1))) / dzc2;
            grad -= zyv / jv * dpdz;
          }
          v[I3(g, i, j, k)] += dtau * (-CP * thbv * mv * grad + tend->v[I3(g, i, j, k)]);
        }
#undef THV
      }
#undef PS
  /* radiation conditions on open normal-velocity faces (kernels.cu:649-688) */
  if (p->bc_x_open)
    for (int k = 0; k < g->nz; ++k)
      for (int j = 0; j < g->ny; ++j) {
        int kk = k + g->ng;
        double u0 = u[I3(g, 0, j, k)];
        if (u0 >= 0.0) u[I3(g, 0, j, k)] = b->ub[kk];
        else {
          double cb = u0 - p->cstar;
          u[I3(g, 0, j, k)] = u0 - dtau * cb * (u[I3(g, 1, j, k)] - u0) / g->dx;
        }
        double un = u[I3(g, g->nx, j, k)];
        if (un <= 0.0) u[I3(g, g->nx, j, k)] = b->ub[kk];
        else {
          double cb = un + p->cstar;
          u[I3(g, g->nx, j, k)] = un - dtau * cb * (un - u[I3(g, g->nx - 1, j, k)]) / g->dx;
        }
      }
  if (p->bc_y_open)
    for (int k = 0; k < g->nz; ++k)
      for (int i = 0; i < g->nx; ++i) {
        double v0 = v[I3(g, i, 0, k)];
        if (v0 >= 0.0) v[I3(g, i, 0, k)] = 0.0;
        else {
          double cb = v0 - p->cstar;
          v[I3(g, i, 0, k)] = v0 - dtau * cb * (v[I3(g, i, 1, k)] - v0) / g->dy;
        }
        double vn = v[I3(g, i, g->ny, k)];
        if (vn <= 0.0) v[I3(g, i, g->ny, k)] = 0.0;
        else {
          double cb = vn + p->cstar;
          v[I3(g, i, g->ny, k)] = vn - dtau * cb * (vn - v[I3(g, i, g->ny - 1, k)]) / g->dy;
        }
      }
  /* neighbour faces for the column divergence (kernels.cu:946-950) */
  bc_x(g, p->bc_x_open, u, g->nx);
  bc_y(g, p->bc_y_open, u, g->ny - 1);
  bc_x(g, p->bc_x_open, v, g->nx - 1);
  bc_y(g, p->bc_y_open, v, g->ny);

  /* vertically implicit w - pi' column solve (kernels.cu:531-645) */
  const int nz = g->nz;
  const double c1 = (1.0 + p->acoustic_beta) * 0.5, c2 = (1.0 - p->acoustic_beta) * 0.5;
#pragma omp parallel
  {
    double* P = dalloc(nz + 1);
    double* E = dalloc(nz + 1);
    double* cs = dalloc(nz + 1);
    double* ds = dalloc(nz + 1);
    double* Wn = dalloc(nz + 1);
    double* Av = dalloc(nz + 1);
    double* Sv = dalloc(nz + 1);
#pragma omp for schedule(static) collapse(2)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        double* w = s->w;
        double* pi = s->pip;
        double* th = s->thp;
        const double J = m->jac[I2(g, i, j)], hxc = m->hx[I2(g, i, j)], hyc = m->hy[I2(g, i, j)];
        Av[0] = 0; Av[nz] = 0; Sv[0] = 0; Sv[nz] = 0;
        for (int k = 1; k < nz; ++k) {
          int kk = k + g->ng;
          size_t c = I3(g, i, j, k);
          Av[k] = aw[c];
          double fac = 1.0 - m->zeta_w[kk] / zt;
          double uw = 0.25 * (u[I3(g, i, j, k - 1)] + u[I3(g, i + 1, j, k - 1)] + u[I3(g, i, j, k)] + u[I3(g, i + 1, j, k)]);
          double vw = 0.25 * (v[I3(g, i, j, k - 1)] + v[I3(g, i, j + 1, k - 1)] + v[I3(g, i, j, k)] + v[I3(g, i, j + 1, k)]);
          Sv[k] = Av[k] * (uw * hxc + vw * hyc) * fac;
        }
        for (int k = 0; k < nz; ++k) {
          int kk = k + g->ng;
          size_t c = I3(g, i, j, k);
          double Kt = kt3[c];
          double mc = m->mapf[I2(g, i, j)];
          double Dh = mc * ((rtjx[I3(g, i + 1, j, k)] * u[I3(g, i + 1, j, k)] - rtjx[c] * u[c]) / g->dx +
                            (rtjy[I3(g, i, j + 1, k)] * v[I3(g, i, j + 1, k)] - rtjy[c] * v[c]) / g->dy);
          double dzc = m->dzeta_c[kk];
          double wk = w[c], wkp = w[I3(g, i, j, k + 1)];
          P[k] = pi[c] + dtau * tend->pip[c] -
                 dtau * Kt * (Dh - (Sv[k + 1] - Sv[k]) / dzc + c2 * (Av[k + 1] * wkp - Av[k] * wk) / dzc);
          E[k] = dtau * Kt * c1 / dzc;
        }
        for (int k = 1; k < nz; ++k) {
          int kk = k + g->ng;
          size_t c = I3(g, i, j, k), cm = I3(g, i, j, k - 1);
          double thvw = b->thbw[c] + 0.5 * (th[cm] + th[c]);
          if (p->moisture) thvw *= 1.0 + EPS61 * 0.5 * (s->qv[cm] + s->qv[c]);
          double G = dtau * CP * thvw * c1 / (J * m->dzeta_w[kk]);
          double A = -G * E[k - 1] * Av[k - 1];
          double B = 1.0 + G * Av[k] * (E[k] + E[k - 1]);
          double C = -G * E[k] * Av[k + 1];
          double buoy = GRAV * 0.5 * (th[cm] + th[c]) / b->thbw[c];
          if (p->moisture) {
            double dqv = 0.5 * (s->qv[cm] + s->qv[c]) - 0.5 * (b->qvb[cm] + b->qvb[c]);
            double qcr = 0.5 * (s->qc[cm] + s->qc[c]) + 0.5 * (s->qr[cm] + s->qr[c]);
            buoy += GRAV * (EPS61 * dqv - qcr);
          }
          double RHS = w[c] + dtau * (buoy + tend->w[c]) -
                       dtau * CP * thvw * c2 * (pi[c] - pi[cm]) / (J * m->dzeta_w[kk]);
          double D = RHS - G * (P[k] - P[k - 1]);
          if (k == 1) {
            cs[k] = C / B;
            ds[k] = D / B;
          } else {
            double mm = B - A * cs[k - 1];
            cs[k] = C / mm;
            ds[k] = (D - A * ds[k - 1]) / mm;
          }
        }
        Wn[nz] = 0;
        double wabove = 0;
        for (int k = nz - 1; k >= 1; --k) {
          double wk = ds[k] - cs[k] * wabove;
          Wn[k] = wk;
          wabove = wk;
        }
        {
          double us = 0.5 * (u[I3(g, i, j, 0)] + u[I3(g, i + 1, j, 0)]);
          double vs = 0.5 * (v[I3(g, i, j, 0)] + v[I3(g, i, j + 1, 0)]);
          Wn[0] = us * hxc + vs * hyc;
        }
        for (int k = 0; k < nz; ++k) {
          size_t c = I3(g, i, j, k);
          double oldpi = pi[c];
          pi[c] = P[k] - E[k] * (Av[k + 1] * Wn[k + 1] - Av[k] * Wn[k]);
          piprev[c] = oldpi;
          double wc = 0.5 * (Wn[k] + Wn[k + 1]);
          th[c] += dtau * (tend->thp[c] - wc * b->dthbdz[c]);
        }
        for (int k = 0; k < nz; ++k) w[I3(g, i, j, k)] = Wn[k];
      }
    free(P); free(E); free(cs); free(ds); free(Wn); free(Av); free(Sv);
  }
  /* pi' ghosts for the next substep (kernels.cu:958-963) */
  bc_x(g, p->bc_x_open, s->pip, g->nx - 1);
  bc_y(g, p->bc_y_open, s->pip, g->ny - 1);
  bc_z_zerograd(g, s->pip);
}

void orc_moisture_stage(const orc_grid* g, const orc_state* s0, const orc_state* tend,
                        double dt, orc_state* out) {
  /* kernels.cu:268-273, over every padded point */
  const size_t n = orc_npts(g);
  for (size_t c = 0; c < n; ++c) {
    out->qv[c] = s0->qv[c] + dt * tend->qv[c];
    out->qc[c] = s0->qc[c] + dt * tend->qc[c];
    out->qr[c] = s0->qr[c] + dt * tend->qr[c];
  }
}

float orc_absmax(const double* f, size_t n) {
  /* kernels.cu:278-289: max |f| in float, NaN ranks above every finite value */
  unsigned int best = 0;
  for (size_t c = 0; c < n; ++c) {
    float v = fabsf((float)f[c]);
    unsigned int bits;
    memcpy(&bits, &v, sizeof(bits));
    if (bits > best) best = bits;
  }
  float out;
  memcpy(&out, &best, sizeof(out));
  return out;
}

double orc_dry_mass(const orc_grid* g, const orc_base* b, const orc_metric* m,
                    const orc_state* s) {
  double total = 0.0;
  for (int k = 0; k < g->nz; ++k) {
    double plane = 0.0;
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        size_t c = I3(g, i, j, k);
        double pi = b->pib[c] + s->pip[c];
        double th = b->thb[c] + s->thp[c];
        double qv = s->qv ? s->qv[c] : 0.0;
        double qt = qv + (s->qc ? s->qc[c] : 0.0) + (s->qr ? s->qr[c] : 0.0);
        double rho = P00 * pow(pi, CV / RD) / (RD * th * (1.0 + EPS61 * qv));
        plane += rho / (1.0 + qt) * m->jac[I2(g, i, j)];
      }
    total += plane * m->dzeta_c[k + g->ng];
  }
  return total * g->dx * g->dy;
}

/* ------------------------------------------------------------- Kessler */
static double fall_speed(double rq, double rho_sfc, double rho, double T) {
  /* terminal velocity, 0.35 factor below freezing (src/physics/kessler.cu:34-56) */
  if (!(rq > 1e-9)) return 0.0;
  return 36.34 * pow(rq, 0.1364) * sqrt(rho_sfc / rho) * (T < TFRZ ? 0.35 : 1.0);
}

void orc_kessler(const orc_grid* g, const orc_base* b, const orc_metric* m, double dt,
                 orc_state* s, double* rain) {
  const int nz = g->nz;
#pragma omp parallel
  {
    double* qrl = dalloc(nz);
    double* rhol = dalloc(nz);
    double* dzl = dalloc(nz);
    double* vr = dalloc(nz);
#pragma omp for schedule(static) collapse(2)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        const double J = m->jac[I2(g, i, j)];
        const double k1 = 0.001, qc0 = 0.001;
        /* 1) sedimentation, first-order upwind, CFL-subcycled (kessler.cu:34-77) */
        double rho_sfc = b->rhob[I3(g, i, j, 0)];
        double vrmax = 0, dzmin = 1e30;
        for (int k = 0; k < nz; ++k) {
          size_t c = I3(g, i, j, k);
          qrl[k] = s->qr[c] > 0.0 ? s->qr[c] : 0.0;
          rhol[k] = b->rhob[c];
          dzl[k] = m->dzeta_c[k + g->ng] * J;
          double T = (b->thb[c] + s->thp[c]) * (b->pib[c] + s->pip[c]);
          vr[k] = fall_speed(rhol[k] * qrl[k], rho_sfc, rhol[k], T);
          if (vr[k] > vrmax) vrmax = vr[k];
          if (dzl[k] < dzmin) dzmin = dzl[k];
        }
        int nsub = 1 + (int)(vrmax * dt / (0.8 * dzmin));
        double dts = dt / (double)nsub;
        double acc = 0;
        for (int sb = 0; sb < nsub; ++sb) {
          double fb = rhol[0] * qrl[0] * vr[0];
          acc += dts * fb;
          for (int k = 0; k < nz; ++k) {
            double ftop = (k + 1 < nz) ? rhol[k + 1] * qrl[k + 1] * vr[k + 1] : 0.0;
            double fbot = rhol[k] * qrl[k] * vr[k];
            qrl[k] += dts * (ftop - fbot) / (rhol[k] * dzl[k]);
          }
          if (sb + 1 < nsub)
            for (int k = 0; k < nz; ++k) {
              size_t c = I3(g, i, j, k);
              double rq = rhol[k] * (qrl[k] > 0.0 ? qrl[k] : 0.0);
              double T = (b->thb[c] + s->thp[c]) * (b->pib[c] + s->pip[c]);
              vr[k] = fall_speed(rq, rho_sfc, rhol[k], T);
            }
        }
        rain[I2(g, i, j)] += acc;
        /* 2+3) conversions, evaporation, mixed-phase saturation adjustment
         * (kessler.cu:89-133) */
        for (int k = 0; k < nz; ++k) {
          size_t c = I3(g, i, j, k);
          double qvk = s->qv[c] > 0.0 ? s->qv[c] : 0.0;
          double qck = s->qc[c] > 0.0 ? s->qc[c] : 0.0;
          double qrk = qrl[k] > 0.0 ? qrl[k] : 0.0;
          double pi = b->pib[c] + s->pip[c];
          double th = b->thb[c] + s->thp[c];
          double T = th * pi;
          double pres = P00 * pow(pi, CP / RD);
          double fl = (T - 233.15) / 40.0;
          fl = dmax(0.0, dmin(1.0, fl));
          double qsw = qsat_water(pres, T);
          double qs = fl * qsw + (1.0 - fl) * qsat_icep(pres, T);
          double Leff = fl * LV + (1.0 - fl) * LS;
          double dqauto = k1 * (qck > qc0 ? qck - qc0 : 0.0);
          double dqacc = 2.2 * qck * pow(qrk > 1e-9 ? qrk : 1e-9, 0.875);
          double dqr = dt * (dqauto + dqacc);
          if (dqr > qck) dqr = qck;
          qck -= dqr;
          qrk += dqr;
          if (qvk < qs && qrk > 0.0) {
            double rq = rhol[k] * qrk;
            double vent = 1.6 + 124.9 * pow(rq, 0.2046);
            double ern = vent * pow(rq, 0.525) / (2.55e8 / (pres * qs) + 5.4e5) * (qs - qvk) / (rhol[k] * qs);
            double dqe = dt * ern;
            if (dqe > qrk) dqe = qrk;
            if (dqe > qs - qvk) dqe = qs - qvk;
            qrk -= dqe;
            qvk += dqe;
            s->thp[c] -= Leff * dqe / (CP * pi);
            th = b->thb[c] + s->thp[c];
            T = th * pi;
            double fl2 = dmax(0.0, dmin(1.0, (T - 233.15) / 40.0));
            qs = fl2 * qsat_water(pres, T) + (1.0 - fl2) * qsat_icep(pres, T);
          }
          double gam = Leff * Leff * qs / (CP * RV * T * T);
          double dq = (qvk - qs) / (1.0 + gam);
          if (dq < 0.0) {
            double evap = -dq;
            if (evap > qck) evap = qck;
            dq = -evap;
          }
          qvk -= dq;
          qck += dq;
          s->thp[c] += Leff * dq / (CP * pi);
          s->qv[c] = qvk > 0.0 ? qvk : 0.0;
          s->qc[c] = qck > 0.0 ? qck : 0.0;
          s->qr[c] = qrk > 0.0 ? qrk : 0.0;
        }
      }
    free(qrl); free(rhol); free(dzl); free(vr);
  }
}

/* ----------------------------------------------- surface layer, PBL, soil */
static const double KAPPA = 0.4, SIGMA = 5.67e-8, S0 = 1361, KM_MAX = 1000, KM_MIN = 0.1;
static const double SOIL_DZ[4] = {0.1, 0.3, 0.6, 1.0};

/* Businger-Dyer stability functions (src/physics/surface.cu:28-41) */
static double psi_mom(double zeta) {
  if (zeta >= 0.0) return -5.0 * dmin(zeta, 2.0);
  double x = pow(1.0 - 16.0 * zeta, 0.25);
  const double halfpi = 1.5707963267948966;
  return 2.0 * log((1.0 + x) * 0.5) + log((1.0 + x * x) * 0.5) - 2.0 * atan(x) + halfpi;
}
static double psi_heat(double zeta) {
  if (zeta >= 0.0) return -5.0 * dmin(zeta, 2.0);
  double x = pow(1.0 - 16.0 * zeta, 0.25);
  return 2.0 * log((1.0 + x * x) * 0.5);
}
static double soil_cap(double w) { return 1.2e6 + 3.2e6 * dmin(dmax(w, 0.0), 0.4); }
static double soil_cond(double w) { return 0.25 + 3.0 * dmin(dmax(w, 0.0), 0.4); }

/* implicit column diffusion, Thomas (surface.cu:61-84); work arrays of nz */
static void column_diffuse(int nz, double dt, const double* rho, const double* rhow,
                           const double* dzc, const double* dzw, const double* Kw, double src0,
                           double* phi, const double* fcg, double* A, double* B, double* C,
                           double* D) {
  for (int k = 0; k < nz; ++k) {
    double a = (k > 0) ? rhow[k] * Kw[k] / dzw[k] : 0.0;
    double c = (k < nz - 1) ? rhow[k + 1] * Kw[k + 1] / dzw[k + 1] : 0.0;
    double mm = rho[k] * dzc[k] / dt;
    A[k] = -a;
    B[k] = mm + a + c;
    C[k] = -c;
    D[k] = mm * phi[k];
    if (fcg) D[k] += fcg[k] - fcg[k + 1];
  }
  D[0] += src0;
  for (int k = 1; k < nz; ++k) {
    double w = A[k] / B[k - 1];
    B[k] -= w * C[k - 1];
    D[k] -= w * D[k - 1];
  }
  phi[nz - 1] = D[nz - 1] / B[nz - 1];
  for (int k = nz - 2; k >= 0; --k) phi[k] = (D[k] - C[k] * phi[k + 1]) / B[k];
}

void orc_sfc_init(const orc_grid* g, orc_sfc* s, const double* tsk, const double* land,
                  const double* lat, const double* lon, const double* soilw,
                  double start_hour, int doy, int nonlocal) {
  /* src/physics/surface.cu:440-482 */
  const size_t n = orc_npts(g), n2 = (size_t)g->NX * g->NY;
  s->km = dalloc(n);
  s->tsk = dalloc(n2); s->tdeep = dalloc(n2); s->land = dalloc(n2); s->lat = dalloc(n2);
  s->lon = dalloc(n2); s->soilw = dalloc(n2); s->cdv = dalloc(n2); s->pblh = dalloc(n2);
  s->t2m = dalloc(n2); s->u10 = dalloc(n2); s->soilt = dalloc(4 * n2);
  s->start_hour = start_hour; s->doy = doy; s->nonlocal = nonlocal;
  for (int j = 0; j < g->ny; ++j)
    for (int i = 0; i < g->nx; ++i) {
      size_t q = I2(g, i, j), src = (size_t)j * g->nx + i;
      s->tsk[q] = tsk[src];
      s->tdeep[q] = tsk[src];
      s->land[q] = land[src];
      s->lat[q] = lat[src];
      s->lon[q] = lon[src];
      s->soilw[q] = soilw[src];
      for (int L = 0; L < 4; ++L) s->soilt[(size_t)L * n2 + q] = tsk[src];
    }
}

void orc_sfc_free(orc_sfc* s) {
  double* ps[] = {s->km, s->tsk, s->tdeep, s->land, s->lat, s->lon, s->soilw,
                  s->cdv, s->pblh, s->t2m, s->u10, s->soilt};
  for (double* q : ps) free(q);
  memset(s, 0, sizeof(*s));
}

static void sfc_scalar_column(const orc_grid* g, const orc_base* b, const orc_metric* m,
                              orc_sfc* sf, double dt, double utc, orc_state* st, int i, int j,
                              double* wk) {
  /* mass column: surface layer + radiation + soil + K profile + implicit
   * scalar mixing (src/physics/surface.cu:87-387) */
  const int nz = g->nz;
  const size_t n2plane = (size_t)g->NX * g->NY;
  double* rho = wk;            double* rhow = rho + nz;     double* dzc = rhow + nz;
  double* dzw = dzc + nz;      double* uc = dzw + nz;       double* vc = uc + nz;
  double* thv = vc + nz;       double* Kw = thv + nz;       double* thcol = Kw + nz;
  double* qvcol = thcol + nz;  double* Tlev = qvcol + nz;   double* epslw = Tlev + nz;
  double* Fup = epslw + nz;    double* Fdn = Fup + nz + 1;  double* radht = Fdn + nz + 1;
  double* swabs = radht + nz;  double* fcg_th = swabs + nz; double* fcg_qv = fcg_th + nz + 1;
  double* tA = fcg_qv + nz + 1; double* tB = tA + nz; double* tC = tB + nz; double* tD = tC + nz;

  size_t c2 = I2(g, i, j);
  const double J = m->jac[c2];
  double lwp = 0;
  for (int k = 0; k < nz; ++k) {
    int kk = k + g->ng;
    size_t c = I3(g, i, j, k);
    rho[k] = b->rhob[c];
    rhow[k] = b->rhobw[c];
    dzc[k] = m->dzeta_c[kk] * J;
    dzw[k] = m->dzeta_w[kk] * J;
    uc[k] = 0.5 * (st->u[I3(g, i, j, k)] + st->u[I3(g, i + 1, j, k)]);
    vc[k] = 0.5 * (st->v[I3(g, i, j, k)] + st->v[I3(g, i, j + 1, k)]);
    thcol[k] = b->thb[c] + st->thp[c];
    qvcol[k] = st->qv[c];
    thv[k] = thcol[k] * (1.0 + EPS61 * qvcol[k]);
    lwp += rho[k] * (st->qc[c] > 0.0 ? st->qc[c] : 0.0) * dzc[k] * 1000.0;
  }
  /* Louis (1979) surface layer (surface.cu:120-161) */
  int onland = sf->land[c2] > 0.5;
  double z0 = onland ? 0.1 : 2e-4;
  double alb = onland ? 0.2 : 0.08;
  double beta;
  if (onland) {
    double f = (sf->soilw[c2] - 0.08) / (0.32 - 0.08);
    f = dmin(1.0, dmax(0.0, f));
    beta = dmax(0.05, f * f);
  } else {
    beta = 1.0;
  }
  double z1 = 0.5 * dzc[0];
  double V1 = sqrt(uc[0] * uc[0] + vc[0] * vc[0]);
  if (V1 < 0.5) V1 = 0.5;
  size_t c0 = I3(g, i, j, 0);
  double pi1 = b->pib[c0] + st->pip[c0];
  double p1 = P00 * pow(pi1, CP / RD);
  double Ts = sf->tsk[c2];
  double pis = pi1 + GRAV * z1 / (CP * thv[0]);
  double ths = Ts / pis;
  double qs_s = qsat_water(p1, Ts);
  double thvs = ths * (1.0 + EPS61 * (beta * qs_s + (1.0 - beta) * qvcol[0]));
  double Rib = GRAV * z1 * (thv[0] - thvs) / (thvs * V1 * V1);
  double a2 = KAPPA / log(z1 / z0);
  a2 *= a2;
  double Fm, Fh;
  if (Rib < 0.0) {
    double sq = sqrt(-Rib * z1 / z0);
    Fm = 1.0 - 9.4 * Rib / (1.0 + 7.4 * 9.4 * a2 * sq);
    Fh = 1.0 - 9.4 * Rib / (1.0 + 5.3 * 9.4 * a2 * sq);
  } else {
    double d = 1.0 + 4.7 * Rib;
    Fm = Fh = 1.0 / (d * d);
  }
  double Cd = a2 * Fm, Ch = a2 * Fh;
  sf->cdv[c2] = Cd * V1;
  /* 2 m / 10 m diagnostics (surface.cu:163-182) */
  double z0h = z0 * 0.1;
  double lnz1z0 = log(z1 / z0);
  double zeta1 = (Rib >= 0.0) ? Rib * lnz1z0 / (1.0 - 5.0 * dmin(Rib, 0.19)) : Rib * lnz1z0;
  zeta1 = dmax(-8.0, dmin(2.0, zeta1));
  double zol = zeta1 / z1;
  double den_m = lnz1z0 - psi_mom(zeta1) + psi_mom(z0 * zol);
  double num_m = log(10.0 / z0) - psi_mom(10.0 * zol) + psi_mom(z0 * zol);
  double r10 = dmax(0.0, dmin(1.2, num_m / dmax(den_m, 0.1)));
  sf->u10[c2] = V1 * r10;
  double den_h = log(z1 / z0h) - psi_heat(zeta1) + psi_heat(z0h * zol);
  double num_h = log(2.0 / z0h) - psi_heat(2.0 * zol) + psi_heat(z0h * zol);
  double r2 = dmax(0.0, dmin(1.2, num_h / dmax(den_h, 0.1)));
  double th2 = ths + (thcol[0] - ths) * r2;
  sf->t2m[c2] = th2 * pi1;
  double shf = Ch * V1 * (ths - thcol[0]);
  double qflx = Ch * V1 * beta * (qs_s - qvcol[0]);
  if (!onland && qflx < 0.0) qflx = 0;
  /* two-stream broadband radiation (surface.cu:188-243) */
  double decl = 0.40928 * sin(6.2832 * (284.0 + sf->doy) / 365.0);
  double latr = sf->lat[c2] * 0.0174533;
  double hsol = utc + sf->lon[c2] / 15.0;
  double H = 0.2618 * (hsol - 12.0);
  double cosz = sin(latr) * sin(decl) + cos(latr) * cos(decl) * cos(H);
  if (cosz < 0.0) cosz = 0;
  for (int k = 0; k < nz; ++k) {
    size_t c = I3(g, i, j, k);
    double pik = b->pib[c] + st->pip[c];
    Tlev[k] = thcol[k] * pik;
    double du = rho[k] * qvcol[k] * dzc[k];
    double dl = rho[k] * (st->qc[c] > 0.0 ? st->qc[c] : 0.0) * dzc[k] * 1000.0;
    epslw[k] = 1.0 - exp(-(0.22 * du + 0.30 * dl));
  }
  Fdn[nz] = 0.0;
  for (int k = nz - 1; k >= 0; --k)
    Fdn[k] = Fdn[k + 1] * (1.0 - epslw[k]) + epslw[k] * SIGMA * Tlev[k] * Tlev[k] * Tlev[k] * Tlev[k];
  double lwd = Fdn[0];
  Fup[0] = 0.97 * SIGMA * Ts * Ts * Ts * Ts + 0.03 * Fdn[0];
  for (int k = 0; k < nz; ++k)
    Fup[k + 1] = Fup[k] * (1.0 - epslw[k]) + epslw[k] * SIGMA * Tlev[k] * Tlev[k] * Tlev[k] * Tlev[k];
  double mu = dmax(cosz, 0.05);
  double cldalb = lwp / (lwp + 60.0);
  double Sdn = S0 * cosz * 0.95 * (1.0 - cldalb);
  for (int k = nz - 1; k >= 0; --k) {
    size_t c = I3(g, i, j, k);
    double du = rho[k] * qvcol[k] * dzc[k];
    double dl = rho[k] * (st->qc[c] > 0.0 ? st->qc[c] : 0.0) * dzc[k] * 1000.0;
    double tau = exp(-(0.008 * du + 0.15 * dl) / mu);
    double ab = Sdn * (1.0 - tau);
    swabs[k] = ab;
    Sdn *= tau;
  }
  double swn = Sdn * (1.0 - alb);
  for (int k = 0; k < nz; ++k) {
    size_t c = I3(g, i, j, k);
    double pik = b->pib[c] + st->pip[c];
    double lwconv = (Fdn[k + 1] - Fdn[k]) + (Fup[k] - Fup[k + 1]);
    double net = lwconv + swabs[k];
    radht[k] = net / (rho[k] * CP * dzc[k]) / pik;
  }
  /* 4-layer implicit soil (surface.cu:245-282) */
  double lwu = 0.97 * SIGMA * Ts * Ts * Ts * Ts;
  double G = swn + 0.97 * lwd - lwu - rho[0] * CP * shf * pi1 - rho[0] * LV * qflx;
  if (onland) {
    double Cso = soil_cap(sf->soilw[c2]), Kso = soil_cond(sf->soilw[c2]);
    double Tso[4], A[4], B[4], C[4], D[4];
    for (int L = 0; L < 4; ++L) Tso[L] = sf->soilt[(size_t)L * n2plane + c2];
    for (int L = 0; L < 4; ++L) {
      double cap = Cso * SOIL_DZ[L] / dt;
      double ku = (L > 0) ? Kso / (0.5 * (SOIL_DZ[L - 1] + SOIL_DZ[L])) : 0.0;
      double kl = (L < 3) ? Kso / (0.5 * (SOIL_DZ[L] + SOIL_DZ[L + 1])) : Kso / SOIL_DZ[L];
      A[L] = -ku;
      C[L] = (L < 3) ? -kl : 0.0;
      B[L] = cap + ku + kl;
      D[L] = cap * Tso[L];
    }
    D[0] += G;
    D[3] += (Kso / SOIL_DZ[3]) * sf->tdeep[c2];
    for (int L = 1; L < 4; ++L) {
      double w = A[L] / B[L - 1];
      B[L] -= w * C[L - 1];
      D[L] -= w * D[L - 1];
    }
    Tso[3] = D[3] / B[3];
    for (int L = 2; L >= 0; --L) Tso[L] = (D[L] - C[L] * Tso[L + 1]) / B[L];
    for (int L = 0; L < 4; ++L) {
      if (Tso[L] < 200.0) Tso[L] = 200;
      if (Tso[L] > 350.0) Tso[L] = 350;
      sf->soilt[(size_t)L * n2plane + c2] = Tso[L];
    }
    sf->tsk[c2] = Tso[0];
  }
  /* eddy diffusivity: local Ri (surface.cu:285-298) or nonlocal Troen-Mahrt
   * with counter-gradient fluxes (surface.cu:304-371) */
#define LOCAL_K(k, out)                                                          \
  do {                                                                           \
    double dz_ = dzw[k];                                                         \
    double du_ = (uc[k] - uc[k - 1]) / dz_, dv_ = (vc[k] - vc[k - 1]) / dz_;     \
    double S2_ = du_ * du_ + dv_ * dv_ + 1e-8;                                   \
    double thvw_ = 0.5 * (thv[k - 1] + thv[k]);                                  \
    double N2_ = GRAV / thvw_ * (thv[k] - thv[k - 1]) / dz_;                     \
    double Ri_ = N2_ / S2_;                                                      \
    double zw_ = m->zeta_w[(k) + g->ng] * J;                                     \
    double l_ = KAPPA * zw_ / (1.0 + KAPPA * zw_ / 150.0);                       \
    if (Ri_ < 0.0) out = l_ * l_ * sqrt(S2_) * sqrt(1.0 - 16.0 * Ri_);           \
    else { double d_ = 1.0 + 5.0 * Ri_; out = l_ * l_ * sqrt(S2_) / (d_ * d_); } \
  } while (0)
  Kw[0] = 0;
  fcg_th[0] = fcg_qv[0] = fcg_th[nz] = fcg_qv[nz] = 0;
  if (sf->nonlocal) {
    double ust = sqrt(Cd) * V1;
    double thv1 = thv[0];
    double wthv0 = shf * (1.0 + EPS61 * qvcol[0]) + EPS61 * thcol[0] * qflx;
    const double Ric = 0.25;
    double hpbl = m->zeta_c[(nz - 1) + g->ng] * J;
    double ws = ust > 0.1 ? ust : 0.1;
    for (int it = 0; it < 3; ++it) {
      double exc = (wthv0 > 0.0) ? 6.8 * wthv0 / ws : 0.0;
      double thv_s = thv1 + exc;
      double prevRb = 0;
      hpbl = m->zeta_c[(nz - 1) + g->ng] * J;
      for (int k = 1; k < nz; ++k) {
        double zc = m->zeta_c[k + g->ng] * J;
        double shear = uc[k] * uc[k] + vc[k] * vc[k] + 0.1;
        double Rbk = GRAV * (thv[k] - thv_s) * zc / (thv1 * shear);
        if (Rbk >= Ric) {
          double zcm = m->zeta_c[(k - 1) + g->ng] * J;
          double f = (Ric - prevRb) / (Rbk - prevRb + 1e-9);
          f = dmin(1.0, dmax(0.0, f));
          hpbl = zcm + f * (zc - zcm);
          break;
        }
        prevRb = Rbk;
      }
      double zc0 = m->zeta_c[g->ng] * J;
      if (hpbl < zc0) hpbl = zc0;
      double wstar = (wthv0 > 0.0) ? cbrt(GRAV / thv1 * wthv0 * hpbl) : 0.0;
      ws = cbrt(ust * ust * ust + 0.6 * wstar * wstar * wstar);
      if (ws < 0.1) ws = 0.1;
    }
    sf->pblh[c2] = hpbl;
    double gth = (wthv0 > 0.0) ? 6.8 * shf / (ws * hpbl) : 0.0;
    double gqv = (wthv0 > 0.0) ? 6.8 * qflx / (ws * hpbl) : 0.0;
    for (int k = 1; k < nz; ++k) {
      double zw = m->zeta_w[k + g->ng] * J;
      double Kv;
      if (wthv0 > 0.0 && zw < hpbl) {
        double zf = zw / hpbl;
        Kv = KAPPA * ws * zw * (1 - zf) * (1 - zf);
        fcg_th[k] = rhow[k] * Kv * gth;
        fcg_qv[k] = rhow[k] * Kv * gqv;
      } else {
        LOCAL_K(k, Kv);
        fcg_th[k] = fcg_qv[k] = 0;
      }
      if (Kv < KM_MIN) Kv = KM_MIN;
      if (Kv > KM_MAX) Kv = KM_MAX;
      Kw[k] = Kv;
      sf->km[I3(g, i, j, k)] = Kv;
    }
  } else {
    sf->pblh[c2] = 0;
    for (int k = 1; k < nz; ++k) {
      double Kv;
      LOCAL_K(k, Kv);
      if (Kv < KM_MIN) Kv = KM_MIN;
      if (Kv > KM_MAX) Kv = KM_MAX;
      Kw[k] = Kv;
      sf->km[I3(g, i, j, k)] = Kv;
      fcg_th[k] = fcg_qv[k] = 0;
    }
  }
#undef LOCAL_K
  column_diffuse(nz, dt, rho, rhow, dzc, dzw, Kw, rho[0] * shf, thcol, fcg_th, tA, tB, tC, tD);
  column_diffuse(nz, dt, rho, rhow, dzc, dzw, Kw, rho[0] * qflx, qvcol, fcg_qv, tA, tB, tC, tD);
  for (int k = 0; k < nz; ++k) {
    size_t c = I3(g, i, j, k);
    double dth = dt * radht[k];
    if (dth > 0.02) dth = 0.02;
    if (dth < -0.02) dth = -0.02;
    st->thp[c] = thcol[k] - b->thb[c] + dth;
    double q = qvcol[k];
    st->qv[c] = q > 0.0 ? q : 0.0;
  }
}

/* momentum columns on u (di=1) or v (dj=1) faces: drag + implicit mixing
 * (surface.cu:390-436) */
static void sfc_face_column(const orc_grid* g, const orc_base* b, const orc_metric* m,
                            const orc_sfc* sf, double dt, double* f, int i, int j, int di,
                            int dj, double* wk) {
  const int nz = g->nz;
  double* rho = wk;       double* rhow = rho + nz; double* dzc = rhow + nz; double* dzw = dzc + nz;
  double* Kw = dzw + nz;  double* phi = Kw + nz;   double* tA = phi + nz;   double* tB = tA + nz;
  double* tC = tB + nz;   double* tD = tC + nz;
  double J = 0.5 * (m->jac[I2(g, i - di, j - dj)] + m->jac[I2(g, i, j)]);
  for (int k = 0; k < nz; ++k) {
    int kk = k + g->ng;
    size_t c = I3(g, i, j, k), cb = I3(g, i - di, j - dj, k);
    rho[k] = 0.5 * (b->rhob[cb] + b->rhob[c]);
    rhow[k] = 0.5 * (b->rhobw[cb] + b->rhobw[c]);
    dzc[k] = m->dzeta_c[kk] * J;
    dzw[k] = m->dzeta_w[kk] * J;
    Kw[k] = (k > 0) ? 0.5 * (sf->km[cb] + sf->km[c]) : 0.0;
    phi[k] = f[c];
  }
  double cdva = 0.5 * (sf->cdv[I2(g, i - di, j - dj)] + sf->cdv[I2(g, i, j)]);
  double src0 = -rho[0] * cdva * phi[0];
  column_diffuse(nz, dt, rho, rhow, dzc, dzw, Kw, src0, phi, NULL, tA, tB, tC, tD);
  for (int k = 0; k < nz; ++k) f[I3(g, i, j, k)] = phi[k];
}

void orc_sfc_step(const orc_grid* g, const orc_base* b, const orc_metric* m, orc_sfc* sf,
                  double dt, double t, orc_state* st) {
  /* src/physics/surface.cu:499-514 */
  double utc = sf->start_hour + t / 3600.0;
  utc = utc - 24.0 * floor(utc / 24.0);
  const int nz = g->nz;
  const size_t wsz = (size_t)(24 * nz + 8);
#pragma omp parallel
  {
    double* wk = dalloc(wsz);
#pragma omp for schedule(static) collapse(2)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) sfc_scalar_column(g, b, m, sf, dt, utc, st, i, j, wk);
#pragma omp for schedule(static) collapse(2)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 1; i < g->nx; ++i) sfc_face_column(g, b, m, sf, dt, st->u, i, j, 1, 0, wk);
#pragma omp for schedule(static) collapse(2)
    for (int j = 1; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) sfc_face_column(g, b, m, sf, dt, st->v, i, j, 0, 1, wk);
    free(wk);
  }
}

/* ------------------------------------------------------------ integrator */
struct orc_integ {
  orc_grid g;
  const orc_base* b;
  const orc_metric* m;
  orc_params p;
  orc_state sn, sstage, swork, tend;
  double *div, *piprev, *mfx, *mfy, *mfz, *rain;
  double *rtjx, *rtjy, *kt3, *aw;
  double* pd[4];
  double* const* lo;
  double* const* hi;
  const double* wgt;
  double t_lo, t_hi;
  orc_sfc* sfc;
};

static void state_alloc(orc_state* s, size_t n) {
  s->u = dalloc(n); s->v = dalloc(n); s->w = dalloc(n); s->thp = dalloc(n);
  s->pip = dalloc(n); s->qv = dalloc(n); s->qc = dalloc(n); s->qr = dalloc(n);
}
static void state_free(orc_state* s) {
  free(s->u); free(s->v); free(s->w); free(s->thp); free(s->pip); free(s->qv); free(s->qc); free(s->qr);
}
static void state_copy(orc_state* d, const orc_state* s, size_t n) {
  memcpy(d->u, s->u, n * 8); memcpy(d->v, s->v, n * 8); memcpy(d->w, s->w, n * 8);
  memcpy(d->thp, s->thp, n * 8); memcpy(d->pip, s->pip, n * 8); memcpy(d->qv, s->qv, n * 8);
  memcpy(d->qc, s->qc, n * 8); memcpy(d->qr, s->qr, n * 8);
}
static void state_swap(orc_state* a, orc_state* b) {
  orc_state t = *a;
  *a = *b;
  *b = t;
}

orc_integ* orc_integ_create(const orc_grid* g, const orc_base* b, const orc_metric* m,
                            const orc_params* p) {
  /* src/dynamics/integrator.cpp:43-69 */
  orc_integ* it = (orc_integ*)calloc(1, sizeof(orc_integ));
  it->g = *g; it->b = b; it->m = m; it->p = *p;
  size_t n = orc_npts(g);
  state_alloc(&it->sn, n); state_alloc(&it->sstage, n); state_alloc(&it->swork, n);
  state_alloc(&it->tend, n);
  it->div = dalloc(n); it->piprev = dalloc(n); it->mfx = dalloc(n); it->mfy = dalloc(n);
  it->mfz = dalloc(n); it->rain = dalloc((size_t)g->NX * g->NY);
  it->rtjx = dalloc(n); it->rtjy = dalloc(n); it->kt3 = dalloc(n); it->aw = dalloc(n);
  for (int q = 0; q < 4; ++q) it->pd[q] = p->pd_moist ? dalloc(n) : NULL;
  orc_acoustic_coef(g, b, m, it->rtjx, it->rtjy, it->kt3, it->aw);
  return it;
}

void orc_integ_free(orc_integ* it) {
  if (!it) return;
  state_free(&it->sn); state_free(&it->sstage); state_free(&it->swork); state_free(&it->tend);
  double* ps[] = {it->div, it->piprev, it->mfx, it->mfy, it->mfz, it->rain,
                  it->rtjx, it->rtjy, it->kt3, it->aw, it->pd[0], it->pd[1], it->pd[2], it->pd[3]};
  for (double* q : ps) free(q);
  free(it);
}

orc_state* orc_integ_state(orc_integ* it) { return &it->sn; }
double* orc_integ_rain(orc_integ* it) { return it->rain; }

void orc_integ_set_bdy(orc_integ* it, double* const* lo, double* const* hi, const double* wgt,
                       double t_lo, double t_hi) {
  it->lo = lo; it->hi = hi; it->wgt = wgt; it->t_lo = t_lo; it->t_hi = t_hi;
}
void orc_integ_set_sfc(orc_integ* it, orc_sfc* sf) { it->sfc = sf; }

void orc_integ_step(orc_integ* it, double dt, double t) {
  /* Wicker-Skamarock RK3 with split-explicit acoustic substeps
   * (src/dynamics/integrator.cpp:71-111) */
  const orc_grid* g = &it->g;
  const size_t n = orc_npts(g);
  const double stage_dt[3] = {dt / 3, dt / 2, dt};
  const int ns = it->p.acoustic_ns > 1 ? it->p.acoustic_ns : 1;
  const int ns_stage[3] = {1, ns / 2 > 1 ? ns / 2 : 1, ns};
  double tf = 0.0;
  if (it->lo) { /* BdyManager::tfrac (boundary.cpp:91-97) */
    if (it->t_hi > it->t_lo) {
      tf = (t - it->t_lo) / (it->t_hi - it->t_lo);
      tf = tf < 0 ? 0 : (tf > 1 ? 1.0 : tf);
    }
  }
  for (int mstage = 0; mstage < 3; ++mstage) {
    orc_state* est = mstage == 0 ? &it->sn : &it->sstage;
    orc_apply_bcs(g, &it->p, est);
    orc_mass_fluxes(g, it->b, it->m, est, it->mfx, it->mfy, it->mfz);
    orc_divergence(g, it->m, it->mfx, it->mfy, it->mfz, it->div);
    orc_tendencies(g, it->b, it->m, &it->p, dt, est, it->mfx, it->mfy, it->mfz, it->div,
                   &it->tend, it->p.pd_moist ? it->pd : NULL);
    if (it->lo) orc_bdy_relax(g, est, it->lo, it->hi, tf, it->wgt, &it->tend);
    state_copy(&it->swork, &it->sn, n);
    memcpy(it->piprev, it->sn.pip, n * sizeof(double));
    double dtau = stage_dt[mstage] / ns_stage[mstage];
    for (int s = 0; s < ns_stage[mstage]; ++s)
      orc_acoustic_substep(g, it->b, it->m, &it->p, dtau, &it->swork, &it->tend, it->piprev,
                           it->rtjx, it->rtjy, it->kt3, it->aw);
    if (it->p.moisture) orc_moisture_stage(g, &it->sn, &it->tend, stage_dt[mstage], &it->swork);
    state_swap(&it->sstage, &it->swork);
  }
  state_swap(&it->sn, &it->sstage);
  if (it->p.moisture && it->p.microphysics) orc_kessler(g, it->b, it->m, dt, &it->sn, it->rain);
  if (it->sfc) orc_sfc_step(g, it->b, it->m, it->sfc, dt, t + dt, &it->sn);
}
