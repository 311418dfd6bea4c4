"""Seeded synthetic inputs in the reference's prep format (version 3).

The reference's file-mode cases (profile = file, terrain = file) read what
tools/prep_gfs.py:320-365 writes from GFS analyses:

  wfe_input.ini      version, nx, ny, nz, np_prof, start, bdy_interval, n_bdy, hours
  wfe_init.bin       float32: the profile tables z, theta, qv, u (np_prof each,
                     100 m spacing); the 2D fields h, fcor, tsk, land, lat, lon,
                     soilw (ny*nx each); the 3D cell-centre fields u, v, theta,
                     Exner, qv (nz*ny*nx each, i fastest)
  wfe_bdy_FFF.bin    float32 u, v, theta, Exner, qv (nz*ny*nx each) for forecast
                     hour FFF = idx * bdy_interval / 3600

(layout read back by src/io/input.cpp:19-73).  This module writes the same
files from analytic, seeded fields instead of network data:

  terrain     a sum of 6-12 Gaussian ridges, h = sum A exp(-(a/La)^2 - (c/Lc)^2)
              in ridge-aligned coordinates (a, c), peaks A up to 3 km, half-widths
              La, Lc in 30-150 km, capped at 3 km
  sounding    US standard lapse rates: T = 288.15 K - 6.5 K/km to 11 km and
              216.65 K above, p from the hydrostatic standard-atmosphere formula
              with 1000 hPa at z = 0 (where the model's base state puts Exner = 1),
              relative humidity 0.8 (1 - z/12 km)^1.25 (0 above 12 km), qv from the
              Tetens saturation mixing ratio, capped at 16 g/kg
  wind        a uniform westerly u0 per member (v = 0)
  noise       theta' with standard deviation theta_sigma (K) and multiplicative
              qv' with standard deviation qv_sigma, both white noise filtered by a
              horizontal Gaussian whose correlation length (e-folding of the
              correlation) is corr_len, then [1 2 1]-smoothed in the vertical and
              rescaled; the noise is in the initial fields only
  boundaries  every boundary file holds the unperturbed fields (constant lateral
              targets), so Davies relaxation pulls the edges toward the
              unperturbed state
  surface     land where the terrain exceeds 20 m or a seeded blob pattern says
              so, soil moisture 0.15-0.35 over land (0.25 over water), skin
              temperature from the lapse rate at the terrain height, lat/lon from
              the inverse Lambert conformal projection of the grid (spherical
              Earth), fcor = 2 Omega sin(lat)

The model places cell centres at z = h + zeta_c (zt - h) / zt
(src/core/metric.cpp); the generator supports the uniform vertical grid
(stretch = none), zeta_c = (k + 1/2) dz, zt = nz dz.
"""

from __future__ import annotations

import os
import shutil
from pathlib import Path

import numpy as np

RD = 287.04
CP = 1004.5
GRAV = 9.81
P00 = 1.0e5
OMEGA = 7.292e-5
EARTH_R = 6.371e6


# --------------------------------------------------------------- geometry
def lambert_latlon(nx, ny, dx, dy, lat0=39.0, lon0=35.0, lat1=35.0, lat2=43.0):
    """Latitude/longitude (degrees, shape (ny, nx)) of the cell centres of a grid
    centred on (lat0, lon0) in a Lambert conformal projection with standard
    parallels lat1, lat2 on a sphere (Snyder 1987, eqs. 15-1 to 15-3, 14-4)."""
    r = np.radians
    p0, p1, p2 = r(lat0), r(lat1), r(lat2)
    if abs(lat1 - lat2) < 1e-9:
        n = np.sin(p1)
    else:
        n = np.log(np.cos(p1) / np.cos(p2)) / np.log(np.tan(np.pi / 4 + p2 / 2) /
                                                     np.tan(np.pi / 4 + p1 / 2))
    F = np.cos(p1) * np.tan(np.pi / 4 + p1 / 2) ** n / n
    rho0 = EARTH_R * F / np.tan(np.pi / 4 + p0 / 2) ** n
    x = (np.arange(nx) + 0.5 - nx / 2.0) * dx
    y = (np.arange(ny) + 0.5 - ny / 2.0) * dy
    X, Y = np.meshgrid(x, y)
    rho = np.sign(n) * np.sqrt(X ** 2 + (rho0 - Y) ** 2)
    theta = np.arctan2(np.sign(n) * X, np.sign(n) * (rho0 - Y))
    lat = 2.0 * np.arctan((EARTH_R * F / rho) ** (1.0 / n)) - np.pi / 2
    lon = r(lon0) + theta / n
    return np.degrees(lat), np.degrees(lon)


def ridges(rng, nx, ny, dx, dy, n_min=6, n_max=12, h_max=3000.0, w_min=30e3, w_max=150e3):
    """Sum of n_min..n_max Gaussian ridges, peak <= h_max, half-widths in [w_min, w_max]."""
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(x, y)
    h = np.zeros((ny, nx))
    for _ in range(int(rng.integers(n_min, n_max + 1))):
        xc, yc = rng.uniform(0, nx * dx), rng.uniform(0, ny * dy)
        amp = rng.uniform(0.2, 1.0) * h_max
        la, lc = rng.uniform(w_min, w_max, size=2)
        ang = rng.uniform(0, np.pi)
        a = (X - xc) * np.cos(ang) + (Y - yc) * np.sin(ang)
        c = -(X - xc) * np.sin(ang) + (Y - yc) * np.cos(ang)
        h += amp * np.exp(-(a / la) ** 2 - (c / lc) ** 2)
    return np.minimum(h, h_max)


# ---------------------------------------------------------------- sounding
def standard_atmosphere(z):
    """Temperature (K) and pressure (Pa): US standard lapse rates, 1000 hPa at z = 0."""
    z = np.asarray(z, dtype=np.float64)
    t0, gam, z11 = 288.15, 6.5e-3, 11000.0
    p0 = P00
    t11 = t0 - gam * z11
    p11 = p0 * (t11 / t0) ** (GRAV / (RD * gam))
    T = np.where(z <= z11, t0 - gam * z, t11)
    p = np.where(z <= z11, p0 * (np.maximum(T, 1.0) / t0) ** (GRAV / (RD * gam)),
                 p11 * np.exp(-GRAV * (z - z11) / (RD * t11)))
    return T, p


def qsat_tetens(T, p):
    """Saturation mixing ratio over water (Tetens, es in hPa)."""
    es = 6.1078 * np.exp(17.27 * (T - 273.15) / (T - 35.86)) * 100.0
    return 0.622 * es / np.maximum(p - es, 1.0)


def sounding(z):
    """theta (K), Exner, qv (kg/kg) at heights z (m)."""
    T, p = standard_atmosphere(z)
    exner = (p / P00) ** (RD / CP)
    theta = T / exner
    rh = 0.8 * np.clip(1.0 - np.asarray(z) / 12000.0, 0.0, 1.0) ** 1.25
    qv = np.minimum(rh * qsat_tetens(T, p), 0.016)
    return theta, exner, qv


# ------------------------------------------------------------------- noise
def correlated_noise(rng, shape, dx, dy, corr_len):
    """Unit-variance noise, Gaussian-correlated horizontally (e-folding length
    corr_len of the correlation), [1 2 1] smoothed in the vertical."""
    nz, ny, nx = shape
    w = rng.standard_normal(shape)
    kx = 2 * np.pi * np.fft.fftfreq(nx, d=dx)
    ky = 2 * np.pi * np.fft.fftfreq(ny, d=dy)
    s = corr_len / 2.0  # Gaussian kernel width: correlation exp(-r^2 / (4 s^2))
    tf = np.exp(-0.5 * s * s * (ky[:, None] ** 2 + kx[None, :] ** 2))
    f = np.real(np.fft.ifft2(np.fft.fft2(w, axes=(1, 2)) * tf[None], axes=(1, 2)))
    if nz > 2:
        g = f.copy()
        g[1:-1] = 0.25 * f[:-2] + 0.5 * f[1:-1] + 0.25 * f[2:]
        f = g
    sd = f.std()
    return f / sd if sd > 0 else f


# ------------------------------------------------------------------ writer
def write_prep(outdir, *, nx, ny, nz, dx, dy, dz, seed, u0=10.0, theta_sigma=0.5,
               qv_sigma=0.05, corr_len=50e3, hours=24, bdy_interval=10800,
               start="2024062100", proj=(39.0, 35.0, 35.0, 43.0), flat=False):
    """Write wfe_input.ini, wfe_init.bin and the wfe_bdy_FFF.bin files into outdir.

    Returns a dict of the generated arrays (float32 as written)."""
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    zt = nz * dz
    h = np.zeros((ny, nx)) if flat else ridges(rng, nx, ny, dx, dy)
    lat, lon = lambert_latlon(nx, ny, dx, dy, *proj)
    fcor = 2 * OMEGA * np.sin(np.radians(lat))
    blob = correlated_noise(rng, (1, ny, nx), dx, dy, 200e3)[0]
    land = ((h > 20.0) | (blob > -0.3)).astype(np.float64)
    soilw = np.where(land > 0.5, 0.25 + 0.1 * np.tanh(correlated_noise(
        rng, (1, ny, nx), dx, dy, 100e3)[0]), 0.25)
    tsk = 288.15 - 6.5e-3 * h + 1.5 * correlated_noise(rng, (1, ny, nx), dx, dy, 80e3)[0]

    npf = int(zt // 100) + 2
    ztab = np.arange(npf) * 100.0
    th_tab, _, qv_tab = sounding(ztab)
    u_tab = np.full(npf, float(u0))

    zc = (np.arange(nz) + 0.5) * dz
    z3 = h[None] + zc[:, None, None] * (zt - h[None]) / zt
    th0, ex0, qv0 = sounding(z3)
    u = np.full((nz, ny, nx), float(u0))
    v = np.zeros((nz, ny, nx))
    thp = theta_sigma * correlated_noise(rng, (nz, ny, nx), dx, dy, corr_len)
    qvp = qv_sigma * correlated_noise(rng, (nz, ny, nx), dx, dy, corr_len)
    th = th0 + thp
    qv = np.maximum(qv0 * (1.0 + qvp), 0.0)

    f32 = np.float32
    with open(out / "wfe_init.bin", "wb") as f:
        for a in (ztab, th_tab, qv_tab, u_tab, h, fcor, tsk, land, lat, lon, soilw,
                  u, v, th, ex0, qv):
            np.ascontiguousarray(a, dtype=f32).tofile(f)
    step_h = int(bdy_interval // 3600)
    hrs = list(range(0, hours + 1, step_h)) if step_h > 0 else [0]
    first = out / f"wfe_bdy_{hrs[0]:03d}.bin"
    with open(first, "wb") as f:
        for a in (u, v, th0, ex0, qv0):
            np.ascontiguousarray(a, dtype=f32).tofile(f)
    for fh in hrs[1:]:
        p = out / f"wfe_bdy_{fh:03d}.bin"
        if p.exists() or p.is_symlink():
            p.unlink()
        try:
            os.symlink(first.name, p)
        except OSError:
            shutil.copyfile(first, p)
    meta = [
        "version = 3",
        f"nx = {nx}", f"ny = {ny}", f"nz = {nz}",
        f"np_prof = {npf}",
        f"start = {start}",
        f"bdy_interval = {bdy_interval}",
        f"n_bdy = {len(hrs)}",
        f"hours = {hours}",
    ]
    (out / "wfe_input.ini").write_text("\n".join(meta) + "\n")
    return {"h": h, "lat": lat, "lon": lon, "land": land, "u0": float(u0)}


def write_case(path, prep_dir, *, nx, ny, nz, dx, dy, dz, dt=60.0, ns=6, t_end=86400.0,
               bdy_width=5, bdy_tau=600.0, proj=(39.0, 35.0, 35.0, 43.0), extra=None):
    """A file-mode case (.ini) over prep_dir: full physics, Kessler, positive-definite
    moisture, open boundaries with Davies relaxation toward the boundary files."""
    kv = {
        "nx": nx, "ny": ny, "nz": nz, "dx": dx, "dy": dy, "dz": repr(float(dz)),
        "proj_lat0": proj[0], "proj_lon0": proj[1], "proj_lat1": proj[2], "proj_lat2": proj[3],
        "dt": dt, "acoustic_ns": ns, "t_end": t_end,
        "profile": "file", "terrain": "file", "input_dir": str(Path(prep_dir).resolve()),
        "physics": "simple", "pbl": "nonlocal",
        "bc_x": "open", "bc_y": "open",
        "bdy_width": bdy_width, "bdy_tau": bdy_tau, "nudge_tau": 0,
        "w_damping": "on", "pd_moist": "on",
        "rayleigh_zd": 0.75 * nz * dz, "rayleigh_alpha": 0.02,
        "out_dir": str(Path(path).with_suffix("")) + "_out",
        "out_interval": 1e9, "diag_interval": 1e9,
    }
    kv.update(extra or {})
    Path(path).write_text("".join(f"{k} = {v}\n" for k, v in kv.items()))
    return Path(path)


ENSEMBLE_GROUPS = ((120, 90), (220, 150), (300, 200))


def write_ensemble(root, *, groups=ENSEMBLE_GROUPS, per_group=8, nz=45, dx=12000.0,
                   zt=20000.0, seed=2024, hours=24, dt=60.0, ns=6, t_end=None,
                   bdy_interval=None):
    """Members of uneven sizes: per_group members on each (nx, ny) of groups, each
    with its own terrain, u0 ~ U(5, 20) m/s and noise seed.  Returns the case
    paths in member order."""
    root = Path(root)
    root.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    dz = zt / nz
    t_end = float(hours * 3600 if t_end is None else t_end)
    bint = int(bdy_interval or hours * 3600)
    cases = []
    m = 0
    for (nx, ny) in groups:
        for _ in range(per_group):
            u0 = float(rng.uniform(5.0, 20.0))
            mseed = int(rng.integers(0, 2 ** 31 - 1))
            prep = root / f"m{m:02d}_prep"
            write_prep(prep, nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dz, seed=mseed, u0=u0,
                       hours=hours, bdy_interval=bint)
            cases.append(write_case(root / f"m{m:02d}.ini", prep, nx=nx, ny=ny, nz=nz, dx=dx,
                                    dy=dx, dz=dz, dt=dt, ns=ns, t_end=t_end))
            m += 1
    return cases


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("outdir")
    ap.add_argument("--ensemble", action="store_true", help="the 24-member uneven ensemble")
    ap.add_argument("--nx", type=int, default=120)
    ap.add_argument("--ny", type=int, default=90)
    ap.add_argument("--nz", type=int, default=45)
    ap.add_argument("--dx", type=float, default=12000.0)
    ap.add_argument("--zt", type=float, default=20000.0)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--u0", type=float, default=10.0)
    ap.add_argument("--hours", type=int, default=24)
    a = ap.parse_args(argv)
    if a.ensemble:
        for p in write_ensemble(a.outdir, seed=a.seed, hours=a.hours):
            print(p)
        return
    prep = Path(a.outdir) / "prep"
    dz = a.zt / a.nz
    write_prep(prep, nx=a.nx, ny=a.ny, nz=a.nz, dx=a.dx, dy=a.dx, dz=dz, seed=a.seed, u0=a.u0,
               hours=a.hours, bdy_interval=a.hours * 3600)
    print(write_case(Path(a.outdir) / "case.ini", prep, nx=a.nx, ny=a.ny, nz=a.nz, dx=a.dx,
                     dy=a.dx, dz=dz))


if __name__ == "__main__":
    main()
