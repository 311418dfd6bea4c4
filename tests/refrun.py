"""Runs of the benchmark configurations through the reference's own build and
through wfe_b200, and the per-field comparison measures the config-level
parity tests use (test infrastructure).

The reference side is oracle/_ref/refdump_f64 (or _f32): the unmodified
reference kernels and Integrator::step compiled from the reference's sources
by oracle/Makefile, driven through its C++ API by oracle/refdump/refdump.cu
(mode=run: set-up as src/main.cpp:261-383, then N steps, dumping the padded
FP64 state after the listed steps).  Both sides use the reference's padded
layout (NZ, NY, NX) = (nz + 7, ny + 6, nx + 6).
"""

from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / "oracle" / "_ref"
CFG = ROOT / "cases"
FIELDS = ["u", "v", "w", "thp", "pip", "qv", "qc", "qr"]


def have_reference(prec: str = "f64") -> bool:
    return (REF / f"refdump_{prec}").exists()


def read_ini(path) -> dict:
    kv = {}
    for line in Path(path).read_text().splitlines():
        for c in "#;":
            if c in line:
                line = line[: line.index(c)]
        if "=" in line:
            k, v = line.split("=", 1)
            if k.strip():
                kv[k.strip()] = v.strip()
    return kv


def reference_run(ini, prec: str, nsteps: int, dumps, outdir, overrides=None) -> dict:
    """{step: {field: padded float64 array (+ "rain" for moist cases)}} of the
    reference build after each step in `dumps`."""
    outdir = Path(outdir)
    cmd = [str(REF / f"refdump_{prec}"), str(ini), str(outdir), "mode=run", f"nsteps={nsteps}",
           "dump=" + ",".join(str(d) for d in sorted(dumps))]
    cmd += [f"{k}={v}" for k, v in (overrides or {}).items()]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed ({r.returncode}): {r.stderr[-2000:]}")
    sizes = dict(ln.split() for ln in (outdir / "manifest.txt").read_text().splitlines())
    out = {}
    for d in dumps:
        st = {}
        for k in FIELDS + ["rain"]:
            name = f"s{d}_{k}"
            if name in sizes:
                st[k] = np.fromfile(outdir / f"{name}.bin", dtype=np.float64)
                assert st[k].size == int(sizes[name]), name
        out[d] = st
    for f in outdir.glob("*.bin"):
        f.unlink()
    return out


def ours_run(ini, prec: str, nsteps: int, dumps, overrides=None, device: int = 0):
    """(case, {step: {field: padded float64 array, "rain": 2D padded}}) of
    wfe_b200 after each step in `dumps`; the case is closed."""
    import wfe_b200 as W

    c = W.Case(ini, overrides, precision=prec, device=device)
    out, s = {}, 0
    for d in sorted(dumps):
        c.run(d - s, c.dt, s * c.dt)
        s = d
        st = {k: c.field(k) for k in W.FIELDS}
        if c.moisture:
            st["rain"] = c.rain()
        out[d] = st
    if nsteps > s:
        c.run(nsteps - s, c.dt, s * c.dt)
    c.sync()
    c.close()
    return c, out


def interior(c, a, k):
    """interior points of a padded field: cells, w levels 0..nz"""
    a3 = np.asarray(a).reshape(c.shape)
    g = c.ng
    nzl = c.nz + 1 if k == "w" else c.nz
    return a3[g:g + nzl, g:g + c.ny, g:g + c.nx]


def rain_interior(c, a):
    a2 = np.asarray(a).reshape(c.NY, c.NX)
    g = c.ng
    return a2[g:g + c.ny, g:g + c.nx]


def measures(a, b, scale=None) -> tuple:
    """(relative L2, max-norm) of a against b; with `scale` both are taken
    against that magnitude instead of b's own (rms and max)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    d = a - b
    if scale is None:
        nb = float(np.sqrt((b * b).sum()))
        mb = float(np.abs(b).max())
        return (float(np.sqrt((d * d).sum())) / nb if nb > 0 else float(np.abs(d).max()),
                float(np.abs(d).max()) / mb if mb > 0 else float(np.abs(d).max()))
    return float(np.sqrt((d * d).mean())) / scale, float(np.abs(d).max()) / scale


def straka_front(thp_interior: np.ndarray, dx: float, xc: float = 25600.0) -> float:
    """Front position of the density current (tools/run_tests.py:45-51): the
    right edge of the surface cells colder than -1 K in the middle row,
    measured from the bubble centre."""
    ny = thp_interior.shape[1]
    sfc = thp_interior[0, ny // 2, :]
    cold = np.where(sfc < -1.0)[0]
    return (cold.max() + 0.5) * dx - xc if len(cold) else 0.0
