"""Shared comparison helpers for the parity tests."""

from __future__ import annotations

from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
CASES = GOLDEN / "cases"


FILE_SMALL = dict(nx=24, ny=20, nz=12, dx=12000.0, dy=12000.0, dz=20000.0 / 12)
FILE_SMALL_STEPS = 65  # crosses the first boundary-file switch at t = 3600 s


def make_file_small(root: Path) -> Path:
    """The small file-mode case of the goldens: 24 x 20 x 12, dx = 12 km, seeded
    synthetic prep inputs (wfe_b200.synth, seed 7, u0 = 12 m/s) with 2 h of
    hourly constant boundary files; returns the case .ini."""
    from wfe_b200 import synth
    root = Path(root)
    prep = root / "file_small_prep"
    synth.write_prep(prep, seed=7, u0=12.0, hours=2, bdy_interval=3600, **FILE_SMALL)
    return synth.write_case(root / "file_small.ini", prep, dt=60.0, bdy_width=3, **FILE_SMALL)


def golden(case: str):
    return np.load(GOLDEN / f"{case}.npz")


def scaled_err(a, b, floor: float = 0.0) -> float:
    """max |a - b| / max(|b|, floor) over the finite entries of b."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    fin = np.isfinite(b)
    if not fin.any():
        return 0.0
    assert np.array_equal(np.isfinite(a), fin), "non-finite pattern differs"
    sc = max(float(np.abs(b[fin]).max()), floor)
    if sc == 0.0:
        return float(np.abs(a[fin]).max())
    return float(np.abs(a[fin] - b[fin]).max() / sc)


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = float(np.sqrt((b * b).sum()))
    d = float(np.sqrt(((a - b) ** 2).sum()))
    return d / nb if nb > 0 else d


def view(case_or_shape, a):
    shape = case_or_shape.shape if hasattr(case_or_shape, "shape") else case_or_shape
    return np.asarray(a).reshape(shape)


def valid_region(case, field: str, open_x: bool, open_y: bool):
    """Boolean mask (NZ, NY, NX) of the points the reference defines after a
    step: interior cells, u faces 0..nx, v faces 0..ny, w levels 0..nz."""
    g = case.grid if hasattr(case, "grid") else case
    m = np.zeros(case.shape, dtype=bool)
    ng = g.ng
    ni = g.nx + (1 if field == "u" else 0)
    nj = g.ny + (1 if field == "v" else 0)
    nk = g.nz + (1 if field == "w" else 0)
    m[ng:ng + nk, ng:ng + nj, ng:ng + ni] = True
    return m


def ghost_ok_mask(case, field: str, open_x: bool, open_y: bool):
    """Every padded point except the ones the reference's open-boundary ghost
    fill writes racily (u at i = -3 for open x, v at j = -3 for open y, which
    receive a store from the neighbouring row's right/top ghost)."""
    m = np.ones(case.shape, dtype=bool)
    if field == "u" and open_x:
        m[:, :, 0] = False
    if field == "v" and open_y:
        m[:, 0, :] = False
    return m
