"""The CPU oracle against golden vectors from the reference's own FP64 build.

The goldens were produced on a B200 by tests/golden/make_golden.py from the
reference compiled from its sources (oracle/Makefile): refdump_f64 drives the
reference's kernels and Integrator through its C++ API; wfe_f64 is the
unmodified reference executable.  Set-up (metric, base state, initial
conditions) must be bit-identical (same host FP64 arithmetic); dynamics may
differ only by the GPU build's fused multiply-adds and device libm, so after
8 RK3 steps the tolerance is 1e-11 of each field's magnitude.
"""

import numpy as np
import pytest

import oracle as O
from helpers import (CASES, FILE_SMALL_STEPS, GOLDEN, ghost_ok_mask, golden, make_file_small,
                     scaled_err)

RUN_CASES = ["bubble_open", "straka_periodic", "schaer_open", "wk82_small", "moist_blob"]
OPS_CASES = ["ops_open", "ops_periodic"]
STEP_TOL = 1e-11
OP_TOL = 1e-12


@pytest.fixture(scope="module", params=RUN_CASES)
def run_case(request):
    name = request.param
    return name, O.Case(CASES / f"{name}.ini"), golden(name)


def test_setup_bit_identical(run_case):
    name, c, G = run_case
    for k in O.METRIC_1D + O.METRIC_2D:
        assert np.array_equal(c.metric[k], G["m_" + k]), k
    assert c.zt == G["m_zt"][0]
    for k in O.BASE_3D + ["ub"]:
        assert np.array_equal(c.base[k], G["b_" + k], equal_nan=True), k
    s0 = c.initial_state()
    for k in O.FIELDS:
        assert np.array_equal(s0[k], G["s0_" + k]), k


def test_steps_match_reference_fp64(run_case):
    name, c, G = run_case
    it = c.integrator()
    it.set_state(c.initial_state())
    for step in range(1, 9):
        it.step(c.dt, (step - 1) * c.dt)
        if step in (1, 8):
            st = it.state()
            for k in O.FIELDS:
                kind = "w" if k == "w" else "c"
                e = scaled_err(c.interior(st[k], kind), c.interior(G[f"s{step}_{k}"], kind))
                assert e <= STEP_TOL, (name, step, k, e)
            if c.params.moisture:
                gr = G[f"s{step}_rain"].reshape(c.grid.NY, c.grid.NX)
                assert np.allclose(it.rain().reshape(c.grid.NY, c.grid.NX), gr, rtol=1e-11,
                                   atol=1e-18)


def test_matches_unmodified_reference_executable(run_case):
    """The unmodified wfe_f64 writes float32 interior snapshots (src/io/writer.cpp);
    the oracle rounded to float32 must agree to a couple of float32 ulps."""
    name, c, G = run_case
    W = np.load(GOLDEN / f"{name}_wfe.npz")
    it = c.integrator()
    s0 = c.initial_state()
    it.set_state(s0)
    for k in ("u", "v", "w", "thp", "pip"):
        kind = "w" if k == "w" else "c"
        ref = W[f"wfe64_{k}_000000"]
        got = c.interior(s0[k], kind).astype(np.float32).ravel()
        assert np.array_equal(got, ref), k
    for step in range(1, 9):
        it.step(c.dt, (step - 1) * c.dt)
    st = it.state()
    for k in ("u", "v", "w", "thp", "pip"):
        kind = "w" if k == "w" else "c"
        ref = W[f"wfe64_{k}_000008"].astype(np.float64)
        got = c.interior(st[k], kind).ravel()
        assert scaled_err(got, ref) <= 2.5e-7, k
    log = bytes(W["wfe64_log"]).decode()
    assert "bitti: 8 adim" in log


@pytest.fixture(scope="module", params=OPS_CASES)
def ops_case(request):
    name = request.param
    return name, O.Case(CASES / f"{name}.ini"), golden(name)


def _state(G, pre):
    return {k: G[f"{pre}_{k}"].copy() for k in O.FIELDS}


def _check_state(c, got, G, pre, fields=O.FIELDS, mask_fn=None, tol=OP_TOL):
    p = c.params
    for k in fields:
        m = ghost_ok_mask(c, k, p.bc_x_open, p.bc_y_open)
        if mask_fn is not None:
            m &= mask_fn(k)
        a = got[k].reshape(c.shape)[m]
        b = G[f"{pre}_{k}"].reshape(c.shape)[m]
        e = scaled_err(a, b)
        assert e <= tol, (pre, k, e)


def test_ops_bcs_fluxes_tendencies(ops_case):
    name, c, G = ops_case
    dt = G["params"][-1]
    s = _state(G, "in")
    c.apply_bcs(s)
    _check_state(c, s, G, "bc", tol=0.0)
    s = _state(G, "bc")
    tend, (mfx, mfy, mfz, div) = c.tendencies(s, dt)
    for nm, a in (("mfx", mfx), ("mfy", mfy), ("mfz", mfz), ("div", div)):
        assert scaled_err(a, G[nm]) <= OP_TOL, nm
    g = c.grid

    def unused(k):  # tendencies at open-boundary faces the acoustic step never reads
        m = np.ones(c.shape, dtype=bool)
        if k == "u" and c.params.bc_x_open:
            m[:, :, g.ng] = False
        if k == "v" and c.params.bc_y_open:
            m[:, g.ng, :] = False
        return m

    _check_state(c, tend, G, "tend", mask_fn=unused)
    if "bdy_wgt" in G.files:
        lo = [G[f"bdy_lo{v}"] for v in range(5)]
        hi = [G[f"bdy_hi{v}"] for v in range(5)]
        c.bdy_relax(s, lo, hi, 0.3, G["bdy_wgt"], tend)
        _check_state(c, tend, G, "tendb", mask_fn=unused)


def test_ops_acoustic(ops_case):
    name, c, G = ops_case
    dt = G["params"][-1]
    coef = c.acoustic_coef()
    for a, nm in zip(coef, ("rtjx", "rtjy", "kt3", "aw")):
        assert np.allclose(a, G["ac_" + nm], rtol=1e-14, atol=0, equal_nan=True), nm
    s = _state(G, "bc")
    tend = _state(G, "tendb" if "bdy_wgt" in G.files else "tend")
    work = {k: v.copy() for k, v in s.items()}
    piprev = s["pip"].copy()
    nsub = int(c.cfg.int("nsub", 3))
    dtau = c.cfg.real("dtau", dt / 6)
    for t in range(nsub):
        c.acoustic_substep(work, tend, piprev, dtau, coef)
        if t == 0:
            _check_state(c, work, G, "ac1")
            assert scaled_err(piprev, G["ac1_piprev"]) <= OP_TOL
    _check_state(c, work, G, "acn")
    assert scaled_err(piprev, G["acn_piprev"]) <= OP_TOL
    if c.params.moisture:
        c.moisture_stage(s, tend, dt, work)
        _check_state(c, work, G, "mst", fields=["qv", "qc", "qr"])


def test_ops_kessler(ops_case):
    name, c, G = ops_case
    dt = G["params"][-1]
    s = _state(G, "bc")
    rain = np.zeros(c.grid.NX * c.grid.NY)
    c.kessler(s, dt, rain)
    _check_state(c, s, G, "kes", tol=1e-11)
    assert scaled_err(rain, G["kes_rain"]) <= 1e-11
    # the synthetic state is supersaturated in places: the column physics acted
    assert np.abs(s["qc"] - G["bc_qc"]).max() > 1e-6


def test_ops_surface_pbl(ops_case):
    name, c, G = ops_case
    dt = G["params"][-1]
    g = c.grid
    n2 = g.nx * g.ny
    sin = G["sfc_in"].reshape(5, n2)
    hour, t0 = 9.0, 1800.0
    for pre, nonlocal_pbl in (("sfc", True), ("sfc2", False)):
        s = _state(G, "bc")
        ph = c.sfc(*sin, hour, 172, nonlocal_pbl)
        ph.step(s, dt, t0)
        ph.step(s, dt, t0 + dt)
        _check_state(c, s, G, pre, fields=["u", "v", "thp", "qv"], tol=1e-11)
        for f in ("tsk", "pblh", "t2m", "u10"):
            assert scaled_err(ph.field(f), G[f"{pre}_{f}"]) <= 1e-11, (pre, f)


def test_file_mode_matches_unmodified_reference_executable(tmp_path):
    """file_small (seeded synthetic prep inputs; Davies boundaries with a
    boundary-file switch at 3600 s, surface layer + nonlocal PBL + soil +
    radiation, Kessler, positive-definite moisture, Lambert map factors) through
    the unmodified wfe_f64 against the oracle's file-mode run."""
    import hashlib
    W = np.load(GOLDEN / "file_small_wfe.npz")
    ini = make_file_small(tmp_path)
    sha = hashlib.sha256((tmp_path / "file_small_prep" / "wfe_init.bin").read_bytes()).digest()
    assert sha == bytes(W["prep_sha256"]), "the generator no longer writes the pinned inputs"
    r = O.FileRun(ini)
    c = r.case
    for k in ("u", "v", "w", "thp", "pip", "qv"):
        kind = "w" if k == "w" else "c"
        got = c.interior(r.s0[k], kind).astype(np.float32).ravel()
        assert np.array_equal(got, W[f"wfe64_{k}_000000"]), k
    for step in range(1, FILE_SMALL_STEPS + 1):
        r.step(c.dt, (step - 1) * c.dt)
        if step in (8, FILE_SMALL_STEPS):
            st = r.it.state()
            for k in O.FIELDS:
                kind = "w" if k == "w" else "c"
                ref = W[f"wfe64_{k}_{step:06d}"].astype(np.float64)
                got = c.interior(st[k], kind).ravel()
                assert scaled_err(got, ref) <= 2.5e-7, (step, k, scaled_err(got, ref))
            g2 = c.grid
            for name in ("tsk", "pblh", "t2m", "u10"):
                ref = W[f"wfe64_{name}_{step:06d}"].astype(np.float64)
                got = r.sfc.field(name).reshape(g2.NY, g2.NX)[3:-3, 3:-3].ravel()
                assert scaled_err(got, ref) <= 2.5e-7, (step, name)
            ref = W[f"wfe64_rain_{step:06d}"].astype(np.float64)
            got = r.it.rain().reshape(g2.NY, g2.NX)[3:-3, 3:-3].ravel()
            assert np.abs(got - ref).max() <= 2.5e-7 * max(np.abs(ref).max(), 1e-12), step
    log = bytes(W["wfe64_log"]).decode()
    assert f"bitti: {FILE_SMALL_STEPS} adim" in log
