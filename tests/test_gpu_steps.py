"""Full RK3 steps of the CUDA path against the oracle, and the reference's
guarantees (GPU).

Tolerances (scaled error = max |diff| / max |oracle| per field):
  FP64 build vs FP64 oracle after 8 steps: <= 1e-10 (rounding only).
  FP32 build vs FP64 oracle after 8 steps: relative L2 <= 1e-4 for u, v, w,
  theta' (<= 1e-3 for pi') and max-norm <= 1e-3 of the field magnitude.
"""

import numpy as np
import pytest

import oracle as O
import wfe_b200 as W
from helpers import CASES, make_file_small, rel_l2, scaled_err

pytestmark = pytest.mark.gpu

RUN_CASES = ["bubble_open", "straka_periodic", "schaer_open", "wk82_small", "moist_blob"]
NSTEPS = 8


def _oracle_run(name, nsteps, overrides=None):
    o = O.Case(CASES / f"{name}.ini", overrides)
    it = o.integrator()
    it.set_state(o.initial_state())
    for s in range(nsteps):
        it.step(o.dt, s * o.dt)
    return o, it


def _interior(c, a, k):
    return c.interior(a, "w" if k == "w" else "c")


@pytest.mark.parametrize("name", RUN_CASES)
def test_fp64_steps_match_oracle(name):
    o, it = _oracle_run(name, NSTEPS)
    c = W.Case(CASES / f"{name}.ini", precision="f64")
    for s in range(NSTEPS):
        c.step(c.dt, s * c.dt)
    for k in W.FIELDS:
        e = scaled_err(_interior(c, c.field(k), k), _interior(o, it.field(k), k))
        assert e <= 1e-10, (name, k, e)
    if c.moisture:
        assert scaled_err(c.rain(), it.rain().reshape(c.NY, c.NX)) <= 1e-10


@pytest.mark.parametrize("name", RUN_CASES)
def test_fp32_steps_within_tolerance(name):
    o, it = _oracle_run(name, NSTEPS)
    c = W.Case(CASES / f"{name}.ini", precision="f32")
    c.run(NSTEPS, c.dt, 0.0)
    c.sync()
    # horizontal winds are judged against the wind-speed scale (in the 2D
    # slabs v is a rounding-level field)
    speed = max(np.abs(_interior(o, it.field(k), k)).max() for k in ("u", "v"))
    for k in ["u", "v", "w", "thp", "pip"]:
        a, b = _interior(c, c.field(k), k), _interior(o, it.field(k), k)
        if np.abs(b).max() == 0:
            assert np.abs(a).max() <= 1e-6, k
            continue
        if k in ("u", "v"):
            rl2 = np.sqrt(((a - b) ** 2).mean()) / speed
            smax = np.abs(a - b).max() / speed
        else:
            rl2, smax = rel_l2(a, b), scaled_err(a, b)
        assert rl2 <= (1e-3 if k == "pip" else 1e-4), (name, k, rl2)
        assert smax <= 1e-3, (name, k, smax)


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_graph_replay_equals_direct_steps(prec):
    a = W.Case(CASES / "wk82_small.ini", precision=prec)
    b = W.Case(CASES / "wk82_small.ini", precision=prec)
    for s in range(7):
        a.step(a.dt, s * a.dt)
    b.run(7, b.dt, 0.0)
    b.sync()
    for k in W.FIELDS:
        assert np.array_equal(a.field(k), b.field(k)), k
    assert np.array_equal(a.rain(), b.rain())
    assert b.launches_per_step() > 0


def test_uv_mirror_symmetry_fp32():
    """x <-> y symmetric set-up: u(k, j, i) == v(k, i, j) to <= 2e-6 relative RMS
    (the reference gates 1e-4, tools/run_tests.py:61-78, and claims 2e-6)."""
    c = W.Case(CASES / "bubble_open.ini", precision="f32")
    c.run(40, c.dt, 0.0)
    u = c.field("u", interior=True)
    v = c.field("v", interior=True)
    rms = np.sqrt((u ** 2).mean())
    assert rms > 1e-3
    asym = np.sqrt(((u - np.transpose(v, (0, 2, 1))) ** 2).mean()) / rms
    assert asym <= 2e-6, asym


@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 1e-6)])
def test_resting_atmosphere_over_terrain(prec, tol):
    """schaer_rest (tools/run_tests.py:83-85): no wind, terrain, stratified:
    |w| and |theta'| stay at rounding level."""
    c = W.Case(CASES / "schaer_open.ini", {"wind_u": 0, "coriolis_f": 0}, precision=prec)
    c.run(60, c.dt, 0.0)
    c.sync()
    assert c.field_absmax("w") <= tol
    assert c.field_absmax("thp") <= tol


def test_positive_definite_moisture_fp32():
    """moist_blob (tools/run_tests.py:97-98): PD transport keeps qv >= 0."""
    c = W.Case(CASES / "moist_blob.ini", precision="f32")
    c.run(200, c.dt, 0.0)
    qv = c.field("qv", interior=True)
    assert qv.min() >= -1e-9, qv.min()
    assert qv.max() > 4e-3


def test_no_spurious_precipitation():
    """Subsaturated moisture with microphysics on: no condensate, no rain."""
    c = W.Case(CASES / "moist_blob.ini", {"microphysics": "on", "qvbub_dq": 0.002},
               precision="f32")
    c.run(50, c.dt, 0.0)
    assert c.field_absmax("qc") == 0.0
    assert c.field_absmax("qr") == 0.0
    assert np.abs(c.rain()).max() == 0.0


def test_dry_mass_fp64_matches_oracle_and_is_reproducible():
    o, it = _oracle_run("straka_periodic", 4)
    c = W.Case(CASES / "straka_periodic.ini", precision="f64")
    for s in range(4):
        c.step(c.dt, s * c.dt)
    m1, m2 = c.dry_mass(), c.dry_mass()
    assert m1 == m2
    ref = o.dry_mass(it.state())
    assert abs(m1 - ref) <= 1e-12 * abs(ref)


def test_watchdog_absmax_reports_nan():
    c = W.Case(CASES / "bubble_open.ini", precision="f32")
    w = c.field("w")
    w[5, 5, 5] = np.nan
    c.set_field("w", w)
    assert c.field_absmax("w") > 1e30 or np.isnan(c.field_absmax("w"))


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_interior_transfers_roundtrip(prec):
    """Writer-layout uploads/downloads (src/io/writer.cpp:89-107) keep ghosts
    and agree with the padded transfers."""
    c = W.Case(CASES / "bubble_open.ini", precision=prec)
    rng = np.random.default_rng(3)
    for k in ("u", "w", "qv"):
        before = c.field(k)
        nzl = c.nz + 1 if k == "w" else c.nz
        a = rng.standard_normal((nzl, c.ny, c.nx)).astype(np.float32)
        c.set_field(k, a, interior=True)
        back = c.field(k, interior=True, dtype=np.float32)
        assert np.array_equal(back, a)
        pad = c.field(k)
        g = c.ng
        assert np.array_equal(pad[g:g + nzl, g:g + c.ny, g:g + c.nx].astype(np.float32), a)
        mask = np.ones(c.shape, bool)
        mask[g:g + nzl, g:g + c.ny, g:g + c.nx] = False
        assert np.array_equal(pad[mask], before[mask])


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_async_snapshot_equals_interior_download(prec):
    c = W.Case(CASES / "wk82_small.ini", precision=prec)
    c.run(3)
    names = list(W.FIELDS) + ["rain"]
    for dt in (np.float32, np.float64):
        bufs = c.snapshot_buffers(names, dtype=dt)
        c.snapshot_begin(bufs)
        c.run(2)  # steps issued after the snapshot do not change it
        c.snapshot_wait()
        c2 = None
        for k in names:
            assert bufs[k].dtype == dt
        # the state 2 steps ago: redo on a twin case for the reference values
        c2 = W.Case(CASES / "wk82_small.ini", precision=prec)
        c2.run(3 if dt is np.float32 else 5)
        for k in W.FIELDS:
            assert np.array_equal(bufs[k], c2.field(k, interior=True, dtype=dt)), k
        assert np.array_equal(bufs["rain"], c2.rain(interior=True).astype(dt))
        c2.close()
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wk82_small", "schaer_open", "bubble_open", "straka_periodic",
                                  "ops_periodic", "moist_blob"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_acoustic_variants_are_bit_identical(name, prec, monkeypatch):
    """The TMA-staged acoustic column kernel (variant 6) and the fused substep
    kernel that computes its tile's u, v faces itself (variants 7-9: three tile
    shapes, ragged tiles where nx is no multiple of the tile width) and the
    column kernel with contiguous level chunks per lane (variants 10-12) and
    the persistent column kernel fed by a pipeline of bulk tensor loads
    (variants 13-15: 32- and 16-column tiles, two and three stages; ragged
    tiles, FP64 tiles in shared memory) give the same values, bit for bit, as
    the u, v kernel + shared-memory column tile kernel (variant 0)."""
    out = {}
    for v in ("0", "6", "7", "8", "9", "10", "11", "12", "13", "14", "15"):
        monkeypatch.setenv("WFE_COLUMN_VARIANT", v)
        c = W.Case(CASES / f"{name}.ini", precision=prec)
        for s in range(4):
            c.step(c.dt, s * c.dt)
        c.run(3, t0=4 * c.dt)
        out[v] = {k: c.field(k) for k in W.FIELDS}
        kt = c.kernel_times()  # one more step, timed per kernel: which kernels ran
        assert ("acoustic_fused" in kt) == (v in ("7", "8", "9")), (v, sorted(kt))
        c.close()
    for v in ("6", "7", "8", "9", "10", "11", "12", "13", "14", "15"):
        for k in W.FIELDS:
            assert np.array_equal(out["0"][k], out[v][k]), (v, k)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wk82_small", "schaer_open", "bubble_open", "straka_periodic",
                                  "ops_periodic", "moist_blob"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_uv_variants_are_bit_identical(name, prec, monkeypatch):
    """The persistent forward u, v kernel fed by bulk tensor loads (variant 1:
    interior faces and the flat generic faces from shared memory, lateral
    edges -- radiation or periodic -- and sloped faces by the global-memory
    path; ragged tiles, terrain, moisture, open and periodic boundaries)
    gives the same values, bit for bit, as the thread-per-face kernel (0),
    and so does that kernel in slab-shaped blocks (2: 32 x 2 x 4)."""
    out = {}
    for v in ("0", "1", "2"):
        monkeypatch.setenv("WFE_UV_VARIANT", v)
        c = W.Case(CASES / f"{name}.ini", precision=prec)
        for s in range(3):
            c.step(c.dt, s * c.dt)
        c.run(3, t0=3 * c.dt)
        out[v] = {k: c.field(k) for k in W.FIELDS}
        c.close()
    for v in ("1", "2"):
        for k in W.FIELDS:
            assert np.array_equal(out["0"][k], out[v][k]), (v, k)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wk82_small", "schaer_open", "straka_periodic", "bubble_open"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_tendency_variants_are_bit_identical(name, prec, monkeypatch):
    """The fused (0) and split (1) tendency kernels, the variant with
    TMA-staged scalar tiles (2: each face flux computed once) and the fused
    kernel with two cells per thread (3) give the same values, bit for bit."""
    ov = {"pd_moist": "off"} if name == "wk82_small" else None
    out = {}
    for v in ("0", "1", "2", "3"):
        monkeypatch.setenv("WFE_TEND_VARIANT", v)
        c = W.Case(CASES / f"{name}.ini", overrides=ov, precision=prec)
        for s in range(4):
            c.step(c.dt, s * c.dt)
        out[v] = {k: c.field(k) for k in W.FIELDS}
        c.close()
    for v in ("1", "2", "3"):
        for k in W.FIELDS:
            assert np.array_equal(out["0"][k], out[v][k]), (v, k)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wk82_small", "moist_blob", "ops_open", "ops_periodic", "file_small"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_tendency_variants_bit_identical_with_limiter_and_relaxation(name, prec, monkeypatch, tmp_path):
    """The fused (0), split (1) and two-cells-per-thread (3) tendency kernels
    where the TMA variant does not run: positive-definite moisture (limited
    fluxes with the upwind cells' outflow ratios, at open and periodic edges),
    diffusion, Davies relaxation and surface physics (the file-mode case)."""
    ini = make_file_small(tmp_path) if name == "file_small" else CASES / f"{name}.ini"
    out = {}
    for v in ("0", "1", "3"):
        monkeypatch.setenv("WFE_TEND_VARIANT", v)
        c = W.Case(ini, precision=prec)
        for s in range(6):
            c.step(c.dt, s * c.dt)
        out[v] = {k: c.field(k) for k in W.FIELDS}
        c.close()
    for v in ("1", "3"):
        for k in W.FIELDS:
            assert np.array_equal(out["0"][k], out[v][k]), (v, k)


@pytest.mark.gpu
def test_watchdog_absmax_begin_end_matches_blocking_call():
    """The non-blocking watchdog (two page-locked slots, read one step behind)
    returns exactly what the blocking field_absmax returns for each step."""
    c = W.Case(CASES / "wk82_small.ini", precision="f32")
    seen = []
    for s in range(1, 5):
        c.run(1, c.dt, (s - 1) * c.dt)
        c.absmax_begin("w", s & 1)
        ref = c.field_absmax("w")
        seen.append((s, ref))
        if s > 1:
            assert c.absmax_end((s - 1) & 1) == seen[-2][1]
    assert c.absmax_end(4 & 1) == seen[-1][1]
    c.close()


@pytest.mark.gpu
def test_cases_of_different_depths_share_the_kernels(monkeypatch):
    """A shallower case set up after a deeper one must not lower the shared-
    memory limit of the kernels the deeper case launches (FP64 column tiles
    of 30 levels need more than the default 48 KB)."""
    monkeypatch.setenv("WFE_COLUMN_VARIANT", "0")
    deep = {"nz": "30"}
    a = W.Case(CASES / "bubble_open.ini", deep, precision="f64")
    ref = W.Case(CASES / "bubble_open.ini", deep, precision="f64")
    ref.run(2)
    ref.sync()
    shallow = W.Case(CASES / "bubble_open.ini", {"nz": "8"}, precision="f64")
    shallow.run(2)
    shallow.sync()
    for s in range(2):
        a.step(a.dt, s * a.dt)
    for k in W.FIELDS:
        assert np.array_equal(a.field(k), ref.field(k)), k
    for c in (a, ref, shallow):
        c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wk82_small", "schaer_open", "moist_blob"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_pipelined_parallel_solve_equals_parallel_solve(name, prec, monkeypatch):
    """The pipelined parallel-solve column kernels with 16 level lanes
    (variants 19-21: tiles streamed into shared memory by a producer warp)
    evaluate the parallel-solve kernel's expressions (variant 16) on the same
    values: the same fields, bit for bit, after five steps."""
    out = {}
    for v in ("16", "19", "20", "21"):
        monkeypatch.setenv("WFE_COLUMN_VARIANT", v)
        c = W.Case(CASES / f"{name}.ini", precision=prec)
        c.run(5, c.dt, 0.0)
        c.sync()
        out[v] = {k: c.field(k) for k in W.FIELDS}
        c.close()
    for v in ("19", "20", "21"):
        for k in W.FIELDS:
            assert np.array_equal(out["16"][k], out[v][k]), (v, k)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wk82_small", "moist_blob", "bubble_open", "schaer_open"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_level_tables_equal_fields(name, prec, monkeypatch):
    """On flat ground the column coefficients (rtjx, rtjy, aw, kt3, theta_b^w,
    dtheta_b/dz, qv_b) and the base state hold one value per level: the
    pipelined column kernels (Thomas 13-15, parallel solve 19-22) read the
    coefficients from per-level tables instead of streaming a box of each per
    tile, and the mass-flux, Kessler and u, v kernels the base state
    (thb, pib, rhob, rhobw).  The same fields, bit for bit, as from the 3D
    fields (WFE_LEVEL_TABLES=0) after five steps, for those variants and the
    plain column tile (0).  With terrain (schaer_open) no table is built."""
    for v in ("0", "13", "14", "15", "19", "20", "21", "22"):
        monkeypatch.setenv("WFE_COLUMN_VARIANT", v)
        out = {}
        for prof in ("1", "0"):
            monkeypatch.setenv("WFE_LEVEL_TABLES", prof)
            c = W.Case(CASES / f"{name}.ini", precision=prec)
            c.run(5, c.dt, 0.0)
            c.sync()
            out[prof] = {k: c.field(k) for k in W.FIELDS}
            var = c.variants()
            assert var["column"] == int(v)
            assert var["level_tables"] == (prof == "1" and name != "schaer_open"), (v, var)
            assert var["base_tables"] == (prof == "1" and name != "schaer_open"), (v, var)
            c.close()
        for k in W.FIELDS:
            assert np.array_equal(out["1"][k], out["0"][k]), (v, k)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("f64", 1e-11), ("f32", 1e-4)])
def test_parallel_solve_columns_with_relaxation_and_surface_physics(prec, tol, monkeypatch, tmp_path):
    """The file-mode case (Davies relaxation, whose slow pi' tendency is one
    more box in the pipelined kernels' stages, surface physics, terrain,
    a Lambert map): the pipelined parallel-solve kernels with 16 level lanes
    (19-21) equal the parallel-solve kernel (16) bit for bit, and every
    parallel-solve variant (16-22) agrees with the Thomas kernel (0) to
    rounding after six steps (relative L2 <= 1e-11 FP64 / 1e-4 FP32)."""
    ini = make_file_small(tmp_path)
    out = {}
    for v in ("0", "16", "17", "18", "19", "20", "21", "22"):
        monkeypatch.setenv("WFE_COLUMN_VARIANT", v)
        c = W.Case(ini, precision=prec)
        c.run(6, c.dt, 0.0)
        c.sync()
        out[v] = {k: c.field(k) for k in W.FIELDS}
        c.close()
    for v in ("19", "20", "21"):
        for k in W.FIELDS:
            assert np.array_equal(out["16"][k], out[v][k]), (v, k)
    ref = out["0"]
    speed = max(np.abs(ref["u"]).max(), np.abs(ref["v"]).max(), 1e-30)
    for v in ("16", "17", "18", "22"):
        for k in W.FIELDS:
            a, b = out[v][k], ref[k]
            if k in ("u", "v"):
                err = np.sqrt(((a - b) ** 2).mean()) / speed
            else:
                err = rel_l2(a, b) if np.abs(b).max() > 0 else np.abs(a).max()
            assert err <= tol, (v, k, err)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wk82_small", "schaer_open", "bubble_open", "straka_periodic",
                                  "ops_periodic", "moist_blob"])
@pytest.mark.parametrize("prec,tol", [("f64", 1e-11), ("f32", 1e-4)])
def test_parallel_solve_column_agrees_to_rounding(name, prec, tol, monkeypatch):
    """The column kernels with the parallel tridiagonal solve (variants 16-18:
    each level lane eliminates its own rows, cyclic reduction over the lanes;
    19-22: the same fed by the pipelined bulk-tensor-load ring) solve the
    same rows as the Thomas-sweep kernels: after seven steps the
    fields agree to rounding -- relative L2 <= 1e-11 (FP64) / 1e-4 (FP32, the
    FP32 step-parity bound against the oracle; measured up to 1.2e-5 on the
    moist convective case) of the field (u, v against the wind-speed
    scale) -- and the FP64 steps stay within 1e-10 of the FP64 oracle."""
    out = {}
    variants = ["0"] + [v for v in ("16", "17", "18", "19", "20", "21", "22")]
    for v in variants:
        monkeypatch.setenv("WFE_COLUMN_VARIANT", v)
        c = W.Case(CASES / f"{name}.ini", precision=prec)
        c.run(7, c.dt, 0.0)
        c.sync()
        out[v] = {k: c.field(k) for k in W.FIELDS}
        kt = c.kernel_times()
        assert "acoustic_column" in kt
        c.close()
    ref = out["0"]
    speed = max(np.abs(ref["u"]).max(), np.abs(ref["v"]).max(), 1e-30)
    for v in variants[1:]:
        for k in W.FIELDS:
            a, b = out[v][k], ref[k]
            if k in ("u", "v"):
                err = np.sqrt(((a - b) ** 2).mean()) / speed
            else:
                err = rel_l2(a, b) if np.abs(b).max() > 0 else np.abs(a).max()
            assert err <= tol, (v, k, err)
    if prec == "f64":
        o, it = _oracle_run(name, 7)
        for k in W.FIELDS:
            c = W.Case(CASES / f"{name}.ini", precision="f64", device=-1)
            e = scaled_err(_interior(c, out["16"][k], k), _interior(o, it.field(k), k))
            c.close()
            assert e <= 1e-10, (k, e)
