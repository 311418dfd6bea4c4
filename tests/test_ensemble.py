"""Batched ensembles of uneven members (one launch per kernel over a member x
tile work list, one CUDA graph per rotation phase).

Members are file-mode cases from the seeded prep generator (full physics,
Davies boundaries, Kessler, positive-definite moisture) with different grid
sizes, terrain, winds and noise.  A member advanced inside an ensemble runs
the same kernel bodies on the same arguments as when it is stepped alone, so
the results must agree bit for bit; the members stepped alone are themselves
checked against the oracle in test_file_mode.py.
"""

import numpy as np
import pytest

import oracle as O
import wfe_b200 as W
from wfe_b200 import synth
from helpers import scaled_err

# (nx, ny, nz, seed, u0): uneven sizes, one shallower member
MEMBERS = [(24, 20, 12, 11, 8.0), (36, 18, 12, 12, 15.0), (20, 30, 10, 13, 19.0)]


def make_members(root, members=MEMBERS, hours=2, bdy_interval=3600):
    cases = []
    for q, (nx, ny, nz, seed, u0) in enumerate(members):
        dims = dict(nx=nx, ny=ny, nz=nz, dx=12000.0, dy=12000.0, dz=20000.0 / nz)
        prep = root / f"m{q}_prep"
        synth.write_prep(prep, seed=seed, u0=u0, hours=hours, bdy_interval=bdy_interval, **dims)
        cases.append(synth.write_case(root / f"m{q}.ini", prep, dt=60.0, bdy_width=3, **dims))
    return cases


@pytest.fixture(scope="module")
def member_cases(tmp_path_factory):
    return make_members(tmp_path_factory.mktemp("ens"))


def test_ensemble_rejects_host_only_members(member_cases):
    cs = [W.Case(p, device=-1) for p in member_cases]
    with pytest.raises(W.WfeError, match="without a device model"):
        W.Ensemble(cs)
    for c in cs:
        c.close()


def test_ensemble_generator_members(tmp_path):
    paths = synth.write_ensemble(tmp_path, groups=((12, 10), (16, 8)), per_group=2, nz=8,
                                 hours=1)
    assert len(paths) == 4
    u0 = []
    for p in paths:
        kv = O.read_ini(p)
        inp = O.load_prep(kv["input_dir"], int(kv["nx"]), int(kv["ny"]), int(kv["nz"]))
        u0.append(inp["prof_u"][0])
        assert kv["physics"] == "simple" and kv["pd_moist"] == "on" and kv["bdy_width"] == "5"
    assert len(set(np.round(u0, 6))) == 4 and all(5.0 <= u <= 20.0 for u in u0)


def _alone(path, prec, n):
    c = W.Case(path, precision=prec)
    c.run(n)
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("mode", ["batched", "members", "sequential", ""])
def test_ensemble_equals_members_alone(member_cases, prec, mode, monkeypatch):
    """batched launches, the members' own graphs on concurrent streams, the
    members' own graphs one after another, and the mode the first run picks
    by timing two steps of each ("")"""
    monkeypatch.setenv("WFE_ENSEMBLE_MODE", mode)
    n = 65  # crosses the boundary-file switch at 3600 s
    mem = [W.Case(p, precision=prec) for p in member_cases]
    ens = W.Ensemble(mem)
    ens.run(n, mem[0].dt)
    ens.sync()
    assert ens.launches_per_step() > 0
    if mode:
        assert ens.variants()["mode"] == mode
    for p, m in zip(member_cases, mem):
        alone = _alone(p, prec, n)
        for k in W.FIELDS:
            a, b = m.field(k), alone.field(k)
            assert np.array_equal(a, b), (p.name, k, scaled_err(a, b))
        assert np.array_equal(m.rain(), alone.rain())
        for name in ("tsk", "pblh", "t2m", "u10"):
            assert np.array_equal(m.field2d(name), alone.field2d(name)), name
        alone.close()
    ens.close()
    for m in mem:
        m.close()


@pytest.mark.gpu
def test_ensemble_direct_steps_equal_graph_run(member_cases):
    n = 6
    a = [W.Case(p, precision="f64") for p in member_cases]
    b = [W.Case(p, precision="f64") for p in member_cases]
    ea, eb = W.Ensemble(a), W.Ensemble(b)
    for s in range(n):
        ea.step(a[0].dt, s * a[0].dt)
    eb.run(n, b[0].dt)
    eb.sync()
    for x, y in zip(a, b):
        for k in W.FIELDS:
            assert np.array_equal(x.field(k), y.field(k)), k
    for e in (ea, eb):
        e.close()
    for m in a + b:
        m.close()


@pytest.mark.gpu
def test_ensemble_member_matches_oracle_fp64(member_cases):
    n = 8
    mem = [W.Case(p, precision="f64") for p in member_cases]
    ens = W.Ensemble(mem)
    ens.run(n, mem[0].dt)
    ens.sync()
    q = 2  # the shallow member
    r = O.FileRun(member_cases[q])
    for s in range(n):
        r.step(r.case.dt, s * r.case.dt)
    st = r.it.state()
    for k in W.FIELDS:
        kind = "w" if k == "w" else "c"
        e = scaled_err(mem[q].interior(mem[q].field(k), kind), r.case.interior(st[k], kind))
        assert e <= 1e-10, (k, e)
    ens.close()
    for m in mem:
        m.close()


@pytest.mark.gpu
def test_ensemble_rejects_mismatched_members(member_cases, tmp_path):
    a = W.Case(member_cases[0], precision="f64")
    b = W.Case(member_cases[1], precision="f32")
    with pytest.raises(W.WfeError, match="precision"):
        W.Ensemble([a, b])
    c = W.Case(member_cases[1], {"acoustic_ns": 4}, precision="f64")
    with pytest.raises(W.WfeError, match="settings"):
        W.Ensemble([a, c])
    for m in (a, b, c):
        m.close()
