"""Variational analysis and analysis nudging on the device (GPU).

  * the 4D-Var gradient (background term + point observations of w and
    theta' at two times and u, theta' interpolated at positions over the
    terrain, chained adjoint runs) against central differences of the cost
    along seeded directions (FP64);
  * incremental 4D-Var recovers a warm bubble missing from the background
    from observations of its evolution: the cost falls by an order of
    magnitude and theta' moves toward the truth;
  * nudging toward an analysis (BdyManager targets lo = hi = xa, interior
    weight 1/tau: src/dynamics/boundary.cpp:24-39) pulls the forecast to the
    analysis; the tangent-linear run refuses the relaxing case, and after
    clear_boundary the steps are bit-identical to those before it relaxed.
"""

import numpy as np
import pytest

import wfe_b200 as W
from wfe_b200 import adjoint as A
from wfe_b200 import analysis as AN
from helpers import CASES

pytestmark = pytest.mark.gpu

SIGMA_B = {"u": 1.0, "v": 1.0, "w": 0.3, "thp": 0.5, "pip": 1e-4}


def _spinup(name, prec, n=4):
    c = W.Case(CASES / f"{name}.ini", precision=prec)
    c.run(n)
    c.sync()
    return c, A.get_fields(c)


def _bubble(c, amp, xc, zc, r):
    """theta' blob of amplitude amp on the cell centres (padded layout)"""
    g = c.ng
    x = (np.arange(c.nx) + 0.5) * c.dx
    z = c.metric("zeta_c")[g:g + c.nz]
    d2 = ((x[None, :] - xc) / r) ** 2 + ((z[:, None] - zc) / r) ** 2
    out = np.zeros(c.shape)
    out[g:g + c.nz, g:g + c.ny, g:g + c.nx] = (amp * np.exp(-d2))[:, None, :]
    return out


def _obs_from(c, model, xt, steps, fields, sigma, rng, every_k=1):
    """perfect observations of the truth run at every `every_k`-th interior
    point of the named fields"""
    times = sorted(set(steps))
    traj, x, t0 = {}, xt, 0
    for t in times:
        x = model.forecast(x, t - t0)
        traj[t], t0 = x, t
    obs = []
    for t in times:
        for f in fields:
            nzl = c.nz + 1 if f == "w" else c.nz
            k, j, i = np.meshgrid(np.arange(0, nzl, every_k), np.arange(c.ny),
                                  np.arange(0, c.nx, every_k), indexing="ij")
            o = AN.Obs.at(c, t, f, i.ravel(), j.ravel(), k.ravel(), np.zeros(i.size), sigma[f])
            o.value = o.sample(traj[t]).copy()
            obs.append(o)
    return obs


def test_4dvar_gradient_matches_central_differences():
    c, xb = _spinup("schaer_open", "f64", 6)
    m = AN.CaseModel(c, every=2)
    rng = np.random.default_rng(21)
    xt = {k: xb[k] + (_bubble(c, 0.5, 8000.0, 2000.0, 1500.0) if k == "thp" else 0.0)
          for k in m.names}
    obs = _obs_from(c, m, xt, [2, 5], ["w", "thp"], {"w": 0.05, "thp": 0.1}, rng, every_k=2)
    # and u, theta' interpolated at positions over the terrain
    xs = rng.uniform(2 * c.dx, (c.nx - 2) * c.dx, 20)
    ys = rng.uniform(1.0 * c.dy, (c.ny - 1) * c.dy, 20)
    zs = rng.uniform(1500.0, 4000.0, 20)
    traj5 = m.forecast(xt, 5)
    for f, sg in (("u", 0.2), ("thp", 0.1)):
        o = AN.Obs.interp(c, 5, f, xs, ys, zs, np.zeros(20), sg)
        o.value = o.sample(traj5) + 0.05 * rng.standard_normal(20)
        obs.append(o)
    v = AN.FourDVar(m, xb, SIGMA_B, obs)
    x0 = {k: xb[k] + 0.1 * SIGMA_B[k] * rng.standard_normal(c.shape) * m.mask(k)
          for k in m.names}
    j, g = v.gradient(x0)
    assert j == pytest.approx(v.cost(x0), rel=1e-12)
    for k in m.names:
        assert np.all(g[k][~m.mask(k)] == 0)
    for r in range(6):
        d = {k: SIGMA_B[k] * rng.standard_normal(c.shape) * m.mask(k) for k in m.names}
        ad = sum(float(np.sum(g[k] * d[k])) for k in m.names)
        gap = {}
        for eps in (1e-4, 1e-5):
            fd = (v.cost({k: x0[k] + eps * d[k] for k in m.names}) -
                  v.cost({k: x0[k] - eps * d[k] for k in m.names})) / (2 * eps)
            gap[eps] = abs(fd - ad) / abs(fd)
        # the O(eps^2) term of the central difference, over a floor of
        # 1e-7 - 2e-5: upwind switches of the advection where the bubble's and
        # the mountain wave's vertical velocities cross 0 make J piecewise
        # smooth, kinks the gradient (the derivative of the branches taken)
        # does not see; the u observations make J the more sensitive to them
        assert gap[1e-4] <= 5e-5 and gap[1e-5] <= 5e-5, (r, gap)
    c.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_4dvar_recovers_a_missing_bubble(prec):
    c, xb = _spinup("schaer_open", prec, 6)
    m = AN.CaseModel(c)
    rng = np.random.default_rng(5)
    blob = _bubble(c, 0.8, 8000.0, 2200.0, 1500.0)
    xt = {k: xb[k] + (blob if k == "thp" else 0.0) for k in m.names}
    obs = _obs_from(c, m, xt, [3, 6], ["w", "thp"], {"w": 0.02, "thp": 0.05}, rng)
    v = AN.FourDVar(m, xb, SIGMA_B, obs)
    r = v.minimise(outer=1, inner=12)
    assert r.cost[-1] < 0.1 * r.cost[0], r.cost
    mk = m.mask("thp")
    eb = np.linalg.norm((xb["thp"] - xt["thp"])[mk])
    ea = np.linalg.norm((r.x["thp"] - xt["thp"])[mk])
    assert ea < 0.5 * eb, (ea, eb)
    c.close()


def test_nudging_toward_an_analysis_and_clearing_it():
    c, xb = _spinup("schaer_open", "f32", 6)
    c.lin_enable()
    blob = _bubble(c, 1.0, 8000.0, 2000.0, 1500.0)
    xa = dict(xb)
    xa["thp"] = xb["thp"] + blob
    mk = AN.control_mask(c, "thp")
    n = 20

    def dist():
        return float(np.linalg.norm((c.field("thp") - xa["thp"])[mk]))

    A.set_fields(c, xb)
    c.run(3)
    ref = {k: c.field(k) for k in A.FIELDS5}
    A.set_fields(c, xb)
    c.run(n)
    free = dist()
    w = AN.nudge(c, xa, tau=5 * c.dt)
    g = c.ng
    assert np.allclose(w[g:g + c.ny, g:g + c.nx], 1.0 / (5 * c.dt))
    A.set_fields(c, xb)
    c.run(n)
    nudged = dist()
    assert nudged < 0.5 * free, (nudged, free)
    # the relaxing case is not linearised; after clear_boundary it is again
    with pytest.raises(W.WfeError):
        c.tl_run(1)
    c.clear_boundary()
    c.lin_zero()
    A.set_fields(c, xb)
    c.tl_run(1)
    # and its steps are the ones it took before it relaxed
    A.set_fields(c, xb)
    c.run(3)
    for k in A.FIELDS5:
        assert np.array_equal(c.field(k), ref[k]), k
    c.close()


def test_correlated_background_on_the_device_model():
    """With Gaussian-correlated background errors (horizontal length 1.5 km,
    and 1.5 levels along the column) the control variable is chi, x = xb +
    B^1/2 chi: on the device model (padded layout with ghost points, the
    staggered u, w masks, GPU tangent-linear and adjoint runs) dJ/dchi agrees
    with central differences of J(chi) along seeded directions, and the
    incremental minimisation lowers J."""
    c, xb = _spinup("schaer_open", "f64", 6)
    m = AN.CaseModel(c, every=2)
    rng = np.random.default_rng(31)
    xt = {k: xb[k] + (_bubble(c, 0.5, 8000.0, 2000.0, 1500.0) if k == "thp" else 0.0)
          for k in m.names}
    obs = _obs_from(c, m, xt, [2, 4], ["w", "thp"], {"w": 0.05, "thp": 0.1}, rng, every_k=2)
    corr = AN.GaussianCorrelation(1500.0, c.dx, c.dy, levels=1.5)
    v = AN.FourDVar(m, xb, SIGMA_B, obs, corr=corr)
    chi = 0.3 * rng.standard_normal(v.pack(xb).size)
    j, g = v.gradient_chi(chi)
    assert j == pytest.approx(v.cost_chi(chi), rel=1e-12)
    for r in range(4):
        d = rng.standard_normal(chi.size)
        ad = float(g @ d)
        eps = 1e-4
        fd = (v.cost_chi(chi + eps * d) - v.cost_chi(chi - eps * d)) / (2 * eps)
        assert abs(fd - ad) <= 5e-5 * abs(fd), (r, fd, ad)
    res = v.minimise(outer=1, inner=8)
    assert res.cost[-1] < 0.5 * res.cost[0], res.cost
    c.close()
