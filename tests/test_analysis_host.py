"""Variational analysis and nudging: host logic (CPU).

The 4D-Var solver of wfe_b200.analysis only talks to a model object, so its
algebra is checked here on small numpy models with exact tangent and adjoint:
  * the chained adjoint gradient (observations at several times, uncontrolled
    points) against central differences of the cost;
  * one Gauss-Newton outer loop with CG run to convergence reproduces the
    closed-form minimiser of the linear problem;
  * outer loops on a nonlinear model lower the cost to a stationary point;
  * argument checks of the observations.
The BdyManager nudging weights of the C ABI (wfe_bdy_weights, host only) are
checked against the oracle's restatement of src/dynamics/boundary.cpp:24-39.
"""

import numpy as np
import pytest

import oracle as O
import wfe_b200 as W
from helpers import CASES
from wfe_b200 import analysis as AN


class QuadMap:
    """x_{n+1} = M x_n + c x_n * x_n on two fields; the last points of each
    field are no input (like ghost points): the step reads them as 0."""

    names = ("a", "b")

    def __init__(self, n=12, c=0.1, seed=3, free=2):
        rng = np.random.default_rng(seed)
        q, _ = np.linalg.qr(rng.standard_normal((2 * n, 2 * n)))
        self.M = 0.9 * q + 0.05 * rng.standard_normal((2 * n, 2 * n))
        self.c, self.n = c, n
        m = np.ones(n, dtype=bool)
        m[n - free:] = False
        self._mask = m

    def mask(self, name):
        return self._mask

    def _vec(self, x):
        return np.concatenate([np.where(self._mask, x[k], 0.0) for k in self.names])

    def _dict(self, v):
        return {"a": v[:self.n].copy(), "b": v[self.n:].copy()}

    def _traj(self, x0, n):
        xs = [self._vec(x0)]
        for _ in range(n):
            x = xs[-1]
            y = self.M @ x + self.c * x * x
            xs.append(np.concatenate([np.where(self._mask, y[:self.n], 0.0),
                                      np.where(self._mask, y[self.n:], 0.0)]))
        return xs

    def forecast(self, x0, n):
        return self._dict(self._traj(x0, n)[-1])

    def tangent(self, x0, dx, n):
        xs = self._traj(x0, n)
        d = self._vec(dx)
        mm = np.concatenate([self._mask, self._mask])
        for s in range(n):
            d = np.where(mm, self.M @ d + 2 * self.c * xs[s] * d, 0.0)
        return self._dict(d)

    def adjoint(self, x0, lam, n):
        xs = self._traj(x0, n)
        mm = np.concatenate([self._mask, self._mask])
        l = np.concatenate([lam[k] for k in self.names])
        for s in range(n - 1, -1, -1):
            l = np.where(mm, l, 0.0)
            l = self.M.T @ l + 2 * self.c * xs[s] * l
        # inputs of nothing receive no gradient
        return self._dict(np.where(mm, l, 0.0))


def _problem(c=0.1, seed=5, steps=(0, 2, 3, 5)):
    m = QuadMap(c=c)
    rng = np.random.default_rng(seed)
    xt = {k: 0.5 * rng.standard_normal(m.n) for k in m.names}
    xb = {k: xt[k] + 0.2 * rng.standard_normal(m.n) for k in m.names}
    obs = []
    for t in steps:
        x = m.forecast(xt, t)
        for f in m.names:
            idx = rng.choice(m.n - 2, size=4, replace=False)
            idx = np.concatenate([idx, idx[:1]])  # a repeated point accumulates
            obs.append(AN.Obs(t, f, idx, x[f][idx] + 0.01 * rng.standard_normal(idx.size),
                              sigma=0.05))
    return m, xt, xb, obs


def test_gradient_matches_finite_differences():
    m, xt, xb, obs = _problem(c=0.15)
    v = AN.FourDVar(m, xb, {"a": 0.3, "b": 0.2}, obs)
    rng = np.random.default_rng(9)
    x0 = {k: xb[k] + 0.1 * rng.standard_normal(m.n) for k in m.names}
    j, g = v.gradient(x0)
    assert j == pytest.approx(v.cost(x0), rel=1e-14)
    for k in m.names:
        assert np.all(g[k][~m.mask(k)] == 0)
    for _ in range(6):
        d = {k: np.where(m.mask(k), rng.standard_normal(m.n), 0.0) for k in m.names}
        eps = 1e-6
        jp = v.cost({k: x0[k] + eps * d[k] for k in m.names})
        jm = v.cost({k: x0[k] - eps * d[k] for k in m.names})
        fd = (jp - jm) / (2 * eps)
        an = sum(float(g[k] @ d[k]) for k in m.names)
        assert abs(fd - an) <= 1e-7 * max(1.0, abs(an)), (fd, an)


def test_linear_problem_minimiser_is_the_closed_form():
    m, xt, xb, obs = _problem(c=0.0)
    sb = {"a": 0.3, "b": 0.2}
    v = AN.FourDVar(m, xb, sb, obs)
    nctl = v.pack(xb).size
    # CG is exact after nctl iterations in exact arithmetic; a few more in FP64
    r = v.minimise(outer=1, inner=3 * nctl, rtol=1e-13)
    # closed form: (B^-1 + G^T R^-1 G) dx = G^T R^-1 (y - G xb)
    G, y, w = [], [], []
    for o in obs:
        rows = []
        for e in range(nctl):
            ev = np.zeros(nctl)
            ev[e] = 1.0
            rows.append(o.sample(m.forecast(v.unpack(ev), o.step)))
        G.append(np.array(rows).T)
        y.append(o.value - o.sample(m.forecast(xb, o.step)))
        w.append(1.0 / o.sigma ** 2)
    G, y, w = np.vstack(G), np.concatenate(y), np.concatenate(w)
    binv = 1.0 / v._sb_vec() ** 2
    dx = np.linalg.solve(np.diag(binv) + G.T @ (w[:, None] * G), G.T @ (w * y))
    xa = v.pack(r.x)
    assert np.allclose(xa, v.pack(xb) + dx, rtol=1e-9, atol=1e-11)
    assert r.cost[-1] < r.cost[0]
    for k in m.names:  # uncontrolled points stay at the background
        assert np.array_equal(r.x[k][~m.mask(k)], xb[k][~m.mask(k)])


def test_gauss_newton_outer_loops_reach_a_stationary_point():
    m, xt, xb, obs = _problem(c=0.2, seed=11)
    v = AN.FourDVar(m, xb, 0.3, obs)
    r = v.minimise(outer=4, inner=40, rtol=1e-10)
    assert all(b <= a * (1 + 1e-12) for a, b in zip(r.cost, r.cost[1:])), r.cost
    _, g0 = v.gradient(xb)
    _, g = v.gradient(r.x)
    n0 = np.sqrt(sum(float(g0[k] @ g0[k]) for k in m.names))
    n1 = np.sqrt(sum(float(g[k] @ g[k]) for k in m.names))
    assert n1 < 1e-6 * n0, (n0, n1)
    # the analysis is closer to the truth than the background
    err = lambda x: np.sqrt(sum(float(np.sum((x[k] - xt[k])[m.mask(k)] ** 2)) for k in m.names))
    assert err(r.x) < 0.5 * err(xb)


def test_observation_checks():
    m = QuadMap()
    xb = {k: np.zeros(m.n) for k in m.names}
    with pytest.raises(ValueError):
        AN.Obs(1, "a", [0, 1], [1.0])
    with pytest.raises(ValueError):
        AN.Obs(1, "a", [0], [1.0], sigma=0.0)
    with pytest.raises(ValueError):
        AN.FourDVar(m, xb, 1.0, [AN.Obs(1, "c", [0], [1.0])])
    with pytest.raises(ValueError):
        AN.FourDVar(m, xb, 1.0, [AN.Obs(1, "a", [m.n], [1.0])])
    with pytest.raises(ValueError):
        AN.FourDVar(m, xb, 1.0, [AN.Obs(-1, "a", [0], [1.0])])
    with pytest.raises(ValueError):
        AN.FourDVar(m, xb, {"a": 1.0, "b": 0.0}, [])


@pytest.mark.parametrize("case,width,tau,nudge_tau", [
    ("bubble_open", 5, 300.0, 0.0), ("bubble_open", 4, 120.0, 3600.0),
    ("schaer_open", 3, 60.0, 900.0), ("straka_periodic", 5, 60.0, 600.0)])
def test_bdy_weights_match_oracle(case, width, tau, nudge_tau):
    c = W.Case(CASES / f"{case}.ini", precision="f64", device=-1)
    o = O.Case(CASES / f"{case}.ini")
    w = c.bdy_weights(width, tau, nudge_tau)
    assert np.array_equal(w.ravel(), o.bdy_weights(width, tau, nudge_tau))
    assert w.shape == (c.NY, c.NX)
    with pytest.raises(W.WfeError):
        c.bdy_weights(width, 0.0, nudge_tau)
    c.close()


def test_control_mask_and_obs_indexing_on_host_case():
    c = W.Case(CASES / "schaer_open.ini", precision="f64", device=-1)
    g = c.ng
    assert AN.control_mask(c, "thp").sum() == c.nx * c.ny * c.nz
    assert AN.control_mask(c, "u").sum() == (c.nx + 1) * c.ny * c.nz
    assert AN.control_mask(c, "v").sum() == c.nx * (c.ny + 1) * c.nz
    assert AN.control_mask(c, "w").sum() == c.nx * c.ny * (c.nz + 1)
    o = AN.Obs.at(c, 2, "thp", [0, c.nx - 1], [1, 2], [3, 0], [1.0, 2.0], 0.5)
    a = np.zeros(c.shape)
    a[3 + g, 1 + g, g] = 1.0
    a[g, 2 + g, c.nx - 1 + g] = 2.0
    assert np.array_equal(o.sample({"thp": a}), [1.0, 2.0])
    assert np.array_equal(o.sigma, [0.5, 0.5])
    with pytest.raises(W.WfeError):  # the relaxation needs the device model
        c.clear_boundary()
    c.close()


def _linear_field(c, field, a, b, cy, d):
    """a + b x + cy y + d zeta at the field's own points, padded layout"""
    g = c.ng
    ex = 0.0 if field == "u" else 0.5
    ey = 0.0 if field == "v" else 0.5
    zeta = c.metric("zeta_w" if field == "w" else "zeta_c")
    x = (np.arange(c.NX) - g + ex) * c.dx
    y = (np.arange(c.NY) - g + ey) * c.dy
    return a + b * x[None, None, :] + cy * y[None, :, None] + d * zeta[:, None, None]


@pytest.mark.parametrize("field", ["thp", "u", "v", "w"])
def test_interp_obs_reproduce_trilinear_fields(field):
    """Trilinear interpolation is exact for a field linear in (x, y, zeta);
    over flat terrain zeta is the height z."""
    c = W.Case(CASES / "bubble_open.ini", precision="f64", device=-1)
    assert np.all(c.metric("h") == 0)
    f = _linear_field(c, field, 1.5, 2e-4, -3e-4, 1e-3)
    rng = np.random.default_rng(4)
    ex = 0.0 if field == "u" else 0.5
    ey = 0.0 if field == "v" else 0.5
    nxp = c.nx + (field == "u")
    nyp = c.ny + (field == "v")
    zl = c.metric("zeta_w" if field == "w" else "zeta_c")[c.ng:c.ng + c.nz + (field == "w")]
    x = (ex + rng.uniform(0, nxp - 1, 50)) * c.dx
    y = (ey + rng.uniform(0, nyp - 1, 50)) * c.dy
    z = rng.uniform(zl[0], zl[-1], 50)
    o = AN.Obs.interp(c, 3, field, x, y, z, np.zeros(50), 0.5)
    assert o.index.shape == (50, 8) and np.allclose(o.weight.sum(axis=1), 1.0)
    expect = 1.5 + 2e-4 * x - 3e-4 * y + 1e-3 * z
    assert np.allclose(o.sample({field: f}), expect, rtol=1e-12, atol=1e-12)
    # the transpose: <H f, r> = <f, H^T r>
    r = rng.standard_normal(50)
    lam = {field: np.zeros(c.shape)}
    o.scatter_into(lam, r)
    assert abs(float(o.sample({field: f}) @ r) - float(np.sum(f * lam[field]))) <= 1e-12 * np.sum(np.abs(f))
    with pytest.raises(ValueError):
        AN.Obs.interp(c, 3, field, [-c.dx], [y[0]], [z[0]], [0.0])
    with pytest.raises(ValueError):
        AN.Obs.interp(c, 3, field, [x[0]], [y[0]], [c.zt * 2], [0.0])
    c.close()


def test_gradient_with_interpolated_observations():
    """weighted observations (rows of points and weights) in the chained
    adjoint gradient, against central differences"""
    m = QuadMap(c=0.15)
    rng = np.random.default_rng(13)
    xb = {k: 0.5 * rng.standard_normal(m.n) for k in m.names}
    idx = np.array([[0, 1], [3, 4], [5, 6], [2, 2]])
    w = np.array([[0.25, 0.75], [0.5, 0.5], [0.9, 0.1], [0.3, 0.7]])
    obs = [AN.Obs(2, "a", idx, rng.standard_normal(4), 0.1, w),
           AN.Obs(4, "b", idx[:3], rng.standard_normal(3), 0.2, w[:3]),
           AN.Obs(4, "a", [1, 7], rng.standard_normal(2), 0.1)]
    v = AN.FourDVar(m, xb, 0.3, obs)
    x0 = {k: xb[k] + 0.1 * rng.standard_normal(m.n) for k in m.names}
    _, g = v.gradient(x0)
    for _ in range(4):
        d = {k: np.where(m.mask(k), rng.standard_normal(m.n), 0.0) for k in m.names}
        eps = 1e-6
        fd = (v.cost({k: x0[k] + eps * d[k] for k in m.names}) -
              v.cost({k: x0[k] - eps * d[k] for k in m.names})) / (2 * eps)
        an = sum(float(g[k] @ d[k]) for k in m.names)
        assert abs(fd - an) <= 1e-7 * max(1.0, abs(an)), (fd, an)
    with pytest.raises(ValueError):
        AN.Obs(1, "a", idx, [1.0, 2.0], 1.0, w)  # one row per observation


def test_gaussian_correlation_is_symmetric_with_unit_variance():
    S = AN.GaussianCorrelation(3000.0, 1000.0, 2000.0)
    rng = np.random.default_rng(17)
    a, b = rng.standard_normal((2, 4, 30, 40))
    assert abs(float(np.sum(S.apply("u", a) * b)) - float(np.sum(a * S.apply("u", b)))) <= 1e-10 * a.size
    w = rng.standard_normal((2, 400, 400))
    inner = S.apply("u", w)[:, 50:-50, 50:-50]
    assert abs(inner.var() - 1.0) < 0.05
    with pytest.raises(ValueError):
        AN.GaussianCorrelation(0.0, 1.0)
    # with vertical correlations (level axis) it stays symmetric
    Sz = AN.GaussianCorrelation(3000.0, 1000.0, 2000.0, levels=2.0)
    a, b = rng.standard_normal((2, 12, 30, 40))
    assert abs(float(np.sum(Sz.apply("u", a) * b)) - float(np.sum(a * Sz.apply("u", b)))) <= 1e-10 * a.size
    wz = rng.standard_normal((60, 60, 60))
    assert abs(Sz.apply("u", wz)[15:-15, 15:-15, 15:-15].var() - 1.0) < 0.1


def test_correlated_linear_minimiser_is_the_closed_form():
    """B^1/2 = sigma S: one outer loop with CG to convergence gives
    x = xb + U (I + U^T G^T R^-1 G U)^-1 U^T G^T R^-1 d"""
    m, xt, xb, obs = _problem(c=0.0)
    S = AN.GaussianCorrelation(2.0, 1.0)
    v = AN.FourDVar(m, xb, {"a": 0.3, "b": 0.2}, obs, corr=S)
    nctl = v.pack(xb).size
    r = v.minimise(outer=1, inner=3 * nctl, rtol=1e-13)
    U = np.array([v._U(e) for e in np.eye(nctl)]).T
    assert np.allclose(U, U.T, atol=1e-14)
    G, y, w = [], [], []
    for o in obs:
        rows = [o.sample(m.forecast(v.unpack(e), o.step)) for e in np.eye(nctl)]
        G.append(np.array(rows).T)
        y.append(o.value - o.sample(m.forecast(xb, o.step)))
        w.append(1.0 / o.sigma ** 2)
    G, y, w = np.vstack(G), np.concatenate(y), np.concatenate(w)
    GU = G @ U
    chi = np.linalg.solve(np.eye(nctl) + GU.T @ (w[:, None] * GU), GU.T @ (w * y))
    assert np.allclose(v.pack(r.x), v.pack(xb) + U @ chi, rtol=1e-9, atol=1e-11)
    assert r.cost[-1] < r.cost[0]
    # correlated increments are smooth: neighbouring points move together
    inc = v.pack(r.x) - v.pack(xb)
    assert np.corrcoef(inc[:-1], inc[1:])[0, 1] > 0.5
    with pytest.raises(ValueError):
        v.gradient(xb)
    with pytest.raises(ValueError):
        v.minimise(x0=xb)


def test_gradient_in_the_control_variable():
    m, xt, xb, obs = _problem(c=0.15)
    v = AN.FourDVar(m, xb, 0.3, obs, corr=AN.GaussianCorrelation(1.5, 1.0))
    rng = np.random.default_rng(23)
    chi = 0.3 * rng.standard_normal(v.pack(xb).size)
    j, g = v.gradient_chi(chi)
    assert j == pytest.approx(v.cost_chi(chi), rel=1e-14)
    for _ in range(4):
        d = rng.standard_normal(chi.size)
        eps = 1e-6
        fd = (v.cost_chi(chi + eps * d) - v.cost_chi(chi - eps * d)) / (2 * eps)
        assert abs(fd - float(g @ d)) <= 1e-7 * max(1.0, abs(fd)), (fd, float(g @ d))
