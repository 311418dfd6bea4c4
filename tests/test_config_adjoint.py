"""Tangent-linear and adjoint runs of the benchmark configurations at full
size and length (GPU).

Schaer mountain waves, 400x4x65 (cases/schaer_400.ini): the 1 h forward run
(900 steps of 4 s) from the initial state, checkpoints every 30 steps, cost
J = sum of w^2 over the box 5-15 km downstream of the ridge (x in
105-115 km) at 2-6 km height.
  * dot-product test <M dx, y> = <dx, M^T y> over the 900 steps, random dx, y
    on every state field: relative gap <= 1e-10 (FP64; measured 5e-15) and
    <= 1e-4 (FP32; measured 2.8e-7);
  * dJ/d(u0, theta'0) from the adjoint against central finite differences
    with eps = 1e-3 relative to the field scales (u: the 10 m/s wind, theta':
    1 K) along 16 seeded random directions: relative gap <= 1e-3 (FP64;
    measured <= 3.4e-4, the O(eps^2) term and the upwind switches where w
    crosses 0); the FP32 adjoint against the FP64 differences along 4 of
    them: <= 1e-3 (measured 3.2e-4).
WK82 160x160x40 (cases/wk82_160.ini) with the linearised Kessler column and
mixed-phase blend, 20 min (200 steps of 6 s) from the initial state, the
positive-definite limiter and w damping off (neither is linearised):
  * dot-product test over the 200 steps on all eight fields: <= 1e-10 (FP64;
    measured 5e-15), <= 1e-4 (FP32; measured 2.7e-7);
  * J = sum w^2 + 1e4 sum qr^2 over a box in the storm against central
    differences with eps = 1e-5 along 4 directions of (u, theta', qv): the
    microphysics' branches (saturation adjustment, the clips to zero) make J
    only piecewise smooth, and points that switch branch under the
    perturbation put a floor under the difference, so the bound is 0.1
    (measured 2e-3 - 4.6e-2).
"""

import numpy as np
import pytest

import wfe_b200 as W
from wfe_b200 import adjoint as A
from helpers import ROOT

pytestmark = pytest.mark.gpu

SCHAER = ROOT / "cases" / "schaer_400.ini"
WK82 = ROOT / "cases" / "wk82_160.ini"


def _dot(a, b, names):
    return sum(float(np.sum(a[k] * b[k])) for k in names)


@pytest.mark.parametrize("prec,tol", [("f64", 1e-10), ("f32", 1e-4)])
def test_schaer_400_dot_product(prec, tol):
    c = W.Case(SCHAER, precision=prec)
    x0 = A.get_fields(c)
    names = A.state_names(c)
    rng = np.random.default_rng(7)
    dx = {k: rng.standard_normal(c.shape) for k in names}
    y = {k: rng.standard_normal(c.shape) for k in names}
    mdx = A.tangent(c, x0, dx, 900)
    mty = A.adjoint(c, x0, y, 900, every=30)
    lhs, rhs = _dot(mdx, y, names), _dot(dx, mty, names)
    assert abs(lhs - rhs) <= tol * max(abs(lhs), abs(rhs)), (lhs, rhs)
    c.close()


def _schaer_gradient(prec):
    c = W.Case(SCHAER, precision=prec)
    x0 = A.get_fields(c)
    names = A.state_names(c)
    mask = A.w_box_mask(c, 105000.0, 115000.0, 2000.0, 6000.0)
    assert mask.sum() > 500
    A.set_fields(c, x0)
    c.run(900)
    wN = c.field("w")
    ybar = {k: np.zeros_like(x0[k]) for k in names}
    ybar["w"] = 2 * np.where(mask, wN, 0.0)
    g = A.adjoint(c, x0, ybar, 900, every=30)
    c.close()
    return x0, names, mask, g


def _schaer_fd(x0, names, mask, ndir, eps=1e-3):
    """central differences of J in FP64 along seeded directions of (u, theta')"""
    c = W.Case(SCHAER, precision="f64")

    def J(x):
        A.set_fields(c, x)
        c.run(900)
        return A.w_box_cost(c.field("w"), mask)

    rng = np.random.default_rng(3)
    out = []
    for _ in range(ndir):
        d = {k: np.zeros_like(x0[k]) for k in names}
        d["u"] = 10.0 * rng.standard_normal(x0["u"].shape)
        d["thp"] = rng.standard_normal(x0["thp"].shape)
        fd = (J({k: x0[k] + eps * d[k] for k in names}) -
              J({k: x0[k] - eps * d[k] for k in names})) / (2 * eps)
        out.append((d, fd))
    c.close()
    return out


def test_schaer_400_gradient_against_finite_differences():
    x0, names, mask, g64 = _schaer_gradient("f64")
    _, _, _, g32 = _schaer_gradient("f32")
    for r, (d, fd) in enumerate(_schaer_fd(x0, names, mask, 16)):
        ad = _dot(g64, d, names)
        assert abs(fd - ad) <= 1e-3 * abs(fd), (r, fd, ad)
        if r < 4:
            ad32 = _dot(g32, d, names)
            assert abs(fd - ad32) <= 1e-3 * abs(fd), (r, fd, ad32)


OV = {"pd_moist": "off", "w_damping": "off"}
SC = {"qv": 1e-3, "qc": 1e-3, "qr": 1e-3}


@pytest.mark.parametrize("prec,tol", [("f64", 1e-10), ("f32", 1e-4)])
def test_wk82_160_moist_dot_product(prec, tol):
    c = W.Case(WK82, OV, precision=prec)
    x0 = A.get_fields(c)
    names = A.state_names(c)
    assert names == A.FIELDS8
    rng = np.random.default_rng(7)
    dx = {k: rng.standard_normal(c.shape) * SC.get(k, 1.0) for k in names}
    y = {k: rng.standard_normal(c.shape) * SC.get(k, 1.0) for k in names}
    mdx = A.tangent(c, x0, dx, 200)
    mty = A.adjoint(c, x0, y, 200, every=30)
    lhs, rhs = _dot(mdx, y, names), _dot(dx, mty, names)
    assert abs(lhs - rhs) <= tol * max(abs(lhs), abs(rhs)), (lhs, rhs)
    c.close()


def test_wk82_160_moist_gradient_against_finite_differences():
    c = W.Case(WK82, OV, precision="f64")
    x0 = A.get_fields(c)
    names = A.state_names(c)
    g_ = c.ng
    mask = np.zeros(c.shape, dtype=bool)
    mask[g_ + 2:g_ + 20, g_ + 60:g_ + 100, g_ + 60:g_ + 100] = True

    def run_cost(x):
        A.set_fields(c, x)
        c.run(200)
        s = A.get_fields(c)
        return (float(np.sum(np.where(mask, s["w"], 0) ** 2) +
                      1e4 * np.sum(np.where(mask, s["qr"], 0) ** 2)), s)

    j0, s = run_cost(x0)
    assert float(s["qr"].max()) > 1e-3  # the storm rains inside the 20 min
    ybar = {k: np.zeros_like(x0[k]) for k in names}
    ybar["w"] = 2 * np.where(mask, s["w"], 0.0)
    ybar["qr"] = 2e4 * np.where(mask, s["qr"], 0.0)
    g = A.adjoint(c, x0, ybar, 200, every=30)
    rng = np.random.default_rng(3)
    eps = 1e-5
    for r in range(4):
        d = {k: np.zeros_like(x0[k]) for k in names}
        d["u"] = rng.standard_normal(x0["u"].shape)
        d["thp"] = rng.standard_normal(x0["thp"].shape)
        d["qv"] = 1e-3 * rng.standard_normal(x0["qv"].shape)
        ad = _dot(g, d, names)
        fd = (run_cost({k: x0[k] + eps * d[k] for k in names})[0] -
              run_cost({k: x0[k] - eps * d[k] for k in names})[0]) / (2 * eps)
        assert abs(fd - ad) <= 0.1 * abs(fd), (r, fd, ad)
    c.close()
