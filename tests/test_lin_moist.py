"""Tangent-linear and adjoint runs with moisture and the Kessler column (GPU).

The moist WK82 sounding (wk82_small: stretched grid, tanh shear, Rayleigh
sponge, Kessler with the mixed-phase blend) with the positive-definite
limiter and w damping off (neither is linearised).  The initial state adds a
cloud and a rain shaft to the spun-up state so that every conversion branch
is live: autoconversion and accretion, rain evaporation in subsaturated air,
condensation and cloud evaporation, the liquid/ice blend aloft, and
sedimentation with several subcycles (dt = 10 s).

  * dot-product test <M dx, y> = <dx, M^T y> over 4 steps with checkpoint
    segments, all eight fields (relative gap <= 1e-10 in FP64, <= 1e-4 in
    FP32), with open and with periodic lateral boundaries;
  * the gradient of J = sum(w^2) + 1e4 sum(qr^2) against central differences
    along 16 seeded directions of (u, theta', qv) with eps = 1e-5 (relative
    gap <= 1e-4).  The microphysics is piecewise smooth (max(q, 0), the
    saturation and evaporation clips, the condensation switch): at eps = 1e-3
    a perturbation moves enough points across a branch that the central
    difference itself is off by up to 1e-2, while at 1e-5 the per-field
    tangent-vs-difference gaps are 1e-6 to 1e-9.  The directions leave qc and
    qr alone, which sit at exactly zero over most of the domain (the kink of
    max(q, 0)).
"""

import numpy as np
import pytest

import wfe_b200 as W
from wfe_b200 import adjoint as A
from helpers import CASES

pytestmark = pytest.mark.gpu

OV = {"pd_moist": "off", "w_damping": "off", "dt": "10", "acoustic_ns": "10"}
PERIODIC = dict(OV, bc_x="periodic", bc_y="periodic")


def _bump(c, i0, j0, k0, ri, rk):
    """cos^2 bump on the padded grid centred at interior (i0, j0, k0)"""
    g = c.ng
    k = np.arange(c.NZ)[:, None, None] - g - k0
    j = np.arange(c.NY)[None, :, None] - g - j0
    i = np.arange(c.NX)[None, None, :] - g - i0
    r = np.sqrt((i / ri) ** 2 + (j / ri) ** 2 + (k / rk) ** 2)
    return np.where(r < 1, np.cos(0.5 * np.pi * r) ** 2, 0.0)


def _moist_state(prec, ov):
    c = W.Case(CASES / "wk82_small.ini", overrides=ov, precision=prec)
    c.run(3)
    c.sync()
    x = A.get_fields(c)
    assert set(x) == set(A.FIELDS8)
    # rain shaft and low cloud in mid-domain, a mixed-phase cloud aloft,
    # moistened air under the shaft
    x["qr"] = x["qr"] + 6e-3 * _bump(c, 8, 8, 4, 4, 4)
    x["qc"] = x["qc"] + 1.5e-3 * _bump(c, 5, 9, 3, 3, 2) + 1e-3 * _bump(c, 10, 6, 11, 3, 2)
    x["qv"] = x["qv"] * (1 + 0.15 * _bump(c, 6, 8, 2, 4, 2))
    A.set_fields(c, x)
    return c, x


def _rand(c, rng, names, scale):
    return {k: rng.standard_normal(c.shape) * scale.get(k, 1.0) for k in names}


def _dot(a, b):
    return sum(float(np.sum(a[k] * b[k])) for k in a)


@pytest.mark.parametrize("ov", [OV, PERIODIC], ids=["open", "periodic"])
@pytest.mark.parametrize("prec,tol", [("f64", 1e-10), ("f32", 1e-4)])
def test_moist_dot_product(ov, prec, tol):
    c, x0 = _moist_state(prec, ov)
    rng = np.random.default_rng(5)
    sc = {"qv": 1e-3, "qc": 1e-3, "qr": 1e-3}
    dx, y = _rand(c, rng, A.FIELDS8, sc), _rand(c, rng, A.FIELDS8, sc)
    n = 4
    mdx = A.tangent(c, x0, dx, n)
    mty = A.adjoint(c, x0, y, n, every=3)
    lhs, rhs = _dot(mdx, y), _dot(dx, mty)
    assert abs(lhs - rhs) <= tol * max(abs(lhs), abs(rhs)), (lhs, rhs)
    # the moisture species carry sensitivity both ways
    for k in ("qv", "qc", "qr"):
        assert np.linalg.norm(mdx[k]) > 0 and np.linalg.norm(mty[k]) > 0, k
    c.close()


def test_moist_gradient_matches_central_differences():
    c, x0 = _moist_state("f64", PERIODIC)
    n = 6

    def cost(f):
        return float(np.sum(f["w"] ** 2) + 1e4 * np.sum(f["qr"] ** 2))

    def J(x):
        A.set_fields(c, x)
        c.run(n)
        return cost(A.get_fields(c))

    A.set_fields(c, x0)
    c.run(n)
    xN = A.get_fields(c)
    ybar = {k: np.zeros_like(x0[k]) for k in A.FIELDS8}
    ybar["w"] = 2 * xN["w"]
    ybar["qr"] = 2e4 * xN["qr"]
    g = A.adjoint(c, x0, ybar, n, every=4)
    assert np.linalg.norm(g["qv"]) > 0 and np.linalg.norm(g["qr"]) > 0
    rng = np.random.default_rng(13)
    for r in range(16):
        d = {k: np.zeros_like(x0[k]) for k in A.FIELDS8}
        d["u"] = rng.standard_normal(c.shape)
        d["thp"] = 0.5 * rng.standard_normal(c.shape)
        d["qv"] = 1e-4 * rng.standard_normal(c.shape)
        ad = _dot(g, d)
        eps = 1e-5
        fd = (J({k: x0[k] + eps * d[k] for k in A.FIELDS8}) -
              J({k: x0[k] - eps * d[k] for k in A.FIELDS8})) / (2 * eps)
        assert abs(fd - ad) <= 1e-4 * abs(fd), (r, fd, ad)
    c.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_moist_tangent_run_advances_the_state_like_the_forward(prec):
    c, x0 = _moist_state(prec, OV)
    c.run(4)
    ref = A.get_fields(c)
    rng = np.random.default_rng(9)
    A.tangent(c, x0, _rand(c, rng, A.FIELDS8, {"qv": 1e-3, "qc": 1e-3, "qr": 1e-3}), 4)
    got = A.get_fields(c)
    for k in A.FIELDS8:
        assert np.array_equal(ref[k], got[k]), k
    c.close()


def test_refuses_positive_definite_moisture():
    c = W.Case(CASES / "wk82_small.ini", precision="f64")
    with pytest.raises(W.WfeError, match="positive-definite"):
        c.lin_enable()
    c.close()
