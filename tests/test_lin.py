"""Tangent-linear and adjoint runs of the dry dynamics (GPU).

Checks, on small dry cases with terrain / open and periodic boundaries /
Coriolis / Rayleigh sponge / diffusion:
  * dot-product test <M dx, y> = <dx, M^T y> over several steps with
    checkpoint segments (relative gap <= 1e-10 in FP64, <= 1e-4 in FP32);
  * the tangent against central finite differences of the forward model
    (FP64, eps = 1e-5 of the perturbation scale: relative L2 <= 1e-6);
  * the gradient of J = sum w^2 over a box against central differences along
    16 seeded random directions of (u0, theta'0): eps = 1e-3 (relative gap
    <= 5e-4, the second-order term of the central difference) and eps = 1e-5
    (<= 1e-6); and through the torch.autograd.Function wrapper.
The finite-difference checks avoid the open-boundary case at rest
(bubble_open): there the radiation faces switch between u = ub and the
radiation update as u crosses 0, a jump the tangent (the derivative of the
branch taken) does not see.  pi' ghost points are not state: no launch reads
or writes them, so they are left out of the comparisons.
"""

import numpy as np
import pytest

import wfe_b200 as W
from wfe_b200 import adjoint as A
from helpers import CASES

pytestmark = pytest.mark.gpu

LIN_CASES = ["schaer_open", "bubble_open", "straka_periodic"]


def _spinup(name, prec, n=4):
    c = W.Case(CASES / f"{name}.ini", precision=prec)
    c.run(n)
    c.sync()
    return c, A.get_fields(c)


def _rand_fields(c, rng, scale=None):
    """random values on every padded point (ghost entries included: the step
    ignores them as inputs, and as outputs they are genuine linear outputs)"""
    return {k: rng.standard_normal(c.shape) * (scale or {}).get(k, 1.0) for k in A.FIELDS5}


def _dot(a, b):
    return sum(float(np.sum(a[k] * b[k])) for k in A.FIELDS5)


@pytest.mark.parametrize("name", LIN_CASES)
@pytest.mark.parametrize("prec,tol", [("f64", 1e-10), ("f32", 1e-4)])
def test_dot_product(name, prec, tol):
    c, x0 = _spinup(name, prec)
    rng = np.random.default_rng(7)
    dx, y = _rand_fields(c, rng), _rand_fields(c, rng)
    n = 5
    mdx = A.tangent(c, x0, dx, n)
    mty = A.adjoint(c, x0, y, n, every=2)
    lhs, rhs = _dot(mdx, y), _dot(dx, mty)
    assert abs(lhs - rhs) <= tol * max(abs(lhs), abs(rhs)), (lhs, rhs)
    c.close()


def _valid(c, k):
    m = np.ones(c.shape, dtype=bool)
    if k == "pip":
        m[:] = False
        g = c.ng
        m[g:g + c.nz, g:g + c.ny, g:g + c.nx] = True
    return m


@pytest.mark.parametrize("name", ["schaer_open", "straka_periodic"])
def test_tangent_matches_finite_differences(name):
    c, x0 = _spinup(name, "f64")
    rng = np.random.default_rng(11)
    scale = {"u": 1.0, "v": 1.0, "w": 0.2, "thp": 0.5, "pip": 1e-4}
    d = _rand_fields(c, rng, scale)
    n = 4
    eps = 1e-5
    mdx = A.tangent(c, x0, d, n)
    res = {}
    for sgn in (1, -1):
        A.set_fields(c, {k: x0[k] + sgn * eps * d[k] for k in A.FIELDS5})
        c.run(n)
        res[sgn] = A.get_fields(c)
    for k in A.FIELDS5:
        m = _valid(c, k)
        fd = (res[1][k] - res[-1][k])[m] / (2 * eps)
        err = np.linalg.norm(fd - mdx[k][m]) / max(np.linalg.norm(fd), 1e-300)
        assert err <= 1e-6, (k, err)
    c.close()


def test_gradient_of_w_box_cost_matches_central_differences():
    c, x0 = _spinup("schaer_open", "f64", 8)
    mask = A.w_box_mask(c, 9000.0, 13000.0, 500.0, 3000.0)
    assert mask.any()
    n = 12
    c_ = c

    def J(x):
        A.set_fields(c_, x)
        c_.run(n)
        return A.w_box_cost(c_.field("w"), mask)

    A.set_fields(c, x0)
    c.run(n)
    wN = c.field("w")
    ybar = {k: np.zeros_like(x0[k]) for k in A.FIELDS5}
    ybar["w"] = 2 * np.where(mask, wN, 0.0)
    g = A.adjoint(c, x0, ybar, n, every=5)
    rng = np.random.default_rng(3)
    for r in range(16):
        d = {k: np.zeros_like(x0[k]) for k in A.FIELDS5}
        d["u"] = rng.standard_normal(x0["u"].shape)
        d["thp"] = 0.5 * rng.standard_normal(x0["thp"].shape)
        ad = _dot(g, d)
        for eps, tol in ((1e-3, 5e-4), (1e-5, 1e-6)):
            fd = (J({k: x0[k] + eps * d[k] for k in A.FIELDS5}) -
                  J({k: x0[k] - eps * d[k] for k in A.FIELDS5})) / (2 * eps)
            assert abs(fd - ad) <= tol * abs(fd), (r, eps, fd, ad)
    c.close()


def test_autograd_function_gradient():
    torch = pytest.importorskip("torch")
    c, x0 = _spinup("bubble_open", "f64", 4)
    n = 6
    xt = {k: torch.tensor(x0[k], requires_grad=True) for k in A.FIELDS5}
    out = A.forecast(c, n, xt, every=3)
    J = (out[2] ** 2).sum() + 0.1 * (out[3] ** 2).sum()
    J.backward()
    ybar = {k: np.zeros_like(x0[k]) for k in A.FIELDS5}
    ybar["w"] = 2 * out[2].detach().numpy()
    ybar["thp"] = 0.2 * out[3].detach().numpy()
    g = A.adjoint(c, x0, ybar, n, every=3)
    # the adjoint accumulates with atomics, so two runs agree to rounding only
    for k in A.FIELDS5:
        a, b = xt[k].grad.numpy(), g[k]
        assert np.linalg.norm(a - b) <= 1e-10 * max(np.linalg.norm(b), 1e-300), k
    assert np.linalg.norm(g["w"]) > 0
    c.close()


@pytest.mark.parametrize("name", ["schaer_open", "straka_periodic"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_tangent_run_advances_the_state_like_the_forward(name, prec):
    """tl_run takes the state x0 -> xN exactly as run does: the column's TL
    launch writes the forward column's outputs itself, bit for bit."""
    c, x0 = _spinup(name, prec)
    A.set_fields(c, x0)
    c.run(4)
    ref = A.get_fields(c)
    A.tangent(c, x0, _rand_fields(c, np.random.default_rng(1)), 4)
    got = A.get_fields(c)
    for k in A.FIELDS5:
        assert np.array_equal(ref[k], got[k]), k
    c.close()


@pytest.mark.parametrize("every", [1, 4, 5, 8, 0])
def test_dot_product_any_checkpoint_interval(every):
    """The adjoint sweep is exact for every checkpoint interval: one step per
    segment, segments of uneven length, a single segment (no separate forward
    run at all), and 0 (the longest interval the device memory holds: here a
    single segment)."""
    c, x0 = _spinup("schaer_open", "f64")
    rng = np.random.default_rng(17)
    dx, y = _rand_fields(c, rng), _rand_fields(c, rng)
    n = 5
    mdx = A.tangent(c, x0, dx, n)
    mty = A.adjoint(c, x0, y, n, every=every)
    lhs, rhs = _dot(mdx, y), _dot(dx, mty)
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs)), (lhs, rhs)
    # the state ends at x_N either way
    A.set_fields(c, x0)
    c.run(n)
    ref = A.get_fields(c)
    A.adjoint(c, x0, y, n, every=every)
    got = A.get_fields(c)
    for k in A.FIELDS5:
        assert np.array_equal(ref[k], got[k]), k
    c.close()


def test_adjoint_across_growing_checkpoint_intervals():
    """Longer segments need a larger undo log; the segment graphs captured for
    the old log are retired with it, so a later call reusing a short segment
    still runs on valid memory and gives the same gradient."""
    c, x0 = _spinup("schaer_open", "f64")
    rng = np.random.default_rng(23)
    y = _rand_fields(c, rng)
    n = 7
    ref = None
    for every in (2, 3, 7, 3, 2):
        g = A.adjoint(c, x0, y, n, every=every)
        if ref is None:
            ref = g
        for k in A.FIELDS5:
            assert np.linalg.norm(g[k] - ref[k]) <= 1e-12 * max(np.linalg.norm(ref[k]), 1e-300), (every, k)
    c.close()
