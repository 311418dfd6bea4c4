"""Forecast gradients through the tangent-linear and adjoint runs.

``Forecast`` is a torch.autograd.Function over a Case: its forward maps
the initial state x0 = (u, v, w, theta', pi'[, qv, qc, qr]) -- the moisture
species when the case carries them -- to the state after ``nsteps`` large
steps; its backward runs the adjoint (wfe_ad_run: checkpoints of the
state every ``every`` steps, recomputation in between) on the incoming
gradients and returns dJ/dx0.  Fields are in the reference's padded layout
(NZ, NY, NX) = (nz+7, ny+6, nx+6), which holds every prognostic point (with
open boundaries the faces u(nx) and v(ny) are prognostic, and the Writer's
interior layout omits them); ghost entries are inputs of nothing (the step
refills them) and receive no gradient.  ``w_box_cost`` is the sensitivity cost of the Schaer
mountain-wave experiment, J = sum of w^2 over a box of the x-z plane.
"""

from __future__ import annotations

import numpy as np

FIELDS5 = ("u", "v", "w", "thp", "pip")
FIELDS8 = FIELDS5 + ("qv", "qc", "qr")


def state_names(case) -> tuple:
    """the prognostic fields of the case's state vector"""
    return FIELDS8 if case.moisture else FIELDS5


def set_fields(case, fields: dict, role: str = "state") -> None:
    for k, a in fields.items():
        case.set_field(k, np.ascontiguousarray(a, dtype=np.float64).reshape(case.shape), role=role)


def get_fields(case, role: str = "state", names=None) -> dict:
    return {k: case.field(k, role=role) for k in (names or state_names(case))}


def w_box_mask(case, x0: float, x1: float, z0: float, z1: float) -> np.ndarray:
    """Padded-layout mask of the w points (levels 0..nz, interior columns) with
    cell-centre x in [x0, x1] and physical height h + zeta_w (zt - h) / zt in
    [z0, z1] (src/core/metric.hpp)."""
    g = case.ng
    zw = case.metric("zeta_w")[g:g + case.nz + 1]
    h = case.metric("h").reshape(case.NY, case.NX)[g:g + case.ny, g:g + case.nx]
    x = (np.arange(case.nx) + 0.5) * case.dx
    z = h[None, :, :] + zw[:, None, None] * (case.zt - h[None, :, :]) / case.zt
    inner = (z >= z0) & (z <= z1) & ((x >= x0) & (x <= x1))[None, None, :]
    m = np.zeros(case.shape, dtype=bool)
    m[g:g + case.nz + 1, g:g + case.ny, g:g + case.nx] = inner
    return m


def w_box_cost(w: np.ndarray, mask: np.ndarray) -> float:
    return float(np.sum(np.where(mask, w, 0.0) ** 2))


def tangent(case, x0: dict, dx0: dict, nsteps: int) -> dict:
    """M dx0 for the nsteps from x0 (the case ends at xN)."""
    case.lin_enable()
    set_fields(case, x0)
    case.lin_zero()
    set_fields(case, dx0, role="lin")
    case.tl_run(nsteps)
    return get_fields(case, role="lin")


def adjoint(case, x0: dict, ybar: dict, nsteps: int, every: int = 30) -> dict:
    """M^T ybar for the nsteps from x0 (the case ends at xN)."""
    case.lin_enable()
    set_fields(case, x0)
    case.lin_zero()
    set_fields(case, ybar, role="lin")
    case.ad_run(nsteps, checkpoint_every=every)
    return get_fields(case, role="lin")


try:
    import torch

    class Forecast(torch.autograd.Function):
        """x0 -> xN of a dry Case; gradients through the adjoint run."""

        @staticmethod
        def forward(ctx, case, nsteps, every, *fields):
            names = state_names(case)
            x0 = {k: t.detach().to("cpu", torch.float64).numpy() for k, t in zip(names, fields)}
            ctx.case, ctx.nsteps, ctx.every, ctx.x0, ctx.names = case, int(nsteps), int(every), x0, names
            case.lin_enable()
            set_fields(case, x0)
            case.run(ctx.nsteps)
            out = get_fields(case)
            ref = fields[0]
            return tuple(torch.from_numpy(out[k]).to(ref.device, ref.dtype) for k in names)

        @staticmethod
        def backward(ctx, *grads):
            ybar = {k: (g.detach().to("cpu", torch.float64).numpy() if g is not None
                        else np.zeros_like(ctx.x0[k])) for k, g in zip(ctx.names, grads)}
            gx = adjoint(ctx.case, ctx.x0, ybar, ctx.nsteps, ctx.every)
            dev = next((g.device for g in grads if g is not None), "cpu")
            return (None, None, None) + tuple(torch.from_numpy(gx[k]).to(dev) for k in ctx.names)

    def forecast(case, nsteps: int, x0: dict, every: int = 30):
        """dict of torch tensors x0 -> tuple of the final state fields (autograd)."""
        return Forecast.apply(case, nsteps, every, *[x0[k] for k in state_names(case)])

except ImportError:  # torch is optional for the numpy entry points
    Forecast = None
