"""Variational analysis and analysis nudging driven by the adjoint.

Strong-constraint 4D-Var over a window of large steps:

    J(x0) = 1/2 sum_f |(x0_f - xb_f) / sb_f|^2
          + 1/2 sum_k |(H_k x(t_k) - y_k) / so_k|^2

x(t) is the model trajectory from x0 (the forward step), xb the background,
sb_f one background standard deviation per prognostic field (diagonal B),
H_k point sampling of one prognostic field at large step t_k and so_k the
observation standard deviation.  The gradient is one chained adjoint sweep:
backwards from the last observation time, H_k^T R_k^-1 (H_k x - y_k) is added
to the adjoint at each observation time and carried to the previous one by
the adjoint run of the steps in between (wfe_ad_run: dJ/dx_end -> dJ/dx_start).

``FourDVar.minimise`` is incremental (Gauss-Newton) 4D-Var: each outer loop
relinearises about the current x0; its inner loop minimises the quadratic
cost of the increment in the control variable chi = B^-1/2 dx by conjugate
gradients, one tangent-linear and one adjoint sweep per iteration (the
Hessian I + B^1/2 M^T H^T R^-1 H M B^1/2 is symmetric positive definite, and
the tangent and adjoint runs are exact transposes of each other).

The reference has no analysis step: it ingests analyses as boundary files and
relaxes toward them with the BdyManager weights, the cos^2 Davies ramp at the
open edges and 1/nudge_tau as the interior analysis-nudging floor
(src/dynamics/boundary.cpp:24-39; the relaxation term of compute_tendencies,
src/dynamics/kernels.cu:292-304, 981-995).  ``nudge`` feeds an analysis back
through that same path: targets lo = hi = xa for (u, v, theta', pi', qv) and
the BdyManager weights, so a forecast from the background relaxes toward the
analysis instead of restarting from it.

Fields are dicts of numpy arrays in the reference's padded layout; the
control points (``control_mask``) are the prognostic points of each field.
The solver only talks to a model object with ``names``, ``mask(name)``,
``forecast(x0, n)``, ``tangent(x0, dx, n)`` and ``adjoint(x0, lam, n)``
(``CaseModel`` wraps a Case), so its algebra is testable without a device.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import adjoint as A

BDY_FIELDS = ("u", "v", "thp", "pip", "qv")


# ------------------------------------------------------------------ model
def control_mask(case, name: str) -> np.ndarray:
    """Prognostic points of one field in the padded layout: cells for the
    scalars, faces i = 0..nx for u, j = 0..ny for v, levels k = 0..nz for w
    (src/core/grid.hpp:22-36).  Ghost points are refilled by each step and are
    inputs of nothing."""
    g = case.ng
    m = np.zeros(case.shape, dtype=bool)
    ex = 1 if name == "u" else 0
    ey = 1 if name == "v" else 0
    ez = 1 if name == "w" else 0
    m[g:g + case.nz + ez, g:g + case.ny + ey, g:g + case.nx + ex] = True
    return m


class CaseModel:
    """The forward, tangent-linear and adjoint runs of a Case as the solver
    sees them.  ``every`` is the adjoint's checkpoint interval (0: the
    largest the device memory allows)."""

    def __init__(self, case, every: int = 0):
        self.case = case
        self.every = int(every)
        self.names = A.state_names(case)
        self._masks = {k: control_mask(case, k) for k in self.names}
        case.lin_enable()

    def mask(self, name: str) -> np.ndarray:
        return self._masks[name]

    def forecast(self, x0: dict, n: int) -> dict:
        A.set_fields(self.case, x0)
        if n > 0:
            self.case.run(n)
        return A.get_fields(self.case, names=self.names)

    def tangent(self, x0: dict, dx: dict, n: int) -> dict:
        if n == 0:
            return {k: np.array(v, dtype=np.float64) for k, v in dx.items()}
        return A.tangent(self.case, x0, dx, n)

    def adjoint(self, x0: dict, lam: dict, n: int) -> dict:
        if n == 0:
            return {k: np.array(v, dtype=np.float64) for k, v in lam.items()}
        return A.adjoint(self.case, x0, lam, n, every=self.every)


# ----------------------------------------------------------- observations
@dataclass
class Obs:
    """Observations of one prognostic field after `step` large steps (0 = the
    start of the window).  Each observation is a point value (`index`: flat
    indices into the padded layout, one per observation) or a weighted sum of
    field values (`index` and `weight` of shape (n_obs, n_points), e.g. the
    trilinear interpolation weights of ``Obs.interp``); values and standard
    deviation(s)."""

    step: int
    field: str
    index: np.ndarray
    value: np.ndarray
    sigma: float | np.ndarray = 1.0
    weight: np.ndarray | None = None

    def __post_init__(self):
        self.value = np.asarray(self.value, dtype=np.float64).ravel()
        idx = np.asarray(self.index, dtype=np.int64)
        if self.weight is None:
            self.index = idx.ravel()
            if self.index.shape != self.value.shape:
                raise ValueError("one value per observed point")
        else:
            w = np.asarray(self.weight, dtype=np.float64)
            if idx.ndim != 2 or w.shape != idx.shape or idx.shape[0] != self.value.size:
                raise ValueError("index and weight: one row of points per observation")
            self.index, self.weight = idx, w
        s = np.broadcast_to(np.asarray(self.sigma, dtype=np.float64), self.value.shape)
        if np.any(s <= 0):
            raise ValueError("observation standard deviations must be positive")
        self.sigma = np.array(s)

    @staticmethod
    def at(case, step: int, field: str, i, j, k, value, sigma=1.0) -> "Obs":
        """observations at interior indices (i, j, k) of `field`"""
        g = case.ng
        i, j, k = (np.asarray(a, dtype=np.int64) for a in (i, j, k))
        idx = ((k + g) * case.NY + (j + g)) * case.NX + (i + g)
        return Obs(step, field, idx, value, sigma)

    @staticmethod
    def interp(case, step: int, field: str, x, y, z, value, sigma=1.0) -> "Obs":
        """Observations at physical positions (x, y in m from the domain's
        corner, z in m above sea level): trilinear interpolation between the
        field's own points in (x, y, zeta), zeta = zt (z - h) / (zt - h) with
        the terrain height h interpolated bilinearly at (x, y) (the Gal-Chen
        map, src/core/metric.cpp).  Cell-centred fields sit at ((i + 1/2) dx,
        (j + 1/2) dy, zeta_c), u on x faces (i dx), v on y faces (j dy), w on
        the zeta_w levels.  Positions outside the field's points raise."""
        g = case.ng
        x, y, z = (np.atleast_1d(np.asarray(a, dtype=np.float64)).ravel() for a in (x, y, z))
        if not (x.shape == y.shape == z.shape):
            raise ValueError("one x, y, z per observation")
        ex = 0.0 if field == "u" else 0.5
        ey = 0.0 if field == "v" else 0.5
        nxp = case.nx + 1 if field == "u" else case.nx
        nyp = case.ny + 1 if field == "v" else case.ny
        zeta = case.metric("zeta_w" if field == "w" else "zeta_c")
        nzp = case.nz + 1 if field == "w" else case.nz
        zlev = zeta[g:g + nzp]

        def axis(pos, d, e, n, name):
            f = pos / d - e
            if np.any(f < 0) or np.any(f > n - 1):
                raise ValueError(f"observation {name} outside the field's points")
            i0 = np.minimum(np.floor(f).astype(np.int64), max(n - 2, 0))
            return i0, f - i0

        i0, tx = axis(x, case.dx, ex, nxp, "x")
        j0, ty = axis(y, case.dy, ey, nyp, "y")
        # terrain height at (x, y) from the cell-centre h (ghost ring included)
        h2 = case.metric("h").reshape(case.NY, case.NX)
        fi, fj = x / case.dx - 0.5, y / case.dy - 0.5
        hi0, hj0 = np.floor(fi).astype(np.int64), np.floor(fj).astype(np.int64)
        hx, hy = fi - hi0, fj - hj0
        hi0, hj0 = hi0 + g, hj0 + g
        h = ((1 - hx) * (1 - hy) * h2[hj0, hi0] + hx * (1 - hy) * h2[hj0, hi0 + 1] +
             (1 - hx) * hy * h2[hj0 + 1, hi0] + hx * hy * h2[hj0 + 1, hi0 + 1])
        zt = case.zt
        zc = zt * (z - h) / (zt - h)
        if np.any(zc < zlev[0]) or np.any(zc > zlev[-1]):
            raise ValueError("observation z outside the field's levels")
        k0 = np.clip(np.searchsorted(zlev, zc, side="right") - 1, 0, nzp - 2)
        tz = (zc - zlev[k0]) / (zlev[k0 + 1] - zlev[k0])
        idx, wts = [], []
        for dk, wk in ((0, 1 - tz), (1, tz)):
            for dj, wj in ((0, 1 - ty), (1, ty)):
                for di, wi in ((0, 1 - tx), (1, tx)):
                    idx.append(((k0 + dk + g) * case.NY + (j0 + dj + g)) * case.NX + (i0 + di + g))
                    wts.append(wk * wj * wi)
        return Obs(step, field, np.stack(idx, axis=1), value, sigma, np.stack(wts, axis=1))

    def sample(self, x: dict) -> np.ndarray:
        v = x[self.field].ravel()[self.index]
        return v if self.weight is None else np.sum(v * self.weight, axis=1)

    def scatter_into(self, lam: dict, r: np.ndarray) -> None:
        """lam[field] += H^T r (repeated indices accumulate)"""
        if self.weight is None:
            np.add.at(lam[self.field].reshape(-1), self.index, r)
        else:
            np.add.at(lam[self.field].reshape(-1), self.index.ravel(),
                      (self.weight * np.asarray(r)[:, None]).ravel())


class GaussianCorrelation:
    """Horizontal background-error correlations for ``FourDVar(corr=...)``:
    S, a separable Gaussian filter of length scale `length` along x (the last
    axis, spacing dx) and y (the axis before it, spacing dy) on every level,
    truncated at three length scales and normalised so that S applied to
    white noise has unit variance.  B^1/2 = sigma S, so B = sigma^2 S S^T
    correlates like a Gaussian of length sqrt(2) * length.  `levels` > 0
    adds a Gaussian of that many levels along the level axis (the axis
    before y, in level indices).  The filter is zero outside the field, which
    keeps S symmetric, as the conjugate-gradient inner loop requires."""

    def __init__(self, length: float, dx: float, dy: float | None = None, levels: float = 0.0):
        if not length > 0 or levels < 0:
            raise ValueError("correlation lengths must be positive")

        def kernel(scale, d):
            n = int(np.ceil(3.0 * scale / d))
            t = np.arange(-n, n + 1) * d
            g = np.exp(-0.5 * (t / scale) ** 2)
            return g / np.sqrt(np.sum(g * g))

        self.gx = kernel(length, dx)
        self.gy = kernel(length, dy if dy is not None else dx)
        self.gz = kernel(levels, 1.0) if levels > 0 else None

    @staticmethod
    def _filter(a: np.ndarray, g: np.ndarray, axis: int) -> np.ndarray:
        """sum over s of g[s] a[i + s] along `axis`, zero outside the field
        (g is symmetric, so this is also the convolution)"""
        a = np.moveaxis(a, axis, -1)
        out = np.zeros_like(a)
        n, m = len(g) // 2, a.shape[-1]
        for s in range(-n, n + 1):
            if abs(s) >= m:
                continue
            w = g[s + n]
            if s >= 0:
                out[..., :m - s] += w * a[..., s:]
            else:
                out[..., -s:] += w * a[..., :m + s]
        return np.moveaxis(out, -1, axis)

    def apply(self, name: str, f: np.ndarray) -> np.ndarray:
        out = self._filter(np.asarray(f, dtype=np.float64), self.gx, -1)
        if out.ndim >= 2:
            out = self._filter(out, self.gy, -2)
        if self.gz is not None and out.ndim >= 3:
            out = self._filter(out, self.gz, -3)
        return out


@dataclass
class Result:
    x: dict
    cost: list = field(default_factory=list)       # J at the start of each outer loop, then at xa
    inner_residual: list = field(default_factory=list)  # CG residual norms, one list per outer loop


# ---------------------------------------------------------------- 4D-Var
class FourDVar:
    """corr: background-error correlations (an object with a symmetric
    ``apply(name, field)``, e.g. GaussianCorrelation); None for a diagonal B.
    With correlations the control variable is chi, x = xb + B^1/2 chi, and
    J_b = |chi|^2 / 2: the minimisation starts from the background and
    ``gradient_chi`` gives the gradient in chi."""

    def __init__(self, model, xb: dict, sigma_b: dict | float, obs: list, corr=None):
        self.m = model
        self.corr = corr
        self.names = tuple(model.names)
        self.xb = {k: np.asarray(xb[k], dtype=np.float64) for k in self.names}
        sb = sigma_b if isinstance(sigma_b, dict) else {k: float(sigma_b) for k in self.names}
        self.sb = {k: float(sb[k]) for k in self.names}
        if any(v <= 0 for v in self.sb.values()):
            raise ValueError("background standard deviations must be positive")
        self.obs = list(obs)
        for o in self.obs:
            if o.field not in self.names:
                raise ValueError(f"observed field {o.field!r} is not prognostic here")
            if o.step < 0:
                raise ValueError("observation steps count from the start of the window")
            n = self.xb[o.field].size
            if o.index.size and (o.index.min() < 0 or o.index.max() >= n):
                raise ValueError("observation index outside the field")
        # segment boundaries: the window start and every observation time
        self.times = sorted({0} | {o.step for o in self.obs})
        self._mask = {k: np.asarray(model.mask(k), dtype=bool) for k in self.names}

    # ---- control vector <-> fields (prognostic points only)
    def pack(self, x: dict) -> np.ndarray:
        return np.concatenate([np.asarray(x[k]).reshape(-1)[self._mask[k].ravel()]
                               for k in self.names])

    def unpack(self, v: np.ndarray) -> dict:
        out, o = {}, 0
        for k in self.names:
            m = self._mask[k]
            a = np.zeros(m.shape)
            n = int(m.sum())
            a[m] = v[o:o + n]
            out[k] = a
            o += n
        return out

    def _U(self, v: np.ndarray) -> np.ndarray:
        """B^1/2 on a packed control vector (symmetric: also its transpose)"""
        if self.corr is None:
            return self._sb_vec() * v
        f = self.unpack(v)
        return self.pack({k: self.sb[k] * self.corr.apply(k, f[k]) for k in self.names})

    def _sb_vec(self) -> np.ndarray:
        return np.concatenate([np.full(int(self._mask[k].sum()), self.sb[k]) for k in self.names])

    def _zeros(self) -> dict:
        return {k: np.zeros_like(self.xb[k]) for k in self.names}

    # ---- nonlinear pieces
    def trajectory(self, x0: dict) -> dict:
        """states at every segment boundary (step -> fields)"""
        traj = {0: {k: np.asarray(x0[k], dtype=np.float64) for k in self.names}}
        x = traj[0]
        for a, b in zip(self.times[:-1], self.times[1:]):
            x = self.m.forecast(x, b - a)
            traj[b] = x
        return traj

    def _obs_at(self, t: int) -> list:
        return [o for o in self.obs if o.step == t]

    def _jo(self, traj: dict) -> float:
        return 0.5 * sum(float(np.sum(((o.sample(traj[o.step]) - o.value) / o.sigma) ** 2))
                         for o in self.obs)

    def cost(self, x0: dict, traj: dict | None = None) -> float:
        """J(x0) with the diagonal B (no correlations)"""
        if self.corr is not None:
            raise ValueError("with correlations J is a function of chi: use cost_chi")
        traj = traj or self.trajectory(x0)
        jb = sum(float(np.sum(((np.asarray(x0[k]) - self.xb[k])[self._mask[k]] / self.sb[k]) ** 2))
                 for k in self.names)
        return 0.5 * jb + self._jo(traj)

    def state_of(self, chi: np.ndarray) -> dict:
        """x = xb + B^1/2 chi"""
        dx = self.unpack(self._U(chi))
        return {k: self.xb[k] + dx[k] for k in self.names}

    def cost_chi(self, chi: np.ndarray, traj: dict | None = None) -> float:
        traj = traj or self.trajectory(self.state_of(chi))
        return 0.5 * float(chi @ chi) + self._jo(traj)

    def gradient_chi(self, chi: np.ndarray) -> tuple:
        """(J, dJ/dchi) = (J, chi + B^1/2 M^T H^T R^-1 (H x - y))"""
        x = self.state_of(chi)
        traj = self.trajectory(x)
        lam = self._adjoint_sweep(traj, lambda o: (o.sample(traj[o.step]) - o.value) / o.sigma ** 2)
        return self.cost_chi(chi, traj), chi + self._U(self.pack(lam))

    def _adjoint_sweep(self, traj: dict, forcing) -> dict:
        """sum_k M_k^T H_k^T forcing(o) over the observations: forcing(o) is the
        weighted residual of each observation set"""
        lam = self._zeros()
        for ti in range(len(self.times) - 1, -1, -1):
            t = self.times[ti]
            for o in self._obs_at(t):
                o.scatter_into(lam, forcing(o))
            if ti > 0:
                t0 = self.times[ti - 1]
                lam = self.m.adjoint(traj[t0], lam, t - t0)
        return lam

    def gradient(self, x0: dict) -> tuple:
        """(J, dJ/dx0) with dJ/dx0 zero off the control points (diagonal B)"""
        if self.corr is not None:
            raise ValueError("with correlations use gradient_chi")
        traj = self.trajectory(x0)
        lam = self._adjoint_sweep(traj, lambda o: (o.sample(traj[o.step]) - o.value) / o.sigma ** 2)
        g = {k: np.where(self._mask[k], lam[k] + (np.asarray(x0[k]) - self.xb[k]) / self.sb[k] ** 2,
                         0.0) for k in self.names}
        return self.cost(x0, traj), g

    # ---- linearised pieces about a trajectory
    def _tangent_sweep(self, traj: dict, dx0: dict) -> dict:
        """H_k M_k dx0 for every observation set (obs id -> values)"""
        out, dx = {}, dx0
        for ti, t in enumerate(self.times):
            if ti > 0:
                t0 = self.times[ti - 1]
                dx = self.m.tangent(traj[t0], dx, t - t0)
            for o in self._obs_at(t):
                out[id(o)] = o.sample(dx)
        return out

    def minimise(self, x0: dict | None = None, outer: int = 2, inner: int = 10,
                 rtol: float = 1e-3) -> Result:
        """Incremental 4D-Var from x0 (default: the background).  Each inner
        loop stops after `inner` CG iterations or when the residual falls
        below rtol times its initial norm."""
        if self.corr is not None and x0 is not None:
            raise ValueError("with correlations the minimisation starts from the background")
        x = {k: np.asarray((x0 or self.xb)[k], dtype=np.float64).copy() for k in self.names}
        res = Result(x=x)
        sbv = self._sb_vec()
        chi_tot = np.zeros_like(sbv)  # with correlations: x = xb + B^1/2 chi_tot
        for _ in range(outer):
            traj = self.trajectory(x)
            res.cost.append(self.cost_chi(chi_tot, traj) if self.corr is not None
                            else self.cost(x, traj))
            # innovations d_k = y_k - H_k x(t_k); background departure in chi
            d = {id(o): o.value - o.sample(traj[o.step]) for o in self.obs}
            bvec = (chi_tot if self.corr is not None
                    else self.pack({k: x[k] - self.xb[k] for k in self.names}) / sbv)

            def hess(v):
                hm = self._tangent_sweep(traj, self.unpack(self._U(v)))
                lam = self._adjoint_sweep(traj, lambda o: hm[id(o)] / o.sigma ** 2)
                return v + self._U(self.pack(lam))

            # A chi = -b + B^1/2 M^T H^T R^-1 d
            lam = self._adjoint_sweep(traj, lambda o: d[id(o)] / o.sigma ** 2)
            rhs = -bvec + self._U(self.pack(lam))
            chi = np.zeros_like(rhs)
            r = rhs.copy()
            p = r.copy()
            rr = float(r @ r)
            norms = [np.sqrt(rr)]
            r0 = norms[0]
            for _ in range(inner):
                if r0 == 0 or np.sqrt(rr) <= rtol * r0:
                    break
                ap = hess(p)
                alpha = rr / float(p @ ap)
                chi += alpha * p
                r -= alpha * ap
                rr_new = float(r @ r)
                norms.append(np.sqrt(rr_new))
                p = r + (rr_new / rr) * p
                rr = rr_new
            res.inner_residual.append(norms)
            chi_tot = chi_tot + chi
            dx = self.unpack(self._U(chi))
            x = {k: x[k] + dx[k] for k in self.names}
        res.x = x
        res.cost.append(self.cost_chi(chi_tot) if self.corr is not None else self.cost(x))
        return res


# --------------------------------------------------------------- nudging
def nudge(case, xa: dict, tau: float, width: int = 0, bdy_tau: float | None = None) -> np.ndarray:
    """Relax the case's forecast toward the analysis xa: BdyManager targets
    lo = hi = xa for (u, v, theta', pi', qv) (absent fields: 0) and the
    reference's weights, 1/tau everywhere with the cos^2 Davies ramp of
    `width` rows and 1/bdy_tau at the open edges.  Returns the weights.
    ``case.clear_boundary()`` switches the relaxation off again (the tangent-
    linear and adjoint runs refuse a case that relaxes)."""
    if not tau > 0:
        raise ValueError("the nudging time scale must be positive")
    w = case.bdy_weights(width, bdy_tau if bdy_tau is not None else tau, tau)
    tg = [np.ascontiguousarray(xa[k], dtype=np.float64) if k in xa else np.zeros(case.shape)
          for k in BDY_FIELDS]
    case.set_boundary(tg, tg, w, 0.0, 1.0)
    return w
