"""wfe_b200: B200-native (sm_100a) WFE dynamical core and column physics.

Python host layer over the C ABI in include/wfe_b200.h (libwfe_b200.so, built
in-tree by wfe_b200.build).  It mirrors the reference's operator interface:

* ``Case(ini, overrides)`` -- src/main.cpp:248-383 set-up (config, metric,
  base state, initial conditions, boundary manager, surface physics);
* ``Case.step(dt, t)`` / ``Case.run(n, dt, t0)`` -- Integrator::step
  (src/dynamics/integrator.cpp:71-111), the latter from captured CUDA graphs;
* ``state()``, ``field()``, ``set_field()``, ``rain()`` -- Integrator::state,
  Field3D upload/download, Integrator::rain;
* ``apply_bcs``, ``compute_tendencies``, ``acoustic_substeps``,
  ``update_moisture_stage``, ``kessler_step``, ``sfc_step``,
  ``set_boundary``, ``set_physics``, ``field_absmax`` -- the kernel API of
  src/dynamics/kernels.hpp:14-71 and src/physics/*.hpp;
* ``Ensemble(members)`` -- members of different grids stepped together
  (batched launches, or the members' own graphs on concurrent streams);
* ``bdy_weights``, ``clear_boundary`` -- BdyManager's relaxation weights
  (src/dynamics/boundary.cpp:24-39) and switching the relaxation off.

Beside it: ``wfe_b200.adjoint`` (tangent-linear and adjoint runs, the
torch.autograd.Function), ``wfe_b200.analysis`` (4D-Var and analysis
nudging), ``wfe_b200.synth`` (prep-format inputs), ``wfe_b200.shard``
(ensemble members over ranks).

Arrays are numpy, in the reference's padded layout (NZ, NY, NX) with ng = 3,
or the Writer's interior layout.  There is no CPU fallback: without the
library or a CUDA device every GPU call raises WfeError.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

__all__ = ["Case", "Ensemble", "WfeError", "load_library", "FIELDS"]

PKG = Path(__file__).resolve().parent
LIBPATH = PKG / "libwfe_b200.so"
FIELDS = ["u", "v", "w", "thp", "pip", "qv", "qc", "qr"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
ROLES = {"state": 0, "tend": 1, "work": 2, "piprev": 3, "lin": 4}
F2D = {"rain": 0, "tsk": 1, "pblh": 2, "t2m": 3, "u10": 4}
METRIC = ["zeta_w", "zeta_c", "dzeta_c", "dzeta_w", "h", "hx", "hy", "hx_u", "hy_v", "jac",
          "fcor", "mapf"]
BASE = ["thb", "pib", "rhob", "dthbdz", "thbw", "rhobw", "thvb", "thvbw", "qvb", "ub"]
ERRORS = {1: "argument", 2: "cuda", 3: "config", 4: "io", 5: "nan", 6: "w_abort"}

SYMBOLS = [
    "wfe_case_create", "wfe_case_create_text", "wfe_ctx_destroy", "wfe_last_error",
    "wfe_get_dims", "wfe_get_spacing", "wfe_get_flags", "wfe_get_metric", "wfe_get_base",
    "wfe_field_upload", "wfe_field_download", "wfe_field2d_download", "wfe_step", "wfe_run",
    "wfe_sync", "wfe_absmax", "wfe_absmax_begin", "wfe_absmax_end", "wfe_dry_mass", "wfe_launches_per_step", "wfe_case_variants", "wfe_op_apply_bcs",
    "wfe_op_tendencies", "wfe_op_acoustic", "wfe_op_moisture_stage", "wfe_op_kessler",
    "wfe_op_sfc", "wfe_set_boundary", "wfe_bdy_weights", "wfe_clear_boundary", "wfe_set_physics", "wfe_time_run", "wfe_kernel_times",
    "wfe_dry_mass_noalloc", "wfe_ensemble_create", "wfe_ensemble_destroy", "wfe_ensemble_run",
    "wfe_ensemble_step", "wfe_ensemble_sync", "wfe_ensemble_time_run",
    "wfe_ensemble_launches_per_step", "wfe_ensemble_variants", "wfe_lin_enable", "wfe_lin_zero",
    "wfe_tl_run", "wfe_ad_run", "wfe_get_run_config", "wfe_snapshot_begin", "wfe_snapshot_wait",
    "wfe_host_alloc", "wfe_host_free",
]


class WfeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"wfe_b200 error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


_lib = None


def load_library(path: str | Path | None = None):
    """Load libwfe_b200.so (raises if it has not been built).  The environment
    variable WFE_B200_LIB names another build of the library to load."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    env = os.environ.get("WFE_B200_LIB")
    p = Path(path) if path else (Path(env) if env else LIBPATH)
    if not p.exists():
        raise WfeError(2, f"{p} not built; run `python -m wfe_b200.build`")
    lib = C.CDLL(str(p))
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    lib.wfe_case_create.argtypes = [C.c_char_p, C.POINTER(C.c_char_p), C.c_int, C.c_int, C.c_int,
                                    C.POINTER(vp)]
    lib.wfe_case_create_text.argtypes = lib.wfe_case_create.argtypes
    lib.wfe_ctx_destroy.argtypes = [vp]
    lib.wfe_last_error.argtypes = [vp]
    lib.wfe_last_error.restype = C.c_char_p
    lib.wfe_get_dims.argtypes = [vp, ip]
    lib.wfe_get_spacing.argtypes = [vp, dp]
    lib.wfe_get_flags.argtypes = [vp, ip]
    lib.wfe_get_metric.argtypes = [vp, C.c_int, dp]
    lib.wfe_get_base.argtypes = [vp, C.c_int, dp]
    lib.wfe_field_upload.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int, C.c_int]
    lib.wfe_field_download.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int, C.c_int]
    lib.wfe_field2d_download.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int]
    lib.wfe_step.argtypes = [vp, C.c_double, C.c_double]
    lib.wfe_run.argtypes = [vp, C.c_int, C.c_double, C.c_double]
    lib.wfe_sync.argtypes = [vp]
    lib.wfe_absmax.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
    lib.wfe_absmax_begin.argtypes = [vp, C.c_int, C.c_int]
    lib.wfe_absmax_end.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
    lib.wfe_dry_mass.argtypes = [vp, dp]
    lib.wfe_launches_per_step.argtypes = [vp]
    lib.wfe_launches_per_step.restype = C.c_long
    lib.wfe_case_variants.argtypes = [vp, ip]
    lib.wfe_op_apply_bcs.argtypes = [vp]
    lib.wfe_op_tendencies.argtypes = [vp, C.c_double, C.c_double]
    lib.wfe_op_acoustic.argtypes = [vp, C.c_double, C.c_int]
    lib.wfe_op_moisture_stage.argtypes = [vp, C.c_double]
    lib.wfe_op_kessler.argtypes = [vp, C.c_double]
    lib.wfe_op_sfc.argtypes = [vp, C.c_double, C.c_double]
    lib.wfe_set_boundary.argtypes = [vp, C.POINTER(dp), C.POINTER(dp), dp, C.c_double,
                                     C.c_double]
    lib.wfe_set_physics.argtypes = [vp, dp, dp, dp, dp, dp, C.c_double, C.c_int, C.c_int]
    lib.wfe_bdy_weights.argtypes = [vp, C.c_int, C.c_double, C.c_double, dp]
    lib.wfe_clear_boundary.argtypes = [vp]
    lib.wfe_time_run.argtypes = [vp, C.c_int, C.c_double, C.c_double, dp]
    lib.wfe_dry_mass_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double] + \
        [vp] * 11
    lib.wfe_kernel_times.argtypes = [vp, C.c_double, C.c_double, C.c_int, dp, ip, C.c_char_p,
                                     C.c_int, ip]
    lib.wfe_snapshot_begin.argtypes = [vp, C.c_int, ip, C.POINTER(vp), C.c_int]
    lib.wfe_snapshot_wait.argtypes = [vp]
    lib.wfe_host_alloc.argtypes = [C.c_size_t]
    lib.wfe_host_alloc.restype = vp
    lib.wfe_host_free.argtypes = [vp]
    lib.wfe_lin_enable.argtypes = [vp]
    lib.wfe_lin_zero.argtypes = [vp]
    lib.wfe_tl_run.argtypes = [vp, C.c_int, C.c_double, C.c_double]
    lib.wfe_ad_run.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_int]
    lib.wfe_ensemble_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(vp)]
    lib.wfe_ensemble_destroy.argtypes = [vp]
    lib.wfe_ensemble_run.argtypes = [vp, C.c_int, C.c_double, C.c_double]
    lib.wfe_ensemble_step.argtypes = [vp, C.c_double, C.c_double]
    lib.wfe_ensemble_sync.argtypes = [vp]
    lib.wfe_ensemble_time_run.argtypes = [vp, C.c_int, C.c_double, C.c_double, dp]
    lib.wfe_ensemble_launches_per_step.argtypes = [vp]
    lib.wfe_ensemble_launches_per_step.restype = C.c_long
    lib.wfe_ensemble_variants.argtypes = [vp, ip]
    if path is None:
        _lib = lib
    return lib


class _PinnedArray:
    """numpy array over page-locked memory from wfe_host_alloc (freed with it)"""

    def __init__(self, lib, shape, dtype):
        self._lib = lib
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self._p = lib.wfe_host_alloc(max(n, 1))
        if not self._p:
            raise WfeError(2, "wfe_host_alloc failed")
        buf = (C.c_char * max(n, 1)).from_address(self._p)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)
        self.array.flags.writeable = True
        # the array keeps this owner alive
        self._finalizer = __import__("weakref").finalize(self.array, lib.wfe_host_free, self._p)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Case:
    """One WFE case on one GPU (or, with device=-1, its host set-up only)."""

    def __init__(self, ini=None, overrides: dict | None = None, *, text: str | None = None,
                 precision: str = "f32", device: int = 0):
        lib = self._lib = load_library()
        ov = [f"{k}={v}".encode() for k, v in (overrides or {}).items()]
        arr = (C.c_char_p * max(1, len(ov)))(*ov)
        h = C.c_void_p()
        prec = {"f32": 0, "f64": 1}[precision]
        if text is not None:
            rc = lib.wfe_case_create_text(text.encode(), arr, len(ov), prec, device, C.byref(h))
        else:
            rc = lib.wfe_case_create(str(ini).encode(), arr, len(ov), prec, device, C.byref(h))
        if rc != 0:
            raise WfeError(rc, lib.wfe_last_error(None).decode())
        self._h = h
        self.precision = precision
        self.device = device
        d = (C.c_int * 7)()
        lib.wfe_get_dims(h, d)
        self.nx, self.ny, self.nz, self.ng, self.NX, self.NY, self.NZ = list(d)
        sp = (C.c_double * 6)()
        lib.wfe_get_spacing(h, sp)
        self.dx, self.dy, self.dz, self.dt, self.t_end, self.zt = list(sp)
        fl = (C.c_int * 10)()
        lib.wfe_get_flags(h, fl)
        (self.moisture, self.microphysics, self.pd_moist, self.bc_x_open, self.bc_y_open,
         self.w_damping, self.file_mode, self.physics_on, self.boundary_on,
         self.acoustic_ns) = [int(x) for x in fl]
        self.shape = (self.NZ, self.NY, self.NX)
        self.npts = self.NX * self.NY * self.NZ

    # ----------------------------------------------------------- plumbing
    def _check(self, rc: int) -> None:
        if rc != 0:
            raise WfeError(rc, self._lib.wfe_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.wfe_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------- set-up
    def metric(self, name: str) -> np.ndarray:
        i = METRIC.index(name)
        out = np.zeros(self.NZ if i < 4 else self.NX * self.NY)
        self._check(self._lib.wfe_get_metric(self._h, i, _dptr(out)))
        return out

    def base(self, name: str) -> np.ndarray:
        i = BASE.index(name)
        out = np.zeros(self.NZ if name == "ub" else self.npts)
        self._check(self._lib.wfe_get_base(self._h, i, _dptr(out)))
        return out

    # ---------------------------------------------------------- field I/O
    def field(self, name: str, role: str = "state", interior: bool = False,
              dtype=np.float64) -> np.ndarray:
        fid = FIELD_ID[name]
        if interior:
            nzl = self.nz + 1 if name == "w" else self.nz
            out = np.zeros((nzl, self.ny, self.nx), dtype=dtype)
        else:
            out = np.zeros(self.shape, dtype=dtype)
        self._check(self._lib.wfe_field_download(
            self._h, ROLES[role], fid, out.ctypes.data_as(C.c_void_p),
            1 if dtype == np.float32 else 0, 1 if interior else 0))
        return out

    def set_field(self, name: str, a, role: str = "state", interior: bool = False) -> None:
        a = np.ascontiguousarray(a)
        if a.dtype not in (np.float32, np.float64):
            a = a.astype(np.float64)
        self._check(self._lib.wfe_field_upload(
            self._h, ROLES[role], FIELD_ID[name], a.ctypes.data_as(C.c_void_p),
            1 if a.dtype == np.float32 else 0, 1 if interior else 0))

    def state(self, role: str = "state", interior: bool = False) -> dict:
        return {k: self.field(k, role, interior) for k in FIELDS}

    def set_state(self, s: dict, role: str = "state") -> None:
        for k, v in s.items():
            self.set_field(k, np.asarray(v).reshape(-1) if v.ndim == 1 else v, role)

    def field2d(self, name: str, interior: bool = False) -> np.ndarray:
        shape = (self.ny, self.nx) if interior else (self.NY, self.NX)
        out = np.zeros(shape)
        self._check(self._lib.wfe_field2d_download(self._h, F2D[name],
                                                   out.ctypes.data_as(C.c_void_p), 0,
                                                   1 if interior else 0))
        return out

    def rain(self, interior: bool = False) -> np.ndarray:
        return self.field2d("rain", interior)

    # ----------------------------------------------------------- stepping
    def step(self, dt: float | None = None, t: float = 0.0) -> None:
        self._check(self._lib.wfe_step(self._h, self.dt if dt is None else dt, t))

    def run(self, nsteps: int, dt: float | None = None, t0: float = 0.0) -> None:
        self._check(self._lib.wfe_run(self._h, nsteps, self.dt if dt is None else dt, t0))

    def sync(self) -> None:
        self._check(self._lib.wfe_sync(self._h))

    def field_absmax(self, name: str = "w") -> float:
        out = C.c_float()
        self._check(self._lib.wfe_absmax(self._h, FIELD_ID[name], C.byref(out)))
        return float(out.value)

    def absmax_begin(self, name: str = "w", slot: int = 0) -> None:
        """enqueue max |field| into page-locked slot 0 or 1 without waiting"""
        self._check(self._lib.wfe_absmax_begin(self._h, FIELD_ID[name], slot))

    def absmax_end(self, slot: int = 0) -> float:
        """wait for slot `slot` of absmax_begin and return its value"""
        out = C.c_float()
        self._check(self._lib.wfe_absmax_end(self._h, slot, C.byref(out)))
        return float(out.value)

    def dry_mass(self) -> float:
        out = C.c_double()
        self._check(self._lib.wfe_dry_mass(self._h, C.byref(out)))
        return float(out.value)

    def time_run(self, nsteps: int, dt: float | None = None, t0: float = 0.0) -> float:
        """device milliseconds of nsteps graph-replayed steps (CUDA events)"""
        ms = C.c_double()
        self._check(self._lib.wfe_time_run(self._h, nsteps, self.dt if dt is None else dt, t0,
                                           C.byref(ms)))
        return float(ms.value)

    def kernel_times(self, dt: float | None = None, t: float = 0.0) -> dict:
        """one direct step with CUDA events around each launch:
        {kernel: (total_ms, launches)}"""
        cap = 32
        ms = (C.c_double * cap)()
        cnt = (C.c_int * cap)()
        names = C.create_string_buffer(1024)
        n = C.c_int()
        self._check(self._lib.wfe_kernel_times(self._h, self.dt if dt is None else dt, t, cap, ms,
                                               cnt, names, 1024, C.byref(n)))
        keys = names.value.decode().split(",") if n.value else []
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(keys)}

    def launches_per_step(self) -> int:
        return int(self._lib.wfe_launches_per_step(self._h))

    def variants(self) -> dict:
        """The tuned kernel variants (-1 before the first step) and whether the
        column coefficients and the base state are read from per-level tables."""
        out = (C.c_int * 4)()
        self._check(self._lib.wfe_case_variants(self._h, out))
        return {"tendencies": out[0], "column": out[1], "uv": out[2], "level_tables": bool(out[3] & 1),
                "base_tables": bool(out[3] & 2)}

    # ------------------------------------------------------ operator API
    def apply_bcs(self) -> None:
        self._check(self._lib.wfe_op_apply_bcs(self._h))

    def compute_tendencies(self, dt: float, t: float = 0.0) -> None:
        self._check(self._lib.wfe_op_tendencies(self._h, dt, t))

    def acoustic_substeps(self, dtau: float, nsub: int = 1) -> None:
        self._check(self._lib.wfe_op_acoustic(self._h, dtau, nsub))

    def update_moisture_stage(self, dt: float) -> None:
        self._check(self._lib.wfe_op_moisture_stage(self._h, dt))

    def kessler_step(self, dt: float) -> None:
        self._check(self._lib.wfe_op_kessler(self._h, dt))

    def sfc_step(self, dt: float, t: float) -> None:
        self._check(self._lib.wfe_op_sfc(self._h, dt, t))

    def set_boundary(self, lo: list, hi: list, wgt, t_lo: float, t_hi: float) -> None:
        keep = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in list(lo) + list(hi)]
        w = np.ascontiguousarray(wgt, dtype=np.float64).ravel()
        DP = C.POINTER(C.c_double)
        plo = (DP * 5)(*[_dptr(a) for a in keep[:5]])
        phi = (DP * 5)(*[_dptr(a) for a in keep[5:]])
        self._check(self._lib.wfe_set_boundary(self._h, plo, phi, _dptr(w), t_lo, t_hi))

    def bdy_weights(self, width: int, tau: float, nudge_tau: float = 0.0) -> np.ndarray:
        """BdyManager::init's relaxation weights (padded NY x NX): Davies ramp
        of `width` rows with 1/tau at open edges, 1/nudge_tau inside"""
        out = np.zeros(self.NY * self.NX, dtype=np.float64)
        self._check(self._lib.wfe_bdy_weights(self._h, int(width), float(tau), float(nudge_tau),
                                              _dptr(out)))
        return out.reshape(self.NY, self.NX)

    def clear_boundary(self) -> None:
        """switch the relaxation of set_boundary off"""
        self._check(self._lib.wfe_clear_boundary(self._h))

    def set_physics(self, tsk, land, lat, lon, soilw, start_hour: float, doy: int,
                    nonlocal_pbl: bool) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in
                (tsk, land, lat, lon, soilw)]
        self._check(self._lib.wfe_set_physics(self._h, *[_dptr(a) for a in arrs], start_hour,
                                              int(doy), int(nonlocal_pbl)))

    # ------------------------------------------------- async snapshots
    def snapshot_buffers(self, names, dtype=np.float32) -> dict:
        """page-locked host arrays (interior layout) for snapshot_begin"""
        out = {}
        for k in names:
            shape = ((self.ny, self.nx) if k in F2D else
                     ((self.nz + 1 if k == "w" else self.nz), self.ny, self.nx))
            out[k] = _PinnedArray(self._lib, shape, dtype).array
        return out

    def snapshot_begin(self, bufs: dict) -> None:
        """pack the named fields on the device and start their copies into the
        arrays of snapshot_buffers (complete after snapshot_wait)"""
        names = list(bufs)
        ids = (C.c_int * len(names))(*[(100 + F2D[k]) if k in F2D else FIELD_ID[k]
                                       for k in names])
        ptrs = (C.c_void_p * len(names))(*[bufs[k].ctypes.data for k in names])
        dt = 1 if next(iter(bufs.values())).dtype == np.float32 else 0
        self._check(self._lib.wfe_snapshot_begin(self._h, len(names), ids, ptrs, dt))

    def snapshot_wait(self) -> None:
        self._check(self._lib.wfe_snapshot_wait(self._h))

    # ---------------------------------------- tangent-linear / adjoint
    def lin_enable(self) -> None:
        """Linearised fields (role "lin") for the tangent-linear and adjoint runs."""
        self._check(self._lib.wfe_lin_enable(self._h))

    def lin_zero(self) -> None:
        self._check(self._lib.wfe_lin_zero(self._h))

    def tl_run(self, nsteps: int, dt: float | None = None, t0: float = 0.0) -> None:
        """state x0 -> xN and lin field dx0 -> M dx0"""
        self._check(self._lib.wfe_tl_run(self._h, nsteps, self.dt if dt is None else dt, t0))

    def ad_run(self, nsteps: int, dt: float | None = None, t0: float = 0.0,
               checkpoint_every: int = 30) -> None:
        """state x0 -> xN; lin field dJ/dxN -> M^T dJ/dxN = dJ/dx0"""
        self._check(self._lib.wfe_ad_run(self._h, nsteps, self.dt if dt is None else dt, t0,
                                         checkpoint_every))

    # -------------------------------------------------------------- index
    def interior(self, a, name: str = "c") -> np.ndarray:
        a3 = np.asarray(a).reshape(self.shape)
        g = self.ng
        nzl = self.nz + 1 if name == "w" else self.nz
        return a3[g:g + nzl, g:g + self.ny, g:g + self.nx]


class Ensemble:
    """Members (Case objects on one device, one precision, same physics
    switches and substep count) advanced together by batched launches: each
    kernel of the step runs once over a member x tile work list, and the step
    is replayed from one CUDA graph per rotation phase.  Replaces the
    reference's one-process-per-member loop (tools/run_ensemble.py:61-64).
    The members stay usable (field(), rain(), dry_mass(), ...) and must stay
    open while the ensemble is."""

    def __init__(self, members: list):
        self._lib = load_library()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m._h for m in self.members])
        h = C.c_void_p()
        rc = self._lib.wfe_ensemble_create(arr, len(self.members), C.byref(h))
        if rc != 0:
            raise WfeError(rc, self._lib.wfe_last_error(None).decode())
        self._h = h

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise WfeError(rc, self._lib.wfe_last_error(None).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.wfe_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def cells(self) -> int:
        return sum(m.nx * m.ny * m.nz for m in self.members)

    def run(self, nsteps: int, dt: float, t0: float = 0.0) -> None:
        self._check(self._lib.wfe_ensemble_run(self._h, nsteps, dt, t0))

    def step(self, dt: float, t: float = 0.0) -> None:
        self._check(self._lib.wfe_ensemble_step(self._h, dt, t))

    def sync(self) -> None:
        self._check(self._lib.wfe_ensemble_sync(self._h))

    def time_run(self, nsteps: int, dt: float, t0: float = 0.0) -> float:
        """device milliseconds of nsteps graph-replayed ensemble steps"""
        ms = C.c_double()
        self._check(self._lib.wfe_ensemble_time_run(self._h, nsteps, dt, t0, C.byref(ms)))
        return float(ms.value)

    def launches_per_step(self) -> int:
        return int(self._lib.wfe_ensemble_launches_per_step(self._h))

    def variants(self) -> dict:
        out = (C.c_int * 3)()
        self._check(self._lib.wfe_ensemble_variants(self._h, out))
        return {"tendencies": out[0], "column_shape": out[1], "persistent": out[2] == 1,
                "mode": {2: "members", 3: "sequential"}.get(out[2], "batched")}
