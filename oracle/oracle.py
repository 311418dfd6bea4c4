"""Python binding of the CPU FP64 oracle -- TEST INFRASTRUCTURE ONLY.

Loads oracle/_build/liboracle.so (built by `make -C oracle oracle`) and exposes
the reference's set-up (src/main.cpp:261-383 for the idealised and file-mode
cases), its operator API (src/dynamics/kernels.hpp, physics/*.hpp) and its
Integrator::step (src/dynamics/integrator.cpp:71-111) on numpy arrays in the
reference's padded layout.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this module; the product never does.
"""

from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBPATH = HERE / "_build" / "liboracle.so"

_dp = C.POINTER(C.c_double)


def build() -> Path:
    if not LIBPATH.exists() or LIBPATH.stat().st_mtime < (HERE / "wfe_oracle.cpp").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    return LIBPATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(build()))
        _lib.orc_npts.restype = C.c_size_t
        _lib.orc_absmax.restype = C.c_float
        _lib.orc_dry_mass.restype = C.c_double
        _lib.orc_base_build.restype = C.c_int
        _lib.orc_integ_create.restype = C.c_void_p
        _lib.orc_integ_state.restype = C.c_void_p
        _lib.orc_integ_state.argtypes = [C.c_void_p]
        _lib.orc_integ_rain.restype = _dp
        _lib.orc_integ_rain.argtypes = [C.c_void_p]
        _lib.orc_integ_step.argtypes = [C.c_void_p, C.c_double, C.c_double]
        _lib.orc_integ_free.argtypes = [C.c_void_p]
        _lib.orc_integ_set_sfc.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_integ_set_bdy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _dp, C.c_double,
                                           C.c_double]
    return _lib


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("ng", C.c_int),
                ("NX", C.c_int), ("NY", C.c_int), ("NZ", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double)]


class Params(C.Structure):
    _fields_ = [("diff_K", C.c_double), ("coriolis_f", C.c_double), ("coriolis_use_ub", C.c_int),
                ("rayleigh_zd", C.c_double), ("rayleigh_alpha", C.c_double),
                ("acoustic_ns", C.c_int), ("acoustic_beta", C.c_double),
                ("acoustic_smdiv", C.c_double), ("bc_x_open", C.c_int), ("bc_y_open", C.c_int),
                ("cstar", C.c_double), ("moisture", C.c_int), ("microphysics", C.c_int),
                ("pd_moist", C.c_int), ("w_damping", C.c_int), ("w_abort", C.c_double)]


METRIC_1D = ["zeta_w", "zeta_c", "dzeta_c", "dzeta_w"]
METRIC_2D = ["h", "hx", "hy", "hx_u", "hy_v", "jac", "fcor", "mapf"]
BASE_3D = ["thb", "pib", "rhob", "dthbdz", "thbw", "rhobw", "thvb", "thvbw", "qvb"]
FIELDS = ["u", "v", "w", "thp", "pip", "qv", "qc", "qr"]


class Metric(C.Structure):
    _fields_ = [(n, _dp) for n in METRIC_1D + METRIC_2D] + [("zt", C.c_double)]


class Base(C.Structure):
    _fields_ = [(n, _dp) for n in BASE_3D] + [("ub", _dp)]


class State(C.Structure):
    _fields_ = [(n, _dp) for n in FIELDS]


class MetricCfg(C.Structure):
    _fields_ = [("stretch", C.c_int), ("dz0", C.c_double), ("dz_ratio", C.c_double),
                ("dz_max", C.c_double), ("terrain", C.c_int), ("h0", C.c_double),
                ("a", C.c_double), ("lam", C.c_double), ("xc", C.c_double), ("yc", C.c_double),
                ("ya", C.c_double), ("coriolis_f", C.c_double), ("h_file", _dp),
                ("fcor_file", _dp), ("mapf_file", _dp)]


class BaseCfg(C.Structure):
    _fields_ = [("profile", C.c_int), ("theta0", C.c_double), ("bv_N", C.c_double),
                ("wind_profile", C.c_int), ("wind_u", C.c_double), ("wind_us", C.c_double),
                ("wind_zs", C.c_double), ("wind_offset", C.c_double), ("np_prof", C.c_int),
                ("prof_z", _dp), ("prof_th", _dp), ("prof_qv", _dp), ("prof_u", _dp)]


class Sfc(C.Structure):
    _fields_ = [(n, _dp) for n in ["km", "tsk", "tdeep", "land", "lat", "lon", "soilw", "cdv",
                                   "pblh", "t2m", "u10", "soilt"]] + \
               [("start_hour", C.c_double), ("doy", C.c_int), ("nonlocal", C.c_int)]


def ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


# ------------------------------------------------------------------- config
def read_ini(path) -> dict:
    """Config::load (src/core/config.cpp:17-31): key = value, '#'/';' comments."""
    kv = {}
    for line in Path(path).read_text(encoding="utf-8-sig").splitlines():
        m = re.search(r"[#;]", line)
        if m:
            line = line[: m.start()]
        if "=" not in line:
            continue
        k, v = line.split("=", 1)
        k, v = k.strip(), v.strip()
        if k:
            kv[k] = v
    return kv


def _atof(s: str) -> float:
    m = re.match(r"\s*[-+]?(\d+\.?\d*|\.\d+)([eE][-+]?\d+)?", s)
    return float(m.group(0)) if m else 0.0


class Cfg:
    def __init__(self, kv: dict):
        self.kv = dict(kv)

    def real(self, k, d):
        return _atof(self.kv[k]) if k in self.kv else float(d)

    def int(self, k, d):
        if k not in self.kv:
            return int(d)
        m = re.match(r"\s*[-+]?\d+", self.kv[k])
        return int(m.group(0)) if m else 0

    def str(self, k, d):
        return self.kv.get(k, d)


# --------------------------------------------------------------------- case
class Case:
    """Reference set-up of one idealised (or file-mode) case, src/main.cpp:261-383."""

    def __init__(self, ini=None, overrides: dict | None = None, kv: dict | None = None,
                 inputs: dict | None = None):
        kv = dict(kv or {})
        if ini is not None:
            kv.update(read_ini(ini))
        kv.update({k: str(v) for k, v in (overrides or {}).items()})
        c = self.cfg = Cfg(kv)
        L = lib()
        self.nx, self.ny, self.nz = c.int("nx", 100), c.int("ny", 100), c.int("nz", 50)
        self.dx, self.dy, self.dz = c.real("dx", 200), c.real("dy", 200), c.real("dz", 200)
        self.dt = c.real("dt", 0.25)
        self.t_end = c.real("t_end", 1000)
        g = self.grid = Grid()
        L.orc_grid_make(C.byref(g), self.nx, self.ny, self.nz, C.c_double(self.dx),
                        C.c_double(self.dy), C.c_double(self.dz))
        self.shape = (g.NZ, g.NY, g.NX)
        self.n = g.NX * g.NY * g.NZ
        self.file_mode = c.str("profile", "isentropic") == "file"
        self.inputs = inputs

        p = self.params = Params()
        p.diff_K = c.real("diff_K", 0)
        p.coriolis_f = c.real("coriolis_f", 0)
        p.coriolis_use_ub = 0 if self.file_mode else 1
        p.rayleigh_zd = c.real("rayleigh_zd", -1)
        p.rayleigh_alpha = c.real("rayleigh_alpha", 0)
        p.acoustic_ns = c.int("acoustic_ns", 6)
        p.acoustic_beta = c.real("acoustic_beta", 0.2)
        p.acoustic_smdiv = c.real("acoustic_smdiv", 0.1)
        p.bc_x_open = int(c.str("bc_x", "periodic") == "open")
        p.bc_y_open = int(c.str("bc_y", "periodic") == "open")
        p.cstar = c.real("cstar", 30)
        p.w_damping = int(c.str("w_damping", "off") == "on")
        p.w_abort = c.real("w_abort", 150)
        p.pd_moist = int(c.str("pd_moist", "off") == "on")
        p.microphysics = int(c.str("microphysics", "on") == "on")

        # metric (src/core/metric.cpp)
        mc = self.metric_cfg = MetricCfg()
        mc.stretch = int(c.str("stretch", "none") == "geometric")
        mc.dz0 = c.real("dz0", self.dz)
        mc.dz_ratio = c.real("dz_ratio", 1.05)
        mc.dz_max = c.real("dz_max", self.dz * 4)
        mc.terrain = {"none": 0, "schaer": 1, "gauss": 2, "file": 3}.get(c.str("terrain", "none"), 0)
        mc.h0 = c.real("mtn_h0", 250)
        mc.a = c.real("mtn_a", 5000)
        mc.lam = c.real("mtn_lambda", 4000)
        mc.xc = c.real("mtn_xc", self.nx * self.dx / 2)
        mc.yc = c.real("mtn_yc", self.ny * self.dy / 2)
        mc.ya = c.real("mtn_ya", mc.a)
        mc.coriolis_f = c.real("coriolis_f", 0)
        self._keep = []
        if self.file_mode:
            for key, attr in (("h", "h_file"), ("fcor", "fcor_file"), ("mapf", "mapf_file")):
                a = np.ascontiguousarray(inputs[key], dtype=np.float64)
                self._keep.append(a)
                setattr(mc, attr, ptr(a))
        self.metric = {}
        m = self.metric_s = Metric()
        for name in METRIC_1D:
            self.metric[name] = np.zeros(g.NZ)
            setattr(m, name, ptr(self.metric[name]))
        for name in METRIC_2D:
            self.metric[name] = np.zeros(g.NX * g.NY)
            setattr(m, name, ptr(self.metric[name]))
        L.orc_metric_build(C.byref(g), C.byref(mc), C.byref(m))
        self.zt = m.zt

        # base state (src/core/base_state.cpp)
        bc = self.base_cfg = BaseCfg()
        bc.profile = {"isentropic": 0, "constant_N": 1, "wk82": 2, "file": 3}[
            c.str("profile", "isentropic")]
        bc.theta0 = c.real("theta0", 300)
        bc.bv_N = c.real("bv_N", 0.01)
        bc.wind_profile = {"tanh": 1, "linear": 2}.get(c.str("wind_profile", "const"), 0)
        bc.wind_u = c.real("wind_u", 0)
        bc.wind_us = c.real("wind_us", 25)
        bc.wind_zs = c.real("wind_zs", 3000)
        bc.wind_offset = c.real("wind_offset", 0)
        if self.file_mode:
            tabs = [np.ascontiguousarray(inputs[k], dtype=np.float64)
                    for k in ("prof_z", "prof_th", "prof_qv", "prof_u")]
            self._keep += tabs
            bc.np_prof = len(tabs[0])
            bc.prof_z, bc.prof_th, bc.prof_qv, bc.prof_u = [ptr(a) for a in tabs]
        self.base = {}
        b = self.base_s = Base()
        for name in BASE_3D:
            self.base[name] = np.zeros(self.n)
            setattr(b, name, ptr(self.base[name]))
        self.base["ub"] = np.zeros(g.NZ)
        b.ub = ptr(self.base["ub"])
        self.has_moisture = bool(L.orc_base_build(C.byref(g), C.byref(bc), C.byref(m), C.byref(b)))
        qv_blob = c.real("qvbub_dq", 0) != 0
        p.moisture = int(self.has_moisture or qv_blob)
        if not p.moisture:
            p.pd_moist = 0

    # ---------------------------------------------------------- helpers
    def zeros(self):
        return np.zeros(self.n)

    def state_struct(self, fields: dict) -> State:
        s = State()
        for k in FIELDS:
            setattr(s, k, ptr(fields[k]))
        return s

    def new_state(self) -> dict:
        return {k: self.zeros() for k in FIELDS}

    def initial_state(self) -> dict:
        """Idealised ICs in main.cpp order: bubble, wind, moisture, qv blob."""
        c, L, g = self.cfg, lib(), self.grid
        s = self.new_state()
        f = C.c_double
        dth = c.real("bubble_dtheta", 0)
        L.orc_ic_bubble(C.byref(g), C.byref(self.metric_s), f(dth),
                        f(c.real("bubble_xc", self.nx * self.dx / 2)),
                        f(c.real("bubble_yc", self.ny * self.dy / 2)),
                        f(c.real("bubble_zc", 2000)), f(c.real("bubble_xr", 2000)),
                        f(c.real("bubble_yr", 2000)), f(c.real("bubble_zr", 2000)), ptr(s["thp"]))
        L.orc_ic_wind(C.byref(g), C.byref(self.base_s), ptr(s["u"]))
        if self.has_moisture:
            L.orc_ic_moisture(C.byref(g), C.byref(self.base_s), ptr(s["qv"]))
        dq = c.real("qvbub_dq", 0)
        L.orc_ic_bubble(C.byref(g), C.byref(self.metric_s), f(dq),
                        f(c.real("qvbub_xc", self.nx * self.dx / 4)),
                        f(c.real("qvbub_yc", self.ny * self.dy / 2)),
                        f(c.real("qvbub_zc", 2000)), f(c.real("qvbub_xr", 2000)),
                        f(c.real("qvbub_yr", 1e9)), f(c.real("qvbub_zr", 2000)), ptr(s["qv"]))
        return s

    # -------------------------------------------------------- operators
    def apply_bcs(self, s: dict) -> None:
        st = self.state_struct(s)
        lib().orc_apply_bcs(C.byref(self.grid), C.byref(self.params), C.byref(st))

    def mass_fluxes(self, s: dict):
        mfx, mfy, mfz, div = (self.zeros() for _ in range(4))
        st = self.state_struct(s)
        L = lib()
        L.orc_mass_fluxes(C.byref(self.grid), C.byref(self.base_s), C.byref(self.metric_s),
                          C.byref(st), ptr(mfx), ptr(mfy), ptr(mfz))
        L.orc_divergence(C.byref(self.grid), C.byref(self.metric_s), ptr(mfx), ptr(mfy),
                         ptr(mfz), ptr(div))
        return mfx, mfy, mfz, div

    def tendencies(self, s: dict, dt: float, tend: dict | None = None):
        mfx, mfy, mfz, div = self.mass_fluxes(s)
        tend = tend if tend is not None else self.new_state()
        pd = None
        if self.params.pd_moist:
            self._pd = [self.zeros() for _ in range(4)]
            pd = (_dp * 4)(*[ptr(a) for a in self._pd])
        st, tt = self.state_struct(s), self.state_struct(tend)
        lib().orc_tendencies(C.byref(self.grid), C.byref(self.base_s), C.byref(self.metric_s),
                             C.byref(self.params), C.c_double(dt), C.byref(st), ptr(mfx),
                             ptr(mfy), ptr(mfz), ptr(div), C.byref(tt), pd)
        return tend, (mfx, mfy, mfz, div)

    def bdy_relax(self, s: dict, lo: list, hi: list, tf: float, wgt, tend: dict) -> None:
        plo = (_dp * 5)(*[ptr(a) for a in lo])
        phi = (_dp * 5)(*[ptr(a) for a in hi])
        st, tt = self.state_struct(s), self.state_struct(tend)
        lib().orc_bdy_relax(C.byref(self.grid), C.byref(st), plo, phi, C.c_double(tf), ptr(wgt),
                            C.byref(tt))

    def acoustic_coef(self):
        out = [self.zeros() for _ in range(4)]
        lib().orc_acoustic_coef(C.byref(self.grid), C.byref(self.base_s), C.byref(self.metric_s),
                                *[ptr(a) for a in out])
        return out

    def acoustic_substep(self, s: dict, tend: dict, piprev, dtau: float, coef=None) -> None:
        coef = coef if coef is not None else self.acoustic_coef()
        st, tt = self.state_struct(s), self.state_struct(tend)
        lib().orc_acoustic_substep(C.byref(self.grid), C.byref(self.base_s),
                                   C.byref(self.metric_s), C.byref(self.params), C.c_double(dtau),
                                   C.byref(st), C.byref(tt), ptr(piprev), *[ptr(a) for a in coef])

    def moisture_stage(self, s0: dict, tend: dict, dt: float, out: dict) -> None:
        a, b, c = (self.state_struct(x) for x in (s0, tend, out))
        lib().orc_moisture_stage(C.byref(self.grid), C.byref(a), C.byref(b), C.c_double(dt),
                                 C.byref(c))

    def kessler(self, s: dict, dt: float, rain) -> None:
        st = self.state_struct(s)
        lib().orc_kessler(C.byref(self.grid), C.byref(self.base_s), C.byref(self.metric_s),
                          C.c_double(dt), C.byref(st), ptr(rain))

    def dry_mass(self, s: dict) -> float:
        st = self.state_struct(s)
        return lib().orc_dry_mass(C.byref(self.grid), C.byref(self.base_s),
                                  C.byref(self.metric_s), C.byref(st))

    def bdy_weights(self, width: int, tau: float, nudge_tau: float):
        w = np.zeros(self.grid.NX * self.grid.NY)
        lib().orc_bdy_weights(C.byref(self.grid), C.byref(self.params), width, C.c_double(tau),
                              C.c_double(nudge_tau), ptr(w))
        return w

    def sfc(self, tsk, land, lat, lon, soilw, hour: float, doy: int, nonlocal_pbl: bool):
        return SfcPBL(self, tsk, land, lat, lon, soilw, hour, doy, nonlocal_pbl)

    def integrator(self) -> "Integrator":
        return Integrator(self)

    # ----------------------------------------------------------- index
    def idx(self, i, j, k):
        g = self.grid
        return ((k + g.ng) * g.NY + (j + g.ng)) * g.NX + (i + g.ng)

    def interior(self, a, field: str = "c"):
        """(nz[+1], ny, nx) interior view as the reference Writer stores it."""
        g = self.grid
        a3 = np.asarray(a).reshape(self.shape)
        nzl = g.nz + 1 if field == "w" else g.nz
        return a3[g.ng:g.ng + nzl, g.ng:g.ng + g.ny, g.ng:g.ng + g.nx]


class SfcPBL:
    def __init__(self, case: Case, tsk, land, lat, lon, soilw, hour, doy, nonlocal_pbl):
        self.case = case
        self.s = Sfc()
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (tsk, land, lat, lon, soilw)]
        lib().orc_sfc_init(C.byref(case.grid), C.byref(self.s), *[ptr(a) for a in arrs],
                           C.c_double(hour), int(doy), int(nonlocal_pbl))

    def step(self, s: dict, dt: float, t: float) -> None:
        st = self.case.state_struct(s)
        c = self.case
        lib().orc_sfc_step(C.byref(c.grid), C.byref(c.base_s), C.byref(c.metric_s),
                           C.byref(self.s), C.c_double(dt), C.c_double(t), C.byref(st))

    def field(self, name: str):
        n = self.case.grid.NX * self.case.grid.NY
        cnt = {"km": self.case.n, "soilt": 4 * n}.get(name, n)
        return np.ctypeslib.as_array(getattr(self.s, name), shape=(cnt,)).copy()

    def __del__(self):
        try:
            lib().orc_sfc_free(C.byref(self.s))
        except Exception:
            pass


class Integrator:
    """Integrator::init/step (src/dynamics/integrator.cpp:43-111) on the CPU."""

    def __init__(self, case: Case):
        self.case = case
        L = lib()
        self.h = L.orc_integ_create(C.byref(case.grid), C.byref(case.base_s),
                                    C.byref(case.metric_s), C.byref(case.params))
        self._bdy = None
        self._sfc = None

    def _state_ptrs(self) -> State:
        return State.from_address(lib().orc_integ_state(self.h))

    def field(self, name: str) -> np.ndarray:
        """Live view of the current state's field (re-fetch after each step)."""
        return np.ctypeslib.as_array(getattr(self._state_ptrs(), name), shape=(self.case.n,))

    def state(self) -> dict:
        return {k: self.field(k).copy() for k in FIELDS}

    def set_state(self, s: dict) -> None:
        for k in FIELDS:
            if k in s:
                self.field(k)[:] = s[k]

    def rain(self) -> np.ndarray:
        g = self.case.grid
        return np.ctypeslib.as_array(lib().orc_integ_rain(self.h), shape=(g.NX * g.NY,)).copy()

    def set_boundary(self, lo: list, hi: list, wgt, t_lo: float, t_hi: float) -> None:
        self._bdy = ([np.ascontiguousarray(a) for a in lo], [np.ascontiguousarray(a) for a in hi],
                     np.ascontiguousarray(wgt))
        plo = (_dp * 5)(*[ptr(a) for a in self._bdy[0]])
        phi = (_dp * 5)(*[ptr(a) for a in self._bdy[1]])
        self._bdy_ptrs = (plo, phi)
        lib().orc_integ_set_bdy(self.h, C.cast(plo, C.c_void_p), C.cast(phi, C.c_void_p),
                                ptr(self._bdy[2]), t_lo, t_hi)

    def set_physics(self, sfc: SfcPBL) -> None:
        self._sfc = sfc
        lib().orc_integ_set_sfc(self.h, C.cast(C.pointer(sfc.s), C.c_void_p))

    def step(self, dt: float, t: float) -> None:
        lib().orc_integ_step(self.h, dt, t)

    def __del__(self):
        try:
            lib().orc_integ_free(self.h)
        except Exception:
            pass


def threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


# ------------------------------------------------------------- file mode
def load_prep(d, nx: int, ny: int, nz: int) -> dict:
    """wfe_input.ini + wfe_init.bin of a prep directory (src/io/input.cpp:19-57)."""
    d = Path(d)
    meta = read_ini(d / "wfe_input.ini")
    assert (int(meta["nx"]), int(meta["ny"]), int(meta["nz"])) == (nx, ny, nz), "grid mismatch"
    assert int(meta.get("version", 1)) >= 3, "input version < 3"
    npf = int(meta.get("np_prof", 0))
    n2, n3 = nx * ny, nx * ny * nz
    raw = np.fromfile(d / "wfe_init.bin", dtype=np.float32).astype(np.float64)
    out, o = {}, 0
    for k, n in (("prof_z", npf), ("prof_th", npf), ("prof_qv", npf), ("prof_u", npf),
                 ("h", n2), ("fcor", n2), ("tsk", n2), ("land", n2), ("lat", n2),
                 ("lon", n2), ("soilw", n2), ("u", n3), ("v", n3), ("th", n3), ("pi", n3),
                 ("qv", n3)):
        out[k] = raw[o:o + n].copy()
        o += n
    assert o == raw.size, "wfe_init.bin is short or corrupt"
    out["dir"] = d
    out["start"] = meta.get("start", "")
    out["bdy_interval"] = _atof(meta.get("bdy_interval", "10800"))
    out["n_bdy"] = int(meta.get("n_bdy", 0))
    return out


def load_bdy(inputs: dict, nx: int, ny: int, nz: int, idx: int) -> list:
    """wfe_bdy_FFF.bin, FFF = idx * bdy_interval / 3600 (src/io/input.cpp:59-73)."""
    fh = int(idx * inputs["bdy_interval"] / 3600)
    raw = np.fromfile(Path(inputs["dir"]) / f"wfe_bdy_{fh:03d}.bin", dtype=np.float32)
    n3 = nx * ny * nz
    assert raw.size == 5 * n3, "boundary file is short or corrupt"
    return [raw[v * n3:(v + 1) * n3].astype(np.float64).reshape(nz, ny, nx) for v in range(5)]


class FileRun:
    """A file-mode case set up and stepped as src/main.cpp:313-383 does: Lambert
    map factor, base state from the profile tables, initial state from
    wfe_init.bin (+ ic_perturb), Davies targets from the boundary files
    (BdyManager, src/dynamics/boundary.cpp:9-97) and the surface scheme."""

    def __init__(self, ini, overrides: dict | None = None):
        kv = read_ini(ini)
        kv.update({k: str(v) for k, v in (overrides or {}).items()})
        c = Cfg(kv)
        nx, ny, nz = c.int("nx", 100), c.int("ny", 100), c.int("nz", 50)
        inp = load_prep(c.str("input_dir", ""), nx, ny, nz)
        mapf = np.zeros(nx * ny)
        lib().orc_lambert_mapf(nx * ny, ptr(np.ascontiguousarray(inp["lat"])),
                               C.c_double(c.real("proj_lat1", 35)),
                               C.c_double(c.real("proj_lat2", 43)), ptr(mapf))
        inp["mapf"] = mapf
        self.inputs = inp
        self.case = cs = Case(kv=kv, inputs=inp)
        g = cs.grid
        s = cs.new_state()
        st = cs.state_struct(s)
        arrs = [np.ascontiguousarray(inp[k]) for k in ("u", "v", "th", "pi", "qv")]
        lib().orc_ic_from_input(C.byref(g), C.byref(cs.base_s), *[ptr(a) for a in arrs],
                                C.byref(st))
        lib().orc_ic_perturb(C.byref(g), C.c_double(c.real("ic_perturb", 0)),
                             C.c_uint(c.int("ens_seed", 0)), ptr(s["thp"]))
        self.s0 = {k: v.copy() for k, v in s.items()}
        self.it = cs.integrator()
        self.it.set_state(s)
        self.wgt = cs.bdy_weights(c.int("bdy_width", 8), c.real("bdy_tau", 600),
                                  c.real("nudge_tau", 0))
        self.idx_hi = 1
        self.lo = self.targets(0)
        self.hi = self.targets(min(1, inp["n_bdy"] - 1))
        self.t_lo, self.t_hi = 0.0, inp["bdy_interval"]
        self.it.set_boundary(self.lo, self.hi, self.wgt, self.t_lo, self.t_hi)
        self.sfc = None
        if c.str("physics", "none") == "simple":
            st_ = inp["start"]
            mo, dd, hh = int(st_[4:6]), int(st_[6:8]), int(st_[8:10])
            cum = [0, 31, 59, 90, 120, 151, 181, 212, 243, 273, 304, 334]
            self.sfc = cs.sfc(inp["tsk"], inp["land"], inp["lat"], inp["lon"], inp["soilw"],
                              float(hh), cum[mo - 1] + dd, c.str("pbl", "local") == "nonlocal")
            self.it.set_physics(self.sfc)

    def targets(self, idx: int) -> list:
        """Padded perturbation targets of boundary file idx (boundary.cpp:51-81)."""
        cs, g = self.case, self.case.grid
        nx, ny, nz = g.nx, g.ny, g.nz
        f = load_bdy(self.inputs, nx, ny, nz, idx)
        out = [cs.zeros() for _ in range(5)]
        v3 = [cs.interior(a) for a in out]  # views (nz, ny, nx) into the padded arrays
        a3 = [np.asarray(a).reshape(cs.shape) for a in out]
        il = np.r_[0, np.arange(nx)]          # u faces 0..nx: centres (i-1, i) clamped
        ir = np.r_[np.arange(nx), nx - 1]
        a3[0][g.ng:g.ng + nz, g.ng:g.ng + ny, g.ng:g.ng + nx + 1] = 0.5 * (f[0][:, :, il] +
                                                                             f[0][:, :, ir])
        jl = np.r_[0, np.arange(ny - 1)]
        v3[1][:] = 0.5 * (f[1][:, jl, :] + f[1])
        v3[2][:] = f[2] - cs.interior(cs.base["thb"])
        v3[3][:] = f[3] - cs.interior(cs.base["pib"])
        v3[4][:] = f[4]
        return out

    def update(self, t: float) -> None:
        """BdyManager::update (boundary.cpp:83-89)."""
        n_bdy = self.inputs["n_bdy"]
        changed = False
        while t >= self.t_hi and self.idx_hi + 1 < n_bdy:
            self.lo = self.hi
            self.idx_hi += 1
            self.hi = self.targets(self.idx_hi)
            self.t_lo = self.t_hi
            self.t_hi += self.inputs["bdy_interval"]
            changed = True
        if changed:
            self.it.set_boundary(self.lo, self.hi, self.wgt, self.t_lo, self.t_hi)

    def step(self, dt: float, t: float) -> None:
        self.update(t)
        self.it.step(dt, t)
