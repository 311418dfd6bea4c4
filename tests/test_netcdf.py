"""NetCDF export of Writer output (wfe_b200.netcdf, the reference's
tools/to_netcdf.py) -- CPU.  A synthetic Writer directory (meta.json, zc.bin,
float32 snapshots in the reference's layout) is exported and read back with
an independent NetCDF reader (scipy.io.netcdf_file, test-only): every value,
dimension, coordinate and attribute must round-trip exactly."""

import json

import numpy as np
import pytest

from wfe_b200 import netcdf


def _writer_dir(d, nx=7, ny=5, nz=4, steps=(0, 10, 20), moist=True):
    d.mkdir()
    vars_ = {"u": nz, "v": nz, "w": nz + 1, "thp": nz, "pip": nz}
    if moist:
        vars_.update({"qv": nz, "qc": nz, "qr": nz, "rain": 1})
    (d / "meta.json").write_text(json.dumps({"nx": nx, "ny": ny, "nz": nz, "dx": 250.0,
                                             "dy": 300.0, "dz": 100.0, "dt": 1.5,
                                             "vars": vars_}))
    rng = np.random.default_rng(4)
    zc = rng.random((nz, ny, nx)).astype(np.float32) * 1e4
    zc.tofile(d / "zc.bin")
    data = {}
    for s in steps:
        for v, lev in vars_.items():
            a = rng.standard_normal(lev * ny * nx).astype(np.float32)
            a.tofile(d / f"{v}_{s:06d}.bin")
            data[(v, s)] = a.reshape((lev, ny, nx) if lev > 1 else (ny, nx))
    return vars_, zc, data


def test_export_round_trips(tmp_path):
    scipy_io = pytest.importorskip("scipy.io")
    steps = (0, 10, 20)
    vars_, zc, data = _writer_dir(tmp_path / "out", steps=steps)
    ini = tmp_path / "case.ini"
    ini.write_text(f"nx = 7\nout_dir = {tmp_path / 'out'}  # trailing comment\n")
    netcdf.main([str(ini), "-o", str(tmp_path / "x.nc")])
    with scipy_io.netcdf_file(tmp_path / "x.nc", "r", mmap=False) as f:
        assert f.version_byte == 2
        assert f.dimensions["time"] == 3 and f.dimensions["zw"] == 5
        assert np.array_equal(f.variables["time"][:], np.array(steps) * 1.5)
        assert np.allclose(f.variables["x"][:], (np.arange(7) + 0.5) * 250.0, rtol=0, atol=0)
        assert np.array_equal(f.variables["y"][:], (np.arange(5) + 0.5) * 300.0)
        assert np.array_equal(f.variables["zc"][:], zc)
        for v, lev in vars_.items():
            var = f.variables[v]
            want = ("time", "zw", "y", "x") if lev == 5 else (
                ("time", "z", "y", "x") if lev == 4 else ("time", "y", "x"))
            assert var.dimensions == want, v
            for q, s in enumerate(steps):
                assert np.array_equal(var[q], data[(v, s)]), (v, s)
            assert var.units.decode() == netcdf.UNITS.get(v, "")
        assert f.title == b"WFE regional forecast"
        assert f.dt_s == 1.5 and f.dx_m == 250.0


def test_dry_case_without_heights(tmp_path):
    scipy_io = pytest.importorskip("scipy.io")
    _writer_dir(tmp_path / "out", moist=False, steps=(0,))
    (tmp_path / "out" / "zc.bin").unlink()
    p = netcdf.export(tmp_path / "out")
    with scipy_io.netcdf_file(p, "r", mmap=False) as f:
        assert "zc" not in f.variables and "qv" not in f.variables
        assert f.variables["w"].shape == (1, 5, 5, 7)
