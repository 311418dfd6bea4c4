"""NetCDF export of a run's snapshots (the reference's tools/to_netcdf.py).

    python -m wfe_b200.netcdf case.ini [-o out.nc]

Collects the Writer output of a case (out_dir of the .ini: meta.json, zc.bin
and the float32 interior snapshots <var>_<step>.bin that the `wfe`
executable and the reference write) into one CF-style NetCDF file: time,
x, y, z coordinates, the cell heights zc, every variable of meta.json over
all snapshot times, with the reference's units and global attributes
(tools/to_netcdf.py:28-78).  The reference builds the file with xarray and
the HDF5-based netCDF4 library (zlib level 3); neither is a dependency here,
so the file is written directly in the NetCDF classic 64-bit-offset format
(CDF-2, no compression), which every NetCDF reader opens.  A variable may
hold at most 4 GiB.
"""

from __future__ import annotations

import argparse
import json
import struct
from pathlib import Path

import numpy as np

UNITS = {"u": "m s-1", "v": "m s-1", "w": "m s-1", "thp": "K", "pip": "1",
         "qv": "kg kg-1", "qc": "kg kg-1", "qr": "kg kg-1", "rain": "mm", "tsk": "K"}

_NC_DIMENSION, _NC_VARIABLE, _NC_ATTRIBUTE = 10, 11, 12
_TYPES = {np.dtype(">i1"): 1, np.dtype("S1"): 2, np.dtype(">i2"): 3, np.dtype(">i4"): 4,
          np.dtype(">f4"): 5, np.dtype(">f8"): 6}


def _pad4(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 4)


def _name(s: str) -> bytes:
    e = s.encode()
    return struct.pack(">i", len(e)) + _pad4(e)


def _attr_value(v):
    if isinstance(v, str):
        e = v.encode()
        return 2, len(e), _pad4(e)
    a = np.atleast_1d(np.asarray(v))
    a = a.astype(">f8") if a.dtype.kind == "f" else a.astype(">i4")
    return _TYPES[a.dtype], a.size, _pad4(a.tobytes())


def _attrs(d: dict) -> bytes:
    if not d:
        return struct.pack(">ii", 0, 0)
    out = struct.pack(">ii", _NC_ATTRIBUTE, len(d))
    for k, v in d.items():
        t, n, b = _attr_value(v)
        out += _name(k) + struct.pack(">ii", t, n) + b
    return out


class Variable:
    """dims: names; dtype: '>f4' / '>f8'; source: a callable giving the data
    (in C order over dims) slab by slab along the first dimension, or an array."""

    def __init__(self, name, dims, dtype, source, attrs=None):
        self.name, self.dims, self.dtype = name, tuple(dims), np.dtype(dtype)
        self.source, self.attrs = source, attrs or {}


def write_classic(path, dims: dict, variables: list, attrs: dict) -> None:
    """Write a NetCDF classic 64-bit-offset file (fixed-size dimensions)."""
    dnames = list(dims)

    def header(begins):
        h = b"CDF\x02" + struct.pack(">i", 0)
        h += struct.pack(">ii", _NC_DIMENSION, len(dims))
        for k in dnames:
            h += _name(k) + struct.pack(">i", dims[k])
        h += _attrs(attrs)
        h += struct.pack(">ii", _NC_VARIABLE, len(variables))
        for v, b in zip(variables, begins):
            h += _name(v.name) + struct.pack(">i", len(v.dims))
            h += b"".join(struct.pack(">i", dnames.index(d)) for d in v.dims)
            h += _attrs(v.attrs)
            size = int(np.prod([dims[d] for d in v.dims], dtype=np.int64)) * v.dtype.itemsize
            if size >= 2 ** 32:
                raise ValueError(f"variable {v.name} exceeds 4 GiB (NetCDF classic format)")
            h += struct.pack(">iiq", _TYPES[v.dtype], size + (-size % 4), b)
        return h

    begins, off = [], len(header([0] * len(variables)))
    for v in variables:
        begins.append(off)
        size = int(np.prod([dims[d] for d in v.dims], dtype=np.int64)) * v.dtype.itemsize
        off += size + (-size % 4)
    with open(path, "wb") as f:
        f.write(header(begins))
        for v, b in zip(variables, begins):
            assert f.tell() == b
            n = 0
            if callable(v.source):
                for slab in v.source():
                    a = np.ascontiguousarray(slab, dtype=v.dtype)
                    f.write(a.tobytes())
                    n += a.nbytes
            else:
                a = np.ascontiguousarray(v.source, dtype=v.dtype)
                f.write(a.tobytes())
                n = a.nbytes
            f.write(b"\0" * (-n % 4))


def read_ini(path) -> dict:
    kv = {}
    for line in Path(path).read_text().splitlines():
        line = line.split("#")[0].split(";")[0]
        if "=" in line:
            k, v = line.split("=", 1)
            kv[k.strip()] = v.strip()
    return kv


def export(outdir, out=None) -> Path:
    """One NetCDF file from the Writer output in `outdir`; returns its path."""
    outdir = Path(outdir)
    meta = json.loads((outdir / "meta.json").read_text())
    nx, ny, nz, dt = meta["nx"], meta["ny"], meta["nz"], meta["dt"]
    steps = sorted(int(p.stem.split("_")[1]) for p in outdir.glob("thp_*.bin"))
    times = np.array([s * dt for s in steps], dtype=np.float64)
    dims = {"time": len(steps), "x": nx, "y": ny, "z": nz}
    var = [Variable("time", ["time"], ">f8", times, {"units": "seconds since model start"}),
           Variable("x", ["x"], ">f8", (np.arange(nx) + 0.5) * meta["dx"], {"units": "m"}),
           Variable("y", ["y"], ">f8", (np.arange(ny) + 0.5) * meta["dy"], {"units": "m"}),
           Variable("z", ["z"], ">f8", np.arange(nz, dtype=np.float64),
                    {"long_name": "model level"})]
    zc = outdir / "zc.bin"
    if zc.exists():
        var.append(Variable("zc", ["z", "y", "x"], ">f4",
                            np.fromfile(zc, dtype=np.float32).reshape(nz, ny, nx),
                            {"units": "m", "long_name": "cell height"}))
    for name, lev in meta["vars"].items():
        files = [outdir / f"{name}_{s:06d}.bin" for s in steps]
        if not all(p.exists() for p in files):
            continue
        if lev == nz:
            vd = ["time", "z", "y", "x"]
        elif lev == nz + 1:
            dims["zw"] = nz + 1
            vd = ["time", "zw", "y", "x"]
        else:
            vd = ["time", "y", "x"]
        count = lev * ny * nx if lev > 1 else ny * nx

        def slabs(files=files, count=count):
            for p in files:
                a = np.fromfile(p, dtype=np.float32)
                if a.size != count:
                    raise ValueError(f"{p}: {a.size} values, expected {count}")
                yield a

        var.append(Variable(name, vd, ">f4", slabs, {"units": UNITS.get(name, "")}))
    path = Path(out) if out else outdir / "wfe_out.nc"
    write_classic(path, dims, var, {"title": "WFE regional forecast", "source": "WFE",
                                    "dx_m": float(meta["dx"]), "dt_s": float(dt)})
    return path


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("case")
    ap.add_argument("-o", "--out", default=None)
    a = ap.parse_args(argv)
    p = export(read_ini(a.case)["out_dir"], a.out)
    print(f"yazildi: {p} ({p.stat().st_size / 1e6:.1f} MB)")


if __name__ == "__main__":
    main()
