"""The reference-surface shim (wfe_b200/shim): the reference's own
src/main.cpp, unchanged, compiled against the shim's headers and linked to
libwfe_b200.so.

CPU: the driver compiles and links (when its source is present), and the
binary needs nothing from the library but the C ABI.
GPU: the FP64 binary (built with -DWFE_DOUBLE, as the reference's FP64
build) writes what the unmodified reference executable wrote for the same
case and steps: its float32 snapshots (tests/golden/*_wfe.npz, from
oracle/_ref/wfe_f64) agree to the float32 rounding of the snapshot (scaled
error <= 2.5e-7 after 8 steps of the idealised cases and 65 steps of the
file-mode case with Davies relaxation, boundary-file switch and surface
physics), and its diagnostics lines match the reference's to 1e-3.
"""

import json
import re
import subprocess

import numpy as np
import pytest

from helpers import CASES, FILE_SMALL_STEPS, GOLDEN, ROOT, make_file_small, scaled_err

SHIM = ROOT / "wfe_b200" / "shim"
BIN = SHIM / "_build"


def _have_main():
    return subprocess.run(["make", "-s", "-C", str(SHIM), "have-main"],
                          capture_output=True).returncode == 0


def test_reference_driver_compiles_against_the_shim(tmp_path):
    if not _have_main():
        pytest.skip("the reference driver source is not present")
    out = tmp_path / "b"
    r = subprocess.run(["make", "-s", "-C", str(SHIM), f"OUT={out}", f"{out}/wfe_refmain_f64",
                        f"{out}/wfe_refmain_f32"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    for prec in ("f32", "f64"):
        exe = out / f"wfe_refmain_{prec}"
        assert exe.exists()
        und = subprocess.run(["nm", "-D", "--undefined-only", str(exe)], capture_output=True,
                             text=True).stdout
        wfe = sorted({ln.split()[-1] for ln in und.splitlines() if ln.split()[-1].startswith("wfe_")})
        assert "wfe_case_create_text" in wfe and "wfe_run" in wfe
        # no C++ symbol of the library: the driver's classes are the shim's own
        assert not [ln for ln in und.splitlines() if "_ZN3wfe" in ln], und


def _dt(ini):
    return float(re.search(r"^dt\s*=\s*([\d.]+)", ini.read_text(), re.M).group(1))


def _run(ini, out, nsteps, dt):
    exe = BIN / "wfe_refmain_f64"
    if not exe.exists():
        pytest.skip("wfe_b200/shim/_build/wfe_refmain_f64 not built")
    r = subprocess.run([str(exe), str(ini), f"out_dir={out}", f"t_end={nsteps * dt}",
                        f"out_interval={dt}", f"diag_interval={dt}"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def _diag(line):
    w = float(re.search(r"\|w\|max=\s*([-\d.]+)", line).group(1))
    t = re.search(r"th'=\[([-+\d.]+),([-+\d.]+)\]", line)
    return w, float(t.group(1)), float(t.group(2))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["bubble_open", "wk82_small"])
def test_shim_driver_matches_unmodified_reference_executable(tmp_path, name):
    W = np.load(GOLDEN / f"{name}_wfe.npz")
    ini = CASES / f"{name}.ini"
    out = tmp_path / "out"
    log = _run(ini, out, 8, _dt(ini))
    meta = json.loads((out / "meta.json").read_text())
    n = 0
    for var in meta["vars"]:
        for step in (0, 8):
            key = f"wfe64_{var}_{step:06d}"
            if key not in W:
                continue
            got = np.fromfile(out / f"{var}_{step:06d}.bin", dtype=np.float32).astype(np.float64)
            assert scaled_err(got, W[key].astype(np.float64), floor=1e-12) <= 2.5e-7, (var, step)
            n += 1
    assert n >= 10
    assert "bitti: 8 adim" in log
    ours = [ln for ln in log.splitlines() if ln.startswith("adim")]
    theirs = [ln for ln in bytes(W["wfe64_log"]).decode().splitlines() if ln.startswith("adim")]
    assert len(ours) == len(theirs) == 8
    for a, b in zip(ours, theirs):
        assert np.allclose(_diag(a), _diag(b), rtol=1e-3, atol=1e-3), (a, b)


@pytest.mark.gpu
def test_shim_driver_file_mode_matches_unmodified_reference_executable(tmp_path):
    W = np.load(GOLDEN / "file_small_wfe.npz")
    ini = make_file_small(tmp_path)
    out = tmp_path / "out"
    log = _run(ini, out, FILE_SMALL_STEPS, 60.0)
    for var in ("u", "v", "w", "thp", "pip", "qv", "qc", "qr", "rain", "tsk", "pblh", "t2m", "u10"):
        for step in (0, 8, FILE_SMALL_STEPS):
            key = f"wfe64_{var}_{step:06d}"
            if key not in W:
                continue
            got = np.fromfile(out / f"{var}_{step:06d}.bin", dtype=np.float32).astype(np.float64)
            assert scaled_err(got, W[key].astype(np.float64), floor=1e-12) <= 2.5e-7, (var, step)
    assert f"bitti: {FILE_SMALL_STEPS} adim" in log
