"""The drop-in executable (wfe_b200/bin/wfe, src/main.cpp on the C ABI).

On a GPU it must write what the unmodified reference executable writes for
the same case and steps: the float32 interior snapshots of the golden runs
(tests/golden/*_wfe.npz, from oracle/_ref/wfe_f64) agree to the float32
rounding of the snapshot (scaled error <= 2.5e-7 after 8 or 65 FP64 steps),
and the stdout diagnostics and closing line keep the reference's format.
"""

import json
import re
import subprocess

import numpy as np
import pytest

from helpers import CASES, FILE_SMALL_STEPS, GOLDEN, ROOT, make_file_small, scaled_err

EXE = ROOT / "wfe_b200" / "bin" / "wfe"


def test_cli_reports_a_bad_case():
    if not EXE.exists():
        pytest.skip("wfe_b200/bin/wfe not built")
    r = subprocess.run([str(EXE), str(CASES / "no_such_case.ini")], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr.strip()


def _run(ini, out, nsteps, dt, extra=()):
    cmd = [str(EXE), str(ini), f"out_dir={out}", f"t_end={nsteps * dt}", f"out_interval={dt}",
           f"diag_interval={dt}", "--fp64", *extra]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def _snap(out, var, step):
    return np.fromfile(out / f"{var}_{step:06d}.bin", dtype=np.float32)


def _diag(line):
    w = float(re.search(r"\|w\|max=\s*([-\d.]+)", line).group(1))
    t = re.search(r"th'=\[([-+\d.]+),([-+\d.]+)\]", line)
    return w, float(t.group(1)), float(t.group(2))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["bubble_open", "wk82_small"])
def test_cli_matches_unmodified_reference_executable(tmp_path, name):
    W = np.load(GOLDEN / f"{name}_wfe.npz")
    dt = float(re.search(r"^dt\s*=\s*([\d.]+)", (CASES / f"{name}.ini").read_text(), re.M).group(1))
    out = tmp_path / "out"
    log = _run(CASES / f"{name}.ini", out, 8, dt)
    meta = json.loads((out / "meta.json").read_text())
    for var in meta["vars"]:
        for step in (0, 8):
            key = f"wfe64_{var}_{step:06d}"
            if key not in W:
                continue
            got = _snap(out, var, step).astype(np.float64)
            ref = W[key].astype(np.float64)
            assert got.shape == ref.shape, var
            assert scaled_err(got, ref, floor=1e-12) <= 2.5e-7, (var, step)
    assert "bitti: 8 adim" in log
    ref_log = bytes(W["wfe64_log"]).decode()
    ours = [ln for ln in log.splitlines() if ln.startswith("adim")]
    theirs = [ln for ln in ref_log.splitlines() if ln.startswith("adim")]
    assert len(ours) == len(theirs) == 8
    for a, b in zip(ours, theirs):
        assert np.allclose(_diag(a), _diag(b), rtol=1e-3, atol=1e-3), (a, b)


@pytest.mark.gpu
def test_cli_file_mode_matches_unmodified_reference_executable(tmp_path):
    W = np.load(GOLDEN / "file_small_wfe.npz")
    ini = make_file_small(tmp_path)
    out = tmp_path / "out"
    log = _run(ini, out, FILE_SMALL_STEPS, 60.0)
    for var in ("u", "v", "w", "thp", "pip", "qv", "qc", "qr", "rain", "tsk", "pblh", "t2m", "u10"):
        for step in (0, 8, FILE_SMALL_STEPS):
            key = f"wfe64_{var}_{step:06d}"
            if key not in W:
                continue
            got = _snap(out, var, step).astype(np.float64)
            ref = W[key].astype(np.float64)
            assert scaled_err(got, ref, floor=1e-12) <= 2.5e-7, (var, step)
    assert f"bitti: {FILE_SMALL_STEPS} adim" in log
