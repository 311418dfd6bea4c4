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


REF_EXE = ROOT / "oracle" / "_ref" / "wfe_f64"


def _run_rc(exe, ini, out, extra, fp64=True):
    cmd = [str(exe), str(ini), f"out_dir={out}", *extra] + (["--fp64"] if fp64 else [])
    return subprocess.run(cmd, capture_output=True, text=True, timeout=600)


@pytest.mark.gpu
def test_cli_watchdog_exit_3_with_emergency_snapshot(tmp_path):
    """|w| above w_abort at the every-10-steps watchdog: the reference prints
    its HATA line, writes the state at that step and exits 3
    (src/main.cpp:429-438)."""
    ini = CASES / "bubble_open.ini"
    dt = float(re.search(r"^dt\s*=\s*([\d.]+)", ini.read_text(), re.M).group(1))
    extra = ["w_abort=0.0001", f"t_end={40 * dt}", f"out_interval={100 * dt}",
             f"diag_interval={100 * dt}"]
    r = _run_rc(EXE, ini, tmp_path / "out", extra)
    assert r.returncode == 3, r.stdout + r.stderr
    assert "esigi asti (adim 10," in r.stderr
    for var in ("u", "v", "w", "thp", "pip"):
        assert (tmp_path / "out" / f"{var}_000010.bin").exists(), var
    assert not (tmp_path / "out" / "w_000020.bin").exists()
    assert "bitti:" not in r.stdout
    w = _snap(tmp_path / "out", "w", 10)
    assert np.isfinite(w).all() and np.abs(w).max() > 1e-4
    if REF_EXE.exists():  # the unmodified reference executable, same case and threshold
        rr = _run_rc(REF_EXE, ini, tmp_path / "ref", extra, fp64=False)
        assert rr.returncode == 3 and "esigi asti (adim 10," in rr.stderr
        wr = _snap(tmp_path / "ref", "w", 10).astype(np.float64)
        assert scaled_err(w.astype(np.float64), wr, floor=1e-12) <= 2.5e-7


@pytest.mark.gpu
def test_cli_nan_exit_2(tmp_path):
    """A non-finite state found by the diagnostics stops the run with exit 2
    and the reference's HATA line (src/main.cpp:440-455).  The NaN is
    injected on the host: bubble_dtheta = nan makes theta' NaN inside the
    bubble of the initial state."""
    ini = CASES / "bubble_open.ini"
    dt = float(re.search(r"^dt\s*=\s*([\d.]+)", ini.read_text(), re.M).group(1))
    extra = ["bubble_dtheta=nan", f"t_end={20 * dt}", f"out_interval={100 * dt}",
             f"diag_interval={dt}"]
    r = _run_rc(EXE, ini, tmp_path / "out", extra)
    assert r.returncode == 2, r.stdout + r.stderr
    assert "NaN/Inf tespit edildi" in r.stderr
    assert [ln for ln in r.stdout.splitlines() if ln.startswith("adim")][-1].split()[1] == "1"
    if REF_EXE.exists():
        rr = _run_rc(REF_EXE, ini, tmp_path / "ref", extra, fp64=False)
        assert rr.returncode == 2 and "NaN/Inf tespit edildi" in rr.stderr
