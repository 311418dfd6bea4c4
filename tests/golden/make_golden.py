"""Generate the golden fixtures that pin the CPU oracle (test infrastructure).

Two steps, run from the repository root:

  python tests/golden/make_golden.py run  --raw <raw dir>
      On a machine with a B200 and the reference built by `make -C oracle ref`
      (oracle/_ref/).  Runs, for every case in tests/golden/cases/:
        * oracle/_ref/refdump_f64 / refdump_f32 (the reference's own kernels and
          Integrator driven through its C++ API; FP64 / FP32 padded dumps),
        * the unmodified reference executable oracle/_ref/wfe_f64 and wfe_f32
          (its src/main.cpp), writing its float32 snapshots every step.
      Raw output goes to --raw.

  python tests/golden/make_golden.py pack --raw <raw dir>
      On any machine, with the raw directory copied back.  Packs a selection of the raw arrays into tests/golden/<case>.npz
      (float64) and the unmodified executables' snapshots into
      tests/golden/<case>_wfe.npz (float32).

  The file-mode case file_small (tests/helpers.py: seeded synthetic prep inputs
  from wfe_b200.synth) runs through the unmodified executables only, for
  FILE_STEPS steps; its snapshots at steps 0, 8 and FILE_STEPS, the logs and the
  SHA-256 of the generated wfe_init.bin go to tests/golden/file_small_wfe.npz.

The cases are small grids so that the pure-CPU oracle finishes in seconds.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

import hashlib

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
CASES = HERE / "cases"
REF = ROOT / "oracle" / "_ref"

RUN_CASES = ["bubble_open", "straka_periodic", "schaer_open", "wk82_small", "moist_blob"]
OPS_CASES = ["ops_open", "ops_periodic"]
NSTEPS = 8
DUMPS = "1,8"
FILE_CASES = ["file_small"]
FILE_STEPS = 65


def read_ini(path: Path) -> dict:
    kv = {}
    for line in path.read_text().splitlines():
        for c in "#;":
            if c in line:
                line = line[: line.index(c)]
        if "=" not in line:
            continue
        k, v = line.split("=", 1)
        if k.strip():
            kv[k.strip()] = v.strip()
    return kv


def sh(cmd, log):
    print("+", " ".join(map(str, cmd)), flush=True)
    with open(log, "w") as f:
        r = subprocess.run([str(c) for c in cmd], stdout=f, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        print(open(log).read()[-3000:])
        raise SystemExit(f"failed ({r.returncode}): {cmd}")


def run(raw: Path) -> None:
    raw.mkdir(parents=True, exist_ok=True)
    for case in RUN_CASES + OPS_CASES:
        ini = CASES / f"{case}.ini"
        kv = read_ini(ini)
        dt = float(kv["dt"])
        for prec in ("f64", "f32"):
            out = raw / f"{case}_{prec}"
            shutil.rmtree(out, ignore_errors=True)
            mode = "ops" if case in OPS_CASES else "run"
            sh([REF / f"refdump_{prec}", ini, out, f"mode={mode}", f"nsteps={NSTEPS}",
                f"dump={DUMPS}"], raw / f"{case}_{prec}.log")
            if mode == "run":
                wout = raw / f"{case}_wfe{prec[1:]}"
                shutil.rmtree(wout, ignore_errors=True)
                sh([REF / f"wfe_{prec}", ini, f"out_dir={wout}", f"out_interval={dt}",
                    f"diag_interval={dt}", f"t_end={NSTEPS * dt}"],
                   raw / f"{case}_wfe{prec[1:]}.log")
    from helpers import make_file_small
    for case in FILE_CASES:
        ini = make_file_small(raw / f"{case}_case")
        dt = float(read_ini(ini)["dt"])
        for prec in ("f64", "f32"):
            wout = raw / f"{case}_wfe{prec[1:]}"
            shutil.rmtree(wout, ignore_errors=True)
            sh([REF / f"wfe_{prec}", ini, f"out_dir={wout}", f"out_interval={dt}",
                f"diag_interval={dt}", f"t_end={FILE_STEPS * dt}"],
               raw / f"{case}_wfe{prec[1:]}.log")


def load_dump(d: Path) -> dict:
    out = {}
    for line in (d / "manifest.txt").read_text().splitlines():
        name, n = line.split()
        a = np.fromfile(d / f"{name}.bin", dtype=np.float64)
        assert a.size == int(n), name
        out[name] = a
    return out


def pack(raw: Path) -> None:
    for case in RUN_CASES + OPS_CASES:
        d64 = load_dump(raw / f"{case}_f64")
        d32 = load_dump(raw / f"{case}_f32")
        keep = {}
        for k, a in d64.items():
            keep[k] = a
        # FP32 reference results, stored as float32 for the FP32-vs-FP64 spread
        for k, a in d32.items():
            if k.startswith(("s8_", "acn_", "tend_", "kes_", "sfc_")):
                keep["f32_" + k] = a.astype(np.float32)
        np.savez_compressed(HERE / f"{case}.npz", **keep)
        if case in RUN_CASES:
            snaps = {}
            for prec in ("64", "32"):
                wdir = raw / f"{case}_wfe{prec}"
                for f in sorted(wdir.glob("*_000000.bin")) + sorted(wdir.glob(f"*_{NSTEPS:06d}.bin")):
                    snaps[f"wfe{prec}_{f.stem}"] = np.fromfile(f, dtype=np.float32)
                snaps[f"wfe{prec}_log"] = np.frombuffer(
                    (raw / f"{case}_wfe{prec}.log").read_bytes(), dtype=np.uint8)
            np.savez_compressed(HERE / f"{case}_wfe.npz", **snaps)
        print(case, "packed")
    for case in FILE_CASES:
        snaps = {}
        for prec in ("64", "32"):
            wdir = raw / f"{case}_wfe{prec}"
            for step in (0, 8, FILE_STEPS):
                for f in sorted(wdir.glob(f"*_{step:06d}.bin")):
                    snaps[f"wfe{prec}_{f.stem}"] = np.fromfile(f, dtype=np.float32)
            snaps[f"wfe{prec}_log"] = np.frombuffer(
                (raw / f"{case}_wfe{prec}.log").read_bytes(), dtype=np.uint8)
        init = raw / f"{case}_case" / f"{case}_prep" / "wfe_init.bin"
        snaps["prep_sha256"] = np.frombuffer(hashlib.sha256(init.read_bytes()).digest(),
                                             dtype=np.uint8)
        np.savez_compressed(HERE / f"{case}_wfe.npz", **snaps)
        print(case, "packed")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["run", "pack"])
    ap.add_argument("--raw", required=True, help="directory of the raw reference outputs")
    ap.add_argument("--only-file", action="store_true", help="the file-mode cases only")
    a = ap.parse_args()
    os.chdir(ROOT)
    if a.only_file:
        RUN_CASES.clear()
        OPS_CASES.clear()
    (run if a.what == "run" else pack)(Path(a.raw))


if __name__ == "__main__":
    main()
