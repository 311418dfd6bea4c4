"""Build the wfe_b200 shared library (and the drop-in `wfe` executable) in-tree.

    python -m wfe_b200.build        # or wfe_b200.build.build()

Compiles wfe_b200/csrc/*.cu and *.cpp with nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) into wfe_b200/libwfe_b200.so, and
wfe_b200/csrc/cli/wfe_main.cpp against it into wfe_b200/bin/wfe.  Objects go to
wfe_b200/_build/; a source is recompiled when it or a header is newer.
"""

from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libwfe_b200.so"
BIN = PKG / "bin" / "wfe"
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def _sources():
    return sorted(p for p in CSRC.iterdir() if p.suffix in (".cu", ".cpp"))


def _headers():
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, hdr_time: float, verbose: bool) -> Path:
    obj = OBJ / (src.name + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_time):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, "-x", "cu" if src.suffix == ".cu" else "c++", "-c", str(src),
           "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    hdr = _headers()
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, hdr, verbose), _sources()))
    newest = max([o.stat().st_mtime for o in objs] + [(CSRC / "exports.map").stat().st_mtime])
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
               "-Xlinker", f"--version-script={CSRC / 'exports.map'}"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    cli = CSRC / "cli" / "wfe_main.cpp"
    if cli.exists() and (not BIN.exists() or BIN.stat().st_mtime < max(LIB.stat().st_mtime,
                                                                      cli.stat().st_mtime)):
        BIN.parent.mkdir(exist_ok=True)
        cmd = [NVCC, "-O2", "-std=c++17", f"-I{ROOT / 'include'}", str(cli), "-o", str(BIN),
               f"-L{PKG}", "-lwfe_b200", f"-Xlinker", f"-rpath={PKG}"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"cli build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
