#!/usr/bin/env python
"""RK3 cell-updates/s of the WFE per-step hot path on B200.

Workload: the WK82-type supercell of cases/wk82_160.ini -- 160 x 160 x 40
cells at 1 km, stretched 20 km column, moist WK82 sounding with straight-line
shear, +3 K bubble, Kessler + mixed-phase microphysics, dt = 6 s with 6
acoustic substeps, FP32 state (the precision the reference runs in).  A "step"
is one large RK3 step (3 stages, 1 + 3 + 6 acoustic substeps, Kessler).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--gpus N > 1 needs N ranks: started under torch.distributed.run (RANK,
WORLD_SIZE, LOCAL_RANK in the environment) it checks that WORLD_SIZE is N;
started without a launcher it runs itself again under
`torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1` and exits
with that run's status.  It never runs fewer ranks than asked.  --dry-run
joins the ranks and reports them without touching a GPU (--backend gloo).

ours       K steps replayed from captured CUDA graphs, timed with CUDA events on
           the library's stream, max over ranks; N > 1 runs one independent
           member per GPU (weak scaling, no collective on the data path).
           Also: a per-kernel CUDA-event profile of one extra step, captured
           as a graph with event nodes around every kernel and replayed
           (roofline of the dominant kernel), an end-to-end run through the C ABI with host
           buffers at the reference driver's I/O cadence, and (rank 0, N = 1)
           the CPU oracle on a bounded sample as the CPU baseline.
reference  the reference's own CUDA implementation, compiled from its sources
           (oracle/_ref/refdump_f32, its Integrator::step through its C++ API)
           on the same GPU, same case, K steps after W warm-up steps.

--workload ensemble24 measures the batched ensemble instead: 24 members in
three groups of 8 on 120x90x45, 220x150x45 and 300x200x45 grids (dx = 12 km,
20 km top, 37 368 000 cells), seeded synthetic prep inputs (wfe_b200.synth:
Gaussian ridges, standard-atmosphere sounding, u0 ~ U(5, 20) m/s, theta' and
qv' noise), full physics (surface layer, nonlocal PBL, soil, radiation,
Kessler), Davies relaxation over 5 rows, positive-definite moisture, dt = 60 s,
6 acoustic substeps, FP32.  value = all members' cells x K / device time of K
graph-replayed batched steps (max over ranks; N > 1 shards members over GPUs
by cell count, no collective on the data path).  The same members stepped one
after another through their own graphs give the serial figure; with
--impl reference the unmodified reference executable (oracle/_ref/wfe_f32)
runs each member for K steps, one after another, and the sum of its own step-
loop wall times is the reference figure.

--workload adjoint measures the cost of the adjoint (and tangent-linear) run
against the forward run on the same WK82 case with the linearised Kessler
column (positive-definite limiter and w damping off, neither linearised):
after W spin-up steps, value = wall time of wfe_ad_run over K steps
(checkpoints every 30 steps, the fields already on the device; the median of
three runs after one that captures the sweep's graphs) / CUDA-event time of
the same K forward steps.  The line also gives the tangent-linear ratio, the
adjoint's with checkpoint_every = 0 (the longest interval the device memory
holds: no recomputation when the whole undo log fits) and the dot-product gap
<M dx, y> - <dx, M^T y> over min(K, 10) steps.  --fp64 runs the FP64 state.
--workload adjoint_schaer measures the same on the dry Schaer mountain-wave
slab (400x4x65, dt = 4 s; K = 900 is its 1 h sensitivity run).
"""

from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
# The autotuner may pick the column kernel with the parallel tridiagonal
# solve, whose solution equals the Thomas sweep's up to rounding (the library
# keeps the bit-identical variants unless this is 0; tests cover both).
os.environ.setdefault("WFE_EXACT_COLUMN", "0")

CASE = ROOT / "cases" / "wk82_160.ini"
# The single-case workloads: the headline WK82 case (configs' moist
# supercell) and the other plain-step configurations, measured the same way
# (--workload).  (case, description, moist, traffic summary)
WORKLOADS = {
    "wk82": ("wk82_160.ini", "WK82 supercell 160x160x40, dx=1 km, 20 km stretched top, moist + "
             "Kessler, dt=6 s, ns=6", True, "traffic_wk82_160.txt"),
    "bubble80": ("warm_bubble_80.ini", "dry warm bubble 80x80x40, dx=dy=dz=250 m, open lateral "
                 "boundaries, Rayleigh layer, dt=1.5 s, ns=6", False, None),
    "straka512": ("straka_512.ini", "Straka density current 512x4x64, dx=dz=100 m, periodic, "
                  "K=75 m2/s, dt=0.5 s, ns=6", False, None),
    "schaer400": ("schaer_400.ini", "Schaer mountain waves 400x4x65, dx=500 m, 20 km top, "
                  "U=10 m/s, N=0.01/s, dt=4 s, ns=6", False, None),
}
WORKLOAD = "wk82"
METRIC = "RK3 cell-updates/s"
PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM = 6650.0  # GB/s, used only when MEASURED_PEAKS.json is absent

# Algorithmic FP32 fields per cell of each kernel (unique fields a launch must
# read or write; moist case, no boundary relaxation).  Bytes = fields x 4.
KERNEL_FIELDS = {
    # u', v' new, w, pi', theta', tw, ttheta, theta_b^w, dtheta_b/dz, rtjx, rtjy,
    # kt3, aw, qv, qc, qr, qv_b (17 reads) + w, pi'_next, theta' (3 writes)
    "acoustic_column": 20,
    # u, v, pi', pi'_prev, theta', theta_b, tu, tv, qv (9 reads) + u, v (2 writes)
    "acoustic_uv": 11,
    # u v w theta' qv qc qr (est) + qv qc qr (time n) + rho_b rho_b^w mfx mfy mfz
    # (15 reads) + tu tv tw ttheta + qv qc qr stage values (7 writes)
    "tendencies": 22,
    "mass_flux": 8,     # u v w rho_b rho_b^w -> mfx mfy mfz
    "kessler": 12,      # theta' pi' qv qc qr theta_b pi_b rho_b -> theta' qv qc qr
    "pd_ratio": 8,
    "fill_ghosts": 0,   # surface-area only
}
# Dry cases: the moisture fields drop out (column: qv qc qr qv_b; u, v: qv;
# tendencies: 3 moisture species read twice and written once).
DRY_KERNEL_FIELDS = dict(KERNEL_FIELDS, acoustic_column=16, acoustic_uv=10, tendencies=13)
# Per cell and step, the reference-set algorithmic bytes (moist + Kessler, ns=6):
# 3 x 19 slow-tendency fields + 10 x 26 acoustic fields + 12 Kessler fields;
# dry: 3 x 10 + 10 x 22.
STEP_FIELDS = 3 * 19 + 10 * 26 + 12
DRY_STEP_FIELDS = 3 * 10 + 10 * 22
# With the column coefficients in per-level tables (a horizontally uniform
# set-up and a pipelined column kernel, variants 13-15 and 19-22) a column
# launch reads none of theta_b^w, dtheta_b/dz, rtjx, rtjy, kt3, aw, qv_b per
# cell: 7 fields fewer (6 dry).
TABLE_FIELDS, DRY_TABLE_FIELDS = 7, 6
PIPE_VARIANTS = set(range(13, 16)) | set(range(19, 23))
# With the base state in per-level tables (a horizontally uniform base state)
# the mass fluxes read neither rho_b nor rho_b^w per cell, Kessler neither
# theta_b, pi_b nor rho_b, the u, v step not theta_b.
BASE_TABLE_FIELDS = {"mass_flux": 2, "kessler": 3, "acoustic_uv": 1}


def use_workload(name: str) -> None:
    global CASE, WORKLOAD
    WORKLOAD = name
    CASE = ROOT / "cases" / WORKLOADS[name][0]


def workload_desc() -> str:
    return WORKLOADS[WORKLOAD][1]


def peaks():
    if PEAKS.exists():
        d = json.loads(PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(gpu)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if "Active" in v and "Not" not in v:
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def _free_port() -> int:
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch_ranks(n: int) -> int:
    """--gpus N > 1 started without a launcher: run this command again as N
    ranks under torch.distributed.run on 127.0.0.1 and return its exit code."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.run(cmd, timeout=3600).returncode


def dist_setup(n, backend="nccl"):
    """Rank, world size and local rank; the process group for N > 1 ranks.
    The world size must be the --gpus count: a mismatch is an error, never a
    silent run on fewer GPUs."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != n:
        raise SystemExit(f"bench.py: --gpus {n} but the launcher started {world} rank(s)")
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def reduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sync_device(world):
    try:
        import torch

        if torch.cuda.is_available():
            torch.cuda.synchronize()
    except Exception:
        pass


def cpu_baseline(seconds: float = 10.0):
    """CPU oracle (FP64, OpenMP over all host cores) on the same workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    o = O.Case(CASE)
    it = o.integrator()
    it.set_state(o.initial_state())
    cells = o.nx * o.ny * o.nz
    n, t0 = 0, time.perf_counter()
    while True:
        it.step(o.dt, n * o.dt)
        n += 1
        el = time.perf_counter() - t0
        if el > seconds or n >= 400:
            break
    return {"value": cells * n / el, "unit": "cell-updates/s", "cores": O.threads(),
            "kind": "port",
            "sample": f"{n} RK3 steps of the full {o.nx}x{o.ny}x{o.nz} case {CASE.name} from t=0, FP64 CPU oracle "
                      f"(oracle/wfe_oracle.cpp, OpenMP), {el:.1f} s"}


def run_reference(args) -> dict:
    exe = ROOT / "oracle" / "_ref" / "refdump_f32"
    if not exe.exists():
        return {"impl": "reference", "unavailable": "oracle/_ref/refdump_f32 not built"}
    cmd = [str(exe), str(CASE), "/tmp/wfe_refbench", "mode=bench", f"warmup={args.warmup}",
           f"steps={args.steps}"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
    m = re.search(r"refbench cells=(\d+) steps=(\d+) ms=([\d.]+)", r.stdout)
    if r.returncode != 0 or not m:
        return {"impl": "reference", "unavailable": f"reference run failed: {r.stderr[-200:]}"}
    cells, steps, ms = int(m.group(1)), int(m.group(2)), float(m.group(3))
    v = cells * steps / (ms / 1000.0)
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "cell-updates/s",
        "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (analytic sounding and initial perturbation of the case, deterministic)",
        "config": {"workload": workload_desc(), "case": f"cases/{CASE.name}",
                   "l2": "per-step working set > L2 (126 MB)" if WORKLOAD == "wk82" else
                         "per-step working set fits in L2 (126 MB)"},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                         "sample": f"{steps} steps of the same case through the reference's own "
                                   "Integrator::step, its CUDA build compiled from its sources "
                                   "for sm_100a (FP32); the reference has no CPU path"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def e2e_run(W, case_ini, steps: int, device: int):
    """End to end through the public API with host buffers, at the reference
    driver's cadence (src/main.cpp:425-467), after three untimed warm-up
    steps through the same calls: initial state uploaded from
    page-locked host buffers, every step the |w| watchdog read back (one step
    behind: wfe_absmax_begin queues step s's reduction, and step s's value is
    read once step s + 1 is queued, so the GPU never waits for the host),
    diagnostics (w, theta', pi', qc, qr) every diag_interval and the full state
    and rain every out_interval downloaded as asynchronous snapshots (packed on
    the device, copied to page-locked buffers while the next steps run)."""
    import numpy as np

    c = W.Case(case_ini, precision="f32", device=device)
    host = c.snapshot_buffers(W.FIELDS)  # page-locked, interior layout
    for k in W.FIELDS:
        host[k][...] = c.field(k, interior=True, dtype=np.float32)
    diag = c.snapshot_buffers(("w", "thp", "pip", "qc", "qr"))
    full = c.snapshot_buffers(list(W.FIELDS) + ["rain"])
    diag_every = max(1, round(120.0 / c.dt))
    out_every = max(1, round(600.0 / c.dt))
    # untimed warm-up through the same calls: the first steps capture the
    # three rotation phases' graphs and the first transfers allocate their
    # staging buffers (one-time set-up, like the warm-up steps of the
    # device-resident measurement); the timed run restarts from the host copy
    # of the initial state
    c.run(3, c.dt, 0.0)
    c.absmax_begin("w", 0)
    c.absmax_end(0)
    c.snapshot_begin(diag)
    c.snapshot_wait()
    c.snapshot_begin(full)
    c.snapshot_wait()
    c.set_field("w", host["w"], interior=True)
    c.sync()
    h2d = d2h = 0
    sync_device(1)
    t0 = time.perf_counter()
    for k, a in host.items():
        c.set_field(k, a, interior=True)
        h2d += a.nbytes
    for s in range(1, steps + 1):
        c.run(1, c.dt, (s - 1) * c.dt)
        c.absmax_begin("w", s & 1)
        d2h += 4
        if s > 1:
            wmax = c.absmax_end((s - 1) & 1)
            if not wmax < 150.0:
                raise RuntimeError(f"|w| watchdog tripped at step {s - 1}: {wmax}")
        # snapshots are packed on the device and copied while later steps run
        if s % diag_every == 0:
            c.snapshot_begin(diag)
            d2h += sum(a.nbytes for a in diag.values())
        if s % out_every == 0 or s == steps:
            c.snapshot_begin(full)
            d2h += sum(a.nbytes for a in full.values())
    wmax = c.absmax_end(steps & 1)
    if not wmax < 150.0:
        raise RuntimeError(f"|w| watchdog tripped at step {steps}: {wmax}")
    c.snapshot_wait()
    c.sync()
    el = time.perf_counter() - t0
    cells = c.nx * c.ny * c.nz
    c.close()
    return cells * steps / el, h2d / steps, d2h / steps, el


ENS_DIR = Path(tempfile.gettempdir()) / "wfe_b200_ensemble24"
ENS_CELLS = 8 * (120 * 90 + 220 * 150 + 300 * 200) * 45
ENS_FIELDS = 3 * 29 + 10 * 27 + 12 + 23  # full physics + Davies + PD, fields per cell-update


def ensemble_members():
    """The 24 member cases (generated once per machine into a temp dir)."""
    from wfe_b200 import synth

    done = ENS_DIR / "done"
    if not done.exists():
        paths = synth.write_ensemble(ENS_DIR, seed=2024, hours=24)
        done.write_text("\n".join(str(p) for p in paths))
    return [Path(p) for p in done.read_text().split()]


ENS_CONFIG = {
    "workload": "batched ensemble: 24 members, 8 each on 120x90x45, 220x150x45, 300x200x45, "
                "dx=12 km, 20 km top, full physics + Kessler + Davies(5) + PD, dt=60 s, ns=6",
    "members": 24, "cells": ENS_CELLS, "precision": "f32",
    "inputs": "wfe_b200.synth.write_ensemble(seed=2024): seeded synthetic prep files",
    "l2": "no flush: per-step working set ~10 GB > L2 (126 MB)",
    "timing": "CUDA events on the ensemble stream around graph replays",
}


def run_reference_ensemble(args) -> dict:
    exe = ROOT / "oracle" / "_ref" / "wfe_f32"
    if not exe.exists():
        return {"impl": "reference", "unavailable": "oracle/_ref/wfe_f32 not built"}
    total_s, cells = 0.0, 0
    for p in ensemble_members():
        kv = dict(ln.split(" = ", 1) for ln in p.read_text().splitlines() if " = " in ln)
        dt = float(kv["dt"])
        r = subprocess.run([str(exe), str(p), f"out_dir=/tmp/wfe_refens/{p.stem}",
                            "out_interval=1e9", "diag_interval=1e9", f"t_end={args.steps * dt}"],
                           capture_output=True, text=True, timeout=1800)
        m = re.search(r"bitti: (\d+) adim, ([\d.]+) s", r.stdout)
        if r.returncode != 0 or not m:
            return {"impl": "reference", "unavailable": f"reference member run failed: {p.name}"}
        total_s += float(m.group(2))
        cells += int(kv["nx"]) * int(kv["ny"]) * int(kv["nz"])
    v = cells * args.steps / total_s
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "cell-updates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": 0, "ms_per_step": total_s * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded prep inputs)", "config": ENS_CONFIG,
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                         "sample": "the unmodified reference executable run once per member, "
                                   "members one after another (its ensemble pattern, "
                                   "tools/run_ensemble.py); wall time of its step loop"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def ensemble_bench(args, rank, world, local):
    import numpy as np
    import wfe_b200 as W
    from wfe_b200 import shard

    paths = ensemble_members()
    sizes = []
    for p in paths:
        kv = dict(ln.split(" = ", 1) for ln in p.read_text().splitlines() if " = " in ln)
        sizes.append(int(kv["nx"]) * int(kv["ny"]) * int(kv["nz"]))
    mine = shard.partition(sizes, world)[rank]
    mem = [W.Case(paths[q], precision="f32", device=local) for q in mine]
    dt = mem[0].dt
    cells = sum(sizes[q] for q in mine)
    ens = W.Ensemble(mem)
    # the first run of 19 or more steps picks the ensemble's mode on real
    # steps (wfe_ensemble_run): that happens in the warm-up, never in the
    # timed region
    warm = max(args.warmup, 20)
    ens.run(warm, dt, 0.0)
    ens.sync()
    sampler = ClockSampler(local)
    time.sleep(0.3)
    barrier(world)
    sync_device(world)
    ms = ens.time_run(args.steps, dt, warm * dt)
    sync_device(world)
    barrier(world)
    clocks = sampler.stop()
    ms_max = reduce_max(ms, world)
    value = sum(sizes) * args.steps / (ms_max / 1000.0)
    launches = ens.launches_per_step()
    variants = ens.variants()

    # serial: the same members stepped one after another through their own graphs
    serial_ms = 0.0
    t_now = (warm + args.steps) * dt
    for m in mem:
        serial_ms += m.time_run(args.steps, dt, t_now)
    serial_ms = reduce_max(serial_ms, world)
    serial_value = sum(sizes) * args.steps / (serial_ms / 1000.0)

    # end to end: initial states from page-locked host buffers, the |w|
    # watchdog of every member each 10 steps (read one block behind, so the
    # next block is queued before the host waits), the final states back to
    # page-locked host buffers (packed on the device)
    e2e = None
    if not args.no_e2e:
        host, out = [], []
        for m in mem:
            hb = m.snapshot_buffers(W.FIELDS)
            for k in W.FIELDS:
                hb[k][...] = m.field(k, interior=True, dtype=np.float32)
            host.append(hb)
            out.append(m.snapshot_buffers(W.FIELDS))
            m.set_field("w", hb["w"], interior=True)  # staging buffers outside the timed region
        h2d = d2h = 0
        sync_device(world)
        t0 = time.perf_counter()
        for m, hs in zip(mem, host):
            for k, a in hs.items():
                m.set_field(k, a, interior=True)
                h2d += a.nbytes
        t = 0.0
        blk = 0
        for s in range(0, args.steps, 10):
            n = min(10, args.steps - s)
            ens.run(n, dt, t)
            t += n * dt
            for m in mem:
                m.absmax_begin("w", blk & 1)
                d2h += 4
            if blk > 0:
                for m in mem:
                    if not m.absmax_end((blk - 1) & 1) < 150.0:
                        raise RuntimeError("|w| watchdog tripped")
            blk += 1
        for m in mem:
            if not m.absmax_end((blk - 1) & 1) < 150.0:
                raise RuntimeError("|w| watchdog tripped")
        for m, ob in zip(mem, out):
            m.snapshot_begin(ob)
            d2h += sum(a.nbytes for a in ob.values())
        for m in mem:
            m.snapshot_wait()
        ens.sync()
        el = reduce_max(time.perf_counter() - t0, world)
        e2e = {"value": sum(sizes) * args.steps / el, "unit": "cell-updates/s",
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps}
    stats = {q: shard.member_stats(m) for q, m in zip(mine, mem)}
    allstats = shard.gather_stats(stats, world, device="cuda" if world > 1 else None)
    ens.close()
    for m in mem:
        m.close()
    if rank == 0:
        hbm, peak_kind = peaks()
        gbs = ENS_FIELDS * 4 * sum(sizes) / (ms_max / args.steps / 1e3) / 1e9 / world
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": warm, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded prep inputs)",
            "config": dict(ENS_CONFIG, parallelism=f"members sharded over {world} GPU(s)"),
            "step_roofline": {"alg_bytes_per_cell": ENS_FIELDS * 4, "achieved_gbs_per_gpu": gbs,
                              "peak": hbm, "peak_kind": peak_kind, "frac": gbs / hbm},
            "serial": {"value": serial_value, "ms_per_step": serial_ms / args.steps,
                       "what": "the same members stepped one after another, each from its own "
                               "captured graphs"},
            "speedup_vs_serial": value / serial_value,
            "variants": variants,
            "gpu_launches": launches * args.steps,
            "clocks": clocks, "e2e": e2e,
            "members_w_max": max(st["w_max"] for st in allstats.values()),
        }
        print(json.dumps(line), flush=True)


# The adjoint workloads: (case, overrides, description).  WK82 runs the
# linearised Kessler column with the two nonlinear switches off; the Schaer
# slab is the dry mountain-wave sensitivity case (1 h = 900 steps of 4 s).
ADJOINT_CASES = {
    "adjoint": ("wk82_160.ini", {"pd_moist": "off", "w_damping": "off"},
                "WK82 supercell 160x160x40, moist + linearised Kessler, dt=6 s, ns=6, "
                "pd_moist=off, w_damping=off"),
    "adjoint_schaer": ("schaer_400.ini", {},
                       "Schaer mountain waves 400x4x65, dry, dx=500 m, 20 km top, dt=4 s, ns=6"),
}


def adjoint_bench(args, device: int) -> dict:
    """Adjoint and tangent-linear cost over the forward (WK82 or Schaer)."""
    import numpy as np
    import wfe_b200 as W
    from wfe_b200 import adjoint as A

    prec = "f64" if args.fp64 else "f32"
    K = args.steps
    ini, over, desc = ADJOINT_CASES[args.workload]
    c = W.Case(ROOT / "cases" / ini, overrides=over, precision=prec, device=device)
    c.run(args.warmup)
    c.sync()
    x0 = A.get_fields(c)
    A.set_fields(c, x0)
    c.sync()
    sampler = ClockSampler(device)
    time.sleep(0.3)
    fwd_ms = c.time_run(K)
    rng = np.random.default_rng(2)
    sc = {"qv": 1e-3, "qc": 1e-3, "qr": 1e-3}
    names = A.state_names(c)
    dx = {k: rng.standard_normal(c.shape) * sc.get(k, 1.0) for k in names}
    y = {k: rng.standard_normal(c.shape) * sc.get(k, 1.0) for k in names}
    c.lin_enable()
    times = {}
    for name in ("ad", "tl", "ad_auto"):
        t = []
        for rep in range(4):  # the first run captures the segment graphs
            A.set_fields(c, x0)
            c.lin_zero()
            A.set_fields(c, dx if name == "tl" else y, role="lin")
            c.sync()
            t0 = time.perf_counter()
            if name == "ad":
                c.ad_run(K, checkpoint_every=30)
            elif name == "ad_auto":
                c.ad_run(K, checkpoint_every=0)
            else:
                c.tl_run(K)
            t.append(time.perf_counter() - t0)
        times[name] = sorted(t[1:])[1] * 1e3  # median of the three later runs
    clocks = sampler.stop()
    m = min(K, 10)
    mdx = A.tangent(c, x0, dx, m)
    mty = A.adjoint(c, x0, y, m, every=5)
    lhs = sum(float(np.sum(mdx[k] * y[k])) for k in names)
    rhs = sum(float(np.sum(dx[k] * mty[k])) for k in names)
    c.close()
    return {
        "metric": "adjoint_cost_over_forward", "value": times["ad"] / fwd_ms, "unit": "x",
        "higher_is_better": False, "n_gpus": 1, "steps": K, "warmup": args.warmup, "dtype": prec,
        "data": "synthetic (analytic initial state, deterministic)",
        "config": {"workload": desc, "case": f"cases/{ini}", "checkpoint_every": 30},
        "statistic": "median of three runs after one that captures the graphs",
        "fwd_ms_per_step": fwd_ms / K, "ad_ms_per_step": times["ad"] / K,
        "tl_ms_per_step": times["tl"] / K, "tl_cost_over_forward": times["tl"] / fwd_ms,
        "ad_auto_checkpoint_cost_over_forward": times["ad_auto"] / fwd_ms,
        "dot_test": {"steps": m, "lhs": lhs, "rhs": rhs,
                     "rel_gap": abs(lhs - rhs) / max(abs(lhs), abs(rhs))},
        "clocks": clocks,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", choices=list(WORKLOADS) + ["ensemble24"] + list(ADJOINT_CASES), default="wk82")
    ap.add_argument("--fp64", action="store_true", help="adjoint workload: FP64 state")
    ap.add_argument("--backend", default="nccl", help="process-group backend for N > 1 ranks")
    ap.add_argument("--dry-run", action="store_true",
                    help="start the ranks, join the process group and report them; no GPU work")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args.gpus))
    rank, world, local = dist_setup(args.gpus, args.backend)
    if args.workload in WORKLOADS:
        use_workload(args.workload)

    if args.dry_run:
        barrier(world)
        if world > 1:
            import torch.distributed as dist

            t = [None] * world
            dist.all_gather_object(t, rank)
            ranks = sorted(t)
        else:
            ranks = [0]
        if rank == 0:
            print(json.dumps({"dry_run": True, "n_gpus": world, "ranks": ranks,
                              "backend": args.backend if world > 1 else None}), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    if args.impl == "reference":
        if rank == 0:
            ref = run_reference_ensemble if args.workload == "ensemble24" else run_reference
            print(json.dumps(ref(args)), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    if args.workload in ADJOINT_CASES:
        if rank == 0:
            print(json.dumps(adjoint_bench(args, local)), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    if args.workload == "ensemble24":
        ensemble_bench(args, rank, world, local)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    import wfe_b200 as W

    c = W.Case(CASE, precision="f32", device=local)
    cells = c.nx * c.ny * c.nz
    c.run(args.warmup, c.dt, 0.0)
    c.sync()
    sampler = ClockSampler(local)
    time.sleep(0.3)
    barrier(world)
    sync_device(world)
    ms = c.time_run(args.steps, c.dt, args.warmup * c.dt)
    sync_device(world)
    barrier(world)
    clocks = sampler.stop()
    ms_max = reduce_max(ms, world)
    value = cells * args.steps * world / (ms_max / 1000.0)
    launches = c.launches_per_step()

    # per-kernel device times of one more step, replayed from a graph with event
    # nodes around each launch
    kt = c.kernel_times(c.dt, (args.warmup + args.steps) * c.dt)
    step_kernel_ms = sum(v[0] for v in kt.values())
    dom = max(kt.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_n) = dom
    avg_ms = dom_ms / dom_n
    moist = WORKLOADS[WORKLOAD][2]
    kf = KERNEL_FIELDS if moist else DRY_KERNEL_FIELDS
    step_fields = STEP_FIELDS if moist else DRY_STEP_FIELDS
    variants = c.variants()
    tables = variants["level_tables"] and variants["column"] in PIPE_VARIANTS
    if tables:
        tab = TABLE_FIELDS if moist else DRY_TABLE_FIELDS
        kf = dict(kf, acoustic_column=kf["acoustic_column"] - tab)
        step_fields -= tab * kt.get("acoustic_column", (0.0, 0))[1]
    if variants["base_tables"]:
        for kname, nf in BASE_TABLE_FIELDS.items():
            if kname in kf and (kname != "kessler" or moist):
                kf = dict(kf, **{kname: kf[kname] - nf})
                step_fields -= nf * kt.get(kname, (0.0, 0))[1]
    alg_bytes = kf.get(dom_name, 0) * 4 * cells
    hbm, peak_kind = peaks()
    achieved = alg_bytes / (avg_ms / 1000.0) / 1e9
    traffic = None
    tname = WORKLOADS[WORKLOAD][3]
    tf = ROOT / "profiles" / tname if tname else None
    tkey = dom_name + ("_tables" if (tables and dom_name == "acoustic_column") or
                       (variants["base_tables"] and dom_name in BASE_TABLE_FIELDS) else "")
    if tf is not None and tf.exists():
        for ln in tf.read_text().splitlines():
            parts = ln.split()
            if len(parts) == 2 and not ln.startswith("#") and parts[0] == tkey:
                traffic = int(parts[1])
    c.close()

    e2e = None
    if not args.no_e2e:
        # three runs, the median: the wall clock of a host-driven loop also
        # sees the host's own scheduling (one stalled host thread idles the GPU)
        runs = [e2e_run(W, CASE, args.steps, local) for _ in range(3)]
        vals = sorted(r[0] for r in runs)
        ev, h2d, d2h = vals[1], runs[0][1], runs[0][2]
        ev = reduce_max(1.0 / ev, world)  # slowest rank
        e2e = {"value": world / ev, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "runs": [round(v) for v in vals],
               "statistic": "median of 3 runs"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (analytic sounding and initial perturbation of the case, deterministic)",
            "config": {"workload": workload_desc(), "case": f"cases/{CASE.name}", "precision": "f32",
                       "parallelism": f"replicas x{world} (one member per GPU)",
                       "l2": "no flush: per-step working set ~270 MB > L2 (126 MB)"
                             if WORKLOAD == "wk82" else
                             "no flush: the per-step working set fits in L2 (126 MB); an "
                             "L2/launch-bound measurement, not an HBM one",
                       "timing": "CUDA events on the library stream around graph replays",
                       "column_solver": "the tuner's fastest column kernel, parallel tridiagonal "
                                        "solve allowed" if os.environ.get("WFE_EXACT_COLUMN") == "0"
                                        else "Thomas sweep (bit-identical variants only)",
                       "variants": variants},
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms,
                         "launches_per_step": dom_n},
            "step_roofline": {"alg_bytes_per_cell": step_fields * 4,
                              "achieved_gbs": step_fields * 4 * cells / (ms_max / args.steps / 1e3) / 1e9,
                              "frac": step_fields * 4 * cells / (ms_max / args.steps / 1e3) / 1e9 / hbm},
            "kernel_ms_per_step": {k: round(v[0], 4) for k, v in kt.items()},
            "kernel_sum_ms": step_kernel_ms,
            "gpu_launches": launches * args.steps,
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
