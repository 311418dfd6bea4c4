"""bench.py's rank handling for --gpus N (CPU, gloo).

--gpus 2 without a launcher must run two ranks (it starts them itself under
torch.distributed.run) and report n_gpus = 2; a launcher that started a
different number of ranks than --gpus asks for is an error, not a silent run
on fewer GPUs.
"""

import json
import os
import subprocess
import sys

from helpers import ROOT


def _bench(args, env=None, timeout=300):
    e = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        e.pop(k, None)
    e.update(env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True,
                          text=True, timeout=timeout, env=e, cwd=ROOT)


def test_two_ranks_started_without_a_launcher():
    r = _bench(["--gpus", "2", "--backend", "gloo", "--dry-run"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["ranks"] == [0, 1] and d["backend"] == "gloo"


def test_world_size_must_match_gpus():
    r = _bench(["--gpus", "2", "--dry-run"], env={"WORLD_SIZE": "1", "RANK": "0",
                                                   "LOCAL_RANK": "0"}, timeout=120)
    assert r.returncode != 0
    assert "--gpus 2" in r.stderr


def test_single_rank_default():
    r = _bench(["--dry-run"], timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert json.loads(r.stdout.strip().splitlines()[-1])["n_gpus"] == 1
