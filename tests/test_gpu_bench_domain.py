"""bench.py's multi-GPU line (the lattice split along t, one slab per rank,
the 16-bit domain solve) run as two ranks under torchrun on the one GPU of
this machine, exchanging through host memory over gloo: no kernel waits on
the other rank.  The line must carry the contract's keys and a converged
solve."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_bench_two_rank_domain_line(cuda):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"),
           "--gpus", "2", "--steps", "2", "--warmup", "1", "--dims", "16,16,16,16", "--transport", "host"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT,
                       env={**os.environ, "OMP_NUM_THREADS": "4"})
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "config", "roofline", "e2e", "clocks", "gpu_launches"):
        assert key in d, key
    assert d["n_gpus"] == 2 and d["scaling"] == "weak" and d["value"] > 0
    assert d["config"]["lattice"] == [16, 16, 16, 32]
    assert d["true_r2"] <= 1e-20 and d["iterations"] > 0
