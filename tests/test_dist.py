"""The multi-process path on CPU: two gloo ranks on 127.0.0.1 exchange only the timing
(max over ranks), and the strong-scaling shard covers every code exactly once."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from qubitserf_b200 import dist
    r, w, local, pg = dist.init_from_env(timeout_s=60)
    assert (r, w, local) == (rank, world, rank) and os.environ["QSFB_DEVICE"] == str(rank)
    m = dist.max_over_ranks(pg, 10.0 + rank)
    s = dist.sum_over_ranks(pg, 1.0)
    dist.barrier(pg)
    mine = dist.shard(list(range(37)), r, w)
    parts = dist.gather_to_root(pg, [10 * i for i in mine], w)
    whole = dist.unshard(parts) if r == 0 else None
    q.put((rank, m, s, mine, whole))
    pg.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [11.0, 11.0]
    assert [o[2] for o in out] == [2.0, 2.0]
    covered = sorted(out[0][3] + out[1][3])
    assert covered == list(range(37))
    # rank 0 rebuilds every code's answer in batch order from the two shards
    assert out[0][4] == [10 * i for i in range(37)] and out[1][4] is None


def test_single_process_defaults(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from qubitserf_b200 import dist
    r, w, local, pg = dist.init_from_env()
    assert (r, w, local, pg) == (0, 1, 0, None)
    assert dist.max_over_ranks(None, 3.5) == 3.5


def test_reference_arm_under_torchrun():
    """`bench.py --impl reference` launched as two ranks: rank 0 alone prints one line."""
    import json
    import subprocess
    import sys
    from conftest import ROOT
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--codes", "64", "--ref-stride", "64"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0
