"""Multi-process plumbing of the field path on CPU (gloo, world size 2):
process-group set-up, barrier, max over ranks, the per-rank point sets of the
weak-scaling run and the block split of a fixed set; and the bench's
torchrun launch contract with two ranks (reference arm: rank 0 prints the
one JSON line, the other rank exits 0 without work)."""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import numpy as np

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from bielcc_b200 import replicas
    from bielcc_b200 import workloads as W

    w, r, local = replicas.env()
    backend = replicas.init(w, local, backend="gloo", timeout_s=60)
    m = replicas.max_over_ranks(w, 1.5 * (r + 1), local)
    replicas.barrier(w)
    cells = W.uv_sphere(8, 16)
    pts = replicas.rank_points(cells, r, n_far=40, n_near=8)
    q.put((r, backend, m, pts, replicas.shard(103, w, r)))
    dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=180) for _ in range(2)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == ["gloo", "gloo"]
    assert [r[2] for r in res] == [3.0, 3.0]
    p0, p1 = res[0][3], res[1][3]
    assert p0.shape == p1.shape == (48, 3) and not np.allclose(p0, p1)
    (a0, b0), (a1, b1) = res[0][4], res[1][4]
    assert a0 == 0 and b0 == a1 and b1 == 103 and abs((b0 - a0) - (b1 - a1)) <= 1


def test_shard_covers_and_balances():
    from bielcc_b200 import replicas

    for n in (0, 1, 7, 64, 1001):
        for ws in (1, 2, 3, 8):
            parts = [replicas.shard(n, ws, r) for r in range(ws)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(ws - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


def test_bench_reference_arm_two_ranks():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="4")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")
