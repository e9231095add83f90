"""CPU tests of the N>1 host path (gloo, world size 2): replicas need no data-path collective,
only the barrier and the max-over-ranks time, and the reference arm runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bench.barrier(world)
    got = bench.max_over_ranks(1.5 + rank, world)
    dist.destroy_process_group()
    with open(os.path.join(out, f"r{rank}.txt"), "w") as f:
        f.write(repr(got))


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        assert float(open(tmp_path / f"r{r}.txt").read()) == 2.5


def test_reference_arm_under_torchrun_prints_once():
    env = dict(os.environ, CSM_REF_BUDGET_S="2", PYTHONPATH=os.path.join(ROOT, "gcsm-bu_b200"))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "3",
           "--config", "c1", "--scale", "0.2"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["value"] >= 0
