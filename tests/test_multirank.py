"""Multi-process host logic of the bench on the CPU (gloo, two ranks): the
max-over-ranks step time, the whole-job rate, per-rank workload shards, and
the reference arm printing one line from rank 0 under torchrun.  The path
has no collective on the data (every rank verifies its own shard)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402
import workload as WL  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(dist, 10.0 + rank, "cpu")
        wl = WL.config_keyset(40, 4, seed=bench.SEED + rank)
        out.put((rank, t, [int(x) for x in wl["sigs"][0][:2]], int(wl["expect"].sum())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_shards_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    assert [g[1] for g in got] == [11.0, 11.0]          # every rank sees the slowest rank's time
    assert got[0][2] != got[1][2]                       # distinct shards
    assert all(g[3] == 35 for g in got)                 # 1 in 8 of 40 corrupted: 35 accepted


def test_whole_job_rate():
    assert bench.whole_job_rate(4096, 2, 10, 2.0) == 4096 * 2 * 10 / 2.0
    assert bench.max_over_ranks(None, 3.5, "cpu") == 3.5


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_prints_one_line():
    env = dict(os.environ)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["cores"] >= 1
