"""The multi-GPU bench path (replicas, no data-path collective) on CPU: two gloo ranks agree on the
slowest rank's time and on the whole-job throughput, and the reference arm prints from rank 0 only."""
import os
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    seconds = [1.5, 2.5][rank]  # rank 1 is the slow replica
    worst = bench.max_over_ranks(seconds, dist, "cpu")
    out[rank] = (worst, bench.replica_value(1000, world, 4, worst))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas_report_the_slowest_rank():
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1] == (2.5, 2 * 1000 * 4 / 2.5)


@pytest.mark.slow
def test_reference_arm_prints_one_line_from_rank_zero_under_torchrun():
    env = dict(os.environ, PYTHONPATH=ROOT)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2", "--master-addr",
           "127.0.0.1", "--master-port", str(30500 + os.getpid() % 1000), os.path.join(ROOT, "bench.py"), "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and '"impl": "reference"' in lines[0]
