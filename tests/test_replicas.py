"""The multi-GPU path of bench.py is replicas only (independent solves, no
data-path collective).  Its host logic runs here on CPU with gloo, world size
2: the step time is the max over ranks and the job throughput counts every
replica; the reference arm prints one line from rank 0 only."""
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
    m = bench.max_over_ranks(ms, dist, device="cpu")
    out[rank] = (m, bench.replicas_throughput(world, 4, m))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, 29517, out), nprocs=world, join=True, start_method="spawn")
    assert out[0][0] == out[1][0] == 150.0
    assert out[0][1] == pytest.approx(2 * 4 / 0.150)


def test_reference_arm_under_two_ranks_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", "29518", os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--workload", "mol60", "--steps", "1", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and '"impl": "reference"' in lines[0]


def test_gpus_flag_spawns_replicas_without_torchrun():
    """`bench.py --gpus 2` started as a plain process (no WORLD_SIZE) starts
    its own two ranks; rank 0 alone prints the line, which names 2 GPUs."""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference",
           "--workload", "mol60", "--steps", "1", "--warmup", "3"]
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    env["OMP_NUM_THREADS"] = "2"
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1 and '"impl": "reference"' in lines[0] and '"n_gpus": 2' in lines[0]
