"""The multi-GPU path of bench.py, run as two gloo ranks on the CPU.

Worlds are sharded across ranks with no exchange on the step path; the only collectives are the whole-job
aggregation (sum of the units all ranks processed over the slowest rank's time) and barriers. The test runs that
aggregation and the per-rank seeding exactly as bench.py does, with rank 1 deliberately slower, and checks that
every rank takes the same collective steps.
"""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world_size, port, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "physicssimulation-agony_b200"))
    import bench
    from ag2d import scenes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world_size),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method="env://", rank=rank, world_size=world_size)
    try:
        r, ws, local = bench.dist_env()
        assert (r, ws, local) == (rank, world_size, rank)
        worlds = 3
        scene_list = scenes.make_c4_worlds(worlds=worlds, seed=bench.rank_seed(rank, worlds), lo=16, hi=64)
        bodies = sum(s.n for s in scene_list)
        steps = 10
        seconds = 0.5 * (rank + 1)   # rank 1 is the slowest
        rate, slowest, total = bench.job_rate(torch, dist, world_size, torch.device("cpu"), bodies * steps, seconds)
        dist.barrier()
        out[rank] = (rate, slowest, total, bodies, [float(s.px.sum()) for s in scene_list])
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation_and_sharding():
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    (rate0, slow0, total0, b0, px0), (rate1, slow1, total1, b1, px1) = out[0], out[1]
    # Every rank computes the same whole-job figures: the sum of all ranks' body-steps over the slowest rank's time.
    assert slow0 == slow1 == 1.0
    assert total0 == total1 == float((b0 + b1) * 10)
    assert rate0 == rate1 == total0 / 1.0
    # The ranks' worlds are disjoint draws (seeds rank * worlds + k).
    assert px0 != px1
