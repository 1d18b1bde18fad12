"""The multi-GPU path of bench.py, run as two gloo ranks on the CPU.

Worlds are sharded across ranks with no exchange on the step path; the only collectives are the whole-job
aggregation (sum of the units all ranks processed over the slowest rank's time) and barriers. The test runs that
aggregation exactly as bench.py does, with rank 1 deliberately slower, and checks that every rank takes the same
collective steps. Each rank builds its share of the job's worlds host-side (greedy body-count balancing, as
bench.py shards the batched-worlds workload); the shares must be disjoint, cover the job and be balanced.
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
        worlds = 8   # per rank: the job is 16 worlds
        share = bench.c4_shard(worlds, rank, world_size)
        scene_list = scenes.make_c4_worlds(worlds=worlds * world_size, seed=0, subset=share)
        counts = scenes.c4_counts(worlds * world_size, 0)
        assert [s.n for s in scene_list] == [int(counts[k]) + 1 for k in share]   # + the ground box
        bodies = sum(s.n for s in scene_list)
        steps = 10
        seconds = 0.5 * (rank + 1)   # rank 1 is the slowest
        rate, slowest, total = bench.job_rate(torch, dist, world_size, torch.device("cpu"), bodies * steps, seconds)
        dist.barrier()
        out[rank] = (rate, slowest, total, bodies, [float(s.px.sum()) for s in scene_list], share,
                     int(sum(int(counts[k]) for k in share)), int(counts.max()))
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation_and_sharding():
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    (rate0, slow0, total0, b0, px0, sh0, load0, big), (rate1, slow1, total1, b1, px1, sh1, load1, _) = out[0], out[1]
    # Every rank computes the same whole-job figures: the sum of all ranks' body-steps over the slowest rank's time.
    assert slow0 == slow1 == 1.0
    assert total0 == total1 == float((b0 + b1) * 10)
    assert rate0 == rate1 == total0 / 1.0
    # The shares are disjoint, cover the job's 16 worlds and are balanced to within one world.
    assert not set(sh0) & set(sh1)
    assert sorted(sh0 + sh1) == list(range(16))
    assert abs(load0 - load1) <= big
    assert px0 != px1
