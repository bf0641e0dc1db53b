"""The multi-GPU (replica) plumbing of bench.py on CPU: two gloo ranks.

`bench.py --gpus N` under torchrun runs one replica per rank, each on its own
scene, with no collective on the data path; the only exchanges are the
barrier and the maximum of the per-rank times.  This test runs that logic
with the gloo backend, world size 2, on 127.0.0.1.
"""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = [12.5, 17.25][rank]
        ms = bench.max_over_ranks(local_ms, dist, "cpu")
        dist.barrier()
        seeds = [None] * world
        dist.all_gather_object(seeds, bench.replica_seed(rank))
        out[rank] = (ms, seeds, bench.aggregate_mpix(world, 4096, ms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_filter_distinct_scenes():
    world, port = 2, _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ms, seeds, mpix = res[r]
        assert ms == 17.25
        assert len(set(seeds)) == world
        assert mpix == pytest.approx(2 * 4096 * 4096 / 17.25e-3 / 1e6)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
