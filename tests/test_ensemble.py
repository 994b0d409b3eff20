"""Multi-rank replica ensembles on CPU: two gloo ranks stand for two GPUs.
Checks the seeds each rank gives its replicas, the max-over-ranks step time
and the ensemble sums of structure functions and Hamiltonians."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_data(rank, R=3, shape=(4, 3, 3)):
    rng = np.random.default_rng(100 + rank)
    sf = rng.normal(size=(R,) + shape) + 1j * rng.normal(size=(R,) + shape)
    h = rng.normal(size=R)
    return {"A,B": sf, "H": h}


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from langevinfts_b200.ensemble import ensemble_sum, max_over_ranks, replica_seeds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        sums, n = ensemble_sum(_rank_data(rank))
        t = max_over_ranks([1.0 + rank, 5.0 - rank])
        out[rank] = (replica_seeds(rank, 3), sums["A,B"], sums["H"], n, t)
    finally:
        dist.destroy_process_group()


def test_two_rank_ensemble():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    seeds = [out[r][0] for r in range(world)]
    assert not set(seeds[0]) & set(seeds[1])
    expect_sf = sum(_rank_data(r)["A,B"].sum(axis=0) for r in range(world))
    expect_h = sum(_rank_data(r)["H"].sum() for r in range(world))
    for r in range(world):
        _, sf, h, n, t = out[r]
        assert n == 6
        np.testing.assert_allclose(sf, expect_sf, rtol=1e-12)
        np.testing.assert_allclose(h, expect_h, rtol=1e-12)
        assert t == [2.0, 5.0]


def test_single_process_fallback():
    from langevinfts_b200.ensemble import ensemble_sum, max_over_ranks
    sums, n = ensemble_sum(_rank_data(0))
    assert n == 3
    np.testing.assert_allclose(sums["A,B"], _rank_data(0)["A,B"].sum(axis=0))
    assert max_over_ranks([1.5]) == [1.5]
