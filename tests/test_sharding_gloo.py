"""Multi-rank host logic on CPU: two gloo ranks reduce their device times to
the max, split the views, agree on the whole-job rate, and sum the gradient
vectors of their views for inverse rendering."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from crisoptix_b200 import sharding


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r "measured" 10 + r ms; everyone must see the slowest rank's time
        ms = sharding.max_over_ranks(10.0 + rank, dist)
        e2e = sharding.max_over_ranks(20.0 - rank, dist)
        rate = sharding.whole_job_rate(1000.0, 5, world, ms)
        views = sharding.assign_views([512 * 512] * 8 + [1280 * 720] * 4 + [1920 * 1080] * 4, world)
        # inverse rendering: 8 views of 512^2 split across ranks, each rank's
        # gradient from its own views (here: view index + 1 per entry), summed
        inv = sharding.assign_views([512 * 512] * 8, world)[rank]
        g_mat = torch.full((321, 7), float(sum(v + 1 for v in inv)))
        g_em = torch.full((256, 3), -float(sum(v + 1 for v in inv)))
        sharding.sum_gradients(g_mat, g_em, dist)
        out[rank] = (ms, e2e, rate, sharding.orbit_offset(rank, world), views, inv,
                     float(g_mat[5, 3]), float(g_em[100, 2]), float(g_mat.sum()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    assert sorted(out.keys()) == [0, 1]
    for r in range(world):
        ms, e2e, rate, _, views, inv, gm, ge, gsum = out[r]
        assert ms == 11.0  # max over ranks, not the rank's own time
        assert e2e == 20.0
        assert rate == pytest.approx(1000.0 * 5 * world / 0.011)
        assert views == out[0][4]  # every rank computes the same split
        assert len(inv) == 4  # 4 of the 8 inverse-rendering views per rank
        # every rank holds the sum over all 8 views: 1 + 2 + ... + 8 = 36
        assert gm == 36.0 and ge == -36.0 and gsum == 36.0 * 321 * 7
    assert sorted(out[0][5] + out[1][5]) == list(range(8))
    assert out[0][3] == 0 and out[1][3] == 30  # distinct views of the 60-frame orbit


def test_assign_views_partitions_and_balances():
    pixels = [512 * 512] * 8 + [1280 * 720] * 4 + [1920 * 1080] * 4
    for world in (1, 2, 3, 4, 8):
        split = sharding.assign_views(pixels, world)
        flat = sorted(v for vs in split for v in vs)
        assert flat == list(range(len(pixels)))
        loads = [sum(pixels[v] for v in vs) for vs in split]
        # LPT bound: no rank exceeds the ideal share by more than the largest view
        assert max(loads) <= sum(pixels) / world + max(pixels)


def test_single_rank_identity():
    assert sharding.max_over_ranks(3.5, None) == 3.5
    g_mat, g_em = torch.ones(3, 7), torch.ones(2, 3)
    a, b = sharding.sum_gradients(g_mat, g_em, None)
    assert a is g_mat and float(a.sum()) == 21.0 and float(b.sum()) == 6.0
    assert sharding.orbit_offset(0, 1) == 0
    with pytest.raises(ValueError):
        sharding.orbit_offset(2, 2)
    with pytest.raises(ValueError):
        sharding.whole_job_rate(1.0, 1, 1, 0.0)
