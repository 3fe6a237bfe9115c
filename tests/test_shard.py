"""The multi-GPU decomposition on CPU: two gloo ranks each take a band of
output rows (shard.row_band) with its halo (shard.band_strip), run the
oracle on it, and gather the bands; the gathered coherence and counts equal
those of the whole region bit for bit, and the max-over-ranks reduction of
a step time is what every rank sees."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from conftest import Case

import tcoh_b200.shard as shard


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, name, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = Case(name)
        kw = c.kwargs()
        band = shard.row_band(c.rows, world, rank)
        slc, amp, valid = shard.band_strip(c.stack.real, c.stack.imag, band, c.window,
                                           phase=c.phase)
        o = oracle.run_oracle(slc, amp, valid, band[1] - band[0], c.cols, **kw)
        parts = [None] * world
        dist.all_gather_object(parts, (band, o["coh"], o["count"]))
        t = torch.tensor([10.0 + rank])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            np.savez(os.path.join(out_dir, "gathered.npz"),
                     coh=np.concatenate([p[1] for p in parts]),
                     count=np.concatenate([p[2] for p in parts]),
                     bands=np.array([p[0] for p in parts]), tmax=t.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 8])
def test_row_bands_cover_the_region(world):
    for rows in (1, 2, 5, 16, 30, 31, 4096):
        bands = [shard.row_band(rows, world, r) for r in range(world)]
        # with more ranks than rows, the surplus ranks (the last ones) get none
        live = [b for b in bands if b is not None]
        assert len(live) == min(rows, world)
        assert all(b is None for b in bands[len(live):])
        assert live[0][0] == 0 and live[-1][1] == rows
        assert all(a[1] == b[0] for a, b in zip(live, live[1:]))
        sizes = [b[1] - b[0] for b in live]
        assert min(sizes) >= 1 and max(sizes) - min(sizes) <= 1


def test_a_rank_without_rows_has_no_strip():
    re = np.zeros((3, 2, 4), np.float32)
    assert shard.row_band(2, 4, 3) is None
    assert shard.band_strip(re, re, shard.row_band(2, 4, 3), (5, 3)) is None
    slc, amp, valid = shard.band_strip(re, re, shard.row_band(2, 4, 1), (5, 3))
    assert valid.shape == (1 + 4, 4 + 2)


def test_two_gloo_ranks_reassemble_the_region(tmp_path):
    name = "topographic"
    world = 2
    mp.start_processes(rank_main, args=(world, free_port(), name, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    g = np.load(tmp_path / "gathered.npz")
    c = Case(name)
    slc, amp, valid = shard.band_strip(c.stack.real, c.stack.imag, (0, c.rows), c.window,
                                       phase=c.phase)
    whole = oracle.run_oracle(slc, amp, valid, c.rows, c.cols, **c.kwargs())
    assert [tuple(b) for b in g["bands"]] == [shard.row_band(c.rows, world, r) for r in range(world)]
    assert np.array_equal(g["count"], whole["count"])
    assert np.array_equal(np.isnan(g["coh"]), np.isnan(whole["coh"]))
    assert np.array_equal(g["coh"][~np.isnan(g["coh"])], whole["coh"][~np.isnan(whole["coh"])])
    assert float(g["tmax"][0]) == 10.0 + world - 1
