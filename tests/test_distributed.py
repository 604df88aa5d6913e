"""Sharding one waveform across ranks (host logic and collectives), on CPU with
the gloo backend and world size 2; the kernels' part is played by the oracle
evaluated on each rank's samples."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fastemriwaveforms_b200 import distributed as D


def test_shard_ranges_tile_the_output():
    for out_len in (1, 7, 100, 100001):
        for world in (1, 2, 3, 8):
            rs = [D.shard_range(out_len, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == out_len
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            sizes = [h - l for l, h in rs]
            assert max(sizes) - min(s for s in sizes if s > 0) <= -(-out_len // world)


def test_restrict_units_and_clip():
    units = np.array([0, 0, 10, 0, 10, 13, 1, 13, 20, 2, 20, 31], np.int32)
    got = D.restrict_units(units, 12, 25).reshape(-1, 3)
    assert got.tolist() == [[0, 12, 13], [1, 13, 20], [2, 20, 25]]
    assert D.clip_seg_start(np.array([0, 13, 20, 31]), 12, 25).tolist() == [12, 13, 20, 25]
    assert D.restrict_units(units, 40, 50).size == 0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from conftest import load_case
        from oracle import oracle as O

        inp, ref = load_case("sum_small_m0.npz")
        out_len = len(ref)
        lo, hi = D.shard_range(out_len, rank, world)
        local = torch.zeros(out_len, dtype=torch.complex128)
        if hi > lo:
            local[lo:hi] = torch.from_numpy(O.mode_sum(inp, window=(lo, hi))[lo:hi])
        full = D.gather_waveform(local, out_len, rank, world)
        # gradients: each rank's partial, summed by the reduction
        g = torch.full((5, 3), float(rank + 1), dtype=torch.complex128) * (1 + 2j)
        r = torch.arange(8, dtype=torch.float64) * (rank + 1)
        D.reduce_gradients([g, r])
        q.put((rank, float(np.abs(full.numpy() - ref).max() / np.abs(ref).max()), g.numpy().tolist(),
               r.numpy().tolist()))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_gather_and_reduce():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, err, g, r in results:
        assert err == 0.0  # the oracle's windows are the oracle's whole waveform, sample for sample
        assert np.allclose(np.array(g), 3 * (1 + 2j))
        assert np.allclose(np.array(r), np.arange(8) * 3.0)
