"""Multi-rank host logic on CPU with the gloo backend (world size 2 and 3)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, size, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=timedelta(seconds=60))
    try:
        from ceep_b200.distributed import allreduce_gradient, gather_tx_split, max_time_ms, shard, tx_range
        res = {}
        items = list(range(23))
        res["shard"] = shard(items, rank, size)
        # S[f, rx, tx] of 13 transmit events split over ranks
        ntx, F, P = 13, 5, 4
        full = torch.arange(F * P * ntx, dtype=torch.float64).reshape(F, P, ntx) * (1 + 1j)
        mine = full[:, :, list(tx_range(ntx, rank, size))]
        res["gather_ok"] = bool(torch.equal(gather_tx_split(mine, ntx, axis=-1), full))
        series = torch.randn(ntx, P, 30, generator=torch.Generator().manual_seed(1))
        res["series_ok"] = bool(torch.equal(gather_tx_split(series[list(tx_range(ntx, rank, size))], ntx, axis=0),
                                            series))
        g = {"eps_r": torch.full((4, 3), float(rank + 1), dtype=torch.float64)}
        res["grad"] = float(allreduce_gradient(g)["eps_r"][0, 0])
        res["tmax"] = max_time_ms(10.0 * (rank + 1))
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("size", [2, 3])
def test_distributed_host_logic(size):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, size, port, q)) for r in range(size)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(size))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = [out[r]["shard"] for r in range(size)]
    assert sorted(sum(shards, [])) == list(range(23))
    assert max(map(len, shards)) - min(map(len, shards)) <= 1
    for r in range(size):
        assert out[r]["gather_ok"] and out[r]["series_ok"]
        assert out[r]["grad"] == sum(range(1, size + 1))
        assert out[r]["tmax"] == 10.0 * size
