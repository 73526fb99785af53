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


# ---------------------------------------------------------------------------
# The product's multi-rank paths, run as gloo ranks on CPU.
# ---------------------------------------------------------------------------
NX, NY, N, T = 30, 28, 4, 70
SRC = [(10, 9), (19, 17), (14, 21), (8, 18), (21, 8)]
FREQS = np.linspace(1e9, 3e9, 7)


def _maps():
    x, y = np.meshgrid(np.arange(NX), np.arange(NY), indexing="ij")
    m = (x - 15) ** 2 + (y - 14) ** 2 <= 6 ** 2
    return np.where(m, 6.0, 1.0), np.where(m, 0.4, 0.0), np.where(m, 18.0, 0.0), np.where(m, 8e-12, 0.0)


def _txsplit_gradient(target, split):
    """Gradient of the S misfit through the FP64 restatement of the solver,
    with this rank's transmit events only when `split` (the Adjoint2D
    reduce_ranks recipe: split_sources, local_columns, allreduce_gradient)."""
    from ceep_b200.distributed import allreduce_gradient, local_columns, split_sources, sum_over_ranks
    from oracle.torch_fdtd2d import TorchFdtd2D, s_misfit_loss
    src = split_sources(SRC)[0] if split else SRC
    t = TorchFdtd2D(NX, NY, 0.5e-3, T, N, src, SRC, 2e9)
    eps, sig, de, tau = (torch.tensor(a, dtype=torch.float64) for a in _maps())
    eps.requires_grad_(True)
    sig.requires_grad_(True)
    de.requires_grad_(True)
    tgt = local_columns(target, len(SRC)) if split else target
    loss, _ = s_misfit_loss(t.run(eps, sig, [(de, tau)]), t.dt, FREQS, tgt)
    loss.backward()
    g = {"eps_r": eps.grad, "sigma": sig.grad, "deps": de.grad}
    if split:
        g = allreduce_gradient(g)
        loss = sum_over_ranks(loss)
    return float(loss.detach()), {k: v.numpy() for k, v in g.items()}


def _target():
    g = torch.Generator().manual_seed(5)
    return 1e-14 * torch.complex(torch.randn(len(FREQS), len(SRC), len(SRC), generator=g, dtype=torch.float64),
                                 torch.randn(len(FREQS), len(SRC), len(SRC), generator=g, dtype=torch.float64))


def _dataset_fake_batch(specs, nx, ny, dx, frequency, n_ant, total_steps, device=None, **kw):
    """CPU stand-in for simulate_batch: values that depend only on the sample id."""
    B, T_ = len(specs), total_steps or 3
    ids = torch.tensor([s.sample_id for s in specs], dtype=torch.float64)
    eps = ids[:, None, None] + torch.zeros(B, nx, ny, dtype=torch.float64)
    series = (ids[:, None, None, None] + 1.0) * torch.ones(B, n_ant, n_ant, T_, dtype=torch.float64)
    return eps, eps * 0.1, eps * 0, series, T_


def _product_worker(rank, size, port, q, tmp):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=timedelta(seconds=120))
    try:
        res = {}
        res["loss"], res["grad"] = _txsplit_gradient(_target(), split=True)
        from ceep_b200 import dataset as ds
        ds.simulate_batch = _dataset_fake_batch
        meta = ds.generate_dataset(n_samples=11, output_dir=tmp, nx=6, ny=6, n_ant=3, total_steps=4, seed=3,
                                   batch=2, device="cpu")
        meta.pop("generation_seconds"), meta.pop("samples_per_second")
        res["meta"] = meta
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_tx_split_gradient_and_sharded_dataset(tmp_path):
    size = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_product_worker, args=(r, size, port, q, str(tmp_path / "ds"))) for r in range(size)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=300) for _ in range(size))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # TX-split gradient == whole-batch gradient, on every rank
    loss1, g1 = _txsplit_gradient(_target(), split=False)
    for r in range(size):
        assert abs(out[r]["loss"] - loss1) <= 1e-12 * abs(loss1)
        for k in g1:
            np.testing.assert_allclose(out[r]["grad"][k], g1[k], rtol=1e-10, atol=1e-12 * np.abs(g1[k]).max())
    # sharded dataset: every sample written once, the same metadata on every rank
    from ceep_b200 import dataset as ds
    files = sorted(os.listdir(tmp_path / "ds" / "s_matrix"))
    assert files == [f"sample_{i:06d}.npy" for i in range(11)]
    for i in range(11):
        assert np.load(tmp_path / "ds" / "s_matrix" / f"sample_{i:06d}.npy")[0, 0, 0] == i + 1.0
    assert out[0]["meta"] == out[1]["meta"] and out[0]["meta"]["ranks"] == 2
    ds.simulate_batch = _dataset_fake_batch
    single = ds.generate_dataset(n_samples=11, output_dir=str(tmp_path / "one"), nx=6, ny=6, n_ant=3,
                                 total_steps=4, seed=3, batch=2, device="cpu")
    assert single["s_matrix_statistics"] == out[0]["meta"]["s_matrix_statistics"]
