"""Host-side logic for running the batched path on several GPUs.

Phantoms are independent and so are the transmit events of one phantom, so
the path shards with no halo exchange (one process per GPU, torch.distributed
over NCCL on NVLink for the few collectives it needs):

* ``shard``               contiguous block of a work list for this rank;
* ``gather_tx_split``     reassemble S[f, rx, tx] (or probe series) of a phantom
                          whose transmit events were split across ranks;
* ``allreduce_gradient``  sum per-rank gradient maps of a TX-split adjoint;
* ``max_time_ms``         the slowest rank's device time, for throughput;
* ``split_sources`` / ``local_columns``  this rank's transmit events of a
                          solver and the matching columns of a full S target;
* ``sum_over_ranks`` / ``gather_objects``  reduce a loss value, collect
                          per-rank host results (dataset statistics).

The product uses them in three places: ``Adjoint2D`` / ``Adjoint3D`` with
``reduce_ranks=True`` (a TX-split gradient: each rank's loss covers its own
transmit events, one all_reduce of the gradient maps), ``generate_dataset``
(samples sharded over ranks, statistics gathered) and ``bench.py --gpus N``
(phantoms sharded over ranks).  None of these touches the data path inside a
time step.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import torch
import torch.distributed as dist


def world() -> Tuple[int, int]:
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(items: Sequence, rank: int, size: int) -> List:
    """Contiguous block of ``items`` for ``rank`` (sizes differ by at most one)."""
    n = len(items)
    lo = rank * n // size
    hi = (rank + 1) * n // size
    return list(items[lo:hi])


def tx_range(ntx: int, rank: int, size: int) -> range:
    return range(rank * ntx // size, (rank + 1) * ntx // size)


def gather_tx_split(local: torch.Tensor, ntx: int, axis: int = -1) -> torch.Tensor:
    """Concatenate per-rank slices along the TX axis (ranks own contiguous TX
    ranges from ``tx_range``); every rank receives the full tensor."""
    rank, size = world()
    if size == 1:
        return local
    local = local.contiguous()
    counts = [len(tx_range(ntx, r, size)) for r in range(size)]
    shape = list(local.shape)
    ax = axis % local.dim()
    parts = []
    for r in range(size):
        shape[ax] = counts[r]
        parts.append(torch.empty(shape, dtype=local.dtype, device=local.device))
    if local.is_complex():
        rl = torch.view_as_real(local).contiguous()
        rparts = [torch.view_as_real(p) for p in parts]
        _all_gather_ragged(rparts, rl)
    else:
        _all_gather_ragged(parts, local)
    return torch.cat(parts, dim=ax)


def _all_gather_ragged(out: List[torch.Tensor], local: torch.Tensor) -> None:
    # pad to a common size so the backend sees equal-shaped buffers
    numel = max(p.numel() for p in out)
    buf = torch.zeros(numel, dtype=local.dtype, device=local.device)
    buf[:local.numel()] = local.reshape(-1)
    recv = [torch.empty_like(buf) for _ in out]
    dist.all_gather(recv, buf)
    for p, r in zip(out, recv):
        p.copy_(r[:p.numel()].reshape(p.shape))


def allreduce_gradient(grads: dict) -> dict:
    """Sum gradient maps over ranks (a TX-split adjoint: each rank's loss term
    covers its own transmit events, the materials are shared)."""
    rank, size = world()
    if size == 1:
        return grads
    for k in sorted(grads):
        dist.all_reduce(grads[k], op=dist.ReduceOp.SUM)
    return grads


def max_time_ms(ms: float, device=None) -> float:
    rank, size = world()
    if size == 1:
        return ms
    t = torch.tensor([ms], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def split_sources(positions: Sequence, rank: int = None, size: int = None):
    """This rank's contiguous block of transmit events: (positions, tx range).
    A solver built with these sources and every probe gives this rank's
    columns S[:, :, tx_range] of the full multistatic matrix."""
    if rank is None or size is None:
        rank, size = world()
    r = tx_range(len(positions), rank, size)
    return [positions[i] for i in r], r


def local_columns(target: torch.Tensor, ntx: int, axis: int = -1, rank: int = None, size: int = None):
    """The slice of a full per-TX array (S target, probe series) along `axis`
    that belongs to this rank's transmit events."""
    if rank is None or size is None:
        rank, size = world()
    r = tx_range(ntx, rank, size)
    idx = [slice(None)] * target.dim()
    idx[axis] = slice(r.start, r.stop)
    return target[tuple(idx)]


def sum_over_ranks(value: torch.Tensor) -> torch.Tensor:
    """Sum of a tensor over ranks (a copy; the input is not modified)."""
    rank, size = world()
    out = value.detach().clone()
    if size > 1:
        dist.all_reduce(out, op=dist.ReduceOp.SUM)
    return out


def gather_objects(obj) -> List:
    """Every rank's `obj` (picklable), in rank order, on every rank."""
    rank, size = world()
    if size == 1:
        return [obj]
    out = [None] * size
    dist.all_gather_object(out, obj)
    return out
