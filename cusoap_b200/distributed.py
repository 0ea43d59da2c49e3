"""Multi-GPU sharding of the SOAP path: one process per GPU, torch.distributed.

Descriptor rows and Jacobian blocks are independent per centre, so each rank
computes a contiguous range of centres with no data-path collective (outputs
stay sharded; ``gather_rows`` brings them to every rank when a caller wants
them together).  Forces of E = sum_c w_c . p_c need one exchange: a rank's
adjoint gives the forces of its own centres' energy on every atom (its
centres' neighbours include atoms of other shards), and one all-reduce (sum)
of the (n_atoms, 3) array completes them.  This is how the reference's
multi-process example shards work across devices (examples/test_mp.py:91-167:
contiguous centre ranges per process, results gathered on the host), with the
force reduction added.  Collectives are NCCL on GPUs, gloo on CPU.
"""
from __future__ import annotations

from typing import Any, Callable, Optional, Sequence, Tuple

import torch
import torch.distributed as dist


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """[lo, hi) of the contiguous block of ``n`` items owned by ``rank``
    (sizes differ by at most one, lower ranks take the extra ones)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of world {world}")
    base, extra = divmod(int(n), world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _world(group) -> Tuple[int, int]:
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def allreduce_sum(t: torch.Tensor, group=None) -> torch.Tensor:
    """In-place sum over the ranks of ``group`` (no-op without a process group)."""
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def sharded_create(soap, system: Any, group=None):
    """This rank's centres [lo, hi) of ``system`` (every atom a centre) and
    their descriptor rows ((0, F) for an empty shard); no collective."""
    rank, world = _world(group)
    n = len(system["atomic_numbers"]) if isinstance(system, dict) else len(system)
    lo, hi = shard_range(n, rank, world)
    if hi > lo:
        rows = soap.create(system, centers=list(range(lo, hi)))
    else:
        rows = torch.zeros((0, soap.get_number_of_features()), dtype=soap.dtype, device=soap.device)
    return lo, hi, rows


def gather_rows(rows: torch.Tensor, n_total: int, group=None) -> torch.Tensor:
    """All ranks' descriptor rows, in centre order, on every rank.

    One all-gather of equal-size shards (each rank's rows padded to the
    largest shard, at most one row of padding), so every rank receives
    n_total rows plus the padding; the padding rows are dropped."""
    rank, world = _world(group)
    if world == 1:
        return rows
    spans = [shard_range(n_total, r, world) for r in range(world)]
    lo, hi = spans[rank]
    if rows.shape[0] != hi - lo:
        raise ValueError(f"rank {rank} holds {rows.shape[0]} rows, its shard is [{lo}, {hi})")
    width = max(b - a for a, b in spans)
    F = rows.shape[1]
    send = torch.zeros((width, F), dtype=rows.dtype, device=rows.device)
    send[:hi - lo] = rows
    recv = torch.empty((world * width, F), dtype=rows.dtype, device=rows.device)
    dist.all_gather_into_tensor(recv, send, group=group)
    return torch.cat([recv[r * width:r * width + (b - a)] for r, (a, b) in enumerate(spans)])


def partial_forces(soap, system: dict, w: torch.Tensor, lo: int, hi: int):
    """(E_part, F_part): the energy sum_{c in [lo, hi)} w . p_c of centres
    lo..hi-1 and minus its gradient on every atom, from one adjoint pass."""
    pos = torch.as_tensor(system["positions"], dtype=torch.float64, device=soap.device).clone().requires_grad_(True)
    sysd = dict(system, positions=pos)
    if hi <= lo:
        return torch.zeros((), dtype=torch.float64, device=soap.device), torch.zeros_like(pos)
    desc = soap.create(sysd, centers=list(range(lo, hi)))
    E = (desc * w.to(desc.dtype)).sum()
    E.backward()
    return E.detach().to(torch.float64), -pos.grad


def sharded_energy_forces(soap, system: dict, w: torch.Tensor, group=None,
                          compute: Optional[Callable] = None):
    """E = sum_c w . p_c over all centres and the forces -dE/dx, with this
    rank computing its centre shard and one all-reduce of (E, forces).
    ``compute(lo, hi) -> (E_part, F_part)`` replaces the GPU adjoint (tests
    drive the reduction with a CPU stand-in)."""
    rank, world = _world(group)
    n = len(system["atomic_numbers"])
    lo, hi = shard_range(n, rank, world)
    E, F = compute(lo, hi) if compute is not None else partial_forces(soap, system, w, lo, hi)
    E = torch.as_tensor(E, dtype=torch.float64, device=F.device).reshape(1).clone()
    F = F.clone()
    allreduce_sum(E, group)
    allreduce_sum(F, group)
    return float(E.item()), F
