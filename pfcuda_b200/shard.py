"""Batch sharding over ranks (one process per GPU).

Matrices are independent, so a batch splits across GPUs with no data exchange
during the factorisation; the reference has no multi-GPU path (its handlers
loop over the batch on one device, bindings/jax_bindings.cu:37-80).  This
module holds the host-side logic:

* ``shard_range``  -- the contiguous slice of a uniform batch a rank owns;
* ``shard_ragged`` -- a balanced assignment of a ragged batch, by the O(n^3)
  work of each matrix (longest-processing-time first, ties to the lower rank);
* ``slog_pfaffian_sharded`` -- each rank factors its slice of a uniform batch
  and, if asked, the per-matrix results are gathered on every rank with one
  all_gather of (log|Pf|, sign) -- 16 or 24 bytes per matrix, the only
  collective, after all compute.

Every rank takes the same collective steps in the same order.  ``compute``
is the per-rank function (log, sign) = compute(A_slice); it defaults to the
engine's ``slog_pfaffian_raw`` and is replaceable so that the host logic can be
exercised on CPU process groups (gloo).
"""
from __future__ import annotations

import heapq

import torch


def shard_range(count: int, world: int, rank: int) -> tuple[int, int]:
    """[lo, hi) of a batch of ``count`` matrices owned by ``rank``: contiguous,
    sizes differing by at most one, the larger shards first."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of world {world}")
    base, extra = divmod(count, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_ragged(orders, world: int) -> list[list[int]]:
    """Indices of a ragged batch per rank, balancing sum(n^3) (the elimination
    work) greedily: largest matrix first, each to the least-loaded rank (lower
    rank on ties).  Deterministic, so every rank computes the same plan."""
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(orders)), key=lambda i: (-int(orders[i]), i))
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(orders[i]) ** 3, r))
    for lst in out:
        lst.sort()
    return out


def _default_compute(A):
    from .api import slog_pfaffian_raw
    return slog_pfaffian_raw(A.contiguous())


def slog_pfaffian_sharded(A: torch.Tensor, group=None, compute=None, gather: bool = True):
    """(log|Pf|, sign) of a (B, n, n) batch, each rank factoring its shard.

    Every rank passes the same full batch shape (its own slice is taken here);
    with ``gather`` the full (B,) results come back on every rank, else only
    the rank's own slice.  Without an initialised process group this is the
    single-GPU call.
    """
    import torch.distributed as dist

    compute = compute or _default_compute
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return compute(A)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    B = A.shape[0]
    lo, hi = shard_range(B, world, rank)
    la, sg = compute(A[lo:hi])
    if not gather:
        return la, sg
    # pad every shard to the largest one so all_gather sees equal sizes; a
    # complex sign travels as its (re, im) pairs
    width = -(-B // world)
    cplx = sg.is_complex()
    sg_r = torch.view_as_real(sg) if cplx else sg
    pad_l = torch.full((width,), float("nan"), dtype=la.dtype, device=la.device)
    pad_s = torch.zeros((width,) + tuple(sg_r.shape[1:]), dtype=sg_r.dtype, device=sg.device)
    pad_l[: hi - lo] = la
    pad_s[: hi - lo] = sg_r
    all_l = [torch.empty_like(pad_l) for _ in range(world)]
    all_s = [torch.empty_like(pad_s) for _ in range(world)]
    dist.all_gather(all_l, pad_l, group=group)
    dist.all_gather(all_s, pad_s, group=group)
    sizes = [shard_range(B, world, r)[1] - shard_range(B, world, r)[0] for r in range(world)]
    out_l = torch.cat([all_l[r][: sizes[r]] for r in range(world)])
    out_s = torch.cat([all_s[r][: sizes[r]] for r in range(world)])
    if cplx:
        out_s = torch.view_as_complex(out_s.contiguous())
    return out_l, out_s
