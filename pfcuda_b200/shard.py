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
  collective, after all compute;
* ``pfaffian_sharded`` -- the same for the small path (2n <= 32);
* ``slog_pfaffian_ragged_sharded`` -- a ragged batch split by ``shard_ragged``,
  each rank running its matrices through one RaggedPlan, the results gathered
  back into the input order;
* ``slog_pfaffian_grad_sharded`` -- the adjoint ct * (1/2) A^-T of each rank's
  slice, the gradients (n^2 values per matrix) gathered if asked.

Every rank takes the same collective steps in the same order.  ``compute``
is the per-rank function; it defaults to the engine's call and is replaceable
so that the host logic can be exercised on CPU process groups (gloo).
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


def _group_info(group):
    import torch.distributed as dist
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return None
    return dist.get_world_size(group), dist.get_rank(group)


def _gather_padded(x: torch.Tensor, counts, group):
    """Concatenation over ranks of each rank's x (counts[r] rows on rank r), in
    rank order, through one all_gather of row blocks padded to the largest
    count.  A complex tensor travels as its (re, im) pairs."""
    import torch.distributed as dist
    world = len(counts)
    width = max(counts) if counts else 0
    cplx = x.is_complex()
    xr = torch.view_as_real(x) if cplx else x
    pad = torch.zeros((width,) + tuple(xr.shape[1:]), dtype=xr.dtype, device=xr.device)
    pad[: xr.shape[0]] = xr
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    out = torch.cat([parts[r][: counts[r]] for r in range(world)])
    return torch.view_as_complex(out.contiguous()) if cplx else out


def _sharded_uniform(A, group, compute, gather):
    """compute(A[lo:hi]) on each rank's contiguous slice; each output (a tensor
    or a tuple of tensors with one leading row per matrix) gathered if asked."""
    info = _group_info(group)
    if info is None:
        return compute(A)
    world, rank = info
    B = A.shape[0]
    lo, hi = shard_range(B, world, rank)
    out = compute(A[lo:hi])
    if not gather:
        return out
    counts = [shard_range(B, world, r)[1] - shard_range(B, world, r)[0] for r in range(world)]
    if isinstance(out, tuple):
        return tuple(_gather_padded(o, counts, group) for o in out)
    return _gather_padded(out, counts, group)


def slog_pfaffian_sharded(A: torch.Tensor, group=None, compute=None, gather: bool = True):
    """(log|Pf|, sign) of a (B, n, n) batch, each rank factoring its shard.

    Every rank passes the same full batch shape (its own slice is taken here);
    with ``gather`` the full (B,) results come back on every rank, else only
    the rank's own slice.  Without an initialised process group this is the
    single-GPU call.
    """
    return _sharded_uniform(A, group, compute or _default_compute, gather)


def pfaffian_sharded(A: torch.Tensor, group=None, compute=None, gather: bool = True):
    """Pf of a (B, n, n) batch with 2n <= 32, each rank computing its shard
    (one pfb_pfaffian launch per rank); gathered as slog_pfaffian_sharded."""
    if compute is None:
        from .api import pfaffian_raw

        def compute(X):
            return pfaffian_raw(X.contiguous())
    return _sharded_uniform(A, group, compute, gather)


def slog_pfaffian_grad_sharded(A: torch.Tensor, ct: torch.Tensor | None = None, group=None, compute=None,
                               gather: bool = True, mode: str = "fp64"):
    """ct * (1/2) A^-T of a (B, n, n) batch, each rank differentiating its shard
    (one pfb_slog_pfaffian_grad call per rank).  ``ct``: one real cotangent per
    matrix of the full batch, or None.  With ``gather`` every rank gets the full
    (B, n, n) gradient (one all_gather of n^2 values per matrix), else its own
    slice."""
    info = _group_info(group)
    B = A.shape[0]
    if compute is None:
        from .grad import slog_pfaffian_grad

        def compute(X, c):
            return slog_pfaffian_grad(X.contiguous(), ct=c, mode=mode)
    if info is None:
        return compute(A, ct)
    world, rank = info
    lo, hi = shard_range(B, world, rank)
    return _sharded_uniform(A, group, lambda X: compute(X, None if ct is None else ct[lo:hi]), gather)


def slog_pfaffian_ragged_sharded(mats, group=None, compute=None, gather: bool = True):
    """(log|Pf|, sign) of a ragged batch split across ranks by shard_ragged.

    Every rank passes the same list; of the other ranks' matrices only the
    order (the shape) is read, so they may be placeholders of the right shape
    (for instance meta tensors).  ``compute`` maps
    the rank's list of matrices to (log, sign) float64 tensors (default:
    slog_pfaffian_ragged).  With ``gather`` the results come back on every rank
    in the input order (one all_gather of 16 bytes per matrix); else the
    rank's own results with their input indices: (log, sign, indices).
    """
    orders = [int(M.shape[-1]) for M in mats]
    if compute is None:
        from .api import slog_pfaffian_ragged as compute
    info = _group_info(group)
    if info is None:
        return compute(list(mats))
    world, rank = info
    plan = shard_ragged(orders, world)
    mine = plan[rank]
    if mine:
        la, sg = compute([mats[i] for i in mine])
    else:
        dev = mats[0].device if len(mats) else torch.device("cpu")
        la = torch.empty(0, dtype=torch.float64, device=dev)
        sg = torch.empty(0, dtype=torch.float64, device=dev)
    idx = torch.tensor(mine, dtype=torch.int64, device=la.device)
    if not gather:
        return la, sg, idx
    counts = [len(p) for p in plan]
    all_l = _gather_padded(la, counts, group)
    all_s = _gather_padded(sg, counts, group)
    order = torch.tensor([i for p in plan for i in p], dtype=torch.int64, device=la.device)
    out_l = torch.empty(len(orders), dtype=all_l.dtype, device=la.device)
    out_s = torch.empty(len(orders), dtype=all_s.dtype, device=la.device)
    out_l[order] = all_l
    out_s[order] = all_s
    return out_l, out_s
