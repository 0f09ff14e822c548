"""Batches of volumes sharded over GPUs, one process per GPU.

Volumes are independent (the per-volume unit is inversion::tv_admm,
src/inversion/tv.rs:63-97), so a batch shards with no exchange between GPUs:

1. every rank computes the same placement, longest-processing-time-first on cost
   N*log2(N)*iterations (``qsm_batch_partition`` in the C ABI, host only);
2. each rank solves the volumes placed on it as one batched call on its own context
   (one CUDA graph per GPU, no collective while solving);
3. the results are gathered on the host of one rank at the end
   (``torch.distributed.gather_object``).

Ranks come from torch.distributed (``RANK`` / ``WORLD_SIZE`` under torchrun); the
process group must be initialised by the caller.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import Grid, QsmError, _lib


def partition(grids: Sequence[Grid], n_parts: int, iterations: Optional[Sequence[int]] = None
              ) -> Tuple[List[int], List[float]]:
    """(part of each volume, total cost of each part) from qsm_batch_partition."""
    lib = _lib.load()
    n = len(grids)
    arr = (_lib.QsmGrid * max(n, 1))()
    for b, g in enumerate(grids):
        arr[b] = g._c()
    it = None
    if iterations is not None:
        if len(iterations) != n:
            raise ValueError("one iteration count per volume")
        it = (C.c_size_t * max(n, 1))(*[int(k) for k in iterations])
    part = (C.c_uint32 * max(n, 1))()
    load = (C.c_double * max(int(n_parts), 1))()
    st = lib.qsm_batch_partition(arr, it, n, int(n_parts), part, load)
    if st != _lib.QSM_OK:
        raise QsmError(st, f"qsm_batch_partition(n={n}, n_parts={n_parts}) failed")
    return [int(part[b]) for b in range(n)], [float(load[k]) for k in range(int(n_parts))]


def share(grids: Sequence[Grid], rank: int, world: int, iterations: Optional[Sequence[int]] = None) -> List[int]:
    """Batch indices placed on `rank`, in batch order."""
    part, _ = partition(grids, world, iterations)
    return [b for b, k in enumerate(part) if k == rank]


def _dist():
    import torch.distributed as dist
    if not dist.is_initialized():
        raise RuntimeError("torch.distributed is not initialised")
    return dist


def gather_volumes(local: dict, n: int, dst: int = 0, group=None) -> Optional[list]:
    """Gather {batch index: result} dicts from every rank onto rank `dst`; returns the n
    results in batch order there and None elsewhere."""
    dist = _dist()
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    bucket = [None] * world if rank == dst else None
    dist.gather_object(local, bucket, dst=dst, group=group)
    if rank != dst:
        return None
    out = [None] * n
    for d in bucket:
        for b, v in d.items():
            if out[b] is not None:
                raise RuntimeError(f"volume {b} solved on two ranks")
            out[b] = v
    missing = [b for b, v in enumerate(out) if v is None]
    if missing:
        raise RuntimeError(f"volumes {missing} were not solved by any rank")
    return out


def tv_admm_sharded(cases, params, *, ctx=None, solve: Optional[Callable] = None, dst: int = 0, group=None):
    """TV-ADMM over a batch sharded across the ranks of the process group.

    cases: the whole batch, the same sequence of (local_field, mask, grid, bdir) on every
    rank.  Each rank solves its placement with inversion.tv_admm_batch on ``ctx`` (or with
    ``solve(sub_cases, params) -> (chis, iterations)`` when given), then the results are
    gathered onto rank ``dst``.  Returns (chis, iterations) in batch order on ``dst`` and
    (None, None) elsewhere, plus this rank's batch indices as a third element."""
    from . import inversion
    dist = _dist()
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    grids = [c[2] for c in cases]
    mine = share(grids, rank, world, [params.max_iter] * len(cases))
    sub = [cases[b] for b in mine]
    if sub:
        if solve is None:
            chis, iters = inversion.tv_admm_batch(sub, params, ctx=ctx)
        else:
            chis, iters = solve(sub, params)
    else:
        chis, iters = [], []
    local = {b: (np.asarray(chis[i]), int(iters[i])) for i, b in enumerate(mine)}
    got = gather_volumes(local, len(cases), dst=dst, group=group)
    if got is None:
        return None, None, mine
    return [g[0] for g in got], [g[1] for g in got], mine
