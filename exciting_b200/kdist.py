"""k-point distribution over processes (one process per GPU).

k-points are independent, as in the reference's MPI split
(src/scf_cycle.f90:237-278, src/force.f90:160-170): each rank owns a
contiguous block of k-points, sets up H/O (and the IBS force) for those only,
and the one reduction of this path -- the 3 x natmtot IBS forces,
MPI_ALLREDUCE at force.f90:170 -- becomes an all-reduce over the process
group (NCCL on GPUs, gloo in the CPU tests).

The block rule follows the documented behaviour of the reference's
``nofset``/``firstofset``/``lastofset`` (src/src_mpi/modmpi.F90:272-463):
N elements over P processes in contiguous blocks, the first N mod P ranks
taking one extra element; a rank without elements gets first = 0,
last = -1 (1-based indices, as in the reference).
"""
from __future__ import annotations

import numpy as np


def nofset(rank: int, n: int, nprocs: int) -> int:
    """Number of elements of process ``rank`` (0-based rank)."""
    if n < 0 or nprocs <= 0 or not 0 <= rank < nprocs:
        raise ValueError("nofset: bad arguments")
    q, r = divmod(n, nprocs)
    return q + (1 if rank < r else 0)


def firstofset(rank: int, n: int, nprocs: int) -> int:
    """1-based index of the first element of process ``rank``; 0 if it has none."""
    if nofset(rank, n, nprocs) == 0:
        return 0
    return 1 + sum(nofset(p, n, nprocs) for p in range(rank))


def lastofset(rank: int, n: int, nprocs: int) -> int:
    """1-based index of the last element of process ``rank``; -1 if it has none."""
    c = nofset(rank, n, nprocs)
    if c == 0:
        return -1
    return firstofset(rank, n, nprocs) + c - 1


def my_kpoints(rank: int, nkpt: int, nprocs: int):
    """0-based k-point indices owned by ``rank``."""
    f = firstofset(rank, nkpt, nprocs)
    if f == 0:
        return []
    return list(range(f - 1, lastofset(rank, nkpt, nprocs)))


def allreduce_forces(forceibs: np.ndarray, group=None, device=None) -> np.ndarray:
    """Sum the per-rank IBS forces over the process group (force.f90:170)."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(forceibs, dtype=np.float64))
    if device is not None:
        t = t.to(device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return np.asfortranarray(t.cpu().numpy())
