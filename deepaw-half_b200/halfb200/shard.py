"""k-point ownership across ranks.

k points are independent units of the path; the reference distributes them
cyclically over MPI ranks (rank r owns k when mod(k-1, size) == r,
src/half_parallel.F90:62-65) and only gathers eigenvalues afterwards.  The
same rule is used here, one process per GPU; no device collective is needed
on the data path.
"""
from __future__ import annotations

import numpy as np


def owned_indices(nk, rank, world):
    """0-based indices of the k points rank `rank` of `world` owns."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank/world")
    return np.arange(nk)[np.arange(nk) % world == rank]


def gather_eigenvalues(local_eig, nk, rank, world, group=None):
    """Assemble the full (nk, nbands) eigenvalue table on every rank from each
    rank's owned rows (host-side, torch.distributed all_gather on CPU tensors;
    used by tests and by callers that need all k points, e.g. occupations)."""
    import torch
    import torch.distributed as dist
    nb = local_eig.shape[1]
    per = int(np.ceil(nk / world))
    buf = torch.zeros((per, nb), dtype=torch.float64)
    buf[:len(local_eig)] = torch.as_tensor(local_eig)
    out = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    full = np.zeros((nk, nb))
    for r in range(world):
        idx = owned_indices(nk, r, world)
        full[idx] = out[r].numpy()[:len(idx)]
    return full
