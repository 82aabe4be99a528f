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


def _allreduce_sum(arrays, group=None):
    """Sum float64 numpy arrays over the group's ranks (host tensors), in place order."""
    import torch
    import torch.distributed as dist
    flat = torch.as_tensor(np.concatenate([np.asarray(a, dtype=np.float64).ravel() for a in arrays]))
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    out, pos = [], 0
    for a in arrays:
        a = np.asarray(a)
        out.append(flat[pos:pos + a.size].numpy().reshape(a.shape).copy())
        pos += a.size
    return out


def sharded_forces(ctx, kpoints, weights, nbands, nelect, sigma, ismear=-1, rank=0, world=1, group=None):
    """The analytic force workload (what Context.forces does in one call) with
    the k points shared over `world` processes, one context each.

    Every term of the force is either a sum over k points or a function of
    such sums, so each rank solves only the k points it owns (the cyclic rule
    of src/half_parallel.F90:62-65) and contributes:
      1. eigenvalues, gathered so that every rank computes the same
         occupations (half_occupations, src/half_energy.F90:41-120);
      2. the non-local force of its k points (half_nonlocal_forces) and the
         smooth plus augmentation density of its states (half_output_density,
         linear in the occupations), both summed over ranks;
    then every rank evaluates the ion-position terms (half_ionic_forces) on
    the summed density.  The reference runs this workload on one rank only
    (app/half_cli.F90:830); with world = 1 this is the same chain as
    half_forces.  Returns a dict with the keys of Context.forces; all ranks
    hold the same values."""
    from .lib import HALF_ERROR_INVALID_ARGUMENT, HalfError, occupations
    ks = np.asarray(kpoints, dtype=np.float64).reshape(-1, 3)
    w = np.asarray(weights, dtype=np.float64)
    nk = len(ks)
    mine = owned_indices(nk, rank, world)
    local_eig, vecs = [], []
    for ik in mine:
        e, v, _, _ = ctx.solve(ks[ik], nbands, vectors=True)
        local_eig.append(e)
        vecs.append(v)
    local = np.array(local_eig).reshape(len(mine), nbands)
    eig = gather_eigenvalues(local, nk, rank, world, group) if world > 1 else local
    occ, band, entropy, mu = occupations(eig, w, nelect, sigma, ismear)
    if sigma > 0 and occ[:, -1].max() > 1e-6:   # app/half_cli.F90:897
        raise HalfError(HALF_ERROR_INVALID_ARGUMENT, "highest computed band is occupied; increase nbands")
    nonlocal_part = np.zeros((ctx.nions, 3))
    for j, ik in enumerate(mine):
        nonlocal_part += ctx.nonlocal_forces(ks[ik], vecs[j], eig[ik], occ[ik], w[ik])
    if len(mine):
        rho, aug = ctx.output_density(ks[mine], w[mine], vecs, occ[mine])
    else:
        rho, aug = np.zeros(ctx.grid_size()), 0.0
    if world > 1:
        nonlocal_part, rho, aug_arr = _allreduce_sum([nonlocal_part, rho, np.array([aug])], group)
        aug = float(aug_arr[0])
    ion = ctx.ionic_forces(rho)
    total = ion["ewald"] + ion["local"] + nonlocal_part + ion["nlcc"] + ion["harris"]
    return {"forces": total, "ewald": ion["ewald"], "local": ion["local"], "nonlocal": nonlocal_part,
            "nlcc": ion["nlcc"], "harris": ion["harris"], "output_density": rho, "band_energy": band,
            "entropy": entropy, "mu": mu, "ewald_energy": ion["ewald_energy"], "local_energy": ion["local_energy"],
            "augmentation_charge": aug, "eigenvalues": eig, "occupations": occ}
