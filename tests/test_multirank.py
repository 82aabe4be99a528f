"""k-point ownership across ranks (host logic of multi-GPU runs), exercised
with two gloo ranks on CPU.  Each rank solves only the k points it owns
(src/half_parallel.F90:62-65 cyclic rule); the eigenvalue table is assembled
afterwards on the host."""
import os
import socket

import numpy as np
import pytest

from halfb200.shard import owned_indices


def test_cyclic_ownership_partition():
    for nk in (1, 4, 7, 64):
        for world in (1, 2, 3, 8):
            seen = np.concatenate([owned_indices(nk, r, world) for r in range(world)])
            assert np.array_equal(np.sort(seen), np.arange(nk))
            for r in range(world):
                assert all(i % world == r for i in owned_indices(nk, r, world))
    with pytest.raises(ValueError):
        owned_indices(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, nk, nb, out):
    import torch.distributed as dist
    from halfb200.shard import gather_eigenvalues, owned_indices
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        table = np.arange(nk * nb, dtype=float).reshape(nk, nb) * 0.5 - 3.0   # stands in for solved eigenvalues
        mine = table[owned_indices(nk, rank, world)]
        full = gather_eigenvalues(mine, nk, rank, world)
        out[rank] = float(np.abs(full - table).max())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nk", [5, 8])
def test_two_rank_gather_gloo(nk):
    import torch.multiprocessing as mp
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, nk, 3, out), nprocs=2, join=True, start_method="spawn")
    assert out[0] == 0.0 and out[1] == 0.0


class FakeContext:
    """Stands in for halfb200.Context on CPU in the sharded-force test: seeded
    per-k eigenproblems, a non-local force and an output density that are
    linear in the occupations and k weights (as the library's are), and
    ion-position terms that are a nonlinear function of the summed density,
    so a helper that applied them before summing would fail the test."""
    nions = 3

    def __init__(self, npw=12):
        self.npw = npw
        r = np.random.default_rng(17)
        self.fpat = r.normal(size=(npw, self.nions, 3))
        self.lmat = r.normal(size=(self.nions * 3, npw))

    def grid_size(self):
        return self.npw

    def solve(self, k, nbands, vectors=False):
        seed = int(abs(hash(tuple(np.round(np.asarray(k, dtype=float), 9)))) % (2 ** 31))
        r = np.random.default_rng(seed)
        a = r.normal(size=(self.npw, self.npw)) + 1j * r.normal(size=(self.npw, self.npw))
        e, v = np.linalg.eigh(a + a.conj().T)
        return e[:nbands], v[:, :nbands], -1.0, -1.0

    def nonlocal_forces(self, k, vectors, eigenvalues, occupations, kweight):
        dens = np.abs(vectors) ** 2                                   # (npw, nb)
        return kweight * np.einsum("b,b,gb,gij->ij", occupations, eigenvalues, dens, self.fpat)

    def output_density(self, kpoints, weights, vectors, occupations):
        rho = np.zeros(self.npw)
        for w, v, o in zip(weights, vectors, occupations):
            rho += w * (np.abs(v) ** 2 @ o)
        return rho, 0.1 * float(np.sum(np.asarray(weights)[:, None] * np.asarray(occupations)))

    def ionic_forces(self, rho):
        loc = (self.lmat @ rho).reshape(self.nions, 3)
        return {"ewald": np.ones((self.nions, 3)), "local": loc, "nlcc": np.tanh(rho.sum()) * loc,
                "harris": np.zeros((self.nions, 3)), "ewald_energy": -5.0, "local_energy": float(rho @ rho)}


KPTS = np.array([[0, 0, 0], [0.25, 0, 0], [0, 0.25, 0.25], [0.25, 0.25, 0.25], [0.5, 0, 0]], dtype=float)
WTS = np.array([0.1, 0.2, 0.3, 0.25, 0.15])


def _force_worker(rank, world, port, out):
    import torch.distributed as dist
    from halfb200.shard import sharded_forces
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = sharded_forces(FakeContext(), KPTS, WTS, 6, 5.0, 0.1, -1, rank=rank, world=world)
        out[rank] = {k: np.asarray(v).tolist() for k, v in r.items()}
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_forces_gloo():
    """k-point-sharded forces on two gloo ranks equal the one-rank chain: the
    eigenvalue gather, the occupations (half_occupations) and the sums of the
    k-linear parts before the ion-position terms."""
    import torch.multiprocessing as mp
    from halfb200.shard import sharded_forces
    ref = sharded_forces(FakeContext(), KPTS, WTS, 6, 5.0, 0.1, -1)
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_force_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    for rank in (0, 1):
        got = out[rank]
        for key in ("forces", "nonlocal", "local", "nlcc", "output_density", "occupations", "eigenvalues"):
            assert np.abs(np.asarray(got[key]) - ref[key]).max() <= 1e-12 * max(1.0, np.abs(ref[key]).max()), key
        for key in ("band_energy", "entropy", "mu", "augmentation_charge", "local_energy"):
            assert abs(float(got[key]) - float(ref[key])) <= 1e-12 * max(1.0, abs(float(ref[key]))), key
    assert np.abs(ref["forces"]).max() > 1e-3
