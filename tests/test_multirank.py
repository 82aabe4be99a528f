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
