"""half_set_positions_noalloc versus half_set_positions.

The allocation-free entry point rebuilds D_ij and dD_ij/dR with every device
scratch buffer in one fixed 32 MiB array, processing the atoms of a species
in chunks that fit it.  Each output element depends only on its own atom, so
the results must be bit-identical to the allocating path; they are observed
through H psi, S psi (D_ij, Q_ij) and the non-local force (dD_ij/dR), over two
calls with different displacements.  This file is collected last so that it
also runs after every other test in one process.
"""
import numpy as np
import pytest

import halfb200
from conftest import workload_files

pytestmark = pytest.mark.gpu

KPT = (0.25, 0.0, 0.25)
NB = 6


def displaced(w, seed, scale=0.03):
    r = np.random.default_rng(seed)
    return np.mod(w.positions + r.normal(0.0, scale, size=w.positions.shape) @ np.linalg.inv(w.lattice), 1.0)


def probe_vectors(ctx, seed):
    n = ctx.npw(KPT)
    r = np.random.default_rng(seed)
    v = r.normal(size=(n, NB)) + 1j * r.normal(size=(n, NB))
    return v / np.linalg.norm(v, axis=0)


def observe(ctx, psi):
    h, s = ctx.apply_hs(KPT, psi)
    eps = np.linspace(-5.0, 3.0, NB)
    occ = np.linspace(1.0, 0.2, NB)
    f = ctx.nonlocal_forces(KPT, psi, eps, occ, 0.5)
    return h, s, f


# hfo2: two species, 48^3 box, all atoms in one chunk.
# si64: 60^3 box, 64 atoms in several chunks of the fixed scratch.
@pytest.mark.parametrize("name", ["hfo2", "si64"])
def test_noalloc_matches_set_positions_over_two_calls(name, inputs_dir):
    w, ch, po = workload_files(name, inputs_dir)
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as ctx:
        psi = probe_vectors(ctx, 5)
        for seed in (1, 2):
            pos = displaced(w, seed)
            ctx.set_positions(pos)
            ref = observe(ctx, psi)
            r0, _ = halfb200.allocation_counts()
            ctx.set_positions(w.positions)          # the next call must redo the work
            r1, d1 = halfb200.allocation_counts()
            assert r1 > r0                          # the allocating path takes device buffers
            ctx.set_positions_noalloc(pos)
            r2, d2 = halfb200.allocation_counts()
            assert (r2 - r1, d2 - d1) == (0, 0)     # this one takes none, cached or new
            got = observe(ctx, psi)
            for a, b in zip(got, ref):
                assert np.array_equal(a, b), np.abs(a - b).max()
        assert np.abs(ref[2]).max() > 1e-4          # dD/dR really entered the forces


def test_noalloc_runs_with_less_free_memory_than_the_allocating_path_needs(inputs_dir):
    """si216v (96^3 box, 212 atoms): half_set_positions needs about 330 MB of
    transient device scratch; the fixed-scratch call succeeds with 256 MiB
    of the device left free."""
    torch = pytest.importorskip("torch")
    w, ch, po = workload_files("si216v", inputs_dir)
    nr = int(np.prod(w.grid))
    allocating_scratch = 24 * nr + w.nions * 160 * 288 * 4 * 8
    headroom = 256 << 20
    assert allocating_scratch > headroom
    pos = displaced(w, 3, scale=0.02)
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as ctx:
        psi = probe_vectors(ctx, 6)
        ctx.set_positions(pos)
        ref = observe(ctx, psi)
        ctx.set_positions_noalloc(w.positions)   # first call on the device: resolves the scratch
        free, _ = torch.cuda.mem_get_info()
        hog = torch.empty(max(0, free - headroom), dtype=torch.uint8, device="cuda")
        try:
            r0, d0 = halfb200.allocation_counts()
            ctx.set_positions_noalloc(pos)
            assert halfb200.allocation_counts() == (r0, d0)
        finally:
            del hog
            torch.cuda.empty_cache()
        got = observe(ctx, psi)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), np.abs(a - b).max()


def test_noalloc_rejects_a_grid_beyond_the_fixed_scratch(tmp_path):
    """A 128 x 120 x 100 box needs 36.9 MB (24 B per point) > 32 MiB:
    HALF_ERROR_CAPACITY with a message naming the limit, and the context is
    left unchanged."""
    from halfb200 import synth
    w = synth.workload("si2")
    w.grid = (128, 120, 100)
    ch, po = synth.write_inputs(w, str(tmp_path))
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as ctx:
        psi = probe_vectors(ctx, 7)
        before = ctx.apply_hs(KPT, psi)
        with pytest.raises(halfb200.HalfError) as e:
            ctx.set_positions_noalloc(displaced(w, 4))
        assert e.value.status == halfb200.HALF_ERROR_CAPACITY
        assert "32 MiB" in e.value.message
        after = ctx.apply_hs(KPT, psi)
        for a, b in zip(after, before):
            assert np.array_equal(a, b)
