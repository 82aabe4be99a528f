"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances: FP64 operator and dense results agree with the oracle to 1e-11
relative (different FFT and summation orders); FP64-mode eigenvalues within
1e-10 eV and mixed-mode eigenvalues within 1e-8 eV of the FP64 dense oracle
once converged; forces within 1e-10 eV/A of the oracle's restatement of the
reference force for the same eigenpairs.
"""
import numpy as np
import pytest

import halfb200
from conftest import rng

pytestmark = pytest.mark.gpu


def ctx_for(files, solver="acc", use_uspp=True):
    w, ch, po = files
    return halfb200.Context(ch, po, w.encut, xc=w.xc, use_uspp=use_uspp, solver=solver)


def test_basis_exact(si2, hfo2, oracle_system):
    from oracle.basis import build_basis
    for files, name in ((si2, "si2"), (hfo2, "hfo2")):
        w = files[0]
        with ctx_for(files) as ctx:
            crystal = oracle_system(name, files).crystal
            for k in [(0, 0, 0), (0.125, 0.25, 0.375)]:
                g, kin = ctx.basis(k)
                b = build_basis(crystal, w.grid, w.encut, k)
                assert np.array_equal(g, b.gvectors)
                assert np.abs(kin - b.kinetic).max() <= 1e-11 * np.abs(b.kinetic).max()


@pytest.mark.parametrize("name", ["si2", "hfo2"])
@pytest.mark.parametrize("k", [(0, 0, 0), (0.125, -0.25, 0.375)])
def test_apply_hs_fp64(name, k, si2, hfo2, oracle_system):
    from oracle import hamiltonian as H
    files = {"si2": si2, "hfo2": hfo2}[name]
    sysm = oracle_system(name, files)
    op = H.prepare(sysm, k)
    r = rng(1)
    psi = r.normal(size=(op.basis.npw, 5)) + 1j * r.normal(size=(op.basis.npw, 5))
    hr, sr = H.apply_hs(op, psi)
    with ctx_for(files) as ctx:
        hg, sg = ctx.apply_hs(k, psi)
    assert np.abs(hg - hr).max() <= 1e-11 * np.abs(hr).max()
    assert np.abs(sg - sr).max() <= 1e-11 * np.abs(sr).max()


@pytest.mark.parametrize("name", ["si2", "hfo2"])
@pytest.mark.parametrize("k", [(0, 0, 0), (0.125, -0.25, 0.375)])
def test_apply_hs_fp32(name, k, si2, hfo2, oracle_system):
    """The mixed mode's operator: FP32 local part, projector part on the
    tensor cores with B split into bf16 planes once per k point (2^-16).  H psi and S psi
    agree with the FP64 oracle to 1e-4 of their largest element, and the
    projector part alone (S psi - psi = B Q B^H psi) to 1e-4 of its own."""
    from oracle import hamiltonian as H
    files = {"si2": si2, "hfo2": hfo2}[name]
    sysm = oracle_system(name, files)
    op = H.prepare(sysm, k)
    r = rng(2)
    psi = r.normal(size=(op.basis.npw, 37)) + 1j * r.normal(size=(op.basis.npw, 37))
    hr, sr = H.apply_hs(op, psi)
    with ctx_for(files) as ctx:
        ctx.set_acc(precision="mixed")
        hg, sg = ctx.apply_hs(k, psi)
    psi32 = psi.astype(np.complex64).astype(np.complex128)
    assert np.abs(hg - hr).max() <= 1e-4 * np.abs(hr).max()
    assert np.abs(sg - sr).max() <= 1e-4 * np.abs(sr).max()
    proj_ref = sr - psi
    proj_gpu = sg - psi32
    assert np.abs(proj_gpu - proj_ref).max() <= 1e-4 * np.abs(proj_ref).max()
    # and it is the FP32 path, not the FP64 one
    assert np.abs(hg - hr).max() > 1e-9 * np.abs(hr).max()


def test_assemble_hs(si2, oracle_system):
    from oracle import hamiltonian as H
    op = H.prepare(oracle_system("si2", si2))
    h, s = H.assemble_dense(op)
    with ctx_for(si2, solver="evd") as ctx:
        hg, sg = ctx.assemble_hs((0, 0, 0))
    assert np.abs(hg - h).max() <= 1e-11 * np.abs(h).max()
    assert np.abs(sg - s).max() <= 1e-12


def test_evd_matches_dense_oracle(si2, oracle_system):
    from oracle import hamiltonian as H
    op = H.prepare(oracle_system("si2", si2))
    w, _, smin, smax = H.solve_dense(op, 16)
    h, s = H.assemble_dense(op)
    with ctx_for(si2, solver="evd") as ctx:
        eg, _, gmin, gmax = ctx.solve((0, 0, 0), 16)
        ev, vec, _, _ = ctx.solve((0, 0, 0), 16, vectors=True)
    assert np.abs(eg - w).max() <= 1e-10
    assert abs(gmin - smin) <= 1e-10 and abs(gmax - smax) <= 1e-10
    assert np.array_equal(ev, eg)
    # eigenpairs of the oracle's dense H, S with the zhegvd normalisation V^H S V = I
    assert np.abs(h @ vec - (s @ vec) * ev[None, :]).max() <= 1e-9
    assert np.abs(vec.conj().T @ s @ vec - np.eye(16)).max() <= 1e-10


def test_index_range_solver(si2, oracle_system):
    from oracle import hamiltonian as H
    op = H.prepare(oracle_system("si2", si2))
    w, _, _, _ = H.solve_dense(op, 8)
    with ctx_for(si2, solver="vasp") as ctx:
        eg, vec, gmin, gmax = ctx.solve((0, 0, 0), 8, vectors=True)
    assert np.abs(eg - w).max() <= 1e-10
    assert gmin == -1.0 and gmax == -1.0
    assert vec.shape == (op.basis.npw, 8)
    h, s = H.assemble_dense(op)
    assert np.abs(h @ vec - (s @ vec) * eg[None, :]).max() <= 1e-9
    assert np.abs(vec.conj().T @ s @ vec - np.eye(8)).max() <= 1e-10


def test_acc_fp64_iterates_match_oracle_acc(hfo2, oracle_system):
    """Same controls, same algorithm: after a fixed number of unconverged
    iterations the Ritz values match the oracle's restatement.  The
    monoclinic cell has no symmetry-degenerate levels, so the iterates are
    well defined (in degenerate spectra the choice of basis inside a
    degenerate eigenspace differs between eigensolver libraries)."""
    from oracle import hamiltonian as H, acc
    op = H.prepare(oracle_system("hfo2", hfo2))
    ref = acc.solve_acc(op, 16, tol=1e-12, max_iterations=8)
    with ctx_for(hfo2) as ctx:
        ctx.set_acc(tol=1e-12, max_iterations=8)
        eg, _, smin, smax = ctx.solve((0, 0, 0), 16)
        info = ctx.info()
    assert smin == -1.0 and smax == -1.0
    assert info["iterations"] == ref.iterations == 8
    print("acc iterate parity", np.abs(eg - ref.eigenvalues).max())
    assert np.abs(eg - ref.eigenvalues).max() <= 1e-9


def test_acc_fp64_converges_to_dense(si2, oracle_system):
    from oracle import hamiltonian as H
    op = H.prepare(oracle_system("si2", si2))
    w, _, _, _ = H.solve_dense(op, 8)
    with ctx_for(si2) as ctx:
        ctx.set_acc(tol=1e-7, max_iterations=400)
        eg, _, _, _ = ctx.solve((0, 0, 0), 8)
        info = ctx.info()
    assert info["converged"] == 1
    assert np.abs(eg - w).max() <= 1e-10


def test_acc_mixed_converges_to_dense(si2, oracle_system):
    from oracle import hamiltonian as H
    op = H.prepare(oracle_system("si2", si2))
    w, _, _, _ = H.solve_dense(op, 8)
    with ctx_for(si2) as ctx:
        ctx.set_acc(tol=1e-7, max_iterations=400, precision="mixed")
        eg, _, _, _ = ctx.solve((0, 0, 0), 8)
        info = ctx.info()
    assert info["converged"] == 1
    assert info["fp64_iterations"] < info["iterations"]
    assert np.abs(eg - w).max() <= 1e-8


def test_mapped_solve_reverse_order(si2, oracle_system):
    """half_solve_kpoint_mapped returns the eigenvectors in the host's G order:
    undoing a reversed host order gives eigenvectors of the oracle's dense
    H, S in HALF order (degenerate levels make a row-by-row comparison of two
    separate solves meaningless)."""
    from oracle import hamiltonian as H
    op = H.prepare(oracle_system("si2", si2))
    h, s = H.assemble_dense(op)
    with ctx_for(si2, solver="evd") as ctx:
        g, _ = ctx.basis((0, 0, 0))
        e0, _, _, _ = ctx.solve((0, 0, 0), 8)
        rev = g[::-1].copy()
        e1, v1, _, _ = ctx.solve_mapped((0, 0, 0), 8, rev)
        with pytest.raises(halfb200.HalfError) as ei:
            ctx.solve_mapped((0, 0, 0), 8, np.concatenate([rev[:1], rev[:-1]]))
        assert ei.value.status == halfb200.HALF_ERROR_INVALID_ARGUMENT
    assert np.abs(e0 - e1).max() <= 1e-12
    v = v1[::-1]
    res = h @ v - (s @ v) * e1[None, :]
    assert np.abs(res).max() <= 1e-9
    assert np.abs(v.conj().T @ s @ v - np.eye(8)).max() <= 1e-10


def test_nonlocal_forces_match_oracle(si2, oracle_system):
    from oracle import hamiltonian as H
    from oracle.forces import nonlocal_forces
    sysm = oracle_system("si2", si2, with_gradient=True)
    op = H.prepare(sysm)
    w, v, _, _ = H.solve_dense(op, 8, vectors=True)
    occ = np.array([2.0, 2.0, 2.0, 2.0, 1.0, 0.5, 0.0, 0.0])
    ref = nonlocal_forces(op.basis, op.species, sysm.dij_atoms, sysm.ddij_atoms, w, occ, 0.7, v)
    with ctx_for(si2) as ctx:
        f = ctx.nonlocal_forces((0, 0, 0), v, w, occ, 0.7)
    assert np.abs(f - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())


def test_guard_bands_find_a_degenerate_level_cut_by_the_band_count(si2, oracle_system):
    """When the band count cuts a degenerate level, the reference iteration may
    converge on a higher level (the residual test accepts any converged
    eigenpairs); the guarded FP64 and the mixed modes carry guard bands and
    must return the lowest m eigenvalues of the dense solve."""
    from oracle import hamiltonian as H
    op = H.prepare(oracle_system("si2", si2))
    w, _, _, _ = H.solve_dense(op, 16)
    cut = [m for m in range(4, 12) if abs(w[m] - w[m - 1]) < 1e-6]
    assert cut, "the Si cell has degenerate levels at Gamma"
    m = cut[0]
    with ctx_for(si2) as ctx:
        for precision, tol in (("fp64_guarded", 1e-10), ("mixed", 1e-8)):
            ctx.set_acc(tol=1e-7, max_iterations=400, precision=precision)
            eg, _, _, _ = ctx.solve((0, 0, 0), m)
            assert ctx.info()["converged"] == 1
            assert np.abs(eg - w[:m]).max() <= tol, (precision, m, eg - w[:m])


def test_guarded_and_mixed_match_dense_on_the_64_atom_cell(inputs_dir):
    """c2-size check (64-atom Si, 11k plane waves, 160 bands, k = (0, 0, 1/4)):
    the 160th band is the first member of a 4-fold level, which the unguarded
    iteration can miss; the guarded modes agree with the dense solve."""
    from conftest import workload_files
    w, ch, po = workload_files("si64", inputs_dir)
    k = tuple(w.kpoints[1])
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as d:
        ref = d.solve(k, w.nbands)[0]
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="acc") as ctx:
        for precision, tol in (("mixed", 1e-8), ("fp64_guarded", 1e-8)):
            ctx.set_acc(tol=2e-5, max_iterations=400, precision=precision)
            e = ctx.solve(k, w.nbands)[0]
            assert ctx.info()["converged"] == 1
            assert np.abs(e - ref).max() <= tol, (precision, np.abs(e - ref).max())


@pytest.mark.parametrize("solver,nb", [("evd", 16), ("vasp", 8)])
def test_dense_64bit_path_matches_oracle(solver, nb, si2, oracle_system, monkeypatch):
    """Large orders (above 16,384 plane waves) solve through the 64-bit solver API:
    Cholesky and two triangular solves, then for eigenvalues alone (and the
    overlap extremes) Householder tridiagonalisation with multisection on
    Sturm counts, for eigenpairs the 64-bit Hermitian evd.
    HALF_DENSE_64BIT_ORDER=0 sends this small cell down that path, which must
    give the oracle's eigenpairs, overlap extremes and S-normalisation like the
    32-bit path."""
    from oracle import hamiltonian as H
    op = H.prepare(oracle_system("si2", si2))
    w, _, smin, smax = H.solve_dense(op, nb)
    h, s = H.assemble_dense(op)
    monkeypatch.setenv("HALF_DENSE_64BIT_ORDER", "0")
    with ctx_for(si2, solver=solver) as ctx:
        eg, _, gmin, gmax = ctx.solve((0, 0, 0), nb)
        ev, vec, _, _ = ctx.solve((0, 0, 0), nb, vectors=True)
    assert np.abs(eg - w).max() <= 1e-10
    assert np.abs(ev - w).max() <= 1e-10
    if solver == "evd":
        assert abs(gmin - smin) <= 1e-10 and abs(gmax - smax) <= 1e-10
    else:
        assert gmin == -1.0 and gmax == -1.0
    assert np.abs(h @ vec - (s @ vec) * ev[None, :]).max() <= 1e-9
    assert np.abs(vec.conj().T @ s @ vec - np.eye(nb)).max() <= 1e-10


@pytest.mark.parametrize("name", ["si2", "hfo2"])
def test_soft_locking_matches_dense(name, si2, hfo2, oracle_system, monkeypatch):
    """Locking in the guard-band modes (on by default; HALF_SOFT_LOCK=0 turns it
    off).  Soft (HALF_HARD_LOCK=0): requested bands whose residual is at or
    below half the tolerance add no correction direction, so the pencils shrink.
    Hard (the default): such bands also leave the Rayleigh-Ritz step and the
    rotations for the rest of the phase.  Either way the converged eigenvalues
    must be the dense solve's, and the operator must see fewer columns than
    without locking."""
    from oracle import hamiltonian as H
    files = {"si2": si2, "hfo2": hfo2}[name]
    w = files[0]
    op = H.prepare(oracle_system(name, files))
    nb = 8 if name == "si2" else w.nbands
    ref, _, _, _ = H.solve_dense(op, nb)
    modes = {"off": ("0", "1"), "soft": ("1", "0"), "hard": ("1", "1")}
    with ctx_for(files) as ctx:
        for precision, tol in (("fp64_guarded", 1e-10), ("mixed", 1e-8)):
            cols = {}
            for mode, (soft, hard) in modes.items():
                monkeypatch.setenv("HALF_SOFT_LOCK", soft)
                monkeypatch.setenv("HALF_HARD_LOCK", hard)
                ctx.set_acc(tol=2e-5 if name == "hfo2" else 1e-7, max_iterations=400, precision=precision)
                e, _, _, _ = ctx.solve((0, 0, 0), nb)
                info = ctx.info()
                assert info["converged"] == 1, (precision, mode)
                assert np.abs(e - ref).max() <= tol, (precision, mode, np.abs(e - ref).max())
                assert np.all(np.diff(e) >= 0), (precision, mode)
                cols[mode] = info["operator_applications"] / max(1, info["iterations"])
            assert cols["soft"] < cols["off"] and cols["hard"] < cols["off"], (precision, cols)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_band_chunk_and_tuning_change_no_result(precision, hfo2):
    """The operator's bands per chunk and the tensor-core GEMM's tile width are
    chosen by the autotuner (block_size 0); every choice must give bit-identical
    H psi and S psi, and repeated mixed solves bit-identical eigenvalues while
    the tuner is still measuring and after it has decided."""
    w = hfo2[0]
    r = rng(4)
    with ctx_for(hfo2) as ctx:
        n = ctx.npw((0, 0, 0))
        psi = r.normal(size=(n, 41)) + 1j * r.normal(size=(n, 41))
        outs = []
        for block in (0, 8, 16, 32, 64, 0, 0, 0, 0):
            ctx.set_acc(block_size=block, precision=precision)
            outs.append(ctx.apply_hs((0, 0, 0), psi))
        for h, s in outs[1:]:
            assert np.array_equal(h, outs[0][0]) and np.array_equal(s, outs[0][1])
        if precision == "mixed":
            ctx.set_acc(tol=2e-5, max_iterations=400, block_size=0, precision="mixed")
            eig = [ctx.solve((0, 0, 0), w.nbands)[0] for _ in range(4)]
            for e in eig[1:]:
                assert np.array_equal(e, eig[0])
