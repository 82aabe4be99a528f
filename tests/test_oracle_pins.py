"""Pins of the CPU oracle against the reference's own known answers and
validation records (CPU only, a few seconds)."""
import numpy as np
import pytest

from oracle.basis import build_basis
from oracle.forces import compute_occupations, gamma_centered_mesh, nonlocal_forces
from oracle.io import Crystal


def si_primitive(volume):
    a = (4 * volume) ** (1 / 3)
    lat = a / 2 * np.array([[0, 1, 1], [1, 0, 1], [1, 1, 0]], float)
    return Crystal("si", lat, ["Si"], [2], np.array([[0, 0, 0], [.25, .25, .25]]))


def test_basis_pins_si_validation_records():
    # docs/validation/si_gamma_basis.json, half_vs_happy_si_slice.json:
    # volume 40.3295268474 A^3, 400 eV, Gamma -> 725 plane waves, kinetic
    # checksum 172858.94956152519 eV (volume given to 12 digits, hence 1e-10).
    c = si_primitive(40.3295268474)
    b = build_basis(c, (56, 56, 56), 400.0)
    assert b.npw == 725
    assert abs(b.kinetic.sum() - 172858.94956152519) / 172858.94956152519 < 1e-10
    # docs/validation/si_arbitrary_kpoint.json: k = [0.125, 0.25, 0.375] -> 733
    assert build_basis(c, (56, 56, 56), 400.0, (0.125, 0.25, 0.375)).npw == 733


def test_basis_ordering_and_fft_index():
    c = si_primitive(40.0)
    b = build_basis(c, (24, 24, 24), 400.0, (0.1, 0.2, 0.3))
    g = b.gvectors.astype(np.int64)
    key = (g[:, 0] + 12) * 576 + (g[:, 1] + 12) * 24 + (g[:, 2] + 12)
    assert np.all(np.diff(key) > 0)                    # n1 -> n2 -> n3 loop order
    idx = np.mod(g[:, 0], 24) * 576 + np.mod(g[:, 1], 24) * 24 + np.mod(g[:, 2], 24)
    assert np.array_equal(idx, b.fft_index)


def test_occupation_known_answers():
    # app/half_energy_check.F90:19-34
    eig = np.array([[0.0, 2.0], [1.0, 3.0]])
    occ, mu, band, ent = compute_occupations(eig, [0.5, 0.5], 2.0, 0.0)
    assert np.abs(occ - np.array([[2.0, 0.0], [2.0, 0.0]])).max() <= 1e-14
    assert abs(mu - 1.0) <= 1e-14 and abs(band - 1.0) <= 1e-14 and abs(ent) <= 1e-14
    eig = np.array([[-1.0, 0.5, 2.0], [-0.8, 0.7, 2.2]])
    w = np.array([0.25, 0.75])
    for ismear in (-1, 0):
        occ, mu, band, ent = compute_occupations(eig, w, 2.0, 0.1, ismear)
        assert abs((w[:, None] * occ).sum() - 2.0) <= 1e-12
        assert ent < 0.0


def test_nonlocal_force_known_answer():
    """app/half_energy_check.F90:58-97: 3 plane waves, 2 projectors, analytic
    force vs central difference of the synthetic energy, tolerance 2e-9."""
    from oracle.paw import SpeciesProjectors
    from oracle.basis import Basis
    q = np.array([[0.2, -0.3, 0.6], [0.7, 0.5, -0.2], [-0.4, 0.8, 0.9]])
    p0 = np.array([[0.4 + 0.1j, 0.1 - 0.2j, -0.3 + 0.2j],
                   [-0.2 + 0.3j, 0.5 + 0.4j, 0.2 + 0.6j]])          # p0[a, g]
    waves = np.array([0.3 - 0.1j, -0.2 + 0.4j, 0.5 + 0.2j])
    dij = np.array([[1.2, 0.15], [0.15, 0.8]])
    qij = np.array([[0.1, 0.02], [0.02, 0.07]])
    eps, focc, kw = 0.37, 1.6, 0.4
    r0 = np.array([0.13, -0.21, 0.08])

    def projectors(pos):
        ph = q @ pos
        return (p0 * (np.cos(ph) - 1j * np.sin(ph))[None, :]).T      # B[g, a]

    basis = Basis((1, 1, 1), np.zeros(3), np.zeros((3, 3), np.int32), q, np.zeros(3), np.zeros(3, np.int64))
    sp = SpeciesProjectors(1, 2, projectors(r0), dij, qij)
    f = nonlocal_forces(basis, [sp], [dij[None]], [None], [eps], [focc], kw, waves[:, None])

    def energy(pos):
        cc = projectors(pos).conj().T @ waves
        return kw * focc * float(np.real(np.vdot(cc, (dij - eps * qij) @ cc)))

    h = 1e-5
    num = np.array([-(energy(r0 + h * e) - energy(r0 - h * e)) / (2 * h) for e in np.eye(3)])
    assert np.abs(f[0] - num).max() <= 2e-9


def test_gamma_centered_mesh():
    pts, w = gamma_centered_mesh(4, 4, 4)
    assert pts.shape == (64, 3) and abs(w.sum() - 1) < 1e-15
    assert np.all(pts <= 0.5) and np.all(pts > -0.5)
    assert np.array_equal(pts[0], [0, 0, 0])



def test_qdep_gradient_matches_central_difference(si2, oracle_system):
    """app/half_force_check.F90:139-153: analytic dD/dR of atom 1 vs central
    difference at fixed Veff, h = 1e-5 A, tolerance 2e-4."""
    from oracle.uspp import build_qdep
    sysm = oracle_system("si2", si2, with_gradient=True)
    c = sysm.crystal
    inv = np.linalg.inv(c.lattice)
    h = 1e-5
    num = np.zeros_like(sysm.ddij_atoms[0][0])
    for a in range(3):
        d = np.zeros(3); d[a] = h
        cp = Crystal(c.name, c.lattice, c.species, c.counts, c.positions.copy())
        cp.positions[0] += d @ inv
        dp = build_qdep(sysm.veff, sysm.shape, sysm.potcars, cp, with_gradient=False)[0][0][0]
        cm = Crystal(c.name, c.lattice, c.species, c.counts, c.positions.copy())
        cm.positions[0] -= d @ inv
        dm = build_qdep(sysm.veff, sysm.shape, sysm.potcars, cm, with_gradient=False)[0][0][0]
        num[:, :, a] = (dp - dm) / (2 * h)
    assert np.abs(sysm.ddij_atoms[0][0] - num).max() <= 2e-4
    assert np.abs(num).max() > 1e-3            # the derivative is not trivially zero


def test_oracle_acc_consistent_with_dense(si2, oracle_system):
    from oracle import hamiltonian as H, acc
    op = H.prepare(oracle_system("si2", si2))
    w, _, smin, smax = H.solve_dense(op, 8)
    r = acc.solve_acc(op, 8, tol=1e-7, max_iterations=300)
    assert r.converged
    assert np.abs(r.eigenvalues - w).max() <= 1e-10
    assert smin > 0.9 and smax < 1.5


def test_matrix_free_equals_dense(si2, oracle_system):
    from oracle import hamiltonian as H
    op = H.prepare(oracle_system("si2", si2), (0.1, 0.2, -0.3))
    h, s = H.assemble_dense(op)
    r = np.random.default_rng(3)
    psi = r.normal(size=(op.basis.npw, 2)) + 1j * r.normal(size=(op.basis.npw, 2))
    hp, sp = H.apply_hs(op, psi)
    assert np.abs(hp - h @ psi).max() <= 1e-12 * np.abs(hp).max()
    assert np.abs(sp - s @ psi).max() <= 1e-12 * np.abs(sp).max()
