"""Band-energy force on the GPU versus central finite differences.

At fixed Veff, fixed plane-wave basis and Fermi-Dirac occupations, the
Mermin band free energy sum_k w_k sum_n f_nk eps_nk + entropy changes with
the atom positions only through the projector phases and D_ij(R); its
derivative is minus the non-local force (src/half_forces.F90:9-73).  The
finite difference is taken with the CPU oracle (dense generalized solves of
the displaced systems, step 1e-3 A) and, independently, with the library's own
dense solver.  Tolerance 1e-5 eV/A.
"""
import numpy as np
import pytest

import halfb200

pytestmark = pytest.mark.gpu

KPTS = np.array([[0.0, 0.0, 0.0], [0.25, 0.0, 0.25]])
WTS = np.array([0.5, 0.5])
NB, SIGMA, NELECT = 10, 0.1, 8.0


def displaced_positions(crystal):
    r = np.random.default_rng(11)
    return crystal.positions + r.normal(0.0, 0.03, size=crystal.positions.shape) @ np.linalg.inv(crystal.lattice)


def oracle_free_energy(sysm, positions):
    from oracle import hamiltonian as H
    from oracle.forces import compute_occupations
    from oracle.io import Crystal
    c = sysm.crystal
    cp = Crystal(c.name, c.lattice, c.species, c.counts, positions)
    s2 = H.make_system(cp, sysm.shape, sysm.values, sysm.potcars, sysm.encut, sysm.use_pbe, True, sysm.veff)
    eig = np.array([H.solve_dense(H.prepare(s2, k), NB)[0] for k in KPTS])
    _, _, band, ent = compute_occupations(eig, WTS, NELECT, SIGMA, -1)
    return band + ent


def test_band_forces_match_oracle_finite_difference(si2, oracle_system):
    w, ch, po = si2
    sysm = oracle_system("si2", si2)
    pos = displaced_positions(sysm.crystal)
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as ctx:
        ctx.set_positions(pos)
        r = ctx.band_forces(KPTS, WTS, NB, NELECT, SIGMA, -1)
    f = r["forces"]
    assert np.abs(f).max() > 1e-3                        # a non-trivial configuration
    lat_inv = np.linalg.inv(sysm.crystal.lattice)
    h = 1e-3
    num = np.zeros_like(f)
    for i in range(sysm.crystal.nions):
        for a in range(3):
            d = np.zeros(3); d[a] = h
            p1 = pos.copy(); p1[i] += d @ lat_inv
            p2 = pos.copy(); p2[i] -= d @ lat_inv
            num[i, a] = -(oracle_free_energy(sysm, p1) - oracle_free_energy(sysm, p2)) / (2 * h)
    print("max |F - F_fd| =", np.abs(f - num).max(), "max |F| =", np.abs(f).max())
    assert np.abs(f - num).max() <= 1e-5


def test_band_forces_match_library_finite_difference(si2):
    w, ch, po = si2
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as ctx:
        lat_inv = np.linalg.inv(ctx.lattice)
        from oracle.io import read_chgcar
        crystal, _, _ = read_chgcar(ch)
        pos = displaced_positions(crystal)
        ctx.set_positions(pos)
        f = ctx.band_forces(KPTS, WTS, NB, NELECT, SIGMA, -1)["forces"]
        h = 1e-3

        def energy(p):
            ctx.set_positions(p)
            r = ctx.band_forces(KPTS, WTS, NB, NELECT, SIGMA, -1)
            return r["band_energy"] + r["entropy"]
        i, a = 1, 2
        d = np.zeros(3); d[a] = h
        p1 = pos.copy(); p1[i] += d @ lat_inv
        p2 = pos.copy(); p2[i] -= d @ lat_inv
        num = -(energy(p1) - energy(p2)) / (2 * h)
    assert abs(f[i, a] - num) <= 1e-5


def test_autograd_backward_is_minus_force(si2):
    torch = pytest.importorskip("torch")
    from halfb200.autograd import band_free_energy
    w, ch, po = si2
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as ctx:
        from oracle.io import read_chgcar
        crystal, _, _ = read_chgcar(ch)
        frac = displaced_positions(crystal)
        cart = torch.tensor(frac @ crystal.lattice, dtype=torch.float64, requires_grad=True)
        e = band_free_energy(cart, ctx, KPTS, WTS, NB, NELECT, SIGMA, -1)
        e.backward()
        ctx.set_positions(frac)
        f = ctx.band_forces(KPTS, WTS, NB, NELECT, SIGMA, -1)["forces"]
    assert np.abs(cart.grad.numpy() + f).max() <= 1e-12
    assert np.isfinite(float(e))
