"""Oracle pins for the ion-position force terms (src/half_energy.F90:122-213,
src/half_local_forces.F90): each analytic force is minus the position
derivative of its energy functional, checked by central differences on the
seeded cells, as the reference's own app/half_force_check.F90 does for dD/dR.
CPU only."""
import dataclasses

import numpy as np
import pytest

from conftest import workload_files


def load(files, with_core_density=False):
    from oracle import hamiltonian as H
    w, ch, po = files
    return w, H.load_system(ch, po, w.encut, use_pbe=(w.xc == "pbe"), use_uspp=True)


def moved(crystal, iat, axis, h):
    pos = crystal.positions.copy()
    d = np.zeros(3); d[axis] = h
    pos[iat] = pos[iat] + d @ np.linalg.inv(crystal.lattice)
    return dataclasses.replace(crystal, positions=pos)


def central(fn, crystal, iat, axis, h=1e-4):
    return -(fn(moved(crystal, iat, axis, h)) - fn(moved(crystal, iat, axis, -h))) / (2 * h)


@pytest.fixture(scope="module")
def si2c(tmp_path_factory):
    return workload_files("si2c", str(tmp_path_factory.mktemp("si2c")))


def test_ewald_force_is_minus_energy_gradient(si2c, hfo2):
    from oracle.ionforces import ewald_energy, ewald_forces
    for files, cases in ((si2c, [(0, 0), (1, 2)]), (hfo2, [(3, 1)])):
        w, sysm = load(files)
        charges = np.repeat([p.zval for p in sysm.potcars], sysm.crystal.counts)
        f = ewald_forces(sysm.crystal, charges)
        assert np.abs(f.sum(axis=0)).max() < 1e-8          # translation invariance
        for iat, a in cases:
            num = central(lambda c: ewald_energy(c, charges)[0], sysm.crystal, iat, a)
            assert abs(f[iat, a] - num) <= 1e-6, (iat, a, f[iat, a], num)


def test_local_force_is_minus_local_energy_gradient(si2c):
    from oracle.ionforces import local_ionic_forces
    w, sysm = load(si2c)
    shape = tuple(sysm.shape)
    f, e = local_ionic_forces(sysm.values, sysm.potcars, sysm.crystal, shape)
    assert np.abs(f).max() > 1e-3
    for iat, a in [(0, 0), (1, 1)]:
        num = central(lambda c: local_ionic_forces(sysm.values, sysm.potcars, c, shape)[1], sysm.crystal, iat, a)
        assert abs(f[iat, a] - num) <= 1e-6, (iat, a, f[iat, a], num)


def test_core_force_is_minus_core_energy_gradient(si2c):
    from oracle.ionforces import core_energy, radial_density_forces, xc_potential
    w, sysm = load(si2c)
    shape = tuple(sysm.shape)
    assert sysm.potcars[0].has_core
    vxc = xc_potential(sysm.values, sysm.potcars, sysm.crystal, shape, w.xc == "pbe")
    f = radial_density_forces(vxc, sysm.potcars, sysm.crystal, shape)
    assert np.abs(f).max() > 1e-4
    for iat, a in [(0, 2), (1, 0)]:
        num = central(lambda c: core_energy(vxc, sysm.potcars, c, shape), sysm.crystal, iat, a)
        assert abs(f[iat, a] - num) <= 1e-7, (iat, a, f[iat, a], num)


def test_smooth_density_counts_the_electrons(si2c):
    from oracle import hamiltonian as H
    from oracle.ionforces import smooth_density
    w, sysm = load(si2c)
    op = H.prepare(sysm)
    e, v, _, _ = H.solve_dense(op, 6, vectors=True)
    occ = np.array([2.0, 2.0, 2.0, 1.0, 1.0, 0.0])
    rho = smooth_density(op.basis, v, occ, 1.0, tuple(sysm.shape))
    # S-orthonormal states: the smooth density alone integrates below sum f (augmentation carries the rest)
    assert 0 < rho.mean() <= occ.sum() + 1e-9


def test_smooth_density_parseval(si2c):
    """Grid mean of the smooth density = sum w f |c|^2 (unnormalised inverse transform)."""
    from oracle import hamiltonian as H
    from oracle.ionforces import smooth_density
    w, sysm = load(si2c)
    op = H.prepare(sysm, (0.25, 0.0, 0.25))
    e, v, _, _ = H.solve_dense(op, 6, vectors=True)
    occ = np.array([2.0, 2.0, 1.5, 1.0, 0.5, 0.0])
    rho = smooth_density(op.basis, v, occ, 0.5, tuple(sysm.shape))
    expect = 0.5 * float(np.sum(occ * np.sum(np.abs(v) ** 2, axis=0)))
    assert abs(rho.mean() - expect) <= 1e-12 * expect


def test_augmentation_density_integrates_to_its_monopole(si2c):
    """The deposited charge is sum_I sum_ab rho_ab M_ab,00 sqrt(4 pi) (the compensation
    shape g_0 is normalised, src/half_uspp.F90:335-342), up to the box quadrature,
    and nothing lands beyond paw_rmax of every atom."""
    from oracle import hamiltonian as H
    from oracle.ionforces import add_augmentation_density, augmentation_occupancy
    from oracle.uspp import species_qdep_tables
    w, sysm = load(si2c)
    op = H.prepare(sysm, (0.0, 0.0, 0.0))
    e, v, _, _ = H.solve_dense(op, 6, vectors=True)
    occ = np.array([2.0, 2.0, 2.0, 1.0, 1.0, 0.0])
    occupancy = augmentation_occupancy(op.species, v, occ, 1.0)
    shape = tuple(sysm.shape)
    n = int(np.prod(shape))
    aug, charge = add_augmentation_density(sysm.potcars, sysm.crystal, shape, occupancy, np.zeros(n))
    expect = 0.0
    for it, pot in enumerate(sysm.potcars):
        t = species_qdep_tables(pot)
        for iat in range(sysm.crystal.counts[it]):
            expect += float(np.sum(occupancy[it][iat] * t["multipole"][:, :, 0])) * np.sqrt(4 * np.pi)
    assert abs(expect) > 1e-3
    assert abs(charge - expect) <= 1e-2 * abs(expect), (charge, expect)
    n1, n2, n3 = shape
    idx = np.arange(n)
    frac = np.stack([(idx % n1) / n1, ((idx // n1) % n2) / n2, (idx // (n1 * n2)) / n3], axis=1)
    near = np.zeros(n, dtype=bool)
    for p in sysm.crystal.positions:
        df = frac - p
        df -= np.sign(df) * np.floor(np.abs(df) + 0.5)
        near |= np.sqrt(((df @ sysm.crystal.lattice) ** 2).sum(axis=1)) <= sysm.potcars[0].paw_rmax
    assert not aug[~near].any() and np.abs(aug[near]).max() > 0
