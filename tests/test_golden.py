"""The oracle against its committed fixtures (tests/golden/golden.json, made by
tests/golden/make_golden.py): the seeded inputs are regenerated and the
cheap parts recomputed, so any drift of the synthetic generator or of the
oracle's restatements shows here.  CPU only.

Tolerances: counts exact; energies and forces 1e-9 (eV, eV/A); densities
1e-9 relative.  The recomputation is deterministic on one machine; the
tolerances leave room for a different BLAS.
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT, workload_files

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))


@pytest.fixture(scope="module")
def si2c(tmp_path_factory):
    return workload_files("si2c", str(tmp_path_factory.mktemp("si2c_golden")))


def load(files):
    from oracle import hamiltonian as H
    w, ch, po = files
    return w, H.load_system(ch, po, w.encut, use_pbe=(w.xc == "pbe"), use_uspp=True)


def test_si2_operator_and_acc(si2):
    from oracle import acc
    from oracle import hamiltonian as H
    g = GOLDEN["si2"]
    w, sysm = load(si2)
    op = H.prepare(sysm)
    assert op.basis.npw == g["npw"]
    assert abs(sysm.veff.mean() - g["veff_mean_eV"]) <= 1e-9
    assert abs(sysm.veff.min() - g["veff_min_eV"]) <= 1e-9 and abs(sysm.veff.max() - g["veff_max_eV"]) <= 1e-9
    assert np.abs(np.asarray(sysm.dij_atoms[0][0]) - np.asarray(g["dij_atom0"])).max() <= 1e-9
    wd, _, smin, smax = H.solve_dense(op, len(g["dense_eigenvalues_eV"]))
    assert np.abs(wd - np.asarray(g["dense_eigenvalues_eV"])).max() <= 1e-9
    assert abs(smin - g["overlap_min"]) <= 1e-9 and abs(smax - g["overlap_max"]) <= 1e-9
    r = acc.solve_acc(op, 8, tol=1e-4, max_iterations=40)
    ga = g["acc_m8_tol1e-4_it40"]
    assert r.iterations == ga["iterations"]
    assert np.abs(r.eigenvalues - np.asarray(ga["eigenvalues_eV"])).max() <= 1e-9
    assert H.prepare(sysm, (0.125, 0.25, 0.375)).basis.npw == g["npw_k_0.125_0.25_0.375"]


def test_si2c_ionic_terms_and_output_density(si2c):
    from oracle import hamiltonian as H
    from oracle import ionforces as I
    g = GOLDEN["si2c_ionic"]
    w, sysm = load(si2c)
    shape = tuple(sysm.shape)
    rng = np.random.default_rng(5)
    out_f = np.asarray(sysm.values) * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, size=len(sysm.values)))
    charges = np.repeat([p.zval for p in sysm.potcars], sysm.crystal.counts)
    assert np.abs(np.asarray(I.ewald_energy(sysm.crystal, charges)) - np.asarray(g["ewald_energy_eV"])).max() <= 1e-9
    assert np.abs(I.ewald_forces(sysm.crystal, charges) - np.asarray(g["ewald_forces"])).max() <= 1e-9
    fl, el = I.local_ionic_forces(out_f, sysm.potcars, sysm.crystal, shape)
    assert abs(el - g["local_energy_eV"]) <= 1e-9 and np.abs(fl - np.asarray(g["local_forces"])).max() <= 1e-9
    vxc = I.xc_potential(sysm.values, sysm.potcars, sysm.crystal, shape, True)
    assert np.abs(I.radial_density_forces(vxc, sysm.potcars, sysm.crystal, shape)
                  - np.asarray(g["nlcc_forces"])).max() <= 1e-9
    fh = I.harris_correction_forces(sysm.values, out_f, sysm.potcars, sysm.crystal, shape, True)
    assert np.abs(fh - np.asarray(g["harris_forces"])).max() <= 1e-9
    op = H.prepare(sysm)
    _, v, _, _ = H.solve_dense(op, 6, vectors=True)
    occ = np.array([2.0, 2.0, 2.0, 1.0, 1.0, 0.0])
    rho = I.smooth_density(op.basis, v, occ, 1.0, shape)
    rho_out, aug = I.add_augmentation_density(sysm.potcars, sysm.crystal, shape,
                                              I.augmentation_occupancy(op.species, v, occ, 1.0), rho)
    gs = g["gamma_6_states"]
    assert abs(rho.mean() - gs["smooth_mean"]) <= 1e-9 * abs(gs["smooth_mean"])
    assert abs(aug - gs["augmentation_charge"]) <= 1e-9 * max(1.0, abs(gs["augmentation_charge"]))
    assert abs(rho_out.sum() - gs["output_density_sum"]) <= 1e-9 * abs(gs["output_density_sum"])
    assert abs(rho_out.max() - gs["output_density_max"]) <= 1e-9 * abs(gs["output_density_max"])
