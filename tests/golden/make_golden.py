"""Generate tests/golden/golden.json from the CPU oracle.

    python tests/golden/make_golden.py

The fixtures pin the oracle's outputs for the seeded synthetic workloads
(inputs are regenerated deterministically by halfb200.synth), so GPU tests
can compare against them without re-running the slow dense solves, and the
CPU suite can detect any drift of the oracle itself.
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "deepaw-half_b200"))

from halfb200 import synth  # noqa: E402
from oracle import acc, hamiltonian as H, ionforces as I  # noqa: E402


def ionic_terms(d):
    """Ion-position force terms on si2c (partial core, PBE) for a seeded +-5 %
    modulation of the input density, and the output density of its 6 lowest
    states at Gamma."""
    w = synth.workload("si2c")
    ch, po = synth.write_inputs(w, d)
    sysm = H.load_system(ch, po, w.encut, use_pbe=True, use_uspp=True)
    shape = tuple(sysm.shape)
    rng = np.random.default_rng(5)
    out_f = np.asarray(sysm.values) * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, size=len(sysm.values)))
    charges = np.repeat([p.zval for p in sysm.potcars], sysm.crystal.counts)
    ew = I.ewald_energy(sysm.crystal, charges)
    fl, el = I.local_ionic_forces(out_f, sysm.potcars, sysm.crystal, shape)
    vxc = I.xc_potential(sysm.values, sysm.potcars, sysm.crystal, shape, True)
    op = H.prepare(sysm)
    _, v, _, _ = H.solve_dense(op, 6, vectors=True)
    occ = np.array([2.0, 2.0, 2.0, 1.0, 1.0, 0.0])
    rho = I.smooth_density(op.basis, v, occ, 1.0, shape)
    occupancy = I.augmentation_occupancy(op.species, v, occ, 1.0)
    rho_out, aug = I.add_augmentation_density(sysm.potcars, sysm.crystal, shape, occupancy, rho)
    return {"ewald_energy_eV": list(ew), "ewald_forces": I.ewald_forces(sysm.crystal, charges).tolist(),
            "local_energy_eV": el, "local_forces": fl.tolist(),
            "nlcc_forces": I.radial_density_forces(vxc, sysm.potcars, sysm.crystal, shape).tolist(),
            "harris_forces": I.harris_correction_forces(sysm.values, out_f, sysm.potcars, sysm.crystal, shape,
                                                        True).tolist(),
            "gamma_6_states": {"smooth_mean": float(rho.mean()), "augmentation_charge": aug,
                               "output_density_sum": float(rho_out.sum()),
                               "output_density_max": float(rho_out.max())}}


def main():
    out = {"generator": "tests/golden/make_golden.py", "note": "oracle outputs on seeded synthetic inputs"}
    with tempfile.TemporaryDirectory() as d:
        for name, nb_dense in (("si2", 16), ("hfo2", 72)):
            w = synth.workload(name)
            ch, po = synth.write_inputs(w, d)
            sysm = H.load_system(ch, po, w.encut, use_pbe=(w.xc == "pbe"), use_uspp=True)
            op = H.prepare(sysm)
            wd, _, smin, smax = H.solve_dense(op, nb_dense)
            rec = {"npw": int(op.basis.npw), "dense_eigenvalues_eV": wd.tolist(), "overlap_min": smin,
                   "overlap_max": smax, "veff_mean_eV": float(sysm.veff.mean()),
                   "veff_min_eV": float(sysm.veff.min()), "veff_max_eV": float(sysm.veff.max()),
                   "dij_atom0": sysm.dij_atoms[0][0].tolist()}
            if name == "si2":
                r = acc.solve_acc(op, 8, tol=1e-4, max_iterations=40)
                rec["acc_m8_tol1e-4_it40"] = {"eigenvalues_eV": r.eigenvalues.tolist(), "iterations": r.iterations,
                                              "max_residual_eV": r.max_residual}
                kop = H.prepare(sysm, (0.125, 0.25, 0.375))
                rec["npw_k_0.125_0.25_0.375"] = int(kop.basis.npw)
            out[name] = rec
        out["si2c_ionic"] = ionic_terms(d)
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()
