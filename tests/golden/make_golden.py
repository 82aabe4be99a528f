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
from oracle import acc, hamiltonian as H  # noqa: E402


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
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()
