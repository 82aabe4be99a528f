"""The band-energy force at the force workload's full size: the 64-atom
Si-like cell with seeded displacements (sigma 0.05 A per component), Gamma
plus 3 k points, 160 bands, 256 electrons, Fermi-Dirac width 0.1 eV.

The analytic non-local force (src/half_forces.F90:9-73: projector phases and
dD_ij/dR) is computed from acc eigenpairs in FP64 mode and in mixed
precision, and compared with
  * the same force from dense FP64 evd eigenpairs (all components), and
  * minus the central difference (step 1e-3 A) of the Mermin band free
    energy sum_k w_k sum_n f_nk eps_nk + entropy from dense evd re-solves of
    the displaced cell at fixed Veff and basis, for a sample of atoms and
    Cartesian components,
to 1e-5 eV/A.  The acc tolerance is 1e-7 eV: the force is first order in the
eigenvector error, which is about residual / gap.
"""
import numpy as np
import pytest

import halfb200
from conftest import workload_files

pytestmark = pytest.mark.gpu

H_STEP = 1e-3
TOL = 1e-5
SAMPLE = [(0, 0), (17, 1), (42, 2)]     # (atom, component)


def _forces(ctx, w):
    return ctx.band_forces(w.kpoints, w.kweights, w.nbands, w.nelect, w.sigma, -1)


@pytest.fixture(scope="module")
def c3(inputs_dir):
    return workload_files("si64d", inputs_dir)


def test_c3_forces_from_acc_match_dense_and_finite_differences(c3):
    w, ch, po = c3
    assert w.nions == 64 and len(w.kpoints) == 4 and w.nbands == 160
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as dctx:
        ref = _forces(dctx, w)
        f_dense = ref["forces"]
        assert ref["occupations"][:, -1].max() < 1e-6      # the band count covers the smearing
        lat_inv = np.linalg.inv(dctx.lattice)
        num = {}
        for i, a in SAMPLE:
            d = np.zeros(3)
            d[a] = H_STEP
            e = []
            for sgn in (1.0, -1.0):
                p = w.positions.copy()
                p[i] += sgn * d @ lat_inv
                dctx.set_positions(p)
                r = _forces(dctx, w)
                e.append(r["band_energy"] + r["entropy"])
            num[(i, a)] = -(e[0] - e[1]) / (2 * H_STEP)
        dctx.set_positions(w.positions)
    assert np.abs(f_dense).max() > 1e-2
    for (i, a), v in num.items():
        assert abs(f_dense[i, a] - v) <= TOL, (i, a, f_dense[i, a], v)
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="acc") as actx:
        for precision in ("fp64", "mixed"):
            actx.set_acc(tol=1e-7, max_iterations=2000, precision=precision)
            r = _forces(actx, w)
            f = r["forces"]
            assert np.abs(r["eigenvalues"] - ref["eigenvalues"])[:, :128].max() <= 1e-8, precision
            assert np.abs(f - f_dense).max() <= TOL, (precision, np.abs(f - f_dense).max())
            for (i, a), v in num.items():
                assert abs(f[i, a] - v) <= TOL, (precision, i, a, f[i, a], v)
