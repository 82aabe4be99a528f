"""Ion-position force terms on the GPU (half_ionic_forces) against the oracle
restatement of src/half_energy.F90:122-210 and src/half_local_forces.F90,
whose own pins (forces = minus the position derivative of their energies)
are in test_ionforces.py.

si2c carries a partial core (PBE), so every term is non-zero there; hfo2 has
no core, so NLCC and Harris must come back exactly zero.  The output density
is the input density with a seeded +-5 % modulation.
Tolerances: Ewald and local forces 1e-9 eV/A, their energies 1e-8 eV; NLCC
1e-8 eV/A; Harris 1e-6 eV/A (a central difference of two V_xc with step
1e-4 in the density, which scales rounding in V_xc by 5e3).
"""
import numpy as np
import pytest

import halfb200
from conftest import workload_files

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def si2c(tmp_path_factory):
    return workload_files("si2c", str(tmp_path_factory.mktemp("si2c")))


def output_density(values, seed=5):
    r = np.random.default_rng(seed)
    return np.asarray(values) * (1.0 + 0.05 * r.uniform(-1.0, 1.0, size=len(values)))


def oracle_terms(sysm, out_f, use_pbe):
    from oracle import ionforces as I
    shape = tuple(sysm.shape)
    charges = np.repeat([p.zval for p in sysm.potcars], sysm.crystal.counts)
    ew = I.ewald_energy(sysm.crystal, charges)
    fl, el = I.local_ionic_forces(out_f, sysm.potcars, sysm.crystal, shape)
    vxc = I.xc_potential(sysm.values, sysm.potcars, sysm.crystal, shape, use_pbe)
    return dict(ewald=I.ewald_forces(sysm.crystal, charges), ewald_e=ew, local=fl, local_energy=el,
                nlcc=I.radial_density_forces(vxc, sysm.potcars, sysm.crystal, shape, use_core=True),
                harris=I.harris_correction_forces(sysm.values, out_f, sysm.potcars, sysm.crystal, shape, use_pbe))


def load(files):
    from oracle import hamiltonian as H
    w, ch, po = files
    return H.load_system(ch, po, w.encut, use_pbe=(w.xc == "pbe"), use_uspp=True)


def check(files, expect_core):
    w, ch, po = files
    sysm = load(files)
    out_f = output_density(sysm.values)
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="acc") as ctx:
        got = ctx.ionic_forces(out_f)
        same = ctx.ionic_forces(None)
    ref = oracle_terms(sysm, out_f, w.xc == "pbe")
    d = {k: float(np.abs(got[k] - ref[k]).max()) for k in ("ewald", "local", "nlcc", "harris")}
    print(w.name, "max |dF|", d, "max |F|", {k: float(np.abs(ref[k]).max()) for k in d})
    assert d["ewald"] <= 1e-9 and d["local"] <= 1e-9
    assert d["nlcc"] <= 1e-8 and d["harris"] <= 1e-6
    for i, key in enumerate(("ewald_energy", "ewald_real", "ewald_reciprocal", "ewald_self", "ewald_background")):
        assert abs(got[key] - ref["ewald_e"][i]) <= 1e-8, key
    assert abs(got["local_energy"] - ref["local_energy"]) <= 1e-8
    assert np.abs(got["ewald"].sum(axis=0)).max() < 1e-8          # translation invariance
    if expect_core:
        assert np.abs(ref["nlcc"]).max() > 1e-4 and np.abs(ref["harris"]).max() > 1e-6
    else:
        assert not got["nlcc"].any() and not got["harris"].any()
    # no output density: the Harris response vanishes and the local force acts on the input density
    assert not same["harris"].any()
    from oracle import ionforces as I
    fl, _ = I.local_ionic_forces(sysm.values, sysm.potcars, sysm.crystal, tuple(sysm.shape))
    assert np.abs(same["local"] - fl).max() <= 1e-9
    assert np.array_equal(same["ewald"], got["ewald"]) and np.array_equal(same["nlcc"], got["nlcc"])


def test_ionic_forces_si2c_partial_core(si2c):
    check(si2c, True)


def test_ionic_forces_hfo2(hfo2):
    check(hfo2, False)


def test_ionic_forces_rejects_wrong_grid(si2c):
    w, ch, po = si2c
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="acc") as ctx:
        with pytest.raises(halfb200.HalfError):
            ctx.ionic_forces(np.ones(10))


def oracle_output_density(sysm, kpts, wts, vecs, occ):
    """Smooth + augmentation density of given states (src/half_local_forces.F90:102-127,
    src/half_uspp.F90:26-111), and the augmentation charge."""
    from oracle import hamiltonian as H
    from oracle import ionforces as I
    shape = tuple(sysm.shape)
    rho = np.zeros(int(np.prod(shape)))
    occupancy = None
    for ik, k in enumerate(kpts):
        op = H.prepare(sysm, k)
        rho += I.smooth_density(op.basis, vecs[ik], occ[ik], wts[ik], shape)
        occupancy = I.augmentation_occupancy(op.species, vecs[ik], occ[ik], wts[ik], occupancy)
    return I.add_augmentation_density(sysm.potcars, sysm.crystal, shape, occupancy, rho)


KPTS = [(0.0, 0.0, 0.0), (0.25, 0.0, 0.25)]
WTS = [0.5, 0.5]


def test_output_density_matches_oracle(si2c):
    """The same eigenvectors through both sides: smooth + augmentation density to
    1e-10 of its maximum, augmentation charge to 1e-10."""
    from oracle import hamiltonian as H
    w, ch, po = si2c
    sysm = load(si2c)
    nb = 8
    vecs = [H.solve_dense(H.prepare(sysm, k), nb, vectors=True)[1] for k in KPTS]
    occ = np.array([[2.0, 2.0, 2.0, 1.5, 1.0, 0.5, 0.0, 0.0], [2.0, 2.0, 1.5, 1.5, 1.0, 0.25, 0.1, 0.0]])
    ref, ref_q = oracle_output_density(sysm, KPTS, WTS, vecs, occ)
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="acc") as ctx:
        got, q = ctx.output_density(KPTS, WTS, vecs, occ)
    print("max |drho|", np.abs(got - ref).max(), "max rho", np.abs(ref).max(), "aug", q, ref_q)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    assert abs(q - ref_q) <= 1e-10 and abs(ref_q) > 1e-4


def test_forces_end_to_end_matches_oracle(si2c):
    """half_forces (dense solves) against the oracle chain: dense solves, occupations,
    non-local force, output density, ion-position terms.  Components to 1e-8 eV/A
    (Harris 1e-6), energies to 1e-8 eV."""
    from oracle import hamiltonian as H
    from oracle import ionforces as I
    from oracle.forces import compute_occupations, nonlocal_forces
    w, ch, po = si2c
    nb, nelect, sigma = 16, 8.0, 0.1
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as ctx:
        r = ctx.forces(KPTS, WTS, nb, nelect, sigma, -1)
    from oracle.hamiltonian import load_system
    sysm = load_system(ch, po, w.encut, use_pbe=(w.xc == "pbe"), use_uspp=True, with_gradient=True)
    eig, vecs, ops = [], [], []
    for k in KPTS:
        op = H.prepare(sysm, k)
        e, v, _, _ = H.solve_dense(op, nb, vectors=True)
        eig.append(e); vecs.append(v); ops.append(op)
    occ, mu, band, ent = compute_occupations(np.array(eig), WTS, nelect, sigma, -1)
    nonloc = np.zeros((sysm.crystal.nions, 3))
    for ik, op in enumerate(ops):
        nonlocal_forces(op.basis, op.species, sysm.dij_atoms, sysm.ddij_atoms, eig[ik], occ[ik], WTS[ik], vecs[ik],
                        forces=nonloc)
    rho_out, q = oracle_output_density(sysm, KPTS, WTS, vecs, occ)
    ref = oracle_terms(sysm, rho_out, w.xc == "pbe")
    d = {"nonlocal": float(np.abs(r["nonlocal"] - nonloc).max())}
    for key in ("ewald", "local", "nlcc", "harris"):
        d[key] = float(np.abs(r[key] - ref[key]).max())
    total = ref["ewald"] + ref["local"] + nonloc + ref["nlcc"] + ref["harris"]
    d["total"] = float(np.abs(r["forces"] - total).max())
    print("max |dF|", d, "max |F|", float(np.abs(total).max()))
    assert max(d[k] for k in ("nonlocal", "ewald", "local", "nlcc")) <= 1e-8
    assert d["harris"] <= 1e-6 and d["total"] <= 1e-6
    assert np.abs(r["output_density"] - rho_out).max() <= 1e-9 * np.abs(rho_out).max()
    assert abs(r["band_energy"] - band) <= 1e-8 and abs(r["mu"] - mu) <= 1e-8
    assert abs(r["ewald_energy"] - ref["ewald_e"][0]) <= 1e-8
    assert abs(r["local_energy"] - ref["local_energy"]) <= 1e-8
    assert abs(r["augmentation_charge"] - q) <= 1e-9


def test_forces_rejects_an_occupied_top_band(si2c):
    w, ch, po = si2c
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as ctx:
        with pytest.raises(halfb200.HalfError):
            ctx.forces(KPTS, WTS, 4, 8.0, 0.1, -1)


def test_device_buffers_give_the_host_results(si2c):
    """half_output_density and half_ionic_forces read device eigenvectors and a device
    density in place; the results are the host-buffer results bit for bit."""
    import ctypes as C
    import torch
    from oracle import hamiltonian as H
    w, ch, po = si2c
    sysm = load(si2c)
    nb = 6
    vecs = [H.solve_dense(H.prepare(sysm, k), nb, vectors=True)[1] for k in KPTS]
    occ = np.array([[2.0, 2.0, 2.0, 1.0, 0.5, 0.0], [2.0, 2.0, 1.5, 1.5, 0.5, 0.0]])
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="acc") as ctx:
        host_rho, host_q = ctx.output_density(KPTS, WTS, vecs, occ)
        ld = max(v.shape[0] for v in vecs)
        block = np.zeros((len(KPTS), nb, ld), dtype=np.complex128)
        for ik, v in enumerate(vecs):
            block[ik, :, :v.shape[0]] = v.T
        dvec = torch.from_numpy(block.view(np.float64).copy()).cuda()
        drho = torch.zeros(host_rho.size, dtype=torch.float64, device="cuda")
        ks = np.ascontiguousarray(np.asarray(KPTS, dtype=np.float64))
        ws = np.ascontiguousarray(np.asarray(WTS, dtype=np.float64))
        oc = np.ascontiguousarray(occ)
        q = C.c_double(0.0)
        err = C.create_string_buffer(256)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        st = ctx.lib.half_output_density(ctx.handle, len(KPTS), p(ks), p(ws), nb, ld, C.c_void_p(dvec.data_ptr()),
                                         p(oc), C.c_void_p(drho.data_ptr()), host_rho.size, C.byref(q), err, 256)
        assert st == halfb200.HALF_SUCCESS, err.value
        torch.cuda.synchronize()
        assert np.array_equal(drho.cpu().numpy(), host_rho) and q.value == host_q
        host_f = ctx.ionic_forces(host_rho)
        outs = [np.zeros((ctx.nions, 3)) for _ in range(4)]
        en = np.zeros(6)
        st = ctx.lib.half_ionic_forces(ctx.handle, C.c_void_p(drho.data_ptr()), host_rho.size, *[p(o) for o in outs],
                                       p(en), err, 256)
        assert st == halfb200.HALF_SUCCESS, err.value
        for o, key in zip(outs, ("ewald", "local", "nlcc", "harris")):
            assert np.array_equal(o, host_f[key]), key


def test_sharded_forces_on_one_rank_is_half_forces(si2c):
    """halfb200.shard.sharded_forces composes the per-k entry points (solve,
    half_occupations, half_nonlocal_forces, half_output_density,
    half_ionic_forces); on one rank it must give what half_forces gives in one
    call, to 1e-10 of each quantity's size."""
    from halfb200.shard import sharded_forces
    w, ch, po = si2c
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="evd") as ctx:
        a = ctx.forces(KPTS, WTS, 16, 8.0, 0.1, -1)
        b = sharded_forces(ctx, KPTS, WTS, 16, 8.0, 0.1, -1)
    for key in ("forces", "ewald", "local", "nonlocal", "nlcc", "harris", "output_density"):
        assert np.abs(a[key] - b[key]).max() <= 1e-10 * max(1.0, np.abs(a[key]).max()), key
    for key in ("band_energy", "entropy", "mu", "ewald_energy", "local_energy", "augmentation_charge"):
        assert abs(a[key] - b[key]) <= 1e-10 * max(1.0, abs(a[key])), key
