"""VASP wave-coefficient export (src/half_vaspwave.F90:94-154).

CPU: the oracle's sort-based permutation equals the reference's own
algorithm (a box lookup table walked gz -> gy -> gx, :143-154), restated here
as a plain loop on the small Si box.  GPU (half_pack_vasp_waves through the C
ABI): bit-exact against the oracle's packing for host and device inputs,
the size query, and the capacity check."""
import numpy as np
import pytest

import halfb200


def reference_loop_permutation(basis):
    nx, ny, nz = basis.shape
    lookup = np.zeros(nx * ny * nz, dtype=np.int64)
    for i, c in enumerate(basis.fft_index):
        lookup[c] = i + 1
    order = []
    for gz in range(nz):
        for gy in range(ny):
            for gx in range(nx):
                j = lookup[gx * ny * nz + gy * nz + gz]
                if j > 0:
                    order.append(j - 1)
    return np.array(order)


@pytest.mark.parametrize("k", [(0.0, 0.0, 0.0), (0.125, 0.25, 0.375)])
def test_permutation_matches_the_reference_loop(si2, oracle_system, k):
    from oracle.basis import build_basis
    from oracle.export import vasp_permutation
    sysm = oracle_system("si2", si2)
    b = build_basis(sysm.crystal, sysm.shape, sysm.encut, k)
    order = vasp_permutation(b)
    assert np.array_equal(order, reference_loop_permutation(b))
    assert np.array_equal(np.sort(order), np.arange(b.npw))


def oracle_inputs(files, oracle_system, name, kpts, nb):
    from oracle.basis import build_basis
    sysm = oracle_system(name, files)
    r = np.random.default_rng(7)
    bases = [build_basis(sysm.crystal, sysm.shape, sysm.encut, k) for k in kpts]
    waves = [r.normal(size=(b.npw, nb)) + 1j * r.normal(size=(b.npw, nb)) for b in bases]
    return bases, waves


@pytest.mark.gpu
def test_pack_vasp_waves_bit_exact(hfo2, oracle_system):
    from oracle.export import pack_vasp_waves
    kpts = [(0.0, 0.0, 0.0), (0.25, 0.0, 0.5), (0.1, 0.2, 0.3)]
    bases, waves = oracle_inputs(hfo2, oracle_system, "hfo2", kpts, 6)
    ref, ref_npw, ref_off = pack_vasp_waves(bases, waves)
    w, ch, po = hfo2
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="acc") as ctx:
        got, npws, offs = ctx.pack_vasp_waves(kpts, waves)
    assert np.array_equal(npws, ref_npw) and np.array_equal(offs, ref_off)
    assert got.dtype == np.float32 and np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
def test_pack_vasp_waves_device_buffers_and_capacity(si2, oracle_system):
    import ctypes as C
    import torch
    from oracle.export import pack_vasp_waves
    kpts = [(0.0, 0.0, 0.0), (0.25, 0.25, 0.0)]
    nb = 4
    bases, waves = oracle_inputs(si2, oracle_system, "si2", kpts, nb)
    ref, ref_npw, ref_off = pack_vasp_waves(bases, waves)
    ld = max(b.npw for b in bases) + 3
    block = np.zeros((len(kpts), nb, ld), dtype=np.complex128)
    for ik, v in enumerate(waves):
        block[ik, :, :v.shape[0]] = v.T
    w, ch, po = si2
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="acc") as ctx:
        dvec = torch.from_numpy(block.view(np.float64).copy()).cuda()
        dout = torch.zeros(ref.size, dtype=torch.float32, device="cuda")
        npws = np.zeros(len(kpts), dtype=np.int32)
        offs = np.zeros(len(kpts), dtype=np.int64)
        ks = np.ascontiguousarray(np.asarray(kpts, dtype=np.float64))
        err = C.create_string_buffer(256)
        st = ctx.lib.half_pack_vasp_waves(ctx.handle, len(kpts), ks.ctypes.data_as(C.c_void_p), nb, ld,
                                          C.c_void_p(dvec.data_ptr()), C.c_void_p(dout.data_ptr()), ref.size,
                                          npws.ctypes.data_as(C.c_void_p), offs.ctypes.data_as(C.c_void_p), err, 256)
        assert st == halfb200.HALF_SUCCESS, err.value
        torch.cuda.synchronize()
        assert np.array_equal(dout.cpu().numpy().view(np.uint32), ref.view(np.uint32))
        st = ctx.lib.half_pack_vasp_waves(ctx.handle, len(kpts), ks.ctypes.data_as(C.c_void_p), nb, ld,
                                          C.c_void_p(dvec.data_ptr()), C.c_void_p(dout.data_ptr()), ref.size - 1,
                                          npws.ctypes.data_as(C.c_void_p), offs.ctypes.data_as(C.c_void_p), err, 256)
        assert st == halfb200.HALF_ERROR_CAPACITY
