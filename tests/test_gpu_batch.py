"""half_solve_kpoints_device: the batched solve writing eigenpairs to device
memory equals per-k half_solve_kpoint results (same algorithm, deterministic),
pads rows beyond each k point's basis with zeros, and rejects a too-small
leading dimension and host buffers."""
import numpy as np
import pytest

import halfb200

pytestmark = pytest.mark.gpu


def test_device_batch_matches_host_solves(si2):
    torch = pytest.importorskip("torch")
    w, ch, po = si2
    ks = np.array([[0.0, 0.0, 0.0], [0.25, 0.0, 0.25], [0.125, 0.25, 0.375]])
    nb = 8
    with halfb200.Context(ch, po, w.encut, xc=w.xc, solver="acc") as ctx:
        ctx.set_acc(tol=1e-8, max_iterations=400, precision="fp64")
        npw = [ctx.npw(k) for k in ks]
        ld = max(npw) + 3
        eig = torch.zeros((len(ks), nb), dtype=torch.float64, device="cuda")
        vec = torch.full((len(ks), nb, ld), 7.0 + 0.0j, dtype=torch.complex128, device="cuda")
        ctx.solve_kpoints_device(ks, nb, eig.data_ptr(), vec.data_ptr(), ld)
        e_dev = eig.cpu().numpy()
        v_dev = vec.cpu().numpy()
        for i, k in enumerate(ks):
            e, v, _, _ = ctx.solve(tuple(k), nb, vectors=True)
            assert np.array_equal(e_dev[i], e)
            assert np.array_equal(v_dev[i, :, :npw[i]], v.T)
            assert np.all(v_dev[i, :, npw[i]:] == 0)
        eig2 = torch.zeros_like(eig)
        ctx.solve_kpoints_device(ks, nb, eig2.data_ptr())
        assert torch.equal(eig2, eig)
        with pytest.raises(halfb200.HalfError) as small:
            ctx.solve_kpoints_device(ks, nb, eig.data_ptr(), vec.data_ptr(), min(npw) - 1)
        assert small.value.status == halfb200.HALF_ERROR_CAPACITY
        host = np.zeros((len(ks), nb))
        with pytest.raises(halfb200.HalfError) as onhost:
            ctx.solve_kpoints_device(ks, nb, host.ctypes.data)
        assert onhost.value.status == halfb200.HALF_ERROR_INVALID_ARGUMENT
