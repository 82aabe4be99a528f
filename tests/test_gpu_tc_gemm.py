"""The tensor-core complex GEMM (half_tc_cgemm) against FP64 products.

Shapes are the mixed mode's: the subspace inner products X^H Y (m x m,
K = plane waves), the rotations X Y (plane waves x m, K = m) and the projector
products, on the 12-atom cell (3411 plane waves, 72 bands with guards) and on
the 216-atom cell (38066 plane waves, 540 bands with guards; >= 5e9
multiply-adds).  The split bf16 product (hi*hi + hi*lo + lo*hi, FP32
accumulation) is accurate to about 2^-16 of sum_k |a_ik| |b_kj|; the test
allows 4e-5 of that sum per element.
"""
import numpy as np
import pytest

import halfb200

TOL = 4e-5


def _torch():
    import torch
    return torch


def _dev(a, dtype):
    """Column-major device copy of a host matrix."""
    torch = _torch()
    return torch.from_numpy(np.asfortranarray(a.astype(dtype))).cuda()


def _op(x, op):
    return x if op == "N" else (x.T if op == "T" else x.conj().T)


def _run(op_a, op_b, m, n, k, lda_pad=0, ldb_pad=0, ldc_pad=0, alpha=1.0 + 0j, beta=0.0 + 0j, c_fp64=False, seed=0,
         on_gpu_ref=False):
    torch = _torch()
    rng = np.random.default_rng(seed)
    ar, ac = (m, k) if op_a == "N" else (k, m)
    br, bc = (k, n) if op_b == "N" else (n, k)
    a = (rng.standard_normal((ar + lda_pad, ac)) + 1j * rng.standard_normal((ar + lda_pad, ac))).astype(np.complex64)
    b = (rng.standard_normal((br + ldb_pad, bc)) + 1j * rng.standard_normal((br + ldb_pad, bc))).astype(np.complex64)
    c0 = (rng.standard_normal((m + ldc_pad, n)) + 1j * rng.standard_normal((m + ldc_pad, n)))
    cdt = np.complex128 if c_fp64 else np.complex64
    c0 = c0.astype(cdt)
    da, db, dc = _dev(a, np.complex64), _dev(b, np.complex64), _dev(c0, cdt)
    halfb200.tc_cgemm(op_a, op_b, m, n, k, alpha, da.data_ptr(), max(1, ar + lda_pad), db.data_ptr(),
                      max(1, br + ldb_pad), beta, dc.data_ptr(), m + ldc_pad, c_fp64)
    torch.cuda.synchronize()
    got = dc.cpu().numpy()[:m]
    A = _op(a[:ar].astype(np.complex128), op_a)
    B = _op(b[:br].astype(np.complex128), op_b)
    if on_gpu_ref:
        tA, tB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
        ref = (alpha * (tA @ tB)).cpu().numpy() + beta * c0[:m].astype(np.complex128)
        mag = (tA.abs() @ tB.abs()).cpu().numpy()
    else:
        ref = alpha * (A @ B) + beta * c0[:m].astype(np.complex128)
        mag = np.abs(A) @ np.abs(B)
    err = np.abs(got - ref)
    bound = TOL * abs(alpha) * mag + 1e-6 * np.abs(beta * c0[:m]) + 1e-30
    ratio = float((err / bound).max())
    # the untouched padding rows of C keep their values
    if ldc_pad:
        assert np.array_equal(dc.cpu().numpy()[m:], c0[m:])
    return ratio, float((err / (np.abs(ref) + 1e-30)).max())


@pytest.mark.gpu
@pytest.mark.parametrize("op_a,op_b", [("C", "N"), ("T", "N"), ("N", "N"), ("N", "T"), ("N", "C"), ("C", "C")])
def test_tc_cgemm_every_operation(op_a, op_b):
    ratio, _ = _run(op_a, op_b, 72, 72, 3411, lda_pad=3, ldb_pad=5, ldc_pad=1)
    assert ratio < 1.0, (op_a, op_b, ratio)


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (5, 3, 7), (130, 17, 33), (129, 257, 16), (200, 300, 1000)])
def test_tc_cgemm_ragged_shapes(m, n, k):
    ratio, _ = _run("C", "N", m, n, k, lda_pad=1, ldb_pad=1, alpha=0.5 - 2j, beta=0.25 + 1j)
    assert ratio < 1.0
    ratio, _ = _run("N", "N", m, n, k, lda_pad=1, ldb_pad=1, alpha=-1.0, beta=1.0)
    assert ratio < 1.0


@pytest.mark.gpu
def test_tc_cgemm_fp64_output_split_k():
    # inner product with K = plane waves: split-K partial sums reduced in FP64
    ratio, _ = _run("C", "N", 144, 144, 3411, c_fp64=True)
    assert ratio < 1.0
    ratio, _ = _run("C", "N", 72, 136, 3411, c_fp64=True, alpha=2.0, beta=-1.0)
    assert ratio < 1.0


@pytest.mark.gpu
def test_tc_cgemm_k_zero_scales_c():
    ratio, _ = _run("N", "N", 40, 24, 0, beta=0.5 + 0.5j)
    assert ratio < 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("op_a,op_b,m,n,k,c_fp64", [
    ("C", "N", 540, 540, 38066, True),     # X^H H X at c4 (split-K, FP64 output)
    ("N", "N", 38066, 540, 540, False),    # X Y rotation at c4 (1.1e10 multiply-adds)
    ("C", "N", 1696, 540, 38066, False),   # B^H X projector coefficients at c4
])
def test_tc_cgemm_large_cell_shapes(op_a, op_b, m, n, k, c_fp64):
    ratio, rel = _run(op_a, op_b, m, n, k, c_fp64=c_fp64, seed=3, on_gpu_ref=True)
    assert ratio < 1.0, (ratio, rel)


@pytest.mark.gpu
def test_tc_cgemm_rejects_host_memory_and_bad_ops():
    a = np.zeros((4, 4), dtype=np.complex64)
    with pytest.raises(halfb200.HalfError) as e:
        halfb200.tc_cgemm("N", "N", 4, 4, 4, 1.0, a.ctypes.data, 4, a.ctypes.data, 4, 0.0, a.ctypes.data, 4)
    assert e.value.status == halfb200.HALF_ERROR_INVALID_ARGUMENT
    torch = _torch()
    d = torch.zeros((4, 4), dtype=torch.complex64, device="cuda")
    with pytest.raises(halfb200.HalfError) as e:
        halfb200.tc_cgemm("X", "N", 4, 4, 4, 1.0, d.data_ptr(), 4, d.data_ptr(), 4, 0.0, d.data_ptr(), 4)
    assert e.value.status == halfb200.HALF_ERROR_INVALID_ARGUMENT
    with pytest.raises(halfb200.HalfError) as e:
        halfb200.tc_cgemm("N", "N", 4, 4, 4, 1.0, d.data_ptr(), 3, d.data_ptr(), 4, 0.0, d.data_ptr(), 4)
    assert e.value.status == halfb200.HALF_ERROR_CAPACITY
