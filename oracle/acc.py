"""The all-band ``acc`` block eigensolver, restated step by step from
src/half_cuda_iterative_solver.cuf:79-310.

Start: m unit vectors at the m lowest-kinetic plane waves in the reference's
heap order (:136-140, 277-310) and a Rayleigh-Ritz (:143, 209-228).  Each
iteration (:146-196): R = HX - eps SX; column norms (only the diagonal of the
reference's R^H R Gram is used, :148-155); bands with norm below
max(1e-2 tol, 1e-12) get the unit seed at plane wave (m+j) mod n (:153-154);
stop when max norm <= tol; P = -R/(|T-eps|+1 eV) or the seed (:42-64);
apply H,S to P; S-orthogonalise P against X (:163-170); normalise P in the S
metric through eigh(P^H S P) with the 1e-14 floor (:173-182); Rayleigh-Ritz on
Z = [X P] with a generalized 2m eigensolve (:184-195).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.linalg as sla

from .hamiltonian import apply_hs


def kinetic_order(kinetic):
    """Heap sort of half_cuda_iterative_solver.cuf:277-310 (0-based result)."""
    kin = np.asarray(kinetic)
    n = len(kin)
    idx = list(range(1, n + 1))           # 1-based heap like the reference
    ind = [0] + idx                       # ind[1..n]
    for i in range(2, n + 1):
        child = i
        while child > 1:
            parent = child // 2
            if kin[ind[parent] - 1] >= kin[ind[child] - 1]:
                break
            ind[parent], ind[child] = ind[child], ind[parent]
            child = parent
    for last in range(n, 1, -1):
        ind[1], ind[last] = ind[last], ind[1]
        parent = 1
        while True:
            child = 2 * parent
            if child > last - 1:
                break
            if child + 1 <= last - 1 and kin[ind[child + 1] - 1] > kin[ind[child] - 1]:
                child += 1
            if kin[ind[parent] - 1] >= kin[ind[child] - 1]:
                break
            ind[parent], ind[child] = ind[child], ind[parent]
            parent = child
    return np.array(ind[1:], dtype=np.int64) - 1


def _gen_eigh(h, s):
    """zhegvd type 1, upper triangles (:242-259)."""
    return sla.eigh(h, s, lower=False, type=1, driver="gvd")


@dataclass
class AccResult:
    eigenvalues: np.ndarray
    vectors: np.ndarray
    iterations: int
    max_residual: float
    converged: bool
    history: list


def solve_acc(op, nbands, tol=1.0e-4, max_iterations=40, apply=None):
    n = op.basis.npw
    m = nbands
    if m < 1 or m > n:
        raise ValueError("invalid ACC target band count")
    if 2 * m > n:
        raise ValueError("ACC solver requires NBANDS <= NPL/2")
    app = apply or (lambda p: apply_hs(op, p))
    kin = op.basis.kinetic
    order = kinetic_order(kin)
    x = np.zeros((n, m), dtype=complex)
    x[order[:m], np.arange(m)] = 1.0
    hx, sx = app(x)
    hs = x.conj().T @ hx; ss = x.conj().T @ sx
    w, y = _gen_eigh(hs, ss)
    x, hx, sx = x @ y, hx @ y, sx @ y
    dw = w.copy()
    history = []
    converged = False
    max_res = np.inf
    it = 0
    for it in range(1, max_iterations + 1):
        r = hx - dw[None, :m] * sx
        norms = np.sqrt(np.maximum(0.0, np.einsum("ij,ij->j", r.conj(), r).real))
        max_res = float(norms.max())
        history.append(max_res)
        seeds = np.where(norms < max(tol * 1e-2, 1e-12), (m + np.arange(m)) % n, -1)
        if max_res <= tol:
            converged = True
            break
        p = -r / (np.abs(kin[:, None] - dw[None, :m]) + 1.0)
        for j in np.nonzero(seeds >= 0)[0]:
            p[:, j] = 0.0
            p[seeds[j], j] = 1.0
        hp, sp = app(p)
        c = x.conj().T @ sp
        p = p - x @ c; hp = hp - hx @ c; sp = sp - sx @ c
        metric = p.conj().T @ sp
        mu, u = sla.eigh(metric, lower=False, driver="evd")
        u = u / np.sqrt(np.maximum(mu, 1.0e-14))[None, :]
        p, hp, sp = p @ u, hp @ u, sp @ u
        z = np.concatenate([x, p], axis=1)
        hz = np.concatenate([hx, hp], axis=1)
        sz = np.concatenate([sx, sp], axis=1)
        hs = z.conj().T @ hz; ss = z.conj().T @ sz
        w, y = _gen_eigh(hs, ss)
        dw = w
        ym = y[:, :m]
        x, hx, sx = z @ ym, hz @ ym, sz @ ym
    iters = min(it, max_iterations)
    return AccResult(dw[:m].copy(), x, iters, max_res, converged, history)
