"""PAW projectors and per-species D/Q tables, restated from src/half_paw.F90.

B[g, (iat, ilm)] = Omega^-1/2 (-i)^l beta_l(|q|) Y_lm(q^) exp(-i q.R_iat)
(half_paw.F90:52-65; GPU twin half_cuda_assembly.cuf:150-170).  beta_l is a
cubic spline on a uniform 100-point grid of spacing gmax/100 with the
reference's end conditions (half_paw.F90:78-107), zeroed for |q| > 0.99 gmax
(:63).  Y_lm are the reference's real harmonics (:109-143).
"""
from __future__ import annotations

from dataclasses import dataclass
import math

import numpy as np


def spline_second(y, xmax):
    """Second-derivative table M (half_paw.F90:78-99)."""
    y = np.asarray(y, dtype=float)
    n = len(y)
    h = xmax / n
    diag = np.zeros(n); rhs = np.zeros(n); upper = np.zeros(n)
    diag[1] = 1.0
    rhs[1] = ((y[2] - y[1]) / h - (y[1] - y[0]) / h) / h
    for i in range(2, n - 2):            # Fortran i=3..n-2
        diag[i] = 4 * h; upper[i] = h
        rhs[i] = 6 * ((y[i + 1] - y[i]) / h - (y[i] - y[i - 1]) / h)
    diag[n - 2] = 1.0
    rhs[n - 2] = ((y[n - 1] - y[n - 2]) / h - (y[n - 2] - y[n - 3]) / h) / h
    for i in range(2, n - 1):            # Fortran i=3..n-1
        w = (h if i <= n - 3 else 0.0) / diag[i - 1]
        diag[i] = diag[i] - w * upper[i - 1]
        rhs[i] = rhs[i] - w * rhs[i - 1]
    m2 = np.zeros(n)
    m2[n - 2] = rhs[n - 2] / diag[n - 2]
    for i in range(n - 3, 0, -1):        # Fortran i=n-2..2
        m2[i] = (rhs[i] - upper[i] * m2[i + 1]) / diag[i]
    m2[0] = 2 * m2[1] - m2[2]
    m2[n - 1] = 2 * m2[n - 2] - m2[n - 3]
    return m2


def spline_eval(y, m2, xmax, x):
    """Vectorised half_paw.F90:101-107 (k clamped to [1, n-1], 1-based)."""
    y = np.asarray(y); m2 = np.asarray(m2)
    x = np.asarray(x, dtype=float)
    n = len(y)
    h = xmax / n
    k = np.clip(np.floor(x / h).astype(np.int64) + 1, 1, n - 1)  # 1-based
    t = (x - (k - 1) * h) / h
    k0 = k - 1
    return ((1 - t) * y[k0] + t * y[k0 + 1]
            + h * h * (((1 - t) ** 3 - (1 - t)) * m2[k0] + (t ** 3 - t) * m2[k0 + 1]) / 6)


def _factorial(n):
    v = 1.0
    for i in range(2, n + 1):
        v *= i
    return v


def assoc_legendre(l, m, x):
    """half_paw.F90:124-137 (Condon-Shortley phase included)."""
    x = np.asarray(x, dtype=float)
    pmm = np.ones_like(x)
    if m > 0:
        fact = 1.0
        s = np.sqrt(np.maximum(0.0, (1 - x) * (1 + x)))
        for _ in range(m):
            pmm = -pmm * fact * s
            fact += 2
    if l == m:
        return pmm
    pmmp1 = x * (2 * m + 1) * pmm
    if l == m + 1:
        return pmmp1
    for ll in range(m + 2, l + 1):
        pll = ((2 * ll - 1) * x * pmmp1 - (ll + m - 1) * pmm) / (ll - m)
        pmm, pmmp1 = pmmp1, pll
    return pmmp1


def real_ylm_x(l, m, x, phi):
    """Real Y_lm from x = cos(theta) (half_paw.F90:109-123, half_uspp.F90:377-384)."""
    am = abs(m)
    p = assoc_legendre(l, am, x)
    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * _factorial(l - am) / _factorial(l + am))
    if m > 0:
        return math.sqrt(2.0) * (-1.0) ** m * norm * p * np.cos(am * phi)
    if m < 0:
        return math.sqrt(2.0) * (-1.0) ** m * norm * p * np.sin(am * phi)
    return norm * p


def lm_list(lps):
    """Channel -> (ich, l, m) expansion, channel-major then m=-l..l (half_paw.F90:39-52)."""
    out = []
    for ich, l in enumerate(lps):
        for m in range(-l, l + 1):
            out.append((ich, l, m))
    return out


def species_tables(pot):
    """Expanded per-species dij, qij (nlm x nlm): nonzero only for equal (l, m)
    (half_paw.F90:41-51)."""
    lm = lm_list(pot.lps)
    nlm = len(lm)
    dij = np.zeros((nlm, nlm)); qij = np.zeros((nlm, nlm))
    for a, (ia, la, ma) in enumerate(lm):
        for b, (ib, lb, mb) in enumerate(lm):
            if la == lb and ma == mb:
                dij[a, b] = pot.dion[ia, ib]
                qij[a, b] = pot.qpaw[ia, ib]
    return dij, qij


@dataclass
class SpeciesProjectors:
    natoms: int
    nlm: int
    B: np.ndarray            # (npw, natoms*nlm) complex128, column (iat*nlm + ilm)
    dij: np.ndarray          # (nlm, nlm) species DION expansion
    qij: np.ndarray          # (nlm, nlm)


def build_projectors(potcars, crystal, basis):
    """build_paw_operators (half_paw.F90:18-76), stored as the GPU column layout
    index = ig + (ilm-1)*n + (iat-1)*n*nlm (half_cuda_assembly.cuf:167)."""
    out = []
    pref = 1.0 / math.sqrt(crystal.volume)
    q = basis.qvectors
    qn = np.sqrt(q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2])
    safe = qn > 1.0e-10
    theta = np.where(safe, np.arccos(np.clip(np.where(safe, q[:, 2] / np.where(safe, qn, 1.0), 1.0), -1.0, 1.0)), 0.0)
    phi = np.where(safe, np.arctan2(q[:, 1], q[:, 0]), 0.0)
    x = np.cos(theta)
    cart = crystal.cartesian()
    ion0 = 0
    for it, pot in enumerate(potcars):
        nat = crystal.counts[it]
        lm = lm_list(pot.lps)
        nlm = len(lm)
        B = np.zeros((basis.npw, nat * nlm), dtype=np.complex128)
        radial = []
        for ich in range(pot.channels):
            m2 = spline_second(pot.pspnl[:, ich], pot.pspnl_gmax)
            r = spline_eval(pot.pspnl[:, ich], m2, pot.pspnl_gmax, qn)
            r = np.where(qn > 0.99 * pot.pspnl_gmax, 0.0, r)
            radial.append(r)
        for ilm, (ich, l, m) in enumerate(lm):
            ilfac = (-1j) ** l
            ylm = real_ylm_x(l, m, x, phi)
            for iat in range(nat):
                rpos = cart[ion0 + iat]
                phase = q[:, 0] * rpos[0] + q[:, 1] * rpos[1] + q[:, 2] * rpos[2]
                B[:, iat * nlm + ilm] = pref * ilfac * radial[ich] * ylm * (np.cos(phase) - 1j * np.sin(phase))
        dij, qij = species_tables(pot)
        out.append(SpeciesProjectors(nat, nlm, B, dij, qij))
        ion0 += nat
    return out
