"""Plane-wave basis, restated from src/half_basis.F90:9-55.

Order: n1 outermost, then n2, then n3, each over [-n/2, (n-1)/2]; a G vector
is kept when hbar^2/2m |k+G|^2 < ENCUT.  ``fft_index`` is the 0-based C-order
box index modulo(n1,s1)*s2*s3 + modulo(n2,s2)*s3 + modulo(n3,s3) (the
reference stores it 1-based, :191-194).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .constants import HSQDTM


@dataclass
class Basis:
    shape: tuple
    kpoint: np.ndarray
    gvectors: np.ndarray   # (npw,3) int32
    qvectors: np.ndarray   # (npw,3) float64, Angstrom^-1
    kinetic: np.ndarray    # (npw,) eV
    fft_index: np.ndarray  # (npw,) int64, 0-based C order

    @property
    def npw(self):
        return len(self.kinetic)


def build_basis(crystal, shape, encut, kpoint=(0.0, 0.0, 0.0)):
    if encut <= 0:
        raise ValueError("ENCUT must be positive")
    s1, s2, s3 = shape
    rec = crystal.reciprocal
    k = np.asarray(kpoint, dtype=float)
    r1 = np.arange(-(s1 // 2), (s1 - 1) // 2 + 1)
    r2 = np.arange(-(s2 // 2), (s2 - 1) // 2 + 1)
    r3 = np.arange(-(s3 // 2), (s3 - 1) // 2 + 1)
    n1, n2, n3 = np.meshgrid(r1, r2, r3, indexing="ij")
    n1, n2, n3 = n1.ravel(), n2.ravel(), n3.ravel()
    frac = np.stack([n1 + k[0], n2 + k[1], n3 + k[2]], axis=1)
    # q = matmul([n+k], reciprocal): row vector times matrix (half_basis.F90:167)
    q = frac[:, 0:1] * rec[0] + frac[:, 1:2] * rec[1] + frac[:, 2:3] * rec[2]
    kin = HSQDTM * (q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2])
    keep = kin < encut
    g = np.stack([n1[keep], n2[keep], n3[keep]], axis=1).astype(np.int32)
    idx = (np.mod(g[:, 0], s1).astype(np.int64) * s2 * s3
           + np.mod(g[:, 1], s2).astype(np.int64) * s3
           + np.mod(g[:, 2], s3).astype(np.int64))
    return Basis(tuple(shape), k, g, q[keep].copy(), kin[keep].copy(), idx)
