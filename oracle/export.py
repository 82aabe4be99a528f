"""Oracle (test infrastructure): the VASP wave-coefficient export of
src/half_vaspwave.F90:94-154, restated in numpy.

* vasp_permutation (:143-154): the basis points in the box's x-fastest order
  (gz outermost, then gy, then gx), i.e. ascending file-order index
  gx + nx*(gy + ny*gz) of each point's box position;
* the packed single-precision array (:117-127): per k point, band-major,
  interleaved (re, im) of the coefficient at order(ig), converted with
  real(., c_float) (round to nearest); offsets in floats, 2*npw*nb per k.

Only tests/ may import this module.
"""
from __future__ import annotations

import numpy as np


def vasp_permutation(basis):
    nx, ny, nz = basis.shape
    idx = np.asarray(basis.fft_index, dtype=np.int64)     # 0-based C order: gx*ny*nz + gy*nz + gz
    gx, rem = np.divmod(idx, ny * nz)
    gy, gz = np.divmod(rem, nz)
    return np.argsort(gx + nx * (gy + ny * gz), kind="stable")


def pack_vasp_waves(bases, waves):
    """(packed float32, npws int32, offsets int64) for per-k (npw, nb) coefficient blocks."""
    npws = np.array([b.npw for b in bases], dtype=np.int32)
    nb = waves[0].shape[1]
    offsets = np.concatenate([[0], np.cumsum(2 * npws.astype(np.int64) * nb)[:-1]]).astype(np.int64)
    parts = []
    for b, w in zip(bases, waves):
        order = vasp_permutation(b)
        c = np.asarray(w)[order, :].T                        # (nb, npw)
        parts.append(np.stack([c.real.astype(np.float32), c.imag.astype(np.float32)], axis=-1).reshape(-1))
    return np.concatenate(parts), npws, offsets
