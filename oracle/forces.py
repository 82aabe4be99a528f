"""Hellmann-Feynman band-energy (non-local PAW) force and occupations.

* ``nonlocal_forces`` restates add_nonlocal_paw_forces (src/half_forces.F90:9-73):
  c = B_I^H psi_n, dc_alpha = B_I^H (i q_alpha psi_n),
  F -= 2 w f Re[((D_I - eps Q) c)^H dc_alpha] + w f Re[c^H dD_I/dR_alpha c].
* ``compute_occupations`` restates src/half_energy.F90:41-120 (zero width,
  Gaussian ISMEAR=0 with erfc, Fermi-Dirac ISMEAR=-1; bisection on mu).
* ``gamma_centered_mesh`` restates src/half_kpoints.F90:52-68, 171-174.
"""
from __future__ import annotations

import math

import numpy as np


def nonlocal_forces(basis, species, dij_atoms, ddij_atoms, eigenvalues, occupations, kweight, vectors,
                    forces=None, split=False):
    nions = sum(s.natoms for s in species)
    if forces is None:
        forces = np.zeros((nions, 3))
    proj = np.zeros_like(forces); aug = np.zeros_like(forces)
    q = basis.qvectors
    occ = np.asarray(occupations)
    eps = np.asarray(eigenvalues)
    ion0 = 0
    for s, dat, ddat in zip(species, dij_atoms, ddij_atoms):
        for iat in range(s.natoms):
            Bi = s.B[:, iat * s.nlm:(iat + 1) * s.nlm]
            for ib in range(len(eps)):
                if occ[ib] == 0.0:
                    continue
                psi = vectors[:, ib]
                c = Bi.conj().T @ psi
                dc = np.stack([Bi.conj().T @ (1j * q[:, a] * psi) for a in range(3)], axis=1)
                metric = dat[iat] - eps[ib] * s.qij
                mc = metric @ c
                for a in range(3):
                    term = -2.0 * kweight * occ[ib] * float(np.real(np.vdot(mc, dc[:, a])))
                    forces[ion0 + iat, a] += term
                    proj[ion0 + iat, a] += term
                    if ddat is not None:
                        term = -kweight * occ[ib] * float(np.real(np.vdot(c, ddat[iat, :, :, a] @ c)))
                        forces[ion0 + iat, a] += term
                        aug[ion0 + iat, a] += term
        ion0 += s.natoms
    if split:
        return forces, proj, aug
    return forces


def compute_occupations(eigenvalues, weights, nelect, sigma, ismear=0):
    """Returns (occupation (nk,nb), mu, band_energy, entropy_term)."""
    eig = np.asarray(eigenvalues, dtype=float)
    w = np.asarray(weights, dtype=float)
    nk, nb = eig.shape
    if abs(w.sum() - 1.0) > 1e-10:
        raise ValueError("k-point weights must sum to one")
    if nelect < -1e-12 or nelect > 2.0 * nb + 1e-12:
        raise ValueError("electrons do not fit in requested bands")
    if ismear not in (-1, 0):
        raise ValueError("supported ISMEAR values are -1 and 0")
    occ = np.zeros((nk, nb))
    if sigma == 0.0:
        states = [(ik, ib) for ik in range(nk) for ib in range(nb)]
        energy = [eig[ik, ib] for ik, ib in states]
        order = sorted(range(len(states)), key=lambda s: energy[s])  # stable like insertion sort
        remaining = nelect; mu = float(eig.min()); pos = 0
        while pos < len(order) and remaining > 1e-13:
            level = energy[order[pos]]
            stop = pos + 1
            tolerance = 1e-10 * max(1.0, abs(level))
            while stop < len(order) and abs(energy[order[stop]] - level) <= tolerance:
                stop += 1
            capacity = sum(2.0 * w[states[order[i]][0]] for i in range(pos, stop))
            frac = min(1.0, max(0.0, remaining / capacity))
            for i in range(pos, stop):
                ik, ib = states[order[i]]
                occ[ik, ib] = 2.0 * frac
            filled = frac * capacity
            if filled > 0:
                mu = level
            remaining -= filled
            pos = stop
        if remaining > 1e-9:
            raise ValueError("not enough bands for electron count")
        return occ, mu, float(np.sum(w[:, None] * occ * eig)), 0.0

    def count(mu):
        x = (eig - mu) / sigma
        if ismear == 0:
            return float(np.sum(w[:, None] * np.vectorize(math.erfc)(x)))
        x = np.clip(x, -700.0, 700.0)
        return float(np.sum(w[:, None] * 2.0 / (1.0 + np.exp(x))))

    lo = eig.min() - max(10.0, 100.0 * sigma)
    hi = eig.max() + max(10.0, 100.0 * sigma)
    for _ in range(256):
        mid = 0.5 * (lo + hi)
        if count(mid) < nelect:
            lo = mid
        else:
            hi = mid
        if hi - lo < 1e-13 * max(1.0, abs(mid)):
            break
    mu = 0.5 * (lo + hi)
    entropy = 0.0
    for ik in range(nk):
        for ib in range(nb):
            x = (eig[ik, ib] - mu) / sigma
            if ismear == 0:
                occ[ik, ib] = math.erfc(x)
                if abs(x) < 20.0:
                    entropy -= sigma * w[ik] * math.exp(-x * x) / math.sqrt(math.pi)
            else:
                x = max(-700.0, min(700.0, x))
                p = 1.0 / (1.0 + math.exp(x))
                occ[ik, ib] = 2.0 * p
                p = max(1e-300, min(1.0 - 1e-16, p))
                entropy += 2.0 * sigma * w[ik] * (p * math.log(p) + (1 - p) * math.log(1 - p))
    return occ, mu, float(np.sum(w[:, None] * occ * eig)), entropy


def gamma_centered_mesh(n1, n2, n3):
    def wrapped(i, n):
        v = i / n
        return v - 1.0 if v > 0.5 else v
    pts = [(wrapped(i1, n1), wrapped(i2, n2), wrapped(i3, n3))
           for i1 in range(n1) for i2 in range(n2) for i3 in range(n3)]
    nk = len(pts)
    return np.array(pts), np.full(nk, 1.0 / nk)
