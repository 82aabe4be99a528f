"""Matrix-free and dense H/S operators and the dense generalized solve.

* ``apply_hs`` restates apply_hs_operator_cuda (src/half_cuda_assembly.cuf:468-519):
  scatter -> unnormalised inverse FFT -> * Veff/N_r -> forward FFT -> gather +
  T psi; S psi = psi; then per species coeff = B^H psi, DY = D_atom coeff,
  QY = Q coeff, H psi += B DY, S psi += B QY.
* ``assemble_dense`` restates assemble_dense_gamma (src/half_dense_solver.F90:53-94):
  circular V(G_i - G_j), kinetic diagonal, B D B^H and I + B Q B^H, hermitised.
* ``solve_dense`` restates solve_dense_gamma (:29-51): overlap extremes from
  zheev(S), then zhegv(H, S) (upper triangles).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.linalg as sla

from .basis import build_basis
from .io import read_chgcar, read_potcar
from .paw import build_projectors
from .potential import build_veff
from .uspp import build_qdep


@dataclass
class System:
    crystal: object
    shape: tuple
    values: np.ndarray
    potcars: list
    encut: float
    use_pbe: bool
    use_uspp: bool
    veff: np.ndarray            # C order, eV
    dij_atoms: list             # per species (natoms, nlm, nlm)
    ddij_atoms: list            # per species (natoms, nlm, nlm, 3) or None


def load_system(chgcar, potcar, encut, use_pbe, use_uspp=True, with_gradient=False):
    """The context the reference builds from files (half_library.F90:51-110 plus
    the ACC path's potential and QDEP set-up, half_cuda_assembly.cuf:402-466)."""
    crystal, shape, values = read_chgcar(chgcar)
    pots = read_potcar(potcar)
    if len(pots) != crystal.ntypes:
        raise ValueError("POTCAR dataset count does not match structure species count")
    veff, _, _ = build_veff(crystal, shape, values, pots, use_pbe)
    return make_system(crystal, shape, values, pots, encut, use_pbe, use_uspp, veff, with_gradient)


def make_system(crystal, shape, values, pots, encut, use_pbe, use_uspp, veff, with_gradient=False):
    from .paw import species_tables
    if use_uspp:
        q = build_qdep(veff, shape, pots, crystal, with_gradient=with_gradient)
        dij = [d for d, _ in q]
        ddij = [dd for _, dd in q]
    else:
        dij = []
        for it, pot in enumerate(pots):
            d, _ = species_tables(pot)
            dij.append(np.repeat(d[None], crystal.counts[it], axis=0))
        ddij = [None] * len(pots)
    return System(crystal, tuple(shape), values, pots, float(encut), use_pbe, use_uspp, veff, dij, ddij)


@dataclass
class KOperator:
    basis: object
    species: list       # SpeciesProjectors
    dij_atoms: list
    veff: np.ndarray
    shape: tuple


def prepare(system, kpoint=(0.0, 0.0, 0.0)):
    basis = build_basis(system.crystal, system.shape, system.encut, kpoint)
    sp = build_projectors(system.potcars, system.crystal, basis)
    return KOperator(basis, sp, system.dij_atoms, system.veff, system.shape)


def apply_hs(op, psi):
    """H psi and S psi for a column block psi (npw, nb)."""
    psi = np.asarray(psi, dtype=np.complex128)
    if psi.ndim == 1:
        psi = psi[:, None]
    b = op.basis
    nr = int(np.prod(op.shape))
    nb = psi.shape[1]
    grid = np.zeros((nb, nr), dtype=complex)
    grid[:, b.fft_index] = psi.T
    g = grid.reshape((nb,) + op.shape)
    g = np.fft.ifftn(g, axes=(1, 2, 3)) * nr                      # CUFFT_INVERSE, unnormalised
    g = g * (op.veff.reshape(op.shape) / nr)[None]
    g = np.fft.fftn(g, axes=(1, 2, 3)).reshape(nb, nr)
    hpsi = g[:, b.fft_index].T + b.kinetic[:, None] * psi
    spsi = psi.copy()
    for s, dat in zip(op.species, op.dij_atoms):
        coeff = s.B.conj().T @ psi                                   # (nat*nlm, nb)
        c = coeff.reshape(s.natoms, s.nlm, nb)
        dy = np.einsum("iab,ibn->ian", dat, c).reshape(-1, nb)
        qy = np.einsum("ab,ibn->ian", s.qij, c).reshape(-1, nb)
        hpsi += s.B @ dy
        spsi += s.B @ qy
    return hpsi, spsi


def assemble_dense(op):
    b = op.basis
    n1, n2, n3 = op.shape
    nr = n1 * n2 * n3
    vg = np.fft.fftn(op.veff.reshape(op.shape).astype(complex)).reshape(-1) / nr
    g = b.gvectors.astype(np.int64)
    d0 = np.mod(g[:, 0][:, None] - g[:, 0][None, :], n1)
    d1 = np.mod(g[:, 1][:, None] - g[:, 1][None, :], n2)
    d2 = np.mod(g[:, 2][:, None] - g[:, 2][None, :], n3)
    h = vg[d0 * n2 * n3 + d1 * n3 + d2]
    h[np.diag_indices(b.npw)] += b.kinetic
    s = np.eye(b.npw, dtype=complex)
    for sp, dat in zip(op.species, op.dij_atoms):
        for iat in range(sp.natoms):
            Bi = sp.B[:, iat * sp.nlm:(iat + 1) * sp.nlm]
            h += Bi @ dat[iat] @ Bi.conj().T
            s += Bi @ sp.qij @ Bi.conj().T
    h = 0.5 * (h + h.conj().T)
    s = 0.5 * (s + s.conj().T)
    return h, s


def solve_dense(op, nbands=None, vectors=False):
    h, s = assemble_dense(op)
    ov = sla.eigh(s, eigvals_only=True, lower=False)
    if vectors:
        w, v = sla.eigh(h, s, lower=False, type=1)
    else:
        w = sla.eigh(h, s, lower=False, type=1, eigvals_only=True)
        v = None
    if nbands is not None:
        w = w[:nbands]
        if v is not None:
            v = v[:, :nbands]
    return w, v, float(ov[0]), float(ov[-1])
