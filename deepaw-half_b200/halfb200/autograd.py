"""torch.autograd binding of the band free energy and its Hellmann-Feynman
gradient.

    E(R) = sum_k w_k sum_n f_nk eps_nk(R) + entropy term     (fixed Veff)

is the Mermin band free energy of src/half_energy.F90:41-120 with the
eigenvalues of the MIMIC_US operator at atom positions R (Cartesian, A).  Its
gradient is minus the non-local PAW force of src/half_forces.F90:9-73
(projector phases + dD_ij/dR); the basis does not move with R, so there is no
Pulay term.  forward() runs the library's half_band_forces: each k point is
solved and its adjoint evaluated on the device while its eigenvectors are
resident, so no eigenvector block ever crosses to the host; backward() only
scales the saved force.
"""
from __future__ import annotations

import numpy as np

try:
    import torch
except ImportError:  # the binding works without torch; only this module needs it
    torch = None


def _require_torch():
    if torch is None:
        raise ImportError("torch is required for halfb200.autograd")


class BandFreeEnergy(torch.autograd.Function if torch is not None else object):
    @staticmethod
    def forward(ctx, positions, context, kpoints, weights, nbands, nelect, sigma, ismear):
        pos = positions.detach().cpu().double().numpy()
        frac = pos @ np.linalg.inv(context.lattice)
        context.set_positions(frac)
        r = context.band_forces(kpoints, weights, nbands, nelect, sigma, ismear)
        ctx.save_for_backward(torch.as_tensor(-r["forces"], dtype=positions.dtype, device=positions.device))
        return torch.as_tensor(r["band_energy"] + r["entropy"], dtype=positions.dtype, device=positions.device)

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return grad_out * grad, None, None, None, None, None, None, None


def band_free_energy(positions, context, kpoints, weights, nbands, nelect, sigma=0.1, ismear=-1):
    """Differentiable band free energy (eV) of Cartesian positions (nions, 3) in A."""
    _require_torch()
    return BandFreeEnergy.apply(positions, context, np.asarray(kpoints, float), np.asarray(weights, float), int(nbands),
                                float(nelect), float(sigma), int(ismear))
