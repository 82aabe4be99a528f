"""Fixed-density effective potential Veff(r) = V_local + V_xc.

Restates the ACC path's GPU builder src/half_cuda_potential.cuf:270-350
(identical in algorithm to the CPU src/half_potential.F90:265-328):
Hartree + ionic local part in reciprocal space, real-space PZ81 LDA or PBE
with spectral gradients and finite-difference functional derivatives
(src/half_xc.F90:10-116).  Output is in C order (i3 fastest), eV.
"""
from __future__ import annotations

import math

import numpy as np

from .constants import AUTOA, EDEPS, FELECT, HATOEV, PI
from .io import reorder_f_to_c
from .paw import spline_eval, spline_second


def reciprocal_grid(shape, rec):
    """G vectors of every box point with the FFT wrap of half_cuda_potential.cuf:34-47."""
    n1, n2, n3 = shape

    def wrap(n):
        i = np.arange(n)
        return np.where(i <= (n - 1) // 2, i, i - n)

    k1, k2, k3 = np.meshgrid(wrap(n1), wrap(n2), wrap(n3), indexing="ij")
    k1 = k1.ravel(); k2 = k2.ravel(); k3 = k3.ravel()
    q = k1[:, None] * rec[0] + k2[:, None] * rec[1] + k3[:, None] * rec[2]
    return q


def _fft(a, shape):
    return np.fft.fftn(a.reshape(shape)).reshape(-1)


def _ifft_unnorm(a, shape):
    return (np.fft.ifftn(a.reshape(shape)) * a.size).reshape(-1)


def lda_pz81(total, volume):
    """half_cuda_potential.cuf:236-259: returns (vxc eV, energy density in Ha/bohr^3 units)."""
    density = total / volume
    rhoau = density * AUTOA ** 3
    vxc = np.zeros_like(total); ed = np.zeros_like(total)
    ok = rhoau > 1.0e-30
    rs = (3.0 / (4 * PI * rhoau[ok])) ** (1.0 / 3.0)
    ex = -0.4582 / rs
    vx = -(4.0 / 3.0) * 0.4582 / rs
    ec = np.empty_like(rs); vc = np.empty_like(rs)
    hi = rs >= 1
    sr = np.sqrt(rs[hi]); denom = 1 + 1.0529 * sr + 0.3334 * rs[hi]
    ec[hi] = -0.1423 / denom
    vc[hi] = ec[hi] * (1 + (7.0 / 6.0) * 1.0529 * sr + (4.0 / 3.0) * 0.3334 * rs[hi]) / denom
    lo = ~hi
    lnrs = np.log(rs[lo])
    ec[lo] = 0.0311 * lnrs - 0.048 + 0.002 * rs[lo] * lnrs - 0.0116 * rs[lo]
    vc[lo] = (0.0311 * lnrs + (-0.048 - 0.0311 / 3) + (2.0 / 3.0) * 0.002 * rs[lo] * lnrs
              + (-0.0232 - 0.002) * rs[lo] / 3)
    vxc[ok] = (vx + vc) * HATOEV
    ed[ok] = (ex + ec) * rhoau[ok]
    return vxc, ed


def _pw92(rs):
    a, a1, b1, b2, b3, b4 = 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294
    sr = np.sqrt(rs)
    q = 2 * a * (b1 * sr + b2 * rs + b3 * rs * sr + b4 * rs * rs)
    la = np.log(1 + 1 / q)
    return -2 * a * (1 + a1 * rs) * la


def pbe_energy_density(density, sigma):
    """half_xc.F90:94-107 (vectorised)."""
    mu, kappa, beta = 0.2195149727645171, 0.804, 0.06672455060314922
    gamma = (1.0 - math.log(2.0)) / (PI * PI)
    n = np.maximum(density, 1.0e-30)
    s = np.maximum(sigma, 0.0)
    rs = (3 / (4 * PI * n)) ** (1.0 / 3.0)
    kf = (3 * PI * PI * n) ** (1.0 / 3.0)
    exlda = -3 * kf / (4 * PI)
    s2 = s / (4 * kf * kf * n * n)
    fx = 1 + kappa - kappa / (1 + mu * s2 / kappa)
    ec = _pw92(rs)
    ks2 = 4 * kf / PI
    t2 = s / (4 * ks2 * n * n)
    aa = beta / gamma / (np.exp(-ec / gamma) - 1)
    at2 = aa * t2
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        r1 = t2 * (1 + at2) / (1 + at2 + at2 * at2)
        inv = 1 / at2
        r2 = (1 / aa) * (1 + inv) / (1 + inv + inv * inv)
    ratio = np.where(t2 == 0, 0.0, np.where(at2 < 1.0e100, r1, r2))
    hh = gamma * np.log(1 + beta / gamma * ratio)
    return n * (exlda * fx + ec + hh)


def build_veff(crystal, shape, values_f, potcars, use_pbe):
    """Return (veff_c, local_r, e_hartree).  values_f is the CHGCAR grid (x fastest)."""
    n = int(np.prod(shape))
    vol = crystal.volume
    rec = crystal.reciprocal
    charge = reorder_f_to_c(values_f, shape)
    rho_g = _fft(charge.astype(complex) / n, shape)
    q = reciprocal_grid(shape, rec)
    g2 = q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2]
    gn = np.sqrt(g2)
    big = g2 > 1.0e-12
    local_g = np.zeros(n, dtype=complex)
    local_g[big] = EDEPS * rho_g[big] / (g2[big] * vol)
    e_h = float(np.sum(0.5 * (np.conj(rho_g[big]) * local_g[big]).real))
    core_g = np.zeros(n, dtype=complex)
    cart = crystal.cartesian()
    ion0 = 0
    for it, pot in enumerate(potcars):
        nrad = len(pot.psp_local)
        m2 = spline_second(pot.psp_local, pot.psp_gmax)
        radial = spline_eval(pot.psp_local, m2, pot.psp_gmax, gn)
        with np.errstate(divide="ignore"):
            radial = np.where(big, radial - 4 * PI * pot.zval * FELECT / np.where(big, g2, 1.0), radial)
        radial = np.where((~big) | (gn > pot.psp_gmax - pot.psp_gmax / nrad), 0.0, radial)
        if pot.has_core:
            m2c = spline_second(pot.pspcor, pot.psp_gmax)
            core = np.where(gn <= pot.psp_gmax - 3 * pot.psp_gmax / nrad,
                            spline_eval(pot.pspcor, m2c, pot.psp_gmax, gn), 0.0)
        else:
            core = np.zeros(n)
        structure = np.zeros(n, dtype=complex)
        for iat in range(crystal.counts[it]):
            r = cart[ion0 + iat]
            phase = q[:, 0] * r[0] + q[:, 1] * r[1] + q[:, 2] * r[2]
            structure += np.cos(phase) - 1j * np.sin(phase)
        local_g += radial * structure / vol
        core_g += core * structure
        ion0 += crystal.counts[it]
    local_r = _ifft_unnorm(local_g, shape).real
    core_r = _ifft_unnorm(core_g, shape).real
    if not use_pbe:
        vxc, _ = lda_pz81(charge + core_r, vol)
        return local_r + vxc, local_r, e_h
    total = charge + core_r
    density = np.maximum(total / vol * AUTOA ** 3, 1.0e-20)   # half_cuda_potential.cuf:116-129
    freq = _fft((total / vol).astype(complex), shape)
    grad = np.zeros((3, n)); sigma = np.zeros(n)
    for a in range(3):
        w = _ifft_unnorm(1j * q[:, a] * freq, shape)
        grad[a] = w.real / n * AUTOA ** 4
        sigma += grad[a] ** 2
    dn = np.maximum(np.abs(density) * 2.0e-5, 1.0e-12)
    nm = np.maximum(density - dn, 1.0e-30); npl = density + dn
    fn = (pbe_energy_density(npl, sigma) - pbe_energy_density(nm, sigma)) / (npl - nm)
    ds = np.maximum(np.abs(sigma) * 2.0e-5, 1.0e-14)
    sm = np.maximum(sigma - ds, 0.0); sp = sigma + ds
    fs = (pbe_energy_density(density, sp) - pbe_energy_density(density, sm)) / (sp - sm)
    fs = np.where(density <= 1.0e-20, 0.0, fs)
    for a in range(3):
        flux = 2 * fs * grad[a]
        fq = _fft(flux.astype(complex), shape)
        w = _ifft_unnorm(1j * q[:, a] * fq, shape)
        fn = fn - AUTOA * w.real / n
    fn = np.where(density <= 1.0e-20, 0.0, fn)
    return local_r + fn * HATOEV, local_r, e_h
