"""MIMIC_US QDEP correction D_ij^I and its position derivative dD_ij^I/dR.

Restates src/half_uspp.F90:112-397 (CPU, with dD/dR and symmetrisation) whose
D part is the same algorithm as the GPU build_uspp_dij_cuda_species
(src/half_cuda_uspp.cuf:124-195):

1. cubic-B-spline coefficients of Veff by spectral prefiltering
   (half_uspp.F90:122-131);
2. 12 Gauss-Legendre x 24 phi directions, yweight = Y_lm w 2pi/24 (:188-200);
3. per atom, V_lm(r) = sum_dir V(R + r n) yweight, radial_v = sum rw r^2 g_l V_lm
   (:204-215); the same with the Cartesian gradient of V for dD/dR (:216-228);
4. D = DION + multipole . radial_v, symmetrised (:229-234, 235-238).
"""
from __future__ import annotations

import math

import numpy as np

from .paw import lm_list, real_ylm_x, species_tables


def radial_weights(r):
    """half_uspp.F90:292-305 (Simpson-like on a non-uniform grid)."""
    r = np.asarray(r, dtype=float)
    n = len(r)
    w = np.zeros(n)
    last = n if n % 2 == 1 else n - 1
    for i in range(0, last - 2, 2):  # Fortran i=1..last-2 step 2
        h0 = r[i + 1] - r[i]; h1 = r[i + 2] - r[i + 1]; s = (h0 + h1) / 6
        w[i] += s * (2 - h1 / h0)
        w[i + 1] += s * (h0 + h1) ** 2 / (h0 * h1)
        w[i + 2] += s * (2 - h0 / h1)
    if n % 2 == 0:
        h0 = r[n - 2] - r[n - 3]; h1 = r[n - 1] - r[n - 2]
        alpha = (2 * h1 * h1 + 3 * h0 * h1) / (6 * (h0 + h1))
        beta = (h1 * h1 + 3 * h0 * h1) / (6 * h0)
        eta = h1 ** 3 / (6 * h0 * (h0 + h1))
        w[n - 1] += alpha; w[n - 2] += beta; w[n - 3] -= eta
    return w


def sph_bessel(l, x):
    """half_uspp.F90:307-319 (series below l+2, upward recursion above)."""
    x = float(x)
    if abs(x) < l + 2:
        den = 1.0
        for i in range(1, l + 1):
            den *= 2 * i + 1
        x2 = x * x
        term = x ** l / den
        v = term
        for k in range(31):
            term = -term * x2 / (2 * (k + 1) * (2 * l + 2 * k + 3))
            v += term
            if abs(term) < 1e-16 * max(1.0, abs(v)):
                break
        return v
    jm = math.sin(x) / x
    if l == 0:
        return jm
    j = math.sin(x) / (x * x) - math.cos(x) / x
    if l == 1:
        return j
    for n in range(1, l):
        jn = (2 * n + 1) * j / x - jm
        jm, j = j, jn
    return j


def sph_bessel_deriv(l, x):
    if l == 0:
        return -sph_bessel(1, x)
    return sph_bessel(l - 1, x) - (l + 1) / x * sph_bessel(l, x)


def bessel_root(l, which):
    """half_uspp.F90:321-333: scan in steps of 0.05 from 1e-4, then bisect."""
    x0 = 1e-4; f0 = sph_bessel(l, x0); found = 0
    while found < which:
        x1 = x0 + 0.05; f1 = sph_bessel(l, x1)
        if f0 * f1 < 0:
            found += 1
            if found == which:
                break
        x0, f0 = x1, f1
    while x1 - x0 > 1e-13:
        root = 0.5 * (x0 + x1)
        if f0 * sph_bessel(l, root) <= 0:
            x1 = root
        else:
            x0 = root; f0 = sph_bessel(l, x0)
    return 0.5 * (x0 + x1)


def gauss_legendre(n):
    """half_uspp.F90:363-375 (Newton on P_n from the Tricomi start)."""
    x = np.zeros(n); w = np.zeros(n)
    m = (n + 1) // 2
    for i in range(1, m + 1):
        z = math.cos(math.pi * (i - 0.25) / (n + 0.5))
        while True:
            p1 = 1.0; p2 = 0.0
            for j in range(1, n + 1):
                p3 = p2; p2 = p1
                p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j
            pp = n * (z * p1 - p2) / (z * z - 1)
            z1 = z; z = z1 - p1 / pp
            if abs(z - z1) < 1e-15:
                break
        x[i - 1] = -z; x[n - i] = z
        w[i - 1] = 2 / ((1 - z * z) * pp * pp); w[n - i] = w[i - 1]
    return x, w


def compensation_coefficients(l, rc, z1, z2):
    """half_uspp.F90:335-342: g'(rc)=0 and int g r^(l+2) = 1."""
    a11 = z1 / rc * sph_bessel_deriv(l, z1)
    a12 = z2 / rc * sph_bessel_deriv(l, z2)
    xg, wg = gauss_legendre(32)
    rg = 0.5 * rc * (xg + 1); wg = 0.5 * rc * wg
    a21 = sum(wg[i] * sph_bessel(l, z1 * rg[i] / rc) * rg[i] ** (l + 2) for i in range(32))
    a22 = sum(wg[i] * sph_bessel(l, z2 * rg[i] / rc) * rg[i] ** (l + 2) for i in range(32))
    det = a11 * a22 - a12 * a21
    return -a12 / det, a11 / det


def gaunt_numeric(l1, m1, l2, m2, l3, m3):
    """half_uspp.F90:353-361 (12 x 24 quadrature of three real harmonics)."""
    xg, wg = gauss_legendre(12)
    g = 0.0
    for it in range(12):
        for ip in range(24):
            phi = 2 * math.pi * ip / 24
            g += (wg[it] * 2 * math.pi / 24 * real_ylm_x(l1, m1, xg[it], phi)
                  * real_ylm_x(l2, m2, xg[it], phi) * real_ylm_x(l3, m3, xg[it], phi))
    return float(g)


def spline_coefficients(veff_c, shape):
    """Cubic B-spline coefficients of Veff (half_uspp.F90:122-131)."""
    n1, n2, n3 = shape
    freq = np.fft.fftn(np.asarray(veff_c, dtype=complex).reshape(shape))
    i1 = np.arange(n1); i2 = np.arange(n2); i3 = np.arange(n3)
    b1 = (2.0 + np.cos(2.0 * np.pi * i1 / n1)) / 3.0
    b2 = (2.0 + np.cos(2.0 * np.pi * i2 / n2)) / 3.0
    b3 = (2.0 + np.cos(2.0 * np.pi * i3 / n3)) / 3.0
    freq = freq / (b1[:, None, None] * b2[None, :, None] * b3[None, None, :])
    work = np.fft.ifftn(freq) * (n1 * n2 * n3)
    return (work.real / (n1 * n2 * n3)).reshape(-1)


def _cubic_weights(t):
    return np.stack([(1 - t) ** 3 / 6, (3 * t ** 3 - 6 * t * t + 4) / 6,
                     (-3 * t ** 3 + 3 * t * t + 3 * t + 1) / 6, t ** 3 / 6], axis=-1)


def _cubic_weights_derivative(t):
    return np.stack([-0.5 * (1 - t) ** 2, 1.5 * t * t - 2.0 * t,
                     -1.5 * t * t + t + 0.5, 0.5 * t * t], axis=-1)


def cubic_sample(coeff, shape, frac, invlat=None):
    """half_uspp.F90:243-277.  Returns values (and the Cartesian gradient when
    invlat is given) at fractional points frac (..., 3)."""
    n = np.array(shape)
    coord = frac * n
    ix = np.floor(coord).astype(np.int64)
    t = coord - ix
    w = [_cubic_weights(t[..., a]) for a in range(3)]
    c = coeff.reshape(shape)
    val = np.zeros(frac.shape[:-1])
    if invlat is not None:
        dw = [_cubic_weights_derivative(t[..., a]) for a in range(3)]
        df = np.zeros(frac.shape[:-1] + (3,))
    for a in range(4):
        ia = np.mod(ix[..., 0] + a - 1, shape[0])
        for b in range(4):
            ib = np.mod(ix[..., 1] + b - 1, shape[1])
            for cc in range(4):
                ic = np.mod(ix[..., 2] + cc - 1, shape[2])
                v = c[ia, ib, ic]
                val += w[0][..., a] * w[1][..., b] * w[2][..., cc] * v
                if invlat is not None:
                    df[..., 0] += dw[0][..., a] * w[1][..., b] * w[2][..., cc] * v * shape[0]
                    df[..., 1] += w[0][..., a] * dw[1][..., b] * w[2][..., cc] * v * shape[1]
                    df[..., 2] += w[0][..., a] * w[1][..., b] * dw[2][..., cc] * v * shape[2]
    if invlat is None:
        return val
    grad = df @ invlat.T   # gradient(alpha) = sum_j df(j) invlat(alpha, j)
    return val, grad


def species_qdep_tables(pot):
    """Shape functions, multipoles and angular weights of one species."""
    lm = lm_list(pot.lps)
    nlm = len(lm)
    lmax = max(2 * l for l in pot.lps)
    naug = (lmax + 1) ** 2
    r = pot.rgrid
    rw = radial_weights(r)
    gshape = np.zeros((len(r), lmax + 1))
    for l in range(lmax + 1):
        z1 = bessel_root(l, 1); z2 = bessel_root(l, 2)
        c1, c2 = compensation_coefficients(l, pot.paw_rmax, z1, z2)
        for ir, rr in enumerate(r):
            if rr <= pot.paw_rmax:
                gshape[ir, l] = c1 * sph_bessel(l, z1 * rr / pot.paw_rmax) + c2 * sph_bessel(l, z2 * rr / pot.paw_rmax)
    laug = []; maug = []
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            laug.append(l); maug.append(m)
    multipole = np.zeros((nlm, nlm, naug))
    for b, (chb, lb, mb) in enumerate(lm):
        for a, (cha, la, ma) in enumerate(lm):
            for k in range(naug):
                l, m = laug[k], maug[k]
                if abs(la - lb) <= l <= la + lb and (la + lb + l) % 2 == 0:
                    moment = np.sum(rw * (pot.wae[:, cha] * pot.wae[:, chb]
                                          - pot.wps[:, cha] * pot.wps[:, chb]) * r ** l)
                    multipole[a, b, k] = gaunt_numeric(la, ma, lb, mb, l, m) * moment
    xg, wg = gauss_legendre(12)
    dirs = []; yw = []
    for it in range(12):
        for m in range(24):
            ph = 2 * math.pi * m / 24
            st = math.sqrt(max(0.0, 1.0 - xg[it] * xg[it]))
            dirs.append((st * math.cos(ph), st * math.sin(ph), xg[it]))
            yw.append([real_ylm_x(laug[k], maug[k], xg[it], ph) * wg[it] * 2 * math.pi / 24
                       for k in range(naug)])
    return dict(nlm=nlm, naug=naug, laug=np.array(laug), rw=rw, gshape=gshape,
                multipole=multipole, dirs=np.array(dirs), yweight=np.array(yw))


def build_qdep(veff_c, shape, potcars, crystal, with_gradient=True):
    """Per species: (dij_atom (natoms,nlm,nlm), ddij_atom (natoms,nlm,nlm,3) or None)."""
    coeff = spline_coefficients(veff_c, shape)
    invlat = np.linalg.inv(crystal.lattice)
    cart = crystal.cartesian()
    out = []
    ion0 = 0
    for it, pot in enumerate(potcars):
        tb = species_qdep_tables(pot)
        dij, _ = species_tables(pot)
        nat = crystal.counts[it]
        nlm = tb["nlm"]
        r = pot.rgrid
        weight_r = tb["rw"] * r * r                       # (nrad,)
        gk = tb["gshape"][:, tb["laug"]]                  # (nrad, naug)
        dij_atom = np.zeros((nat, nlm, nlm))
        ddij_atom = np.zeros((nat, nlm, nlm, 3)) if with_gradient else None
        for iat in range(nat):
            pts = cart[ion0 + iat][None, None, :] + r[:, None, None] * tb["dirs"][None, :, :]
            frac = np.mod(pts @ invlat, 1.0)
            if with_gradient:
                val, grad = cubic_sample(coeff, shape, frac, invlat)
            else:
                val = cubic_sample(coeff, shape, frac)
            vlm = val @ tb["yweight"]                     # (nrad, naug)
            radial_v = np.sum(weight_r[:, None] * gk * vlm, axis=0)
            d = dij + np.einsum("abk,k->ab", tb["multipole"], radial_v)
            dij_atom[iat] = 0.5 * (d + d.T)
            if with_gradient:
                for alpha in range(3):
                    vg = grad[..., alpha] @ tb["yweight"]
                    rg = np.sum(weight_r[:, None] * gk * vg, axis=0)
                    dd = np.einsum("abk,k->ab", tb["multipole"], rg)
                    ddij_atom[iat, :, :, alpha] = 0.5 * (dd + dd.T)
        out.append((dij_atom, ddij_atom))
        ion0 += nat
    return out
