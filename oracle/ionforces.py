"""Oracle (test infrastructure): the ion-position force terms that the
reference's `--forces` path adds to the non-local force
(app/half_cli.F90:947-955), restated in numpy.

* Ewald energy and its analytic force (src/half_energy.F90:122-210);
* local ionic force on a density, with the matching energy
  (src/half_local_forces.F90:11-56);
* non-linear core correction force (src/half_local_forces.F90:58-100);
* the frozen-input Harris response through the core density
  (src/half_local_forces.F90:129-161), with the radial-density force it
  contracts (:163-191);
* the smooth output density of the eigenstates (src/half_local_forces.F90:102-127);
* the MIMIC_US augmentation occupancy and density (src/half_uspp.F90:26-111).

Only tests/ may import this module.
"""
from __future__ import annotations

import math

import numpy as np

from .constants import FELECT, PI
from .io import reorder_f_to_c
from .potential import build_veff, reciprocal_grid


def spline_second(y, xmax):
    """half_local_forces.F90:213-223 (uniform grid, natural-end tridiagonal)."""
    y = np.asarray(y, dtype=float)
    n = len(y)
    h = xmax / n
    diag = np.zeros(n); rhs = np.zeros(n); upper = np.zeros(n)
    diag[1] = 1.0
    rhs[1] = ((y[2] - y[1]) / h - (y[1] - y[0]) / h) / h
    for i in range(2, n - 2):                     # 1-based 3..n-2
        diag[i] = 4 * h; upper[i] = h
        rhs[i] = 6 * ((y[i + 1] - y[i]) / h - (y[i] - y[i - 1]) / h)
    diag[n - 2] = 1.0
    rhs[n - 2] = ((y[n - 1] - y[n - 2]) / h - (y[n - 2] - y[n - 3]) / h) / h
    for i in range(2, n - 1):                     # 1-based 3..n-1
        w = (h if i <= n - 3 else 0.0) / diag[i - 1]
        diag[i] -= w * upper[i - 1]
        rhs[i] -= w * rhs[i - 1]
    m2 = np.zeros(n)
    m2[n - 2] = rhs[n - 2] / diag[n - 2]
    for i in range(n - 3, 0, -1):                 # 1-based n-2..2
        m2[i] = (rhs[i] - upper[i] * m2[i + 1]) / diag[i]
    m2[0] = 2 * m2[1] - m2[2]
    m2[n - 1] = 2 * m2[n - 2] - m2[n - 3]
    return m2


def spline_eval(y, m2, xmax, x):
    """half_local_forces.F90:224-228 (vectorised, k clamped to [1, n-1] 1-based)."""
    y = np.asarray(y); m2 = np.asarray(m2); x = np.asarray(x, dtype=float)
    n = len(y)
    h = xmax / n
    k = np.clip(np.floor(x / h).astype(np.int64) + 1, 1, n - 1)   # 1-based
    t = (x - (k - 1) * h) / h
    y0, y1, m0, m1 = y[k - 1], y[k], m2[k - 1], m2[k]
    return (1 - t) * y0 + t * y1 + h * h * (((1 - t) ** 3 - (1 - t)) * m0 + (t ** 3 - t) * m1) / 6


def _smallest_singular(matrix):
    return float(np.sqrt(max(0.0, np.linalg.eigvalsh(matrix @ matrix.T).min())))


def _ewald_setup(crystal, eta, tolerance):
    alpha = math.sqrt(PI) / crystal.volume ** (1.0 / 3.0) if eta is None else eta
    scale = math.sqrt(-math.log(tolerance))
    rcut, gcut = scale / alpha, 2 * alpha * scale
    rb = math.ceil(rcut / _smallest_singular(crystal.lattice)) + 1
    gb = math.ceil(gcut / _smallest_singular(crystal.reciprocal)) + 1
    return alpha, rcut, gcut, rb, gb


def _images(b):
    r = np.arange(-b, b + 1)
    return np.stack(np.meshgrid(r, r, r, indexing="ij"), axis=-1).reshape(-1, 3).astype(float)


def ewald_energy(crystal, charges, eta=None, tolerance=1e-11):
    """half_energy.F90:122-162: (total, real, reciprocal, self, background)."""
    charges = np.asarray(charges, dtype=float)
    alpha, rcut, gcut, rb, gb = _ewald_setup(crystal, eta, tolerance)
    pos = crystal.cartesian()
    rv = _images(rb) @ crystal.lattice
    re = 0.0
    for i in range(len(pos)):
        for j in range(len(pos)):
            d = pos[i] - pos[j] + rv
            dist = np.sqrt((d * d).sum(axis=1))
            sel = (dist > 1e-13) & (dist <= rcut)
            re += charges[i] * charges[j] * float(np.sum(np.array([math.erfc(alpha * x) for x in dist[sel]]) / dist[sel]))
    re *= 0.5 * FELECT
    gv = _images(gb) @ crystal.reciprocal
    gn = np.sqrt((gv * gv).sum(axis=1))
    sel = (gn > 1e-13) & (gn <= gcut)
    gv, gn = gv[sel], gn[sel]
    phase = gv @ pos.T
    sr = (charges[None, :] * np.cos(phase)).sum(axis=1)
    si = -(charges[None, :] * np.sin(phase)).sum(axis=1)
    ge = 2 * PI * FELECT / crystal.volume * float(np.sum(np.exp(-gn * gn / (4 * alpha * alpha)) * (sr * sr + si * si) / (gn * gn)))
    se = -FELECT * alpha / math.sqrt(PI) * float(np.sum(charges * charges))
    be = -FELECT * PI * float(charges.sum()) ** 2 / (2 * alpha * alpha * crystal.volume)
    return re + ge + se + be, re, ge, se, be


def ewald_forces(crystal, charges, eta=None, tolerance=1e-11):
    """half_energy.F90:164-210."""
    charges = np.asarray(charges, dtype=float)
    alpha, rcut, gcut, rb, gb = _ewald_setup(crystal, eta, tolerance)
    pos = crystal.cartesian()
    n = len(pos)
    forces = np.zeros((n, 3))
    rv = _images(rb) @ crystal.lattice
    for i in range(n):
        for j in range(n):
            d = pos[i] - pos[j] + rv
            dist = np.sqrt((d * d).sum(axis=1))
            sel = (dist > 1e-13) & (dist <= rcut)
            ds, dd = dist[sel], d[sel]
            screen = np.array([math.erfc(alpha * x) for x in ds]) / ds ** 3 + \
                2 * alpha * np.exp(-(alpha * ds) ** 2) / (math.sqrt(PI) * ds ** 2)
            forces[i] += FELECT * charges[i] * charges[j] * (screen[:, None] * dd).sum(axis=0)
    gv = _images(gb) @ crystal.reciprocal
    gn = np.sqrt((gv * gv).sum(axis=1))
    sel = (gn > 1e-13) & (gn <= gcut)
    gv, gn = gv[sel], gn[sel]
    phase = gv @ pos.T                                        # (G, ions)
    sr = (charges[None, :] * np.cos(phase)).sum(axis=1)
    si = -(charges[None, :] * np.sin(phase)).sum(axis=1)
    pref = 4 * PI * FELECT / crystal.volume * np.exp(-gn * gn / (4 * alpha * alpha)) / (gn * gn)
    for i in range(n):
        w = pref * charges[i] * (sr * np.sin(phase[:, i]) + si * np.cos(phase[:, i]))
        forces[i] += (w[:, None] * gv).sum(axis=0)
    return forces


def _grid(crystal, shape):
    q = reciprocal_grid(shape, crystal.reciprocal)
    g2 = (q * q).sum(axis=1)
    return q, g2, np.sqrt(g2)


def _radial_forces(field_g, table, gmax, cut_points, crystal, counts_slice, shape, q, g2, gn, scale, coulomb_z=None):
    """sum over the box of -q * radial * Im(conj(f(G)) e^{-i G.R_I}) * scale, per atom;
    radial = spline(table) (minus the Coulomb tail when coulomb_z is given)."""
    m2 = spline_second(table, gmax)
    n = len(table)
    sel = (g2 > 1e-12) & (gn <= gmax - cut_points * gmax / n)
    radial = spline_eval(table, m2, gmax, gn[sel])
    if coulomb_z is not None:
        radial = radial - 4 * PI * coulomb_z * FELECT / g2[sel]
    qs, fs = q[sel], field_g[sel]
    pos = crystal.cartesian()
    out, energy = [], 0.0
    for iat in counts_slice:
        phase = qs @ pos[iat]
        e = np.cos(phase) - 1j * np.sin(phase)
        prod = np.conj(fs) * e
        term = radial * scale * prod.imag
        out.append(-(term[:, None] * qs).sum(axis=0))
        energy += float(np.sum(radial * scale * prod.real))
    return out, energy


def local_ionic_forces(values_f, potcars, crystal, shape):
    """half_local_forces.F90:11-56: (forces, energy) on the density values_f
    (CHGCAR convention, x fastest)."""
    n = int(np.prod(shape))
    rho = reorder_f_to_c(values_f, shape)
    rho_g = np.fft.fftn(rho.reshape(shape).astype(complex)).reshape(-1) / n
    q, g2, gn = _grid(crystal, shape)
    forces = np.zeros((crystal.nions, 3))
    energy = 0.0
    ion0 = 0
    for it, pot in enumerate(potcars):
        idx = range(ion0, ion0 + crystal.counts[it])
        f, e = _radial_forces(rho_g, pot.psp_local, pot.psp_gmax, 1, crystal, idx, shape, q, g2, gn,
                              1.0 / crystal.volume, coulomb_z=pot.zval)
        forces[ion0:ion0 + crystal.counts[it]] = f
        energy += e
        ion0 += crystal.counts[it]
    return forces, energy


def radial_density_forces(potential_c, potcars, crystal, shape, use_core=True):
    """half_local_forces.F90:163-191 with the potential in C order (the
    reference's nlcc_forces :58-100 is the same sum with the XC potential)."""
    n = int(np.prod(shape))
    pot_g = np.fft.fftn(np.asarray(potential_c).reshape(shape).astype(complex)).reshape(-1) / n
    q, g2, gn = _grid(crystal, shape)
    forces = np.zeros((crystal.nions, 3))
    ion0 = 0
    for it, pot in enumerate(potcars):
        table = pot.pspcor if use_core else pot.psprho
        if table is not None:
            idx = range(ion0, ion0 + crystal.counts[it])
            f, _ = _radial_forces(pot_g, table, pot.psp_gmax, 3, crystal, idx, shape, q, g2, gn, 1.0)
            forces[ion0:ion0 + crystal.counts[it]] = f
        ion0 += crystal.counts[it]
    return forces


def core_energy(potential_c, potcars, crystal, shape):
    """sum_I sum_G radial_core(G) Re(conj(v(G)) e^{-i G.R_I}): the functional whose
    position derivative is minus radial_density_forces (finite-difference pin)."""
    n = int(np.prod(shape))
    pot_g = np.fft.fftn(np.asarray(potential_c).reshape(shape).astype(complex)).reshape(-1) / n
    q, g2, gn = _grid(crystal, shape)
    total, ion0 = 0.0, 0
    for it, pot in enumerate(potcars):
        if pot.pspcor is not None:
            _, e = _radial_forces(pot_g, pot.pspcor, pot.psp_gmax, 3, crystal,
                                  range(ion0, ion0 + crystal.counts[it]), shape, q, g2, gn, 1.0)
            total += e
        ion0 += crystal.counts[it]
    return total


def xc_potential(values_f, potcars, crystal, shape, use_pbe):
    """V_xc of a density in C order: Veff minus its Hartree and local parts."""
    veff, local_r, _ = build_veff(crystal, shape, values_f, potcars, use_pbe)
    return veff - local_r


def harris_correction_forces(input_f, output_f, potcars, crystal, shape, use_pbe, t=1.0e-4):
    """half_local_forces.F90:129-161: the core-density force of the XC response
    (V_xc(n_in + t dn) - V_xc(n_in - t dn)) / (2 t), dn = n_out - n_in.  The
    reference takes the vxc_out argument of build_veff_* (:151-157), so the
    Hartree potential, linear in the density, does not enter."""
    delta = np.asarray(output_f) - np.asarray(input_f)
    vplus = xc_potential(np.asarray(input_f) + t * delta, potcars, crystal, shape, use_pbe)
    vminus = xc_potential(np.asarray(input_f) - t * delta, potcars, crystal, shape, use_pbe)
    return radial_density_forces((vplus - vminus) / (2 * t), potcars, crystal, shape, use_core=True)


def smooth_density(basis, vectors, occupations, kweight, shape):
    """half_local_forces.F90:102-127: sum w f |psi(r)|^2 in file order (x fastest);
    psi(r) by the unnormalised inverse transform of the plane-wave coefficients."""
    n = int(np.prod(shape))
    acc = np.zeros(n)
    for b, f in enumerate(occupations):
        if f == 0.0:
            continue
        grid = np.zeros(n, dtype=complex)
        grid[basis.fft_index] = vectors[:, b]
        psi = np.fft.ifftn(grid.reshape(shape)).reshape(-1) * n
        acc += kweight * f * np.abs(psi) ** 2
    return acc.reshape(shape).transpose(2, 1, 0).reshape(-1)   # C order -> x fastest


def augmentation_occupancy(projectors, vectors, occupations, kweight, occupancy=None):
    """half_uspp.F90:26-47: occupancy[it][iat, a, b] += w f Re(conj(c_a) c_b), c = B_I^H psi;
    projectors from oracle.paw.build_projectors (column iat*nlm + ilm)."""
    if occupancy is None:
        occupancy = [np.zeros((sp.natoms, sp.nlm, sp.nlm)) for sp in projectors]
    for it, sp in enumerate(projectors):
        for iat in range(sp.natoms):
            bi = sp.B[:, iat * sp.nlm:(iat + 1) * sp.nlm]
            for ib, f in enumerate(occupations):
                if f == 0.0:
                    continue
                c = bi.conj().T @ vectors[:, ib]
                occupancy[it][iat] += kweight * f * np.real(np.conj(c)[:, None] * c[None, :])
    return occupancy


def _anint(x):
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def add_augmentation_density(potcars, crystal, shape, occupancy, density_f):
    """half_uspp.F90:49-111: (density_f + augmentation, integrated charge); every box
    point within paw_rmax of an atom (minimum image) gets
    Omega sum_lm [sum_ab occ_ab M_ab,lm] g_l(r) Y_lm."""
    from .paw import real_ylm_x
    from .uspp import bessel_root, compensation_coefficients, species_qdep_tables, sph_bessel
    out = np.array(density_f, dtype=float, copy=True)
    n1, n2, n3 = shape
    n = n1 * n2 * n3
    before = out.sum() / n
    idx = np.arange(n)
    frac = np.stack([(idx % n1) / n1, ((idx // n1) % n2) / n2, (idx // (n1 * n2)) / n3], axis=1)
    ion0 = 0
    for it, pot in enumerate(potcars):
        t = species_qdep_tables(pot)
        naug = t["naug"]
        lmax = int(round(math.sqrt(naug))) - 1
        rc = pot.paw_rmax
        shapes = []
        for l in range(lmax + 1):
            z1, z2 = bessel_root(l, 1), bessel_root(l, 2)
            c1, c2 = compensation_coefficients(l, rc, z1, z2)
            shapes.append((z1, z2, c1, c2))
        for iat in range(crystal.counts[it]):
            coeff = np.einsum("ab,abk->k", occupancy[it][iat], t["multipole"])
            df = frac - crystal.positions[ion0 + iat]
            df = df - _anint(df)
            cart = df @ crystal.lattice
            r = np.sqrt((cart * cart).sum(axis=1))
            sel = np.nonzero(r <= rc)[0]
            rs, cs = r[sel], cart[sel]
            safe = rs > 1e-14
            theta = np.where(safe, np.arccos(np.clip(cs[:, 2] / np.where(safe, rs, 1.0), -1.0, 1.0)), 0.0)
            phi = np.where(safe, np.arctan2(cs[:, 1], cs[:, 0]), 0.0)
            x = np.cos(theta)
            value = np.zeros(len(sel))
            k = 0
            for l in range(lmax + 1):
                z1, z2, c1, c2 = shapes[l]
                g = np.array([c1 * sph_bessel(l, z1 * rr / rc) + c2 * sph_bessel(l, z2 * rr / rc) for rr in rs])
                for m in range(-l, l + 1):
                    value += coeff[k] * g * real_ylm_x(l, m, x, phi)
                    k += 1
            out[sel] += crystal.volume * value
        ion0 += crystal.counts[it]
    return out, out.sum() / n - before
