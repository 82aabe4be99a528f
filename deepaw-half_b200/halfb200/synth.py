"""Seeded synthetic inputs in the reference's text formats (CHGCAR, POTCAR).

The workloads stand in for real VASP inputs (which are licensed and absent):

* ``si2``     2-atom diamond Si-like cell, a = 5.43 A, 24^3 box, 400 eV, LDA,
              Gamma, 16 bands;
* ``hfo2``    12-atom monoclinic HfO2-like cell (4 heavy s,p,d + 8 light s,p),
              48^3 box, ~3400 plane waves, PBE, Gamma, 64 bands;
* ``si64``    64-atom Si-like supercell, a = 10.86 A, 60^3 box, ~11,000 plane
              waves, PBE, Gamma-centred 4x4x4 mesh, 160 bands;
* ``si64d``   si64 with N(0, 0.05 A) displacements, Gamma + 3 k, 160 bands,
              Fermi-Dirac width 0.1 eV (force workload);
* ``si216v``  216-atom Si-like supercell with 4 seeded vacancies (212 atoms),
              a = 16.29 A, 96^3 box, ~38,000 plane waves, PBE, Gamma + 7 k,
              480 bands.

Per species: s and p channels (plus d for the heavy species) with two
projectors each, beta_l(r) = A r^l exp(-r^2/0.6^2) (1, r^2) cut at 1.9 A and
Bessel-transformed onto the 100-point reciprocal grid; DION and QPAW are
seeded random symmetric blocks per l with eigenvalues in [-5, 5] eV and
[0.05, 0.4]; the partial waves are seeded smooth radial functions whose AE-PS
difference vanishes at paw_rmax.  Density: atom-centred Gaussians
(sigma = 0.8 A) plus a uniform background, normalised to the valence count.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np
from scipy.special import spherical_jn

NPSPTS, NPSNL = 1000, 100
PSP_GMAX = 60.0        # A^-1, local-part grid extent
PSPNL_GMAX = 16.0      # A^-1, projector grid extent
RC_PROJ = 1.9          # A, projector cut radius
PAW_RMAX = 1.9
NMAX = 160             # PAW radial grid points
FELECT = 2.0 * 13.605826 * 0.529177249


@dataclass
class SpeciesSpec:
    element: str
    zval: float
    lps: list            # one entry per channel (two channels per l)
    amp: float = 2.0
    rloc: float = 1.0    # erf width of the ionic local potential
    v0: float = 20.0     # short-range repulsive Gaussian (eV)
    core: float = 0.0    # partial core charge (electrons) for the non-linear core correction; 0 = none


@dataclass
class Workload:
    name: str
    lattice: np.ndarray
    species: list        # SpeciesSpec per type
    counts: list
    positions: np.ndarray  # fractional, type-major
    grid: tuple
    encut: float
    xc: str              # "lda" | "pbe"
    nbands: int
    kpoints: np.ndarray
    kweights: np.ndarray
    sigma: float = 0.0
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def nions(self):
        return int(sum(self.counts))

    @property
    def nelect(self):
        return float(sum(s.zval * c for s, c in zip(self.species, self.counts)))


def _diamond_conventional():
    fcc = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])
    return np.concatenate([fcc, fcc + 0.25])


def _supercell(frac, n):
    out = []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                out.append((frac + np.array([i, j, k])) / n)
    return np.concatenate(out)


def _hfo2_positions():
    def orbit(x, y, z):
        return [(x, y, z), (-x, y + .5, -z + .5), (-x, -y, -z), (x, -y + .5, z + .5)]
    hf = orbit(0.2758, 0.0404, 0.2089)
    o = orbit(0.0703, 0.3317, 0.3446) + orbit(0.4423, 0.7582, 0.4789)
    return np.mod(np.array(hf + o), 1.0)


def _mesh(n):
    def wrapped(i, m):
        v = i / m
        return v - 1.0 if v > 0.5 else v
    pts = np.array([(wrapped(a, n), wrapped(b, n), wrapped(c, n))
                    for a in range(n) for b in range(n) for c in range(n)])
    return pts, np.full(len(pts), 1.0 / len(pts))


SI = SpeciesSpec("Si", 4.0, [0, 0, 1, 1])


def workload(name, seed=None):
    """Build one of the named synthetic workloads (positions, box, k set)."""
    base = {"si2": 11, "hfo2": 12, "si64": 13, "si64d": 14, "si216v": 15, "si2c": 16}
    if name not in base:
        raise KeyError(name)
    seed = 20261203 + base[name] if seed is None else seed
    rng = np.random.default_rng(seed)
    if name == "si2c":   # the Si cell with a partial core (non-linear core correction), displaced atoms
        a = 5.43
        lat = a / 2 * np.array([[0, 1, 1], [1, 0, 1], [1, 1, 0]], dtype=float)
        spec = SpeciesSpec("Si", 4.0, [0, 0, 1, 1], core=1.5)
        return Workload(name, lat, [spec], [2], np.array([[0.01, -0.02, 0.015], [.25, .26, .24]]), (24, 24, 24),
                        400.0, "pbe", 16, np.zeros((1, 3)), np.ones(1), seed=seed)
    if name == "si2":
        a = 5.43
        lat = a / 2 * np.array([[0, 1, 1], [1, 0, 1], [1, 1, 0]], dtype=float)
        return Workload(name, lat, [SI], [2], np.array([[0, 0, 0], [.25, .25, .25]]), (24, 24, 24),
                        400.0, "lda", 16, np.zeros((1, 3)), np.ones(1), seed=seed)
    if name == "hfo2":
        a, b, c, beta = 5.117, 5.175, 5.291, math.radians(99.22)
        lat = np.array([[a, 0, 0], [0, b, 0], [c * math.cos(beta), 0, c * math.sin(beta)]])
        heavy = SpeciesSpec("Hf", 5.0, [0, 0, 1, 1, 2, 2], amp=2.0, rloc=1.1, v0=25.0)
        light = SpeciesSpec("O", 3.0, [0, 0, 1, 1], amp=1.6, rloc=0.8, v0=15.0)
        return Workload(name, lat, [heavy, light], [4, 8], _hfo2_positions(), (48, 48, 48),
                        490.0, "pbe", 64, np.zeros((1, 3)), np.ones(1), seed=seed)
    if name in ("si64", "si64d"):
        a = 10.86
        lat = a * np.eye(3)
        pos = _supercell(_diamond_conventional(), 2)
        if name == "si64":
            k, w = _mesh(4)
            return Workload(name, lat, [SI], [64], pos, (60, 60, 60), 245.0, "pbe", 160, k, w, seed=seed)
        disp = rng.normal(0.0, 0.05, size=pos.shape)
        pos = np.mod(pos + disp @ np.linalg.inv(lat), 1.0)
        k = np.array([[0, 0, 0], [0.25, 0, 0], [0, 0.25, 0.25], [0.25, 0.25, 0.25]])
        return Workload(name, lat, [SI], [64], pos, (60, 60, 60), 245.0, "pbe", 160, k,
                        np.full(4, 0.25), sigma=0.1, seed=seed)
    a = 16.29
    lat = a * np.eye(3)
    pos = _supercell(_diamond_conventional(), 3)
    vac = rng.choice(len(pos), size=4, replace=False)
    pos = np.delete(pos, vac, axis=0)
    k = np.array([[0, 0, 0], [.5, 0, 0], [0, .5, 0], [0, 0, .5], [.5, .5, 0], [.5, 0, .5], [0, .5, .5],
                  [.5, .5, .5]])
    return Workload(name, lat, [SI], [212], pos, (96, 96, 96), 247.0, "pbe", 480, k, np.full(8, 1 / 8),
                    seed=seed, extra={"vacancies": sorted(int(v) for v in vac)})


# --------------------------------------------------------------------------- POTCAR

def _rand_sym(rng, n, lo, hi):
    q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    ev = rng.uniform(lo, hi, size=n)
    return (q * ev) @ q.T


def species_dataset(spec, rng):
    """Radial tables of one synthetic dataset (all in the POTCAR's units)."""
    lps = list(spec.lps)
    nch = len(lps)
    # reciprocal projectors: beta(q) = 4 pi int r^2 j_l(q r) beta(r) dr
    r = np.linspace(0.0, RC_PROJ, 2001)
    wr = np.full(len(r), r[1] - r[0]); wr[0] *= 0.5; wr[-1] *= 0.5
    qg = PSPNL_GMAX * np.arange(NPSNL) / NPSNL
    rr = np.linspace(0.0, RC_PROJ, NPSNL)
    pspnl = np.zeros((NPSNL, nch)); psprnl = np.zeros((NPSNL, nch))
    seen = {}
    for ich, l in enumerate(lps):
        which = seen.get(l, 0); seen[l] = which + 1
        br = spec.amp * r ** l * np.exp(-r * r / 0.36) * (r * r if which else 1.0)
        jl = spherical_jn(l, np.outer(qg, r))
        pspnl[:, ich] = 4 * np.pi * (jl * (r * r * br)[None, :] * wr[None, :]).sum(axis=1)
        psprnl[:, ich] = spec.amp * rr ** l * np.exp(-rr * rr / 0.36) * (rr * rr if which else 1.0)
    dion = np.zeros((nch, nch)); qpaw = np.zeros((nch, nch))
    for l in sorted(set(lps)):
        idx = [i for i, x in enumerate(lps) if x == l]
        k = len(idx)
        dion[np.ix_(idx, idx)] = _rand_sym(rng, k, -5.0, 5.0)
        qpaw[np.ix_(idx, idx)] = _rand_sym(rng, k, 0.05, 0.4)
    qloc = PSP_GMAX * np.arange(NPSPTS) / NPSPTS
    with np.errstate(divide="ignore", invalid="ignore"):
        coul = np.where(qloc > 0, 4 * np.pi * spec.zval * FELECT * (1 - np.exp(-qloc ** 2 * spec.rloc ** 2 / 4))
                        / np.where(qloc > 0, qloc ** 2, 1.0),
                        np.pi * spec.zval * FELECT * spec.rloc ** 2)
    a_sr = 0.7
    local = coul + spec.v0 * np.pi ** 1.5 * a_sr ** 3 * np.exp(-qloc ** 2 * a_sr ** 2 / 4)
    psprho = spec.zval * np.exp(-qloc ** 2 * 0.3)
    # partial core density in the POTCAR's reciprocal convention (value at q=0 = core electrons);
    # deterministic, so datasets without a core draw the same random numbers as before
    pspcor = spec.core * np.exp(-qloc ** 2 * 0.15) if spec.core > 0 else None
    rgrid = 0.002 * np.exp(np.arange(NMAX) * math.log(2.0 / 0.002) / (NMAX - 1))
    wps = np.zeros((NMAX, nch)); wae = np.zeros((NMAX, nch))
    seen = {}
    for ich, l in enumerate(lps):
        which = seen.get(l, 0); seen[l] = which + 1
        wps[:, ich] = rgrid ** (l + 1) * np.exp(-rgrid ** 2 / 0.8) * (1.0 + 0.3 * which)
        bump = np.where(rgrid < PAW_RMAX, rgrid ** (l + 1) * (1 - (rgrid / PAW_RMAX) ** 2) ** 2, 0.0)
        wae[:, ich] = wps[:, ich] + rng.uniform(-0.3, 0.3) * bump
    return dict(element=spec.element, zval=spec.zval, lps=lps, pspnl=pspnl, psprnl=psprnl, dion=dion,
                qpaw=qpaw, local=local, psprho=psprho, pspcor=pspcor, rgrid=rgrid, wps=wps, wae=wae)


def _block(values, per_line=5):
    v = np.asarray(values, dtype=float).ravel()
    lines = []
    for i in range(0, len(v), per_line):
        lines.append(" " + " ".join(f"{x:.16E}" for x in v[i:i + per_line]))
    return "\n".join(lines)


def potcar_text(ds):
    nch = len(ds["lps"])
    out = [f"  PAW_PBE {ds['element']} 03Dec2026 synthetic",
           f"  {ds['zval']:.16f}",
           " parameters from PSCTR are:",
           f"   VRHFIN ={ds['element']}: synthetic",
           "   LEXCH  = PE",
           f"   POMASS =   28.085; ZVAL   =  {ds['zval']:.6f}    mass and valenz",
           "   ENMAX  =  245.000; ENMIN  =  184.000 eV",
           " END of PSCTR-controll parameters",
           " local part",
           f"  {PSP_GMAX:.16f}",
           _block(ds["local"]),
           " gradient corrections used for XC",
           "     2"]
    if ds.get("pspcor") is not None:
        out += [" core charge-density (partial)", _block(ds["pspcor"])]
    out += [" atomic pseudo charge-density",
           _block(ds["psprho"]),
           f"  {PSPNL_GMAX:.16f}"]
    lps = ds["lps"]
    i = 0
    while i < nch:
        l = lps[i]
        j = i
        while j < nch and lps[j] == l:
            j += 1
        npro = j - i
        out.append(" Non local part")
        out.append(f"    {l}    {npro}    {RC_PROJ:.6f}")
        out.append(_block(ds["dion"][i:j, i:j]))
        for c in range(i, j):
            out.append(" Reciprocal Space Part")
            out.append(_block(ds["pspnl"][:, c]))
            out.append(" Real Space Part")
            out.append(_block(ds["psprnl"][:, c]))
        i = j
    out += [" PAW radial sets",
            f"    {NMAX}    {PAW_RMAX:.16f}",
            " (5E20.12)",
            " augmentation charges (non sperical)",
            _block(ds["qpaw"]),
            " grid",
            _block(ds["rgrid"]),
            " aepotential",
            _block(-2.0 * ds["zval"] * FELECT / (ds["rgrid"] + 0.1)),
            " core charge-density",
            _block(np.zeros(NMAX)),
            " pspotential valence only",
            _block(-ds["zval"] * FELECT / (ds["rgrid"] + 0.5))]
    for c in range(nch):
        out.append(" pseudo wavefunction")
        out.append(_block(ds["wps"][:, c]))
        out.append(" ae wavefunction")
        out.append(_block(ds["wae"][:, c]))
    out.append(" End of Dataset")
    return "\n".join(out) + "\n"


# --------------------------------------------------------------------------- CHGCAR

def density_grid(w):
    """rho * Omega on the box, returned in file order (x fastest)."""
    n1, n2, n3 = w.grid
    lat = w.lattice
    vol = abs(np.linalg.det(lat))
    f1 = np.arange(n1) / n1; f2 = np.arange(n2) / n2; f3 = np.arange(n3) / n3
    F1, F2, F3 = np.meshgrid(f1, f2, f3, indexing="ij")
    sig = 0.8
    rho = np.zeros((n1, n2, n3))
    # minimum-image Gaussians plus as many neighbouring images as a 4.5 sigma
    # reach needs along each cell height
    heights = [vol / np.linalg.norm(np.cross(lat[(i + 1) % 3], lat[(i + 2) % 3])) for i in range(3)]
    reach = [max(0, int(math.ceil(4.5 * sig / h - 0.5))) for h in heights]
    for p in w.positions:
        d1 = F1 - p[0]; d1 -= np.round(d1)
        d2 = F2 - p[1]; d2 -= np.round(d2)
        d3 = F3 - p[2]; d3 -= np.round(d3)
        for a in range(-reach[0], reach[0] + 1):
            for b in range(-reach[1], reach[1] + 1):
                for c in range(-reach[2], reach[2] + 1):
                    x = (d1 + a)[..., None] * lat[0] + (d2 + b)[..., None] * lat[1] + (d3 + c)[..., None] * lat[2]
                    rho += np.exp(-(x * x).sum(-1) / (2 * sig * sig))
    values = rho / rho.mean() * 0.75 + 0.25          # mean 1
    values *= w.nelect                               # rho*Omega averaged over the box = N_e
    return values.transpose(2, 1, 0).ravel()         # x fastest


def chgcar_text(w):
    names = " ".join(s.element for s in w.species)
    counts = " ".join(str(c) for c in w.counts)
    lines = [f"synthetic {w.name} seed {w.seed}", "   1.00000000000000"]
    for v in w.lattice:
        lines.append("  " + " ".join(f"{x:.16f}" for x in v))
    lines += ["   " + names, "   " + counts, "Direct"]
    for p in w.positions:
        lines.append("  " + " ".join(f"{x:.16f}" for x in p))
    lines.append("")
    lines.append(f"  {w.grid[0]}  {w.grid[1]}  {w.grid[2]}")
    lines.append(_block(density_grid(w)))
    return "\n".join(lines) + "\n"


def write_inputs(w, directory):
    """Write CHGCAR and POTCAR for workload w; returns their paths."""
    os.makedirs(directory, exist_ok=True)
    rng = np.random.default_rng(w.seed + 1000)
    ch = os.path.join(directory, f"CHGCAR.{w.name}")
    po = os.path.join(directory, f"POTCAR.{w.name}")
    with open(po, "w") as fh:
        for spec in w.species:
            fh.write(potcar_text(species_dataset(spec, rng)))
    with open(ch, "w") as fh:
        fh.write(chgcar_text(w))
    return ch, po
