"""Text CHGCAR / POTCAR readers restated from the reference.

* ``read_chgcar`` follows src/half_chgcar.F90:133-219 (POSCAR header, optional
  element line, Direct/Cartesian, grid line, x-fastest values).
* ``read_potcar`` follows src/half_potcar.F90:24-205 (PSCTR tags, local part,
  optional local sections, non-local projector blocks, PAW radial sets).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

NPSPTS = 1000  # half_potcar.F90:10
NPSNL = 100
NPSRNL = 100


@dataclass
class Crystal:
    """crystal_t (half_types.F90:9-21); lattice rows are lattice vectors."""
    name: str
    lattice: np.ndarray          # (3,3), row i = vector i, Angstrom
    species: list                # element names per type
    counts: list                 # atoms per type
    positions: np.ndarray        # (nions,3) fractional, type-major order

    @property
    def nions(self):
        return int(sum(self.counts))

    @property
    def ntypes(self):
        return len(self.counts)

    @property
    def volume(self):
        # half_types.F90:259-263 (abs(det))
        return abs(float(np.linalg.det(self.lattice)))

    @property
    def reciprocal(self):
        # half_types.F90:262: 2*pi*transpose(inverse(lattice)); row i = b_i
        return 2.0 * np.pi * np.linalg.inv(self.lattice).T

    def cartesian(self):
        return self.positions @ self.lattice


@dataclass
class Potcar:
    """potcar_t (half_types.F90:41-56), only the fields the path reads."""
    header: str = ""
    element: str = ""
    zval: float = 0.0
    psp_gmax: float = 0.0
    psp_local: np.ndarray = None
    pspcor: np.ndarray = None
    psprho: np.ndarray = None
    pspnl_gmax: float = 0.0
    lps: list = field(default_factory=list)
    dion: np.ndarray = None
    pspnl: np.ndarray = None       # (NPSNL, channels)
    psprnl: np.ndarray = None
    nmax: int = 0
    paw_rmax: float = 0.0
    qpaw: np.ndarray = None
    rgrid: np.ndarray = None
    wae: np.ndarray = None         # (nmax, channels)
    wps: np.ndarray = None

    @property
    def has_core(self):
        return self.pspcor is not None

    @property
    def channels(self):
        return len(self.lps)


def _floats(tokens):
    return np.array([float(t.replace("D", "E").replace("d", "e")) for t in tokens])


def read_chgcar(path):
    """Return (Crystal, grid shape, values in file order [x fastest])."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    pos = 0
    name = lines[pos].strip(); pos += 1
    scale = float(lines[pos].split()[0]); pos += 1
    if scale <= 0:
        raise ValueError("only positive POSCAR scale is supported")
    lat = np.array([[float(x) for x in lines[pos + i].split()[:3]] for i in range(3)]) * scale
    pos += 3
    words = lines[pos].split(); pos += 1

    def is_int(w):
        try:
            int(w)
            return True
        except ValueError:
            return False

    if all(is_int(w) for w in words):
        species = [f"Type{i + 1}" for i in range(len(words))]
        counts = [int(w) for w in words]
    else:
        species = words
        counts = [int(w) for w in lines[pos].split()]; pos += 1
    mode = lines[pos]; pos += 1          # the reference tests column 1 only
    if mode[:1].lower() == "s":
        mode = lines[pos]; pos += 1
    cart = mode[:1].lower() in ("c", "k")
    nions = sum(counts)
    posn = np.array([[float(x) for x in lines[pos + i].split()[:3]] for i in range(nions)])
    pos += nions
    if cart:
        posn = posn @ np.linalg.inv(lat)
    while not lines[pos].strip():
        pos += 1
    shape = tuple(int(x) for x in lines[pos].split()[:3]); pos += 1
    ngrid = shape[0] * shape[1] * shape[2]
    toks = []
    while len(toks) < ngrid:
        toks.extend(lines[pos].split()); pos += 1
    values = _floats(toks[:ngrid])
    return Crystal(name, lat, species, counts, posn), shape, values


class _Lines:
    def __init__(self, path):
        with open(path) as fh:
            self.lines = fh.read().split("\n")
        self.pos = 0

    def eof(self):
        return self.pos >= len(self.lines)

    def line(self):
        if self.eof():
            raise ValueError("unexpected end of POTCAR")
        s = self.lines[self.pos]
        self.pos += 1
        return s

    def nonblank(self):
        while True:
            s = self.line()
            if s.strip():
                return s

    def values(self, n):
        """Fortran list-directed read of n values starting at the next line."""
        toks = []
        while len(toks) < n:
            toks.extend(self.line().replace(",", " ").split())
        return _floats(toks[:n])


def _tag(line, tag):
    at = line.find(tag)
    if at < 0:
        return None
    eq = line[at:].find("=")
    if eq < 0:
        return None
    return line[at + eq + 1:].lstrip()


def read_potcar(path):
    """Return the list of Potcar datasets in file order (half_potcar.F90:24-49)."""
    rd = _Lines(path)
    out = []
    while True:
        try:
            header = rd.nonblank()
        except ValueError:
            break
        if "End of Dataset" in header:
            continue
        out.append(_read_dataset(rd, header.strip()))
    return out


def _read_dataset(rd, header):
    p = Potcar(header=header)
    words = header.split()
    p.element = words[1] if len(words) >= 2 else ""
    p.zval = float(rd.values(1)[0])
    while True:  # PSCTR, half_potcar.F90:65-78
        s = rd.line()
        if "end of psctr" in s.lower():
            break
        v = _tag(s, "ZVAL")
        if v is not None:
            try:
                p.zval = float(v.split(";")[0].split()[0])
            except (ValueError, IndexError):
                pass
        v = _tag(s, "VRHFIN")
        if v is not None:
            tok = ""
            for ch in v:
                if ch in " :;\t":
                    break
                tok += ch
            p.element = tok
    s = rd.nonblank()
    if "local part" not in s.lower():
        raise ValueError("expected POTCAR local part")
    p.psp_gmax = float(rd.values(1)[0])                         # half_potcar.F90:86
    p.psp_local = rd.values(NPSPTS)
    while True:                                                 # half_potcar.F90:90-106
        s = rd.nonblank().lower()
        if "gradient" in s:
            rd.line()
        elif "core charge-density (partial)" in s:
            p.pspcor = rd.values(NPSPTS)
        elif "kinetic energy density" in s:
            rd.values(NPSPTS)
        elif "atomic pseudo charge-density" in s:
            p.psprho = rd.values(NPSPTS)
            break
        else:
            raise ValueError("unknown POTCAR local-data selector")
    p.pspnl_gmax = float(rd.values(1)[0])                       # half_potcar.F90:117
    lps, dblocks, gcols, rcols = [], [], [], []
    while True:                                                 # half_potcar.F90:119-144
        s = rd.nonblank().lower()
        if "paw radial sets" in s:
            break
        if "non local part" not in s:
            raise ValueError("expected non-local projector block")
        hdr = rd.values(3)
        lval, npro = int(hdr[0]), int(hdr[1])
        flat = rd.values(npro * npro)
        dblocks.append((len(lps), flat.reshape(npro, npro)))   # row-major (:132)
        for _ in range(npro):
            lps.append(lval)
            if "reciprocal space part" not in rd.nonblank().lower():
                raise ValueError("expected reciprocal projector")
            gcols.append(rd.values(NPSNL))
            if "real space part" not in rd.nonblank().lower():
                raise ValueError("expected real projector")
            rcols.append(rd.values(NPSRNL))
    n = len(lps)
    p.lps = lps
    p.dion = np.zeros((n, n))
    for off, blk in dblocks:
        k = blk.shape[0]
        p.dion[off:off + k, off:off + k] = blk
    p.pspnl = np.array(gcols).T.copy()
    p.psprnl = np.array(rcols).T.copy()
    hdr = rd.values(2)                                          # half_potcar.F90:154
    p.nmax, p.paw_rmax = int(hdr[0]), float(hdr[1])
    rd.line()                                                   # format line
    if "augmentation charges" not in rd.nonblank().lower():
        raise ValueError("expected augmentation charges")
    p.qpaw = rd.values(n * n).reshape(n, n)                     # row_major (:207-213)
    p.rgrid = np.zeros(p.nmax)
    p.wae = np.zeros((p.nmax, n))
    p.wps = np.zeros((p.nmax, n))
    while True:                                                 # half_potcar.F90:163-200
        key = rd.nonblank().strip().lower()
        if "occupancies in atom" in key or "uccopancies in atom" in key:
            rd.values(n * n)
        elif key == "grid":
            p.rgrid = rd.values(p.nmax)
        elif key == "aepotential":
            rd.values(p.nmax)
        elif "core charge-density (pseudized)" in key:
            rd.values(p.nmax)
        elif "core charge-density" in key:
            rd.values(p.nmax)
        elif "local pseudopotential core" in key:
            rd.values(p.nmax)
        elif "pspotential valence only" in key:
            rd.values(p.nmax)
        elif "kinetic energy-density" in key or "mkinetic energy-density" in key:
            rd.values(p.nmax)
        elif "pseudo wavefunction" in key:
            p.wps[:, 0] = rd.values(p.nmax)
            rd.nonblank()
            p.wae[:, 0] = rd.values(p.nmax)
            for i in range(1, n):
                rd.nonblank()
                p.wps[:, i] = rd.values(p.nmax)
                rd.nonblank()
                p.wae[:, i] = rd.values(p.nmax)
            break
        elif key[:1] == "t":
            rd.values(n * n)
        else:
            raise ValueError("unknown POTCAR PAW selector: " + key)
    while not rd.eof():
        if "End of Dataset" in rd.line():
            break
    return p


def reorder_f_to_c(values, shape):
    """half_potential.F90:330-344: x-fastest file order -> C order (i3 fastest)."""
    n1, n2, n3 = shape
    return np.asarray(values).reshape(n3, n2, n1).transpose(2, 1, 0).reshape(-1).copy()
