"""ctypes binding of libhalf: every C entry point of include/half.h and
include/half_b200.h, with numpy arrays in and out.

Status codes are raised as HalfError(status, message).  There is no
fallback: if libhalf.so is missing or cannot be loaded, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HALF_SUCCESS = 0
HALF_ERROR_INVALID_ARGUMENT = 1
HALF_ERROR_IO = 2
HALF_ERROR_INVALID_HANDLE = 3
HALF_ERROR_CAPACITY = 4
HALF_ERROR_UNAVAILABLE = 5
HALF_ERROR_INTERNAL = 6

XC = {"lda": 1, "pbe": 2}
BACKEND = {"auto": 0, "cpu": 1, "cuda": 2}
SOLVER = {"evd": 1, "evj": 2, "vasp": 3, "evx": 3, "acc": 4}
PRECISION = {"fp64": 0, "mixed": 1, "fp64_guarded": 2}

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def library_path():
    return os.path.join(os.path.dirname(_HERE), "lib", "libhalf.so")


class HalfError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"HALF status {status}: {message}")
        self.status = status
        self.message = message


class SolveInfo(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("iterations", C.c_int32), ("fp64_iterations", C.c_int32),
                ("converged", C.c_int32), ("npw", C.c_int64), ("operator_applications", C.c_int64),
                ("max_residual_eV", C.c_double), ("setup_ms", C.c_double), ("solve_ms", C.c_double),
                ("operator_ms", C.c_double), ("device_ms", C.c_double), ("local_ms", C.c_double),
                ("local_bytes", C.c_double), ("local_columns", C.c_int64), ("kernel_launches", C.c_int64),
                ("sweep_ms", C.c_double), ("sweep_columns", C.c_int64), ("adjoint_ms", C.c_double),
                ("tensor_ms", C.c_double), ("tensor_flops", C.c_double), ("tensor_launches", C.c_int64),
                ("reserved", C.c_uint64 * 1)]


class RequestGeometry(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("flags", C.c_uint32), ("nions", C.c_int32), ("ntypes", C.c_int32),
                ("grid", C.c_int32 * 3), ("reserved_i32", C.c_int32), ("lattice", C.c_double * 9),
                ("species", C.POINTER(C.c_int32)), ("positions_fractional", C.POINTER(C.c_double)),
                ("reserved", C.c_uint64 * 8)]


_P = C.c_void_p
_ERR = [C.c_char_p, C.c_int]
_SIGS = {
    "half_get_abi_version": (C.c_int, []),
    "half_get_version_string": (C.c_char_p, []),
    "half_get_capabilities": (C.c_int, []),
    "half_escn_health": (C.c_int, [C.c_char_p, C.c_int] + _ERR),
    "half_escn_predict": (C.c_int, [C.c_char_p, _P, _P, C.c_int] + _ERR),
    "half_create_from_files": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double, C.c_int, C.c_int, _P] + _ERR),
    "half_create_from_files_backend": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double, C.c_int, C.c_int, C.c_int,
                                                 C.c_int, _P] + _ERR),
    "half_create_from_escn": (C.c_int, [C.c_char_p, C.c_char_p, _P, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_int, C.c_int, _P] + _ERR),
    "half_destroy": (C.c_int, [C.c_int64] + _ERR),
    "half_set_request_geometry": (C.c_int, [C.c_int64, _P] + _ERR),
    "half_get_request_geometry": (C.c_int, [C.c_int64, _P, _P, _P, _P, C.c_int64, _P, C.c_int64, _P] + _ERR),
    "half_get_system_info": (C.c_int, [C.c_int64, _P, _P, _P, _P, _P] + _ERR),
    "half_get_basis_size": (C.c_int, [C.c_int64, _P, _P] + _ERR),
    "half_get_basis": (C.c_int, [C.c_int64, _P, C.c_int64, _P, _P] + _ERR),
    "half_assemble_hs": (C.c_int, [C.c_int64, _P, C.c_int64, _P, _P] + _ERR),
    "half_apply_hs": (C.c_int, [C.c_int64, _P, C.c_int, C.c_int64, _P, _P, _P] + _ERR),
    "half_solve_kpoint": (C.c_int, [C.c_int64, _P, C.c_int, _P, _P, C.c_int64, _P, _P] + _ERR),
    "half_solve_kpoint_mapped": (C.c_int, [C.c_int64, _P, C.c_int, C.c_int64, _P, _P, _P, C.c_int64, _P, _P] + _ERR),
    "half_set_acc_controls": (C.c_int, [C.c_int64, C.c_double, C.c_int, C.c_int, C.c_int] + _ERR),
    "half_get_last_solve_info": (C.c_int, [C.c_int64, _P] + _ERR),
    "half_solve_kpoints": (C.c_int, [C.c_int64, C.c_int, _P, C.c_int, _P] + _ERR),
    "half_solve_kpoints_device": (C.c_int, [C.c_int64, C.c_int, _P, C.c_int, C.c_void_p, C.c_void_p, C.c_int64]
                                  + _ERR),
    "half_set_positions": (C.c_int, [C.c_int64, _P] + _ERR),
    "half_set_positions_noalloc": (C.c_int, [C.c_int64, _P] + _ERR),
    "half_nonlocal_forces": (C.c_int, [C.c_int64, _P, C.c_int, C.c_int64, _P, _P, _P, C.c_double, _P] + _ERR),
    "half_band_forces": (C.c_int, [C.c_int64, C.c_int, _P, _P, C.c_int, C.c_double, C.c_double, C.c_int, _P, _P, _P,
                                   _P] + _ERR),
    "half_ionic_forces": (C.c_int, [C.c_int64, _P, C.c_int64, _P, _P, _P, _P, _P] + _ERR),
    "half_output_density": (C.c_int, [C.c_int64, C.c_int, _P, _P, C.c_int, C.c_int64, _P, _P, _P, C.c_int64, _P]
                            + _ERR),
    "half_pack_vasp_waves": (C.c_int, [C.c_int64, C.c_int, _P, C.c_int, C.c_int64, _P, _P, C.c_int64, _P, _P]
                             + _ERR),
    "half_occupations": (C.c_int, [C.c_int, C.c_int, _P, _P, C.c_double, C.c_double, C.c_int, _P, _P] + _ERR),
    "half_forces": (C.c_int, [C.c_int64, C.c_int, _P, _P, C.c_int, C.c_double, C.c_double, C.c_int, _P, _P, _P, _P]
                    + _ERR),
    "half_get_allocation_counts": (C.c_int, [_P, _P] + _ERR),
    "half_tc_cgemm": (C.c_int, [C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, _P, C.c_void_p, C.c_int64, C.c_void_p,
                                C.c_int64, _P, C.c_void_p, C.c_int64, C.c_int] + _ERR),
}


def load_library(path=None):
    """Load libhalf.so (once) and declare every exported signature."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or library_path()
    if not os.path.exists(p):
        raise OSError(f"libhalf.so not built: {p} (run deepaw-half_b200/build.py)")
    lib = C.CDLL(p)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(status, err):
    if status != HALF_SUCCESS:
        raise HalfError(status, err.value.decode(errors="replace"))


def abi_version():
    return load_library().half_get_abi_version()


def version_string():
    return load_library().half_get_version_string().decode()


def capabilities():
    return load_library().half_get_capabilities()


def occupations(eigenvalues, weights, nelect, sigma, ismear=-1):
    """half_occupations: (occupations (nk, nb), band energy, entropy term, mu).
    A host routine; needs no context or GPU."""
    eig = np.ascontiguousarray(np.asarray(eigenvalues, dtype=np.float64))
    if eig.ndim != 2:
        raise ValueError("eigenvalues must be (nk, nbands)")
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
    occ = np.zeros_like(eig)
    en = np.zeros(3)
    err = C.create_string_buffer(512)
    _check(load_library().half_occupations(eig.shape[0], eig.shape[1], _ptr(eig), _ptr(w), float(nelect),
                                           float(sigma), int(ismear), _ptr(occ), _ptr(en), err, 512), err)
    return occ, en[0], en[1], en[2]


def allocation_counts():
    """(device buffers taken, cudaMalloc calls) since the library was loaded."""
    lib = load_library()
    err = C.create_string_buffer(128)
    r, d = C.c_int64(0), C.c_int64(0)
    _check(lib.half_get_allocation_counts(C.byref(r), C.byref(d), err, 128), err)
    return int(r.value), int(d.value)


def tc_cgemm(op_a, op_b, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, c_ptr, ldc, c_fp64=False):
    """C = alpha op(A) op(B) + beta C on the library's tensor-core kernel.
    a_ptr, b_ptr, c_ptr: device addresses of column-major complex64 data
    (complex128 for C when c_fp64); op_a / op_b in 'N', 'T', 'C'."""
    lib = load_library()
    err = C.create_string_buffer(512)
    al = np.array([alpha.real, alpha.imag], dtype=np.float64)
    be = np.array([beta.real, beta.imag], dtype=np.float64)
    st = lib.half_tc_cgemm(op_a.encode(), op_b.encode(), m, n, k, _ptr(al), C.c_void_p(a_ptr), lda,
                           C.c_void_p(b_ptr), ldb, _ptr(be), C.c_void_p(c_ptr), ldc, int(bool(c_fp64)), err, 512)
    _check(st, err)


class Context:
    """One libhalf context (half_create_from_files_backend)."""

    def __init__(self, chgcar, potcar, encut, xc="pbe", use_uspp=True, backend="cuda", solver="acc"):
        self.lib = load_library()
        self.handle = C.c_int64(0)
        err = C.create_string_buffer(512)
        st = self.lib.half_create_from_files_backend(
            str(chgcar).encode(), str(potcar).encode(), float(encut), XC[xc], 1 if use_uspp else 0,
            BACKEND[backend], SOLVER[solver], C.byref(self.handle), err, 512)
        _check(st, err)
        ni, nt = C.c_int(0), C.c_int(0)
        grid = (C.c_int * 3)()
        lat = (C.c_double * 9)()
        vol = C.c_double(0)
        _check(self.lib.half_get_system_info(self.handle, C.byref(ni), C.byref(nt), grid, lat, C.byref(vol), err, 512),
               err)
        self.nions, self.ntypes = ni.value, nt.value
        self.grid = tuple(grid)
        self.lattice = np.array(list(lat)).reshape(3, 3)
        self.volume = vol.value

    # -------------------------------------------------------------- helpers
    def _err(self):
        return C.create_string_buffer(512)

    @staticmethod
    def _k(k):
        return np.ascontiguousarray(np.asarray(k, dtype=np.float64).reshape(3))

    def close(self):
        if self.handle.value:
            err = self._err()
            _check(self.lib.half_destroy(self.handle, err, 512), err)
            self.handle = C.c_int64(0)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None and self.handle.value:
                self.lib.half_destroy(self.handle, None, 0)
        except Exception:
            pass

    # -------------------------------------------------------------- ABI v1
    def basis(self, k=(0, 0, 0)):
        err = self._err()
        kk = self._k(k)
        n = C.c_int64(0)
        _check(self.lib.half_get_basis_size(self.handle, _ptr(kk), C.byref(n), err, 512), err)
        g = np.zeros((n.value, 3), dtype=np.int32)
        kin = np.zeros(n.value)
        _check(self.lib.half_get_basis(self.handle, _ptr(kk), n.value, _ptr(g), _ptr(kin), err, 512), err)
        return g, kin

    def npw(self, k=(0, 0, 0)):
        err = self._err()
        kk = self._k(k)
        n = C.c_int64(0)
        _check(self.lib.half_get_basis_size(self.handle, _ptr(kk), C.byref(n), err, 512), err)
        return n.value

    def solve(self, k, nbands, vectors=False):
        err = self._err()
        kk = self._k(k)
        eig = np.zeros(nbands)
        smin, smax = C.c_double(0), C.c_double(0)
        vec = None
        ld = 0
        if vectors:
            ld = self.npw(k)
            vec = np.zeros((nbands, ld), dtype=np.complex128)   # column-major (ld x nbands)
        _check(self.lib.half_solve_kpoint(self.handle, _ptr(kk), nbands, _ptr(eig), _ptr(vec), ld, C.byref(smin),
                                          C.byref(smax), err, 512), err)
        return eig, (vec.T if vec is not None else None), smin.value, smax.value

    def solve_mapped(self, k, nbands, host_gvec):
        err = self._err()
        kk = self._k(k)
        hg = np.ascontiguousarray(np.asarray(host_gvec, dtype=np.int32))
        n = hg.shape[0]
        eig = np.zeros(nbands)
        vec = np.zeros((nbands, n), dtype=np.complex128)
        smin, smax = C.c_double(0), C.c_double(0)
        _check(self.lib.half_solve_kpoint_mapped(self.handle, _ptr(kk), nbands, n, _ptr(hg), _ptr(eig), _ptr(vec), n,
                                                 C.byref(smin), C.byref(smax), err, 512), err)
        return eig, vec.T, smin.value, smax.value

    def apply_hs(self, k, psi):
        err = self._err()
        kk = self._k(k)
        psi = np.asarray(psi, dtype=np.complex128)
        if psi.ndim == 1:
            psi = psi[:, None]
        n, nb = psi.shape
        x = np.ascontiguousarray(psi.T)           # column-major (n x nb)
        h = np.zeros_like(x)
        s = np.zeros_like(x)
        _check(self.lib.half_apply_hs(self.handle, _ptr(kk), nb, n, _ptr(x), _ptr(h), _ptr(s), err, 512), err)
        return h.T, s.T

    def assemble_hs(self, k):
        err = self._err()
        kk = self._k(k)
        n = self.npw(k)
        h = np.zeros((n, n), dtype=np.complex128)
        s = np.zeros((n, n), dtype=np.complex128)
        _check(self.lib.half_assemble_hs(self.handle, _ptr(kk), n, _ptr(h), _ptr(s), err, 512), err)
        return h.T, s.T

    # -------------------------------------------------------------- extensions
    def set_acc(self, tol=1e-4, max_iterations=40, block_size=0, precision="fp64"):
        """ACC controls; block_size 0 lets the library's autotuner pick the bands per chunk."""
        err = self._err()
        _check(self.lib.half_set_acc_controls(self.handle, float(tol), int(max_iterations), int(block_size),
                                              PRECISION[precision], err, 512), err)

    def info(self):
        err = self._err()
        s = SolveInfo()
        s.struct_size = C.sizeof(SolveInfo)
        _check(self.lib.half_get_last_solve_info(self.handle, C.byref(s), err, 512), err)
        return {f: getattr(s, f) for f, _ in SolveInfo._fields_ if f not in ("reserved", "struct_size")}

    def solve_kpoints(self, kpoints, nbands):
        err = self._err()
        ks = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
        eig = np.zeros((len(ks), nbands))
        _check(self.lib.half_solve_kpoints(self.handle, len(ks), _ptr(ks), nbands, _ptr(eig), err, 512), err)
        return eig

    def solve_kpoints_device(self, kpoints, nbands, eigenvalues_ptr, vectors_ptr=None, ld=0):
        """half_solve_kpoints_device: eigenvalues (nk x nbands, float64) and
        optionally eigenvectors (nk blocks of ld x nbands, complex128,
        column-major) written to device memory at the given addresses (for
        example ``tensor.data_ptr()`` of CUDA tensors)."""
        err = self._err()
        ks = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
        _check(self.lib.half_solve_kpoints_device(self.handle, len(ks), _ptr(ks), nbands, C.c_void_p(eigenvalues_ptr),
                                                  C.c_void_p(vectors_ptr) if vectors_ptr else None, ld, err, 512),
               err)

    def set_positions(self, positions_fractional):
        err = self._err()
        p = np.ascontiguousarray(np.asarray(positions_fractional, dtype=np.float64).reshape(-1, 3))
        _check(self.lib.half_set_positions(self.handle, _ptr(p), err, 512), err)

    def set_positions_noalloc(self, positions_fractional):
        """``set_positions`` through the entry point that allocates no device
        memory (fixed 32 MiB scratch; HALF_ERROR_CAPACITY beyond it)."""
        err = self._err()
        p = np.ascontiguousarray(np.asarray(positions_fractional, dtype=np.float64).reshape(-1, 3))
        _check(self.lib.half_set_positions_noalloc(self.handle, _ptr(p), err, 512), err)

    def nonlocal_forces(self, k, vectors, eigenvalues, occupations, kweight):
        err = self._err()
        kk = self._k(k)
        v = np.ascontiguousarray(np.asarray(vectors, dtype=np.complex128).T)   # (nb, n) = column-major n x nb
        nb, n = v.shape
        e = np.ascontiguousarray(np.asarray(eigenvalues, dtype=np.float64))
        o = np.ascontiguousarray(np.asarray(occupations, dtype=np.float64))
        f = np.zeros((self.nions, 3))
        _check(self.lib.half_nonlocal_forces(self.handle, _ptr(kk), nb, n, _ptr(v), _ptr(e), _ptr(o), float(kweight),
                                             _ptr(f), err, 512), err)
        return f

    def band_forces(self, kpoints, weights, nbands, nelect, sigma, ismear=-1):
        err = self._err()
        ks = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
        f = np.zeros((self.nions, 3))
        eig = np.zeros((len(ks), nbands))
        occ = np.zeros((len(ks), nbands))
        en = np.zeros(3)
        _check(self.lib.half_band_forces(self.handle, len(ks), _ptr(ks), _ptr(w), nbands, float(nelect), float(sigma),
                                         int(ismear), _ptr(f), _ptr(eig), _ptr(occ), _ptr(en), err, 512), err)
        return dict(forces=f, eigenvalues=eig, occupations=occ, band_energy=en[0], entropy=en[1], mu=en[2])

    def ionic_forces(self, output_density=None):
        """Ewald, local, NLCC and Harris forces (each (nions, 3), eV/A) and the
        Ewald / local energies; output_density in file order (x fastest,
        rho * Omega), None = the context's own density."""
        err = self._err()
        d = None
        n = 0
        if output_density is not None:
            d = np.ascontiguousarray(np.asarray(output_density, dtype=np.float64).reshape(-1))
            n = d.size
        out = {k: np.zeros((self.nions, 3)) for k in ("ewald", "local", "nlcc", "harris")}
        en = np.zeros(6)
        _check(self.lib.half_ionic_forces(self.handle, _ptr(d) if d is not None else None, n, _ptr(out["ewald"]),
                                          _ptr(out["local"]), _ptr(out["nlcc"]), _ptr(out["harris"]), _ptr(en),
                                          err, 512), err)
        out.update(ewald_energy=en[0], ewald_real=en[1], ewald_reciprocal=en[2], ewald_self=en[3],
                   ewald_background=en[4], local_energy=en[5])
        return out

    def grid_size(self):
        return int(np.prod(self.grid))

    def output_density(self, kpoints, weights, vectors, occupations):
        """Smooth + augmentation density (file order) of given states: vectors is a
        list of (npw_k, nbands) arrays, occupations (nk, nbands)."""
        err = self._err()
        ks = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
        nb = int(np.asarray(vectors[0]).shape[1])
        ld = max(int(np.asarray(v).shape[0]) for v in vectors)
        block = np.zeros((len(ks), nb, ld), dtype=np.complex128)      # per k: column-major ld x nb
        for ik, v in enumerate(vectors):
            v = np.asarray(v, dtype=np.complex128)
            block[ik, :, :v.shape[0]] = v.T
        occ = np.ascontiguousarray(np.asarray(occupations, dtype=np.float64).reshape(len(ks), nb))
        n = self.grid_size()
        rho = np.zeros(n)
        aug = C.c_double(0.0)
        _check(self.lib.half_output_density(self.handle, len(ks), _ptr(ks), _ptr(w), nb, ld, _ptr(block), _ptr(occ),
                                            _ptr(rho), n, C.byref(aug), err, 512), err)
        return rho, aug.value

    def pack_vasp_waves(self, kpoints, vectors):
        """VASP-ordered single-precision coefficients: (packed float32, npws, offsets);
        vectors is a list of (npw_k, nbands) arrays (host memory)."""
        err = self._err()
        ks = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
        nb = int(np.asarray(vectors[0]).shape[1])
        ld = max(int(np.asarray(v).shape[0]) for v in vectors)
        block = np.zeros((len(ks), nb, ld), dtype=np.complex128)
        for ik, v in enumerate(vectors):
            v = np.asarray(v, dtype=np.complex128)
            block[ik, :, :v.shape[0]] = v.T
        npws = np.zeros(len(ks), dtype=np.int32)
        offsets = np.zeros(len(ks), dtype=np.int64)
        _check(self.lib.half_pack_vasp_waves(self.handle, len(ks), _ptr(ks), nb, ld, _ptr(block), None, 0, _ptr(npws),
                                             _ptr(offsets), err, 512), err)
        packed = np.zeros(int(2 * nb * npws.astype(np.int64).sum()), dtype=np.float32)
        _check(self.lib.half_pack_vasp_waves(self.handle, len(ks), _ptr(ks), nb, ld, _ptr(block), _ptr(packed),
                                             packed.size, _ptr(npws), _ptr(offsets), err, 512), err)
        return packed, npws, offsets

    def forces(self, kpoints, weights, nbands, nelect, sigma, ismear=-1):
        """The analytic --forces workload: total force, its five components, the
        output density and the energies."""
        err = self._err()
        ks = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
        f = np.zeros((self.nions, 3))
        comp = np.zeros((5, self.nions, 3))
        rho = np.zeros(self.grid_size())
        en = np.zeros(6)
        _check(self.lib.half_forces(self.handle, len(ks), _ptr(ks), _ptr(w), int(nbands), float(nelect), float(sigma),
                                    int(ismear), _ptr(f), _ptr(comp), _ptr(rho), _ptr(en), err, 512), err)
        return dict(forces=f, ewald=comp[0], local=comp[1], **{"nonlocal": comp[2]}, nlcc=comp[3], harris=comp[4],
                    output_density=rho, band_energy=en[0], entropy=en[1], mu=en[2], ewald_energy=en[3],
                    local_energy=en[4], augmentation_charge=en[5])
