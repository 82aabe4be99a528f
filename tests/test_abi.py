"""C-ABI boundary checks that need no GPU: the library loads, exports every
symbol the headers declare, and follows the reference's error conventions
(src/half_c_api.F90:627-665, tests/test_c_api.c of the reference)."""
import ctypes as C
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import halfb200
from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", "half.h"), os.path.join(ROOT, "include", "half_b200.h")]


def declared_symbols():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(half_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = halfb200.load_library()
    syms = declared_symbols()
    assert len(syms) == 33   # 18 of ABI v1 + 15 additive extensions
    for s in syms:
        assert hasattr(lib, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", halfb200.library_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (half_[a-z0-9_]+)", out))
    assert set(syms) <= exported


def test_version_and_capabilities():
    assert halfb200.abi_version() == 1
    assert halfb200.version_string() == "0.6.0"
    caps = halfb200.capabilities()
    assert caps & ~0x3F == 0          # only the six defined capability bits


def test_invalid_handle_conventions():
    lib = halfb200.load_library()
    err = C.create_string_buffer(128)
    assert lib.half_destroy(12345, err, 128) == halfb200.HALF_ERROR_INVALID_HANDLE
    assert b"invalid" in err.value
    assert lib.half_destroy(0, err, 128) == halfb200.HALF_ERROR_INVALID_HANDLE
    assert lib.half_destroy(-5, err, 128) == halfb200.HALF_ERROR_INVALID_HANDLE
    k = (C.c_double * 3)(0, 0, 0)
    g = (C.c_int32 * 3)(0, 0, 0)
    e = C.c_double(0)
    v = (C.c_double * 2)()
    smin, smax = C.c_double(0), C.c_double(0)
    st = lib.half_solve_kpoint_mapped(12345, k, 1, 1, g, C.byref(e), v, 1, C.byref(smin), C.byref(smax), err, 128)
    assert st == halfb200.HALF_ERROR_INVALID_HANDLE
    assert lib.half_set_request_geometry(12345, None, err, 128) == halfb200.HALF_ERROR_INVALID_HANDLE
    assert lib.half_get_request_geometry(12345, None, None, None, None, 0, None, 0, None, err, 128) == \
        halfb200.HALF_ERROR_INVALID_HANDLE
    assert lib.half_set_acc_controls(12345, 1e-4, 40, 16, 0, err, 128) == halfb200.HALF_ERROR_INVALID_HANDLE


def test_invalid_selectors_and_truncation():
    lib = halfb200.load_library()
    h = C.c_int64(7)
    err = C.create_string_buffer(128)
    st = lib.half_create_from_files_backend(b"", b"", 400.0, 2, 1, 99, 1, C.byref(h), err, 128)
    assert st == halfb200.HALF_ERROR_INVALID_ARGUMENT and h.value == 0
    for backend, solver, xc in ((0, 5, 2), (0, 0, 2), (3, 1, 2), (0, 1, 3)):
        st = lib.half_create_from_files_backend(b"a", b"b", 400.0, xc, 1, backend, solver, C.byref(h), err, 128)
        assert st == halfb200.HALF_ERROR_INVALID_ARGUMENT
    small = C.create_string_buffer(8)
    lib.half_destroy(99, small, 8)
    assert len(small.value) == 7                     # truncated to capacity - 1, NUL terminated
    assert lib.half_destroy(99, None, 0) == halfb200.HALF_ERROR_INVALID_HANDLE   # capacity 0: no write
    st = lib.half_escn_health(b"http://127.0.0.1:1", 1, err, 128)
    assert st == halfb200.HALF_ERROR_UNAVAILABLE


def test_cpu_backend_unavailable_and_missing_files(tmp_path):
    lib = halfb200.load_library()
    h = C.c_int64(0)
    err = C.create_string_buffer(256)
    st = lib.half_create_from_files_backend(b"x", b"y", 400.0, 2, 1, 1, 1, C.byref(h), err, 256)
    assert st == halfb200.HALF_ERROR_UNAVAILABLE
    st = lib.half_create_from_files_backend(b"x", b"y", -1.0, 2, 1, 2, 4, C.byref(h), err, 256)
    assert st == halfb200.HALF_ERROR_INVALID_ARGUMENT


C_PROGRAM = r"""
#include "half.h"
#include "half_b200.h"
#include <stdio.h>
#include <string.h>
int main(void) {
  char error[128];
  half_handle handle = 0;
  const double gamma[3] = {0.0, 0.0, 0.0};
  const int32_t gzero[3] = {0, 0, 0};
  double eigenvalue = 0.0, smin = 0.0, smax = 0.0;
  double _Complex eigenvector = 0.0;
  if (half_get_abi_version() != HALF_ABI_VERSION) return 1;
  if (strcmp(half_get_version_string(), "0.6.0") != 0) return 2;
  if (half_get_capabilities() & ~(HALF_CAP_CPU | HALF_CAP_CUDA | HALF_CAP_MPI | HALF_CAP_HDF5 |
                                  HALF_CAP_SPGLIB | HALF_CAP_ESCN_API)) return 3;
  if (half_destroy(4242, error, sizeof error) != HALF_ERROR_INVALID_HANDLE) return 4;
  if (strstr(error, "invalid") == NULL) return 5;
  if (half_solve_kpoint_mapped(4242, gamma, 1, 1, gzero, &eigenvalue, &eigenvector, 1, &smin, &smax,
                               error, sizeof error) != HALF_ERROR_INVALID_HANDLE) return 6;
  if (half_create_from_files_backend("", "", 400.0, HALF_XC_PBE, 1, 99, HALF_SOLVER_EVD, &handle,
                                     error, sizeof error) != HALF_ERROR_INVALID_ARGUMENT) return 7;
  if (half_set_request_geometry(4242, NULL, error, sizeof error) != HALF_ERROR_INVALID_HANDLE) return 8;
  if (half_get_request_geometry(4242, NULL, NULL, NULL, NULL, 0, NULL, 0, NULL, error, sizeof error) !=
      HALF_ERROR_INVALID_HANDLE) return 9;
  if (half_set_acc_controls(4242, 1e-4, 40, 16, HALF_PRECISION_MIXED, error, sizeof error) !=
      HALF_ERROR_INVALID_HANDLE) return 10;
  puts("ok");
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_consumer_links_and_runs(tmp_path):
    """A C99 caller built against include/half.h links libhalf.so and sees the
    reference's error conventions."""
    src = tmp_path / "consumer.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "consumer"
    libdir = os.path.dirname(halfb200.library_path())
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L", libdir, "-lhalf", "-Wl,-rpath," + libdir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.strip() == "ok"


# Root of the reference source tree, from the environment (HALF_REFERENCE_ROOT);
# the test below is skipped when it is unset or lacks tests/test_c_api.c.
REFERENCE_ROOT = os.environ.get("HALF_REFERENCE_ROOT", "")
REFERENCE_C_API_TEST = os.path.join(REFERENCE_ROOT, "tests", "test_c_api.c") if REFERENCE_ROOT else ""


@pytest.mark.skipif(not REFERENCE_C_API_TEST or not os.path.exists(REFERENCE_C_API_TEST) or shutil.which("gcc") is None,
                    reason="HALF_REFERENCE_ROOT does not point at the reference sources")
def test_reference_c_api_test_passes_unchanged(tmp_path):
    """The reference's own tests/test_c_api.c, compiled from where it lies,
    passes against this library (only where the reference tree is given)."""
    exe = tmp_path / "ref_c_api"
    libdir = os.path.dirname(halfb200.library_path())
    r = subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), REFERENCE_C_API_TEST,
                        "-o", str(exe), "-L", libdir, "-lhalf", "-Wl,-rpath," + libdir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)


def test_force_and_export_entries_reject_a_stale_handle():
    """The additive force, density and export entries follow the ABI's handle
    convention before reading any other argument (src/half_c_api.F90:636-640)."""
    lib = halfb200.load_library()
    err = C.create_string_buffer(128)
    calls = [
        lambda: lib.half_ionic_forces(12345, None, 0, None, None, None, None, None, err, 128),
        lambda: lib.half_output_density(12345, 1, None, None, 1, 1, None, None, None, 0, None, err, 128),
        lambda: lib.half_forces(12345, 1, None, None, 1, 8.0, 0.1, -1, None, None, None, None, err, 128),
        lambda: lib.half_pack_vasp_waves(12345, 1, None, 1, 1, None, None, 0, None, None, err, 128),
    ]
    for call in calls:
        err.value = b"stale"
        assert call() == halfb200.HALF_ERROR_INVALID_HANDLE
        assert err.value == b"invalid HALF context handle"


def test_occupations_match_the_oracle_and_known_answers():
    """half_occupations (host routine, no GPU) against app/half_energy_check.F90:19-34
    and the oracle restatement of src/half_energy.F90:41-120 on seeded spectra."""
    from oracle.forces import compute_occupations
    occ, band, ent, mu = halfb200.occupations([[0.0, 2.0], [1.0, 3.0]], [0.5, 0.5], 2.0, 0.0)
    assert np.abs(occ - np.array([[2.0, 0.0], [2.0, 0.0]])).max() <= 1e-14
    assert abs(mu - 1.0) <= 1e-14 and abs(band - 1.0) <= 1e-14 and abs(ent) <= 1e-14
    r = np.random.default_rng(3)
    for nk, nb, nelect, sigma, ismear in ((4, 12, 9.0, 0.1, -1), (3, 10, 7.5, 0.05, 0), (2, 8, 6.0, 0.0, -1)):
        eig = np.sort(r.normal(0.0, 3.0, size=(nk, nb)), axis=1)
        w = r.uniform(0.5, 1.0, size=nk)
        w /= w.sum()
        occ, band, ent, mu = halfb200.occupations(eig, w, nelect, sigma, ismear)
        o2, mu2, band2, ent2 = compute_occupations(eig, w, nelect, sigma, ismear)
        assert np.abs(occ - o2).max() <= 1e-12 and abs(band - band2) <= 1e-11
        assert abs(ent - ent2) <= 1e-12 and abs(mu - mu2) <= 1e-11
        assert abs((w[:, None] * occ).sum() - nelect) <= 1e-10
    with pytest.raises(halfb200.HalfError):
        halfb200.occupations([[0.0, 1.0]], [0.7], 2.0, 0.1)        # weights must sum to one
    with pytest.raises(halfb200.HalfError):
        halfb200.occupations([[0.0, 1.0]], [1.0], 5.0, 0.1)        # more electrons than bands hold
