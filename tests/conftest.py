"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU.

The binding (and with it libhalf.so and the CUDA toolkit's cuBLAS) is loaded
before anything imports torch.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "deepaw-half_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

import halfb200  # noqa: E402  (load the library first)

try:
    halfb200.load_library()
except OSError:
    pass


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_present():
    try:
        return halfb200.capabilities() & 2 != 0
    except OSError:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_present():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def inputs_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("inputs"))


_CACHE = {}


def workload_files(name, directory):
    """Write (once per session) the synthetic CHGCAR/POTCAR of a workload."""
    from halfb200 import synth
    key = (name, directory)
    if key not in _CACHE:
        w = synth.workload(name)
        ch, po = synth.write_inputs(w, directory)
        _CACHE[key] = (w, ch, po)
    return _CACHE[key]


@pytest.fixture(scope="session")
def si2(inputs_dir):
    return workload_files("si2", inputs_dir)


@pytest.fixture(scope="session")
def hfo2(inputs_dir):
    return workload_files("hfo2", inputs_dir)


_SYS = {}


@pytest.fixture(scope="session")
def oracle_system():
    """Oracle System objects keyed by (name, with_gradient)."""
    from oracle import hamiltonian as H

    def get(name, files, with_gradient=False):
        key = (name, with_gradient)
        if key not in _SYS:
            w, ch, po = files
            _SYS[key] = H.load_system(ch, po, w.encut, use_pbe=(w.xc == "pbe"), use_uspp=True,
                                      with_gradient=with_gradient)
        return _SYS[key]
    return get


def rng(seed=0):
    return np.random.default_rng(seed)
