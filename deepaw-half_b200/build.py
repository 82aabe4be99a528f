"""Build libhalf.so (the C-ABI library) in-tree for sm_100a.

    python deepaw-half_b200/build.py [--force]

Compiles every csrc/*.cu and csrc/*.cpp with nvcc
(-gencode arch=compute_100a,code=sm_100a -lineinfo -O3) into _build/ and
links deepaw-half_b200/lib/libhalf.so against the CUDA toolkit's cuBLAS and
cuSOLVER.  Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libhalf.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
          "-I" + CSRC, "-I" + INCLUDE]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def cuda_lib_dir(nv):
    return os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nv))), "lib64")


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(nv, src, obj, force):
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header()):
        return None
    cmd = [nv] + ARCH + COMMON + ["-c", src, "-o", obj]
    if src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"] if os.environ.get("HALF_PTXAS_VERBOSE") else []
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    return r.stderr.strip() or None


def build(force=False, verbose=True):
    nv = nvcc()
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    objs = [os.path.join(BUILD, os.path.basename(s) + ".o") for s in srcs]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        futs = {ex.submit(_compile, nv, s, o, force): s for s, o in zip(srcs, objs)}
        for f in cf.as_completed(futs):
            msg = f.result()
            if msg and verbose:
                print(f"[{os.path.basename(futs[f])}] {msg}", file=sys.stderr)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        libdir = cuda_lib_dir(nv)
        cmd = [nv] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-L" + libdir, "-lcublas", "-lcusolver", "-Xlinker", "-rpath," + libdir]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
