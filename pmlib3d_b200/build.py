"""Builds the in-tree CUDA library ``libpmgpu.so`` for sm_100a with nvcc.

The library is a few translation units compiled in parallel (``csrc/pmgpu.cu``
with the plans, particle kernels and C ABI; ``csrc/passes_*.cu`` with the FFT
pass kernels, one per precision and component count), without relocatable
device code, linked against a static CUDA runtime so it loads into any process
that has the NVIDIA driver, with or without PyTorch.  Objects go to
``pmlib3d_b200/_build``; a unit is recompiled when it or any header is newer
than its object.
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
OUT = os.path.join(HERE, "libpmgpu.so")
BUILD = os.path.join(HERE, "_build")
UNITS = ([os.path.join(CSRC, "pmgpu.cu")] + sorted(glob.glob(os.path.join(CSRC, "passes_*.cu"))) +
         [os.path.join(CSRC, "output.cu")])
HEADERS = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))) + [
    os.path.join(os.path.dirname(HERE), "include", "pmlib_gpu.h")]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def compile_flags(extra=()):
    return [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", *extra]


def _obj(unit: str) -> str:
    return os.path.join(BUILD, os.path.splitext(os.path.basename(unit))[0] + ".o")


def _deps(unit: str) -> list:
    """The unit and the project headers it includes (nvcc -M), all headers if that fails."""
    r = subprocess.run([nvcc(), "-std=c++17", "-M", unit], capture_output=True, text=True)
    if r.returncode != 0:
        return [unit, *HEADERS]
    words = r.stdout.replace("\\\n", " ").split()
    own = {os.path.realpath(h) for h in HEADERS}
    return [unit] + [w for w in words if os.path.realpath(w) in own]


def _stale(unit: str) -> bool:
    o = _obj(unit)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return any(os.path.getmtime(f) > t for f in _deps(unit) if os.path.exists(f))


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in [*UNITS, *HEADERS] if os.path.exists(f))


def _compile(unit: str, verbose: bool):
    cmd = [nvcc(), *compile_flags(["-Xptxas", "-v"] if verbose else []), "-c", "-o", _obj(unit) + ".tmp", unit]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode == 0:
        os.replace(_obj(unit) + ".tmp", _obj(unit))
    return unit, r


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    todo = [u for u in UNITS if force or _stale(u)]
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda u: _compile(u, verbose), todo))
    for unit, r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {os.path.basename(unit)}")
        if verbose:
            sys.stderr.write(f"== {os.path.basename(unit)}\n" + r.stderr)
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", OUT + ".tmp", *[_obj(u) for u in UNITS]]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libpmgpu.so")
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
