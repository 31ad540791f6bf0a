"""Builds the in-tree CUDA library ``_lib/libcuregot_b200.so`` for sm_100a.

Every ``csrc/*.cu`` file is compiled by nvcc (in parallel) with
``-gencode arch=compute_100a,code=sm_100a -lineinfo`` and linked into one
shared library that exports the C ABI declared in ``include/curegot_b200.h``.
The library links cuSOLVER (dense FP64 Cholesky of the Schur complement).

Usage: ``python -m curegot_backward_b200.build`` (or ``build()`` from Python).
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(ROOT, "_build", "obj")
LIB_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIB_DIR, "libcuregot_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _nvcc() -> str:
    p = shutil.which("nvcc") or os.path.join(CUDA_HOME, "bin", "nvcc")
    return p


def _flags(extra=()):
    # C++20: the SPLR solve is a coroutine (csrc/task.cuh)
    return [*ARCH, "-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC",
            "-Xcompiler", "-Wno-subobject-linkage",
            "-I", INCLUDE, "-I", CSRC, *extra]


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "curegot_b200.h"))
    return hs


def _compile(src: str, verbose: bool, extra=()) -> str:
    os.makedirs(OBJ, exist_ok=True)
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    newest_dep = max(os.path.getmtime(h) for h in _headers() + [src])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep and not extra:
        return obj
    cmd = [_nvcc(), *_flags(extra), "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None, extra=()) -> str:
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, extra), srcs))
    os.makedirs(LIB_DIR, exist_ok=True)
    newest = max(os.path.getmtime(o) for o in objs)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest and not extra:
        return LIB
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *ARCH, "-shared", "-o", tmp, *objs,
           "-L", os.path.join(CUDA_HOME, "lib64"), "-lcusolver", "-lcusparse", "-lcublas",
           "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64")]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


def ptxas_report() -> str:
    """Registers / spills / shared memory per kernel (nvcc -Xptxas -v)."""
    out = []
    for src in _sources():
        cmd = [_nvcc(), *_flags(["-Xptxas", "-v"]), "-c", src, "-o", os.devnull]
        r = subprocess.run(cmd, capture_output=True, text=True)
        out.append(f"== {os.path.basename(src)}\n{r.stderr}")
    return "\n".join(out)


if __name__ == "__main__":
    if "--ptxas" in sys.argv:
        print(ptxas_report())
    else:
        print(build(verbose="-v" in sys.argv))
