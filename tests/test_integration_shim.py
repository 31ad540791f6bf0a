"""The reference-side shim of INTEGRATION.md compiles and links (CPU only).

The two C++ blocks (backward_context_b200.h, solvers_b200.cpp) are taken
from INTEGRATION.md as written, compiled against include/curegot_b200.h and
linked into a shared library with libcuregot_b200.so.  When a reference
checkout is available ($REFERENCE_ROOT, or a `reference` directory beside
this repository), a caller compiled against the reference's own
src/solvers.h is linked against that library: a definition whose signature
differs from the reference's declaration leaves an undefined symbol and
fails the link.  Nothing is executed on a GPU.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
LIB_DIR = os.path.join(ROOT, "curegot_backward_b200", "_lib")


def _blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    out = {}
    for body in re.findall(r"```cpp\n(.*?)```", text, flags=re.S):
        first = body.splitlines()[0]
        m = re.match(r"// (\S+) --", first)
        if m:
            out[m.group(1)] = body
    return out


def _reference_root():
    env = os.environ.get("REFERENCE_ROOT")
    cand = env or os.path.join(os.path.dirname(ROOT), "reference")
    return cand if os.path.isfile(os.path.join(cand, "src", "solvers.h")) else None


def _run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    assert r.returncode == 0, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"


@pytest.fixture(scope="module")
def shim_lib(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIB_DIR, "libcuregot_b200.so")):
        pytest.skip("native library not built")
    blocks = _blocks()
    assert {"backward_context_b200.h", "solvers_b200.cpp"} <= set(blocks)
    d = tmp_path_factory.mktemp("shim")
    for name, body in blocks.items():
        (d / name).write_text(body)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", str(d), "-I",
           os.path.join(CUDA_HOME, "include")]
    _run(["g++", "-std=c++17", "-fPIC", "-Wall", "-Werror", *inc, "-c", "solvers_b200.cpp",
          "-o", "solvers_b200.o"], d)
    _run(["g++", "-shared", "-o", "libshim.so", "solvers_b200.o", "-L", LIB_DIR,
          "-lcuregot_b200", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
          f"-Wl,-rpath,{LIB_DIR}", "-Wl,--no-undefined"], d)
    return d, inc


def test_shim_compiles_and_links_with_the_library(shim_lib):
    d, _ = shim_lib
    nm = subprocess.run(["nm", "-DC", str(d / "libshim.so")], capture_output=True, text=True)
    for fn in ("cuda_sinkhorn_bcd(", "cuda_sinkhorn_splr(", "cuda_sinkhorn_splr_bwd("):
        assert fn in nm.stdout


def test_shim_matches_the_reference_declarations(shim_lib):
    ref = _reference_root()
    if ref is None:
        pytest.skip("no reference checkout to read src/solvers.h from")
    d, inc = shim_lib
    caller = (
        f'#include "{os.path.join(ref, "src", "solvers.h")}"\n'
        '#include "backward_context_b200.h"\n'
        "int main(int argc, char**) {\n"
        "  if (argc < 100) return 0;  // link-time check only: never called\n"
        "  int niter = 0; bool conv = false;\n"
        "  cuda_sinkhorn_bcd(nullptr, nullptr, nullptr, nullptr, 0.1, 1, 1e-8, 1, 1, &niter);\n"
        "  cuda_sinkhorn_splr(nullptr, nullptr, nullptr, nullptr, 0.1, 1, 1e-8, 1, 2, &niter,\n"
        "                     0.1, 1e-3, 30, 3, 0);\n"
        "  SPLRBackwardContext ctx(2, 4);\n"
        "  cuda_sinkhorn_splr_bwd(nullptr, nullptr, nullptr, nullptr, 0.1, 1, 1e-8, 1, 2, &niter,\n"
        "                         0.1, 1e-3, 30, 3, 0, nullptr, nullptr, true, true, &ctx,\n"
        "                         &conv, false, false);\n"
        "  return ctx.is_valid() ? 0 : 1;\n"
        "}\n")
    (d / "caller.cpp").write_text(caller)
    _run(["g++", "-std=c++17", *inc, "caller.cpp", "-o", "caller", "-L", str(d), "-lshim",
          "-L", LIB_DIR, "-lcuregot_b200", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
          f"-Wl,-rpath,{d}", f"-Wl,-rpath,{LIB_DIR}"], d)
