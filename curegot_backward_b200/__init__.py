"""B200-native entropic optimal-transport engine behind the curegot API.

Namespaces mirror the reference package (benben-cd/curegot_backward,
curegot/__init__.py:1-43 and src/bindings.cpp:83-137):

    curegot_backward_b200.numpy   sinkhorn_bcd, sinkhorn_splr      (host arrays)
    curegot_backward_b200.torch   sinkhorn_bcd, sinkhorn_splr, sinkhorn_splr_bwd,
                                  SPLRBackwardContext, splr_ot, splr_ot_with_info,
                                  splr_ot_batch, SPLROT, solve_backward
    curegot_backward_b200.tests   test_T_computation_sparsify,
                                  test_sparse_cholesky_solve

``import curegot_backward_b200 as curegot`` is the drop-in spelling.  All
numerical work runs in the sm_100a CUDA library ``_lib/libcuregot_b200.so``
through its C ABI (``include/curegot_b200.h``); there is no CPU fallback.
"""

from __future__ import annotations

import sys as _sys
import types as _types

from . import _native, _solvers
from ._context import SPLRBackwardContext
from . import backward, autograd
from .autograd import SPLROT, splr_ot, splr_ot_batch, splr_ot_with_info
from .backward import solve_backward

__version__ = "0.1.0"


def _namespace(name: str, doc: str, members: dict) -> _types.ModuleType:
    mod = _types.ModuleType(f"{__name__}.{name}", doc)
    for k, v in members.items():
        setattr(mod, k, v)
    _sys.modules[mod.__name__] = mod
    return mod


numpy = _namespace("numpy", "NumPy interface.", {
    "sinkhorn_bcd": _solvers.numpy_sinkhorn_bcd,
    "sinkhorn_splr": _solvers.numpy_sinkhorn_splr,
})

torch = _namespace("torch", "PyTorch interface.", {
    "sinkhorn_bcd": _solvers.torch_sinkhorn_bcd,
    "sinkhorn_splr": _solvers.torch_sinkhorn_splr,
    "sinkhorn_splr_bwd": _solvers.torch_sinkhorn_splr_bwd,
    "SPLRBackwardContext": SPLRBackwardContext,
    "splr_ot": splr_ot,
    "splr_ot_with_info": splr_ot_with_info,
    "splr_ot_batch": splr_ot_batch,
    "SPLROT": SPLROT,
    "solve_backward": solve_backward,
})

tests = _namespace("tests", "Test functions.", {
    "test_T_computation_sparsify": _solvers.test_T_computation_sparsify,
    "test_sparse_cholesky_solve": _solvers.test_sparse_cholesky_solve,
})

CuregotError = _native.CuregotError
