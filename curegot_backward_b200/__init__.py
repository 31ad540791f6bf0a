"""B200-native entropic optimal-transport engine behind the curegot API.

Namespaces mirror the reference package (benben-cd/curegot_backward,
curegot/__init__.py:1-43 and src/bindings.cpp:83-137):

    curegot_backward_b200.numpy   sinkhorn_bcd, sinkhorn_splr      (host arrays)
    curegot_backward_b200.torch   sinkhorn_bcd, sinkhorn_splr, sinkhorn_splr_bwd,
                                  SPLRBackwardContext, splr_ot, splr_ot_with_info,
                                  splr_ot_batch, SPLROT, solve_backward
    curegot_backward_b200.tests   test_T_computation_sparsify,
                                  test_sparse_cholesky_solve

``import curegot_backward_b200 as curegot`` is the drop-in spelling; with
``curegot_backward_b200/compat`` on ``sys.path`` (or after
``install_reference_names()``) the reference's own names work unchanged:
``import curegot``, ``from curegot.torch import splr_ot``, and the
repo-root modules ``backward_core``, ``splr_backward``, ``splr_autograd``.  All
numerical work runs in the sm_100a CUDA library ``_lib/libcuregot_b200.so``
through its C ABI (``include/curegot_b200.h``); there is no CPU fallback.
"""

from __future__ import annotations

import sys as _sys
import types as _types

from . import _native, _solvers
from ._context import SPLRBackwardContext
from . import backward, autograd, points
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

def set_bcd_cluster_path(enabled: bool = True) -> None:
    """Enable (default) or disable the cluster-resident Sinkhorn solver for
    problems whose cost matrix fits one thread-block cluster's shared memory;
    disabled, every problem uses the multi-CTA row/column passes."""
    _native.call("cg_bcd_set_cluster_path", 1 if enabled else 0)


def set_bcd_staging(enabled: bool = True) -> None:
    """Enable or disable (default) the shared-memory staging of the Sinkhorn
    passes: long rows and column strips stream through per-warp rings filled
    by bulk asynchronous copies.  Results are bitwise the same either way; on
    B200 the register path measured faster, so staging is off by default."""
    _native.call("cg_bcd_set_staging", 1 if enabled else 0)


def set_bcd_shifted_lse(enabled: bool = True) -> None:
    """Shifted log-sum-exp sums in the Sinkhorn passes (default on): after
    the first pass, each row / column sums relative to its previous LSE when
    the other side's duals moved by less than 40 base-2 units, with no running
    maximum.  Off, every pass keeps the running maximum.  Results agree to
    rounding."""
    _native.call("cg_bcd_set_shifted_lse", 1 if enabled else 0)


def set_bcd_l2_prefetch(chunks: int) -> None:
    """L2 prefetch distance of the Sinkhorn passes, in warp loop steps
    (0 = off, at most 64).  A hint only: results are bitwise the same for
    every setting."""
    _native.call("cg_bcd_set_l2_prefetch", int(chunks))


_DIRSOLVE = {"auto": 0, "dense": 1, "sparse": 2, "peel": 3}


def set_direction_solver(mode: str = "auto") -> None:
    """Choose the SPLR direction-solve path for this process: "dense" (Schur
    complement + dense FP64 Cholesky), "sparse" (cuSOLVER sparse Cholesky of
    the full sparsified Hessian in an AMD order), "peel" (fill-free
    elimination of the nodes outside the graph's 2-core, then the dense Schur
    path on the core) or "auto" (per sparsity pattern: "peel" when the core's
    Schur complement is at most half the dense one, else "dense")."""
    if mode not in _DIRSOLVE:
        raise ValueError(f"direction solver must be one of {sorted(_DIRSOLVE)}, got {mode!r}")
    _native.call("cg_splr_set_direction_solver", _DIRSOLVE[mode])


def last_direction_solver() -> str | None:
    """Path of the last SPLR direction solve on this thread."""
    v = _native.lib().cg_splr_last_direction_solver()
    return {0: "dense", 1: "sparse", 2: "peel"}.get(v)


def install_reference_names() -> str:
    """Put the reference's import names on sys.path: ``curegot`` (with
    ``curegot.numpy/torch/tests/autograd/backward/_backward_core``) and the
    reference's repo-root modules ``backward_core``, ``splr_backward`` and
    ``splr_autograd``, all served by this package.  Returns the directory
    added."""
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "compat")
    if path not in _sys.path:
        _sys.path.insert(0, path)
    return path
