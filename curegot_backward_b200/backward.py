"""Implicit-gradient backward of the SPLR entropic-OT plan.

Public entry point ``solve_backward`` with the reference's contract
(curegot/backward.py:47-144): given the optimal plan T, the upstream
gradient G = dL/dT, the backward context from ``sinkhorn_splr_bwd`` and the
regularisation eta, solve the reduced-Hessian system Q(T*) lambda = mu by
PCG and assemble dL/dM.  The whole solve runs in the native adjoint kernels
(one fused pass over T per PCG iteration, PCG scalars on the device); there
is no Python-side PCG loop.
"""

from __future__ import annotations

import ctypes

import torch

from . import _native

__all__ = ["solve_backward", "solve_backward_batch", "select_preconditioner"]

_VALID_PRECONDITIONERS = ("diag", "splr", "none")
_MODE = {"none": _native.CG_PRECOND_NONE, "diag": _native.CG_PRECOND_DIAG,
         "splr": _native.CG_PRECOND_SPLR}


def select_preconditioner(ctx, preconditioner):
    """Validate a preconditioner name against the context; returns its mode id.

    ``"diag"`` needs the native diagonal (set up by ``sinkhorn_splr_bwd``),
    ``"splr"`` applies factor solve + rank-2 correction, ``"none"`` is plain
    CG.  Any other value raises ValueError (reference backward.py:47-69).
    """
    if preconditioner == "diag":
        if not bool(ctx.has_diagonal_preconditioner):
            raise RuntimeError("SPLRBackwardContext: diagonal preconditioner not set up")
        return _MODE["diag"]
    if preconditioner in ("splr", "none"):
        return _MODE[preconditioner]
    raise ValueError(f"invalid preconditioner '{preconditioner}'; expected one of: "
                     f"{' | '.join(_VALID_PRECONDITIONERS)}")


def solve_backward(T, G, ctx, eta, *, preconditioner="diag", tol=1e-12, max_iter=2000):
    """Solve the backward system and assemble the implicit gradient dL/dM.

    Returns a dict with ``lambda`` ([n+m-1], reduced gauge beta_m = 0),
    ``grad`` ([n, m] = dL/dM), ``iterations``, ``converged`` and the
    ``preconditioner`` used.  A zero right-hand side returns lambda = 0 with
    zero iterations; a PCG breakdown (p^T A p <= 0) raises RuntimeError.
    """
    if T.dim() != 2:
        raise ValueError("T must be a 2D tensor")
    if G.shape != T.shape:
        raise ValueError("G must have the same shape as T")
    mode = select_preconditioner(ctx, preconditioner)
    n, m = int(T.shape[0]), int(T.shape[1])
    if not T.is_cuda:
        raise RuntimeError("solve_backward: T must be a CUDA tensor (no CPU fallback)")
    dev = T.device
    Td = T.detach().to(dtype=torch.float64).contiguous()
    Gd = G.detach().to(device=dev, dtype=torch.float64).contiguous()
    lam = torch.empty(n + m - 1, dtype=torch.float64, device=dev)
    grad = torch.empty((n, m), dtype=torch.float64, device=dev)
    iters = ctypes.c_int(0)
    conv = ctypes.c_int(0)
    handle = ctx._handle if ctx is not None and hasattr(ctx, "_handle") else None
    with torch.cuda.device(dev):
        _native.call("cg_backward_f64", Td.data_ptr(), Gd.data_ptr(), handle, float(eta), mode,
                     float(tol), int(max_iter), n, m, lam.data_ptr(), grad.data_ptr(),
                     ctypes.byref(iters), ctypes.byref(conv),
                     torch.cuda.current_stream(dev).cuda_stream)
    return {"lambda": lam, "grad": grad, "iterations": int(iters.value),
            "converged": bool(conv.value), "preconditioner": preconditioner}


def solve_backward_batch(T, G, ctxs, eta, *, preconditioner="diag", tol=1e-12, max_iter=2000):
    """solve_backward for B problems of one shape in one native call
    (cg_backward_batch_f64): T, G [B, n, m]; ctxs: the B backward contexts
    (may be None with preconditioner="none").  Returns ``lambda`` [B, n+m-1],
    ``grad`` [B, n, m], and per-problem ``iterations`` / ``converged`` lists;
    each problem's values are those of solve_backward.  The "splr"
    preconditioner is not batched."""
    if T.dim() != 3 or G.shape != T.shape:
        raise ValueError("T and G must be [B, n, m] tensors of one shape")
    if preconditioner not in ("diag", "none"):
        raise ValueError("solve_backward_batch: preconditioner must be 'diag' or 'none'")
    if not T.is_cuda:
        raise RuntimeError("solve_backward_batch: T must be a CUDA tensor (no CPU fallback)")
    B, n, m = (int(x) for x in T.shape)
    if preconditioner == "diag" and ctxs is None:
        raise ValueError("solve_backward_batch: preconditioner 'diag' needs the contexts")
    if ctxs is not None and len(ctxs) != B:
        raise ValueError("solve_backward_batch: one context per problem")
    modes = [select_preconditioner(c, preconditioner) for c in ctxs] if ctxs is not None else \
        [select_preconditioner(None, preconditioner)]
    mode = modes[0]
    dev = T.device
    Td = T.detach().to(dtype=torch.float64).contiguous()
    Gd = G.detach().to(device=dev, dtype=torch.float64).contiguous()
    lam = torch.empty((B, n + m - 1), dtype=torch.float64, device=dev)
    grad = torch.empty((B, n, m), dtype=torch.float64, device=dev)
    iters = (ctypes.c_int * B)()
    conv = (ctypes.c_int * B)()
    handles = None
    if ctxs is not None and mode != 0:
        handles = (ctypes.c_void_p * B)(*[c._handle.value for c in ctxs])
    with torch.cuda.device(dev):
        _native.call("cg_backward_batch_f64", Td.data_ptr(), Gd.data_ptr(), handles, float(eta),
                     mode, float(tol), int(max_iter), B, n, m, lam.data_ptr(), grad.data_ptr(),
                     iters, conv, torch.cuda.current_stream(dev).cuda_stream)
    return {"lambda": lam, "grad": grad, "iterations": list(iters),
            "converged": [bool(x) for x in conv], "preconditioner": preconditioner}
