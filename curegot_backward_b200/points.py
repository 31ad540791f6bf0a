"""Sinkhorn on a cost recomputed from point clouds on the tensor cores.

The cost is never stored:

    M_ij = max(0, s * ((|x_i|^2 + |y_j|^2) - 2 x_i . y_j))      (FP32)

X (n x d) and Y (m x d) are BF16 (1 <= d <= 64); x_i . y_j is accumulated in
FP32 by tcgen05 MMAs and the squared norms in FP32 from the same BF16
values.  ``s`` defaults to 1/d, the mean over features (M_ij = mean_k
(x_ik - y_jk)^2 up to rounding).  No reference counterpart: the reference
solvers take a materialised M (src/solvers.h:4-9); this is the BF16-input /
FP32-compute cost variant of the differentiation configuration, and
``cost_from_points`` is the same computation written out as a matrix.
"""
from __future__ import annotations

import ctypes

import torch

from . import _native


def _check_points(X, Y):
    if not (torch.is_tensor(X) and torch.is_tensor(Y)):
        raise TypeError("X and Y must be torch tensors")
    if X.dtype != torch.bfloat16 or Y.dtype != torch.bfloat16:
        raise TypeError("X and Y must be torch.bfloat16")
    if X.dim() != 2 or Y.dim() != 2 or X.shape[1] != Y.shape[1]:
        raise ValueError("X (n x d) and Y (m x d) must be matrices with the same d")
    if not (X.is_cuda and Y.is_cuda) or X.device != Y.device:
        raise ValueError("X and Y must be on the same CUDA device")
    d = int(X.shape[1])
    if not 1 <= d <= 64:
        raise ValueError("feature dimension must be in [1, 64]")
    return X.contiguous(), Y.contiguous(), int(X.shape[0]), int(Y.shape[0]), d


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def cost_from_points(X, Y, scale=None):
    """The FP32 cost matrix the tensor-core passes see (n x m, on X's device)."""
    X, Y, n, m, d = _check_points(X, Y)
    s = 1.0 / d if scale is None else float(scale)
    M = torch.empty((n, m), dtype=torch.float32, device=X.device)
    with torch.cuda.device(X.device):
        _native.call("cg_points_cost_bf16", X.data_ptr(), Y.data_ptr(), n, m, d, s, M.data_ptr(),
                     _stream(X.device))
    return M


def sinkhorn_bcd_points(X, Y, a, b, reg, tol=1e-8, max_iter=100000, scale=None,
                        precision="mixed"):
    """Sinkhorn BCD with the cost recomputed from X, Y in every pass.

    Returns {"niter", "dual" (FP64 [n + m]: alpha then beta), "fast_iters"}.
    The stopping rule is the row-marginal error ||T 1 - a||_2 < tol of an
    iterate; ``precision="mixed"`` runs SFU exponentials until the estimate
    is below tol / 2, then FP64 passes confirm."""
    X, Y, n, m, d = _check_points(X, Y)
    if precision not in ("mixed", "fp64"):
        raise ValueError("precision must be 'mixed' or 'fp64'")
    if not reg > 0:
        raise ValueError("reg must be positive")
    dev = X.device
    a = torch.as_tensor(a, dtype=torch.float64, device=dev).contiguous()
    b = torch.as_tensor(b, dtype=torch.float64, device=dev).contiguous()
    if a.numel() != n or b.numel() != m:
        raise ValueError("a must have n entries and b m entries")
    s = 1.0 / d if scale is None else float(scale)
    dual = torch.empty(n + m, dtype=torch.float64, device=dev)
    niter = ctypes.c_int(0)
    fast = ctypes.c_int(0)
    mode = _native.CG_POINTS_MIXED if precision == "mixed" else _native.CG_POINTS_FP64
    with torch.cuda.device(dev):
        _native.call("cg_bcd_points_bf16", X.data_ptr(), Y.data_ptr(), n, m, d, s, a.data_ptr(),
                     b.data_ptr(), float(reg), int(max_iter), float(tol), mode,
                     ctypes.byref(niter), dual.data_ptr(), ctypes.byref(fast), _stream(dev))
    return {"niter": niter.value, "dual": dual, "fast_iters": fast.value}


def cost_normalisers(X, Y):
    """(max, lower median) of the unscaled cost c_ij = max(0, |x_i|^2 + |y_j|^2
    - 2 x_i . y_j) as the tensor-core tiles compute it, without storing it.
    ``sinkhorn_bcd_points(..., scale=1 / max)`` is the "M / max" cost;
    ``scale=1 / median`` the "M / median" one."""
    X, Y, n, m, d = _check_points(X, Y)
    mx = ctypes.c_double(0.0)
    md = ctypes.c_double(0.0)
    with torch.cuda.device(X.device):
        _native.call("cg_points_cost_stats_bf16", X.data_ptr(), Y.data_ptr(), n, m, d,
                     ctypes.byref(mx), ctypes.byref(md), _stream(X.device))
    return mx.value, md.value
