"""Solver entry points mirroring the reference's pybind11 bindings.

``curegot.torch.sinkhorn_bcd / sinkhorn_splr / sinkhorn_splr_bwd`` follow
src/solvers_torch.cpp (tensor in, tensor out, converted to FP64 CUDA and back
to the input's options); ``curegot.numpy.*`` follow src/solvers_numpy.cpp
(host arrays in and out).  Signatures, defaults, kwargs and error messages
match the reference; one keyword is added: ``precision="fp64"`` (default,
the reference's arithmetic) or ``"mixed"`` (FP32 cost matrix, FP64 duals).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native

_PRECISIONS = ("fp64", "mixed")


def _stream_of(dev: torch.device) -> int:
    return torch.cuda.current_stream(dev).cuda_stream


def _target_device(t: torch.Tensor) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("curegot_backward_b200: a CUDA device is required (no CPU fallback)")
    if t.is_cuda:
        return t.device
    return torch.device("cuda", torch.cuda.current_device())


def _check_shapes(M, a, b, kind="tensor"):
    if M.dim() != 2:
        raise RuntimeError(f"M must be a 2D {kind}")
    if a.dim() != 1 or b.dim() != 1:
        raise RuntimeError(f"a and b must be 1D {kind}s")
    n, m = int(M.shape[0]), int(M.shape[1])
    if a.shape[0] != n or b.shape[0] != m:
        raise RuntimeError("Shape mismatch: M is [n x m], a should be length n, "
                           "b should be length m")
    return n, m


def _precision(kwargs) -> str:
    p = kwargs.get("precision", "fp64")
    if p not in _PRECISIONS:
        raise ValueError(f"precision must be one of {_PRECISIONS}, got {p!r}")
    return p


def _x0(kwargs, n, m, dev, kind="tensor"):
    if "x0" not in kwargs or kwargs["x0"] is None:
        return None
    x0 = kwargs["x0"]
    if not isinstance(x0, torch.Tensor):
        x0 = torch.as_tensor(np.asarray(x0, dtype=np.float64))
    if x0.dim() != 1 or x0.shape[0] != n + m:
        raise RuntimeError(f"x0 must be a 1D {kind} of length n + m")
    return x0.to(device=dev, dtype=torch.float64).contiguous()


def _verbose_report(name, n, m, reg, tol, max_iter, niter):
    print(f"{name} (CUDA implementation) completed")
    print(f"Input shape: [{n} x {m}]")
    print(f"Regularization parameter: {reg}")
    print(f"Tolerance: {tol}")
    print(f"Max iterations: {max_iter}")
    print(f"Actual iterations: {niter}")
    if niter == max_iter:
        print("Warning: Maximum iterations reached without convergence")


def _bcd_device(M, a, b, reg, tol, max_iter, x0, precision, want_plan=True):
    """Core device call: M/a/b already on one CUDA device, contiguous."""
    dev = M.device
    n, m = int(M.shape[0]), int(M.shape[1])
    opts = dict(device=dev, dtype=torch.float64)
    P = torch.empty((n, m), **opts) if want_plan else None
    dual = torch.empty(n + m, **opts)
    niter = ctypes.c_int(0)
    fn = "cg_bcd_mixed" if precision == "mixed" else "cg_bcd_f64"
    with torch.cuda.device(dev):
        _native.call(fn, M.data_ptr(), a.data_ptr(), b.data_ptr(),
                     P.data_ptr() if P is not None else None, float(reg), int(max_iter),
                     float(tol), n, m, ctypes.byref(niter),
                     x0.data_ptr() if x0 is not None else None, dual.data_ptr(),
                     _stream_of(dev))
    return int(niter.value), P, dual


def torch_sinkhorn_bcd(M, a, b, reg, tol=1e-6, max_iter=1000, verbose=0, **kwargs):
    """Sinkhorn BCD (reference src/solvers_torch.cpp:20-135)."""
    n, m = _check_shapes(M, a, b)
    src_dtype, src_device = M.dtype, M.device
    dev = _target_device(M)
    precision = _precision(kwargs)
    mdt = torch.float32 if precision == "mixed" else torch.float64
    Md = M.detach().to(device=dev, dtype=mdt).contiguous()
    ad = a.detach().to(device=dev, dtype=torch.float64).contiguous()
    bd = b.detach().to(device=dev, dtype=torch.float64).contiguous()
    x0 = _x0(kwargs, n, m, dev)
    niter, P, dual = _bcd_device(Md, ad, bd, reg, tol, max_iter, x0, precision)
    if verbose > 0:
        _verbose_report("torch_sinkhorn_bcd", n, m, reg, tol, max_iter, niter)
    return {"niter": niter, "plan": P.to(device=src_device, dtype=src_dtype),
            "dual": dual.to(device=src_device, dtype=src_dtype)}


def numpy_sinkhorn_bcd(M, a, b, reg, tol=1e-6, max_iter=1000, verbose=0, **kwargs):
    """Sinkhorn BCD with host arrays (reference src/solvers_numpy.cpp:13-110)."""
    M = np.asarray(M, dtype=np.float64)
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n, m = _check_shapes(torch.from_numpy(M), torch.from_numpy(a), torch.from_numpy(b),
                         kind="array")
    if "x0" in kwargs and kwargs["x0"] is not None:
        x0 = np.asarray(kwargs["x0"], dtype=np.float64)
        if x0.ndim != 1 or x0.shape[0] != n + m:
            raise RuntimeError("x0 must be a 1D array of length n + m")
    precision = _precision(kwargs)
    dev = _target_device(torch.empty(0))
    mdt = torch.float32 if precision == "mixed" else torch.float64
    Md = torch.from_numpy(np.ascontiguousarray(M)).to(device=dev, dtype=mdt)
    ad = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    bd = torch.from_numpy(np.ascontiguousarray(b)).to(dev)
    x0 = _x0(kwargs, n, m, dev, kind="array")
    niter, P, dual = _bcd_device(Md, ad, bd, reg, tol, max_iter, x0, precision)
    if verbose > 0:
        _verbose_report("sinkhorn_bcd", n, m, reg, tol, max_iter, niter)
    return {"niter": niter, "plan": P.cpu().numpy(), "dual": dual.cpu().numpy()}
