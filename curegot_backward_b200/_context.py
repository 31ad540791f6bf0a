"""SPLRBackwardContext: Python handle of the native backward context.

Mirrors the pybind class of the reference (src/solvers_torch.cpp:296-705):
same method / property names, argument checks and error messages.  The
debug/benchmark profiling methods of the reference are not provided.
"""

from __future__ import annotations

import ctypes

import torch

from . import _native


class SPLRBackwardContext:
    """Opaque backward context of the SPLR solver.

    Owns the factorization of the last forward iteration's sparsified Hessian
    and the rank-2 BFGS materials, and applies B^{-1} (or the diagonal D_A^{-1})
    as a preconditioner for the backward PCG.
    """

    def __init__(self, handle: int, device: torch.device, expose_point: bool):
        self._h = ctypes.c_void_p(handle)
        self._device = device
        self._expose_point = expose_point
        self._info = None

    # -- lifetime -------------------------------------------------------------
    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _native.lib().cg_ctx_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def _handle(self):
        if self._h is None or not self._h.value:
            raise RuntimeError("SPLRBackwardContext: invalid context")
        return self._h

    def _query(self) -> _native.CtxInfo:
        info = _native.CtxInfo()
        _native.call("cg_ctx_info", self._handle, ctypes.byref(info))
        return info

    def _stream(self):
        return torch.cuda.current_stream(self._device).cuda_stream

    def _check_r(self, r):
        info = self._query()
        if not info.valid:
            raise RuntimeError("SPLRBackwardContext: invalid context")
        if not isinstance(r, torch.Tensor) or r.dim() != 1 or r.shape[0] != info.dim:
            raise RuntimeError(
                "SPLRBackwardContext: r must be a 1D tensor of length n + m - 1")
        if not r.is_cuda:
            raise RuntimeError("SPLRBackwardContext: r must be a CUDA tensor")
        return r.to(dtype=torch.float64).contiguous(), info

    # -- preconditioners ------------------------------------------------------
    def apply_preconditioner(self, r):
        """Compute z = B^{-1} r (factor solve + rank-2 Woodbury correction)."""
        r, info = self._check_r(r)
        z = torch.empty(info.dim, dtype=torch.float64, device=r.device)
        with torch.cuda.device(r.device):
            _native.call("cg_ctx_apply", self._handle, r.data_ptr(), z.data_ptr(),
                         _native.CG_PRECOND_SPLR, self._stream())
        return z

    def apply_diagonal_preconditioner(self, r):
        """Compute z = D_A^{-1} r with D_A = diag(A) of the context CSR."""
        if not self.has_diagonal_preconditioner:
            raise RuntimeError("SPLRBackwardContext: diagonal preconditioner not set up")
        r, info = self._check_r(r)
        z = torch.empty(info.dim, dtype=torch.float64, device=r.device)
        with torch.cuda.device(r.device):
            _native.call("cg_ctx_apply", self._handle, r.data_ptr(), z.data_ptr(),
                         _native.CG_PRECOND_DIAG, self._stream())
        return z

    def setup_diagonal_preconditioner(self):
        with torch.cuda.device(self._device):
            _native.call("cg_ctx_setup_diag", self._handle, self._stream())

    @property
    def has_diagonal_preconditioner(self) -> bool:
        return bool(self._query().has_diag)

    # -- properties -----------------------------------------------------------
    @property
    def reg(self) -> float:
        return float(self._query().reg)

    @property
    def dim(self) -> int:
        return int(self._query().dim)

    @property
    def low_rank_enabled(self) -> bool:
        return bool(self._query().low_rank)

    @property
    def is_fallback(self) -> bool:
        return bool(self._query().fallback)

    @property
    def adopted_forward_state(self) -> bool:
        return bool(self._query().adopted)

    @property
    def ys(self) -> float:
        return float(self._query().ys)

    @property
    def is_valid(self) -> bool:
        return bool(self._query().valid)

    # -- array copies ---------------------------------------------------------
    def _copy(self, what: int, length: int, dtype):
        out = torch.empty(length, dtype=dtype, device=self._device)
        with torch.cuda.device(self._device):
            _native.call("cg_ctx_copy", self._handle, what, out.data_ptr(), self._stream())
        return out

    def inv_diag(self):
        if not self.has_diagonal_preconditioner:
            raise RuntimeError("SPLRBackwardContext: diagonal preconditioner not set up")
        return self._copy(_native.CG_CTX_INV_DIAG, self.dim, torch.float64)

    def csr_values(self):
        return self._copy(_native.CG_CTX_CSR_VALUES, int(self._query().nnz), torch.float64)

    def csr_colind(self):
        return self._copy(_native.CG_CTX_CSR_COLIND, int(self._query().nnz), torch.int32)

    def csr_rowptr(self):
        return self._copy(_native.CG_CTX_CSR_ROWPTR, self.dim + 1, torch.int32)

    def secant_s(self):
        if not self.low_rank_enabled:
            raise RuntimeError(
                "SPLRBackwardContext: low-rank correction is disabled, s is unavailable")
        return self._copy(_native.CG_CTX_SECANT_S, self.dim, torch.float64)

    def secant_y(self):
        if not self.low_rank_enabled:
            raise RuntimeError(
                "SPLRBackwardContext: low-rank correction is disabled, y is unavailable")
        return self._copy(_native.CG_CTX_SECANT_Y, self.dim, torch.float64)

    def ctx_point(self):
        if not self._expose_point:
            raise RuntimeError("SPLRBackwardContext: context point unavailable "
                               "(call with return_validation=True)")
        return self._copy(_native.CG_CTX_POINT, self.dim, torch.float64)

    def __repr__(self):
        try:
            i = self._query()
            return (f"SPLRBackwardContext(dim={i.dim}, nnz={i.nnz}, reg={i.reg}, "
                    f"low_rank={bool(i.low_rank)}, fallback={bool(i.fallback)})")
        except Exception:
            return "SPLRBackwardContext(<released>)"
