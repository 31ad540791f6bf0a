"""Continuous-batching OT serving engine (Python handle of cg_engine_*).

    eng = OTEngine(budget_bytes=120e9)
    rid = eng.submit(M, a, b, eta=0.05, algo="bcd", tol=1e-8)
    results = eng.poll(wait_ms=100)      # list of dicts: id, tag, niter, latency, ...

Requests take CUDA tensors (device-resident inputs, results written to a
device dual tensor) or CPU tensors / NumPy arrays (the engine copies them in
and the duals back out; pinned memory makes those copies asynchronous).  An
FP32 cost matrix selects the mixed-precision passes (FP32 M, FP64 duals,
FP64-confirmed stopping test); FP64 selects the plain FP64 passes.

Start serving processes with CUDA_MODULE_LOADING=EAGER: under lazy loading
the first launch of each kernel variant (pass templates, cuSOLVER size
classes) happens mid-stream and held every stream of the process for
0.3-1 s on a fresh machine.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native

_ALGOS = {"bcd": _native.CG_ALGO_BCD, "splr": _native.CG_ALGO_SPLR}


class OTEngine:
    def __init__(self, budget_bytes=120e9, max_batch=64, splr_workers=16, chunk=8, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("OTEngine: a CUDA device is required (no CPU fallback)")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None
                                   else torch.device(device).index)
        self._h = ctypes.c_void_p(0)
        with torch.cuda.device(self.device):
            _native.call("cg_engine_create", int(budget_bytes), int(max_batch),
                         int(splr_workers), int(chunk), ctypes.byref(self._h))
        self._keep = {}

    def submit(self, M, a, b, *, eta, algo="bcd", tol=1e-8, max_iter=100000, dual_out=None,
               tag=0):
        """Enqueue one OT solve; returns its id.  Buffers are kept alive until polled."""
        if algo not in _ALGOS:
            raise ValueError(f"algo must be one of {tuple(_ALGOS)}")
        if isinstance(M, np.ndarray):
            M = torch.from_numpy(np.ascontiguousarray(M))
        if isinstance(a, np.ndarray):
            a = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
        if isinstance(b, np.ndarray):
            b = torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64))
        if M.dim() != 2 or a.dim() != 1 or b.dim() != 1 or a.shape[0] != M.shape[0] \
                or b.shape[0] != M.shape[1]:
            raise ValueError("submit: M must be [n, m], a [n], b [m]")
        if M.dtype not in (torch.float32, torch.float64):
            raise ValueError("submit: M must be float32 (mixed) or float64 (plain)")
        host = not M.is_cuda
        if (a.is_cuda == host) or (b.is_cuda == host):
            raise ValueError("submit: M, a, b must all be on the host or all on the device")
        M = M.contiguous()
        a = a.to(torch.float64).contiguous()
        b = b.to(torch.float64).contiguous()
        n, m = int(M.shape[0]), int(M.shape[1])
        if dual_out is None:
            dual_out = torch.empty(n + m, dtype=torch.float64,
                                   device="cpu" if host else self.device,
                                   pin_memory=host)
        req = _native.Request(_ALGOS[algo], n, m, int(M.dtype == torch.float32), int(host),
                              int(max_iter), float(eta), float(tol), M.data_ptr(), a.data_ptr(),
                              b.data_ptr(), dual_out.data_ptr(), int(tag))
        rid = ctypes.c_uint64(0)
        _native.call("cg_engine_submit", self._h, ctypes.byref(req), ctypes.byref(rid))
        self._keep[rid.value] = (M, a, b, dual_out)
        return rid.value

    def poll(self, max_results=4096, wait_ms=0):
        """Finished results (dicts with duals, iteration counts and timings)."""
        buf = (_native.Result * max_results)()
        cnt = ctypes.c_int(0)
        _native.call("cg_engine_poll", self._h, buf, max_results, int(wait_ms),
                     ctypes.byref(cnt))
        out = []
        for r in buf[: cnt.value]:
            M, a, b, dual = self._keep.pop(r.id, (None, None, None, None))
            out.append({"id": r.id, "tag": r.tag, "status": r.status, "niter": r.niter,
                        "converged": bool(r.converged), "fast_iters": r.fast_iters,
                        "last_err": r.last_err, "t_submit": r.t_submit, "t_admit": r.t_admit,
                        "t_done": r.t_done, "dual": dual})
        return out

    def cancel(self, rid):
        """Cancel a submitted request; its result comes back from poll() with
        status CG_ERR_CANCELLED.  Raises if the id is unknown or finished."""
        _native.call("cg_engine_cancel", self._h, int(rid))

    def stats(self):
        s = _native.EngineStats()
        _native.call("cg_engine_stats", self._h, ctypes.byref(s))
        return {k: getattr(s, k) for k, _ in s._fields_}

    @staticmethod
    def clock():
        return _native.lib().cg_engine_clock()

    def close(self):
        if self._h is not None and self._h.value:
            _native.lib().cg_engine_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
