"""The allocation-free FP64 BCD entry point (cg_bcd_f64_noalloc), called
through the C ABI and compared with the allocating entry point cg_bcd_f64.

Tolerance: the two entry points run the same kernels with the same launch
geometry, so results must agree to the BCD parity bar used everywhere else
(identical niter, duals within 1e-10 relative, plan within 1e-12 absolute).
The file name sorts last so the test also runs after every other GPU test.
"""
import ctypes

import numpy as np
import pytest
import torch

from curegot_backward_b200 import _native

pytestmark = pytest.mark.gpu

DUAL_RTOL = 1e-10
PLAN_ATOL = 1e-12
CU_MEMPOOL_ATTR_USED_MEM_HIGH = 8


def _problem(n, m, seed):
    rng = np.random.default_rng(seed)
    X, Y = rng.uniform(size=(n, 6)), rng.uniform(size=(m, 6))
    M = ((X[:, None, :] - Y[None, :, :]) ** 2).mean(-1)
    a = rng.uniform(0.5, 1.5, size=n); a /= a.sum()
    b = rng.uniform(0.5, 1.5, size=m); b /= b.sum()
    return M, a, b


def _solve(fn, M, a, b, reg, tol, max_iter, dev):
    n, m = M.shape
    Md = torch.tensor(M, device=dev)
    ad, bd = torch.tensor(a, device=dev), torch.tensor(b, device=dev)
    P = torch.empty((n, m), dtype=torch.float64, device=dev)
    dual = torch.empty(n + m, dtype=torch.float64, device=dev)
    niter = ctypes.c_int(-1)
    stream = torch.cuda.current_stream(dev).cuda_stream
    status = getattr(_native.lib(), fn)(
        Md.data_ptr(), ad.data_ptr(), bd.data_ptr(), P.data_ptr(), reg, max_iter, tol, n, m,
        ctypes.byref(niter), None, dual.data_ptr(), stream)
    _native.check(fn, status)
    torch.cuda.synchronize(dev)
    return {"niter": niter.value, "plan": P.cpu().numpy(), "dual": dual.cpu().numpy()}


def _assert_same(got, ref):
    assert got["niter"] == ref["niter"], (got["niter"], ref["niter"])
    scale = max(np.abs(ref["dual"]).max(), 1e-300)
    assert np.abs(got["dual"] - ref["dual"]).max() <= DUAL_RTOL * scale
    assert np.abs(got["plan"] - ref["plan"]).max() <= PLAN_ATOL


def test_two_calls_in_a_row_match_allocating_entry(cuda_dev):
    cases = [(_problem(512, 640, 11), 0.05, 1e-8), (_problem(300, 2000, 12), 0.02, 1e-9)]
    got = [_solve("cg_bcd_f64_noalloc", *p, reg, tol, 3000, cuda_dev) for p, reg, tol in cases]
    for (p, reg, tol), g in zip(cases, got):
        ref = _solve("cg_bcd_f64", *p, reg, tol, 3000, cuda_dev)
        _assert_same(g, ref)
        assert np.linalg.norm(g["plan"].sum(1) - p[1]) < tol


def test_small_problem_matches_pass_path(cuda_dev):
    """64 x 80: cg_bcd_f64 would take the cluster path; with it disabled the
    two entry points run the same passes.  The marginal error is also checked
    against the oracle's evaluation of the returned duals."""
    import curegot_backward_b200 as cg
    import oracle
    M, a, b = _problem(64, 80, 14)
    got = _solve("cg_bcd_f64_noalloc", M, a, b, 0.05, 1e-8, 3000, cuda_dev)
    cg.set_bcd_cluster_path(False)
    try:
        ref = _solve("cg_bcd_f64", M, a, b, 0.05, 1e-8, 3000, cuda_dev)
    finally:
        cg.set_bcd_cluster_path(True)
    _assert_same(got, ref)
    o = oracle.bcd(M, a, b, 0.05, tol=1e-8, max_iter=3000)
    assert got["niter"] == o["niter"]
    P = np.exp((got["dual"][:64, None] + got["dual"][None, 64:] - M) / 0.05)
    assert np.linalg.norm(P.sum(1) - a) < 1e-8


@pytest.mark.parametrize("n,m", [(16384, 64), (64, 16384), (16384, 16384)])
def test_largest_accepted_shapes_fit_the_scratch(cuda_dev, n, m):
    """The scratch carve depends on the SM count through the column-pass
    splits and the row-pass CTAs; the extreme shapes inside the documented
    n, m <= 16384 limit must be accepted and agree with cg_bcd_f64.  Inputs
    stay on the device, no plan is written, and a few iterations at tol 0
    keep the 2 GB case short."""
    L = _native.lib()
    g = torch.Generator(device=cuda_dev).manual_seed(n + 7 * m)
    M = torch.rand((n, m), dtype=torch.float64, device=cuda_dev, generator=g)
    a = torch.full((n,), 1.0 / n, dtype=torch.float64, device=cuda_dev)
    b = torch.full((m,), 1.0 / m, dtype=torch.float64, device=cuda_dev)
    stream = torch.cuda.current_stream(cuda_dev).cuda_stream
    out = {}
    for fn in ("cg_bcd_f64_noalloc", "cg_bcd_f64"):
        dual = torch.empty(n + m, dtype=torch.float64, device=cuda_dev)
        niter = ctypes.c_int(-1)
        status = getattr(L, fn)(M.data_ptr(), a.data_ptr(), b.data_ptr(), None, 0.1, 3, 0.0,
                                n, m, ctypes.byref(niter), None, dual.data_ptr(), stream)
        _native.check(fn, status)
        torch.cuda.synchronize(cuda_dev)
        out[fn] = (niter.value, dual.cpu().numpy())
    (n0, d0), (n1, d1) = out["cg_bcd_f64_noalloc"], out["cg_bcd_f64"]
    assert n0 == n1 == 3
    assert np.abs(d0 - d1).max() <= DUAL_RTOL * max(np.abs(d1).max(), 1e-300)
    del M
    torch.cuda.empty_cache()


class _PoolProbe:
    """High-water mark of a stream-ordered memory pool (driver API)."""

    def __init__(self, pool):
        self.cu = ctypes.CDLL("libcuda.so.1")
        self.pool = pool

    @classmethod
    def default_pool(cls, ordinal):
        cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int()
        assert cu.cuDeviceGet(ctypes.byref(dev), ordinal) == 0
        pool = ctypes.c_void_p()
        assert cu.cuDeviceGetDefaultMemPool(ctypes.byref(pool), dev) == 0
        return cls(pool)

    @classmethod
    def library_pool(cls, ordinal):
        pool = ctypes.c_void_p()
        _native.call("cg_memory_pool", ordinal, ctypes.byref(pool))
        return cls(pool)

    def reset(self):
        zero = ctypes.c_uint64(0)
        assert self.cu.cuMemPoolSetAttribute(self.pool, CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                             ctypes.byref(zero)) == 0

    def high(self):
        v = ctypes.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                             ctypes.byref(v)) == 0
        return v.value


def test_no_pool_allocation(cuda_dev):
    M, a, b = _problem(700, 900, 13)
    ordinal = cuda_dev.index or 0
    probes = [_PoolProbe.library_pool(ordinal), _PoolProbe.default_pool(ordinal)]

    def highs_after(fn):
        torch.cuda.synchronize(cuda_dev)
        for p in probes:
            p.reset()
        base = [p.high() for p in probes]
        _solve(fn, M, a, b, 0.05, 1e-8, 2000, cuda_dev)
        return base, [p.high() for p in probes]

    # the probe sees the allocating entry point's workspace (library pool) ...
    base, after = highs_after("cg_bcd_f64")
    assert after[0] > base[0]
    # ... and nothing from the allocation-free one, in either pool
    base, after = highs_after("cg_bcd_f64_noalloc")
    assert after == base


def test_rejects_sizes_above_the_scratch_limit(cuda_dev):
    L = _native.lib()
    n, m = 16385, 4
    M = torch.zeros((n, m), dtype=torch.float64, device=cuda_dev)
    a = torch.full((n,), 1.0 / n, dtype=torch.float64, device=cuda_dev)
    b = torch.full((m,), 1.0 / m, dtype=torch.float64, device=cuda_dev)
    niter = ctypes.c_int(-1)
    launches = L.cg_launch_count()
    status = L.cg_bcd_f64_noalloc(M.data_ptr(), a.data_ptr(), b.data_ptr(), None, 0.05, 100,
                                  1e-8, n, m, ctypes.byref(niter), None, None,
                                  torch.cuda.current_stream(cuda_dev).cuda_stream)
    assert status == _native.CG_ERR_INVALID_ARG
    assert b"16384" in L.cg_last_error()
    assert L.cg_launch_count() == launches
    assert niter.value == -1
