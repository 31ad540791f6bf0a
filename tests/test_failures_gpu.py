"""Failure handling, exercised without faulting the GPU.

Every failure here is made on the host or by an input value:
  * non-finite inputs (NaN in M, a or b) reach the solvers' stopping tests;
    Sinkhorn returns CG_ERR_NONFINITE, SPLR takes the reference's break on a
    non-finite objective (src/sinkhorn_splr.cu:1128: converged = false), and
    the serving engine reports CG_ERR_NONFINITE for that request only;
  * a direction-solve failure is injected on the host (cg_test_inject_failure):
    the status the solver reads back is replaced, nothing on the device is
    touched, and the call returns CG_ERR_NOT_SPD;
  * the tensor-core completion wait of the points solver is given a zero poll
    limit, so every first wait gives up at once; the kernel drains the MMAs,
    frees its tensor memory and the call returns CG_ERR_TIMEOUT; the next call
    with the default limit gives the normal result;
  * engine requests are cancelled while queued and while admitted.
"""
import ctypes
import time

import numpy as np
import pytest
import torch

import curegot_backward_b200 as cg
from curegot_backward_b200 import _native, _solvers, points
from curegot_backward_b200.serving import OTEngine
from curegot_backward_b200.synthetic import StreamSpec, stream_problem

pytestmark = pytest.mark.gpu


def _problem(n, m, seed=0):
    rng = np.random.default_rng(seed)
    X, Y = rng.uniform(size=(n, 8)), rng.uniform(size=(m, 8))
    M = ((X[:, None, :] - Y[None, :, :]) ** 2).mean(-1)
    return M, np.full(n, 1.0 / n), np.full(m, 1.0 / m)


@pytest.mark.parametrize("n,m", [(48, 40), (700, 900)])  # cluster path, pass path
@pytest.mark.parametrize("where", ["M", "a"])
def test_bcd_nonfinite_input(cuda_dev, n, m, where):
    M, a, b = _problem(n, m)
    if where == "M":
        M[n // 2, m // 3] = np.nan
    else:
        a[3] = np.nan
    with pytest.raises(_native.CuregotError) as e:
        cg.numpy.sinkhorn_bcd(M, a, b, 0.05, tol=1e-8, max_iter=2000)
    assert e.value.status == _native.CG_ERR_NONFINITE
    # the library stays usable: the clean problem solves normally
    M2, a2, b2 = _problem(n, m)
    out = cg.numpy.sinkhorn_bcd(M2, a2, b2, 0.05, tol=1e-8, max_iter=2000)
    assert out["niter"] < 2000


def test_bcd_mixed_nonfinite_input(cuda_dev):
    M, a, b = _problem(600, 500)
    Md = torch.tensor(M, device=cuda_dev, dtype=torch.float32)
    Md[10, 10] = float("nan")
    ad, bd = torch.tensor(a, device=cuda_dev), torch.tensor(b, device=cuda_dev)
    with pytest.raises(_native.CuregotError) as e:
        _solvers._bcd_device(Md, ad, bd, 0.05, 1e-8, 5000, None, "mixed", want_plan=False)
    assert e.value.status == _native.CG_ERR_NONFINITE


def test_splr_nonfinite_takes_the_reference_break(cuda_dev):
    M, a, b = _problem(120, 90)
    M[5, 7] = np.nan
    Md = torch.tensor(M, device=cuda_dev)
    ad, bd = torch.tensor(a, device=cuda_dev), torch.tensor(b, device=cuda_dev)
    out = _solvers._splr_device(Md, ad, bd, 0.05, 1e-8, 300, 0, None, "fp64",
                                min(10.0 / 90, 1.0), 1e-3, 30, 3, want_plan=False)
    assert out["niter"] == 0 and not out["converged"]
    # the autograd API treats it as non-convergence, as the reference does
    with pytest.raises(RuntimeError):
        cg.torch.splr_ot(Md, ad, bd, eta=0.05, tol=1e-8, max_iter=300)


def test_injected_direction_solve_failure(cuda_dev):
    M, a, b = _problem(150, 130, seed=2)
    _native.call("cg_test_inject_failure", _native.CG_INJECT_DIRECTION_SOLVE, 1)
    try:
        with pytest.raises(_native.CuregotError) as e:
            cg.numpy.sinkhorn_splr(M, a, b, 0.05, tol=1e-8, max_iter=300)
        assert e.value.status == _native.CG_ERR_NOT_SPD
    finally:
        _native.call("cg_test_inject_failure", _native.CG_INJECT_DIRECTION_SOLVE, 0)
    out = cg.numpy.sinkhorn_splr(M, a, b, 0.05, tol=1e-8, max_iter=300)
    assert out["niter"] < 300
    with pytest.raises(_native.CuregotError):
        _native.call("cg_test_inject_failure", 99, 1)


def test_points_wait_timeout_then_normal(cuda_dev):
    g = torch.Generator(device=cuda_dev).manual_seed(5)
    n, m, d = 300, 260, 32
    X = torch.rand(n, d, device=cuda_dev, generator=g).to(torch.bfloat16)
    Y = torch.rand(m, d, device=cuda_dev, generator=g).to(torch.bfloat16)
    a = torch.full((n,), 1.0 / n, dtype=torch.float64, device=cuda_dev)
    b = torch.full((m,), 1.0 / m, dtype=torch.float64, device=cuda_dev)
    ref = points.sinkhorn_bcd_points(X, Y, a, b, 0.05, tol=1e-8, max_iter=3000)
    _native.call("cg_points_set_wait_limit", 0)
    try:
        with pytest.raises(_native.CuregotError) as e:
            points.sinkhorn_bcd_points(X, Y, a, b, 0.05, tol=1e-8, max_iter=3000)
        assert e.value.status == _native.CG_ERR_TIMEOUT
        with pytest.raises(_native.CuregotError) as e:
            points.cost_from_points(X, Y)
        assert e.value.status == _native.CG_ERR_TIMEOUT
    finally:
        _native.call("cg_points_set_wait_limit", -1)
    again = points.sinkhorn_bcd_points(X, Y, a, b, 0.05, tol=1e-8, max_iter=3000)
    assert again["niter"] == ref["niter"]
    assert torch.equal(again["dual"], ref["dual"])


def _drain(eng, count, timeout_s=120.0):
    got = {}
    t0 = time.time()
    while len(got) < count:
        assert time.time() - t0 < timeout_s, "engine results did not arrive"
        for r in eng.poll(wait_ms=100):
            got[r["tag"]] = r
    return got


def test_engine_nonfinite_request_is_isolated(cuda_dev):
    specs = [StreamSpec(k, 200 + 37 * k, 180 + 29 * k, 8, 0.05, "splr" if k % 3 == 2 else "bcd",
                        77 + k, 0.0) for k in range(6)]
    probs = [stream_problem(s, device=cuda_dev) for s in specs]
    bad = {1, 2}  # one Sinkhorn, one SPLR request
    eng = OTEngine(budget_bytes=8e9, max_batch=8, splr_workers=2, chunk=4)
    try:
        for k, (s, (M, a, b)) in enumerate(zip(specs, probs)):
            if k in bad:
                M = M.clone()
                M[3, 4] = float("nan")
            eng.submit(M, a, b, eta=s.eta, algo=s.algo, tol=1e-8, tag=k)
        got = _drain(eng, len(specs))
        assert eng.stats()["in_use_bytes"] == 0
    finally:
        eng.close()
    for k in range(len(specs)):
        if k in bad:
            assert got[k]["status"] == _native.CG_ERR_NONFINITE, (k, got[k])
        else:
            assert got[k]["status"] == 0, (k, got[k])
            assert got[k]["converged"]


def test_engine_injected_direction_failure(cuda_dev):
    s = StreamSpec(0, 300, 250, 8, 0.05, "splr", 91, 0.0)
    M, a, b = stream_problem(s, device=cuda_dev)
    eng = OTEngine(budget_bytes=8e9, max_batch=4, splr_workers=1, chunk=4)
    _native.call("cg_test_inject_failure", _native.CG_INJECT_DIRECTION_SOLVE, 1)
    try:
        eng.submit(M, a, b, eta=s.eta, algo="splr", tol=1e-8, tag=0)
        got = _drain(eng, 1)
        assert got[0]["status"] == _native.CG_ERR_NOT_SPD
        eng.submit(M, a, b, eta=s.eta, algo="splr", tol=1e-8, tag=1)
        got = _drain(eng, 1)
        assert got[1]["status"] == 0 and got[1]["converged"]
    finally:
        _native.call("cg_test_inject_failure", _native.CG_INJECT_DIRECTION_SOLVE, 0)
        eng.close()


def test_engine_cancel_queued_and_admitted(cuda_dev):
    """One Sinkhorn slot and one SPLR worker: a long Sinkhorn request (tol 0)
    and a long SPLR request are admitted, a second Sinkhorn request waits in
    the queue.  Cancelling all three returns each with CG_ERR_CANCELLED; the
    engine then serves a normal request and holds no memory."""
    big = StreamSpec(0, 1024, 1024, 8, 0.01, "bcd", 3, 0.0)
    sp = StreamSpec(1, 1500, 1400, 8, 0.01, "splr", 4, 0.0)
    small = StreamSpec(2, 200, 210, 8, 0.05, "bcd", 5, 0.0)
    pb, ps, pm = (stream_problem(x, device=cuda_dev) for x in (big, sp, small))
    eng = OTEngine(budget_bytes=8e9, max_batch=1, splr_workers=1, chunk=4)
    try:
        r_big = eng.submit(*pb, eta=big.eta, algo="bcd", tol=0.0, max_iter=400000, tag=0)
        r_sp = eng.submit(*ps, eta=sp.eta, algo="splr", tol=1e-14, max_iter=5000, tag=1)
        r_q = eng.submit(*pm, eta=small.eta, algo="bcd", tol=1e-8, tag=2)
        t0 = time.time()
        while True:  # both long requests admitted
            st = eng.stats()
            if st["active_bcd"] >= 1 and st["active_splr"] >= 1:
                break
            assert time.time() - t0 < 30
            time.sleep(0.01)
        eng.cancel(r_q)  # still queued behind the one Sinkhorn slot
        eng.cancel(r_big)
        eng.cancel(r_sp)
        got = _drain(eng, 3, timeout_s=60.0)
        for k in range(3):
            assert got[k]["status"] == _native.CG_ERR_CANCELLED, (k, got[k])
        with pytest.raises(_native.CuregotError):
            eng.cancel(r_q)  # finished: unknown now
        eng.submit(*pm, eta=small.eta, algo="bcd", tol=1e-8, tag=3)
        got = _drain(eng, 1)
        assert got[3]["status"] == 0 and got[3]["converged"]
        assert eng.stats()["in_use_bytes"] == 0
    finally:
        eng.close()
