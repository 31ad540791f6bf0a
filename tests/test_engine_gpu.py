"""Serving engine: every result is the same alone and in the mix, meets the
FP64-checked 1e-8 marginal error, and admission respects the HBM budget."""
import numpy as np
import pytest
import torch

import curegot_backward_b200 as cg
from curegot_backward_b200.serving import OTEngine
from curegot_backward_b200.synthetic import StreamSpec, stream_problem

pytestmark = pytest.mark.gpu


def specs():
    rng = np.random.default_rng(0)
    out = []
    for k in range(14):
        n = int(np.exp(rng.uniform(np.log(48), np.log(700))))
        m = int(np.exp(rng.uniform(np.log(48), np.log(700))))
        algo = "splr" if k % 4 == 3 else "bcd"
        out.append(StreamSpec(k, n, m, int(rng.choice([8, 32])),
                              float(rng.choice([0.1, 0.05, 0.01])), algo, 1000 + k, 0.0))
    return out


def alone(s, M, a, b):
    """The same request through an engine that serves nothing else."""
    eng = OTEngine(budget_bytes=8e9, max_batch=6, splr_workers=2, chunk=4)
    try:
        eng.submit(M, a, b, eta=s.eta, algo=s.algo, tol=1e-8, tag=0)
        while True:
            res = eng.poll(wait_ms=100)
            if res:
                assert res[0]["status"] == 0
                return res[0]["dual"].to(M.device)
    finally:
        eng.close()


@pytest.mark.parametrize("host", [False, True])
def test_same_alone_and_in_the_mix(cuda_dev, host):
    ss = specs()
    probs = [(s,) + stream_problem(s, device=cuda_dev) for s in ss]
    eng = OTEngine(budget_bytes=8e9, max_batch=6, splr_workers=2, chunk=4)
    try:
        for k, (s, M, a, b) in enumerate(probs):
            if host:
                eng.submit(M.cpu().pin_memory(), a.cpu().pin_memory(), b.cpu().pin_memory(),
                           eta=s.eta, algo=s.algo, tol=1e-8, tag=k)
            else:
                eng.submit(M, a, b, eta=s.eta, algo=s.algo, tol=1e-8, tag=k)
        got = {}
        while len(got) < len(probs):
            for r in eng.poll(wait_ms=100):
                assert r["status"] == 0
                got[r["tag"]] = r
        st = eng.stats()
        assert st["in_use_bytes"] == 0 and st["completed"] == len(probs)
    finally:
        eng.close()
    for k, (s, M, a, b) in enumerate(probs):
        dual = got[k]["dual"].to(cuda_dev)
        ref = alone(s, M, a, b)
        assert torch.equal(dual, ref), (k, s)
        al, be = dual[: s.n], dual[s.n:]
        P = torch.exp((al[:, None] + be[None, :] - M.double()) / s.eta)
        # rows and all m columns, for both algorithms (SPLR in the engine
        # stops on the full marginal error, gauge column included)
        assert float(torch.linalg.norm(P.sum(1) - a)) <= 1e-8, (k, s)
        assert float(torch.linalg.norm(P.sum(0) - b)) <= 1e-8, (k, s)


def test_admission_rejects_oversized(cuda_dev):
    s = StreamSpec(0, 2048, 2048, 8, 0.1, "bcd", 5, 0.0)
    M, a, b = stream_problem(s, device=cuda_dev)
    eng = OTEngine(budget_bytes=1e4, max_batch=4, splr_workers=1, chunk=4)
    try:
        eng.submit(M, a, b, eta=s.eta, algo="bcd")
        res = []
        while not res:
            res = eng.poll(wait_ms=100)
        assert res[0]["status"] == cg._native.CG_ERR_ADMISSION
    finally:
        eng.close()


def test_engine_splr_gauge_correction(cuda_dev):
    """The engine's SPLR stops at the first iterate where the full marginal
    error (gauge column included) is below tol, either directly or after the
    gauge column is made exact: never later than the plain full-marginal
    stop of cg_splr_mixed, and every result meets 1e-8 on rows and on all
    columns."""
    from curegot_backward_b200 import _solvers
    rng = np.random.default_rng(4)
    ss = [StreamSpec(k, int(rng.integers(150, 900)), int(rng.integers(150, 900)), 8,
                     float(rng.choice([0.1, 0.05, 0.01])), "splr", 500 + k, 0.0) for k in range(6)]
    probs = [(s,) + stream_problem(s, device=cuda_dev) for s in ss]
    eng = OTEngine(budget_bytes=8e9, max_batch=4, splr_workers=3, chunk=4)
    try:
        for k, (s, M, a, b) in enumerate(probs):
            eng.submit(M, a, b, eta=s.eta, algo="splr", tol=1e-8, tag=k)
        got = {}
        while len(got) < len(probs):
            for r in eng.poll(wait_ms=100):
                assert r["status"] == 0 and r["converged"]
                got[r["tag"]] = r
    finally:
        eng.close()
    saved = 0
    for k, (s, M, a, b) in enumerate(probs):
        plain = _solvers._splr_device(M, a, b, s.eta, 1e-8, 1000, 0, None, "mixed",
                                      min(10.0 / min(s.n, s.m), 1.0), 1e-3, 30, 3,
                                      want_plan=False)
        assert got[k]["niter"] <= plain["niter"], (k, s)
        saved += plain["niter"] - got[k]["niter"]
        dual = got[k]["dual"].to(cuda_dev)
        assert float(dual[-1]) == 0.0  # the reference's gauge
        al, be = dual[: s.n], dual[s.n:]
        P = torch.exp((al[:, None] + be[None, :] - M.double()) / s.eta)
        err = torch.sqrt(torch.linalg.norm(P.sum(1) - a) ** 2 + torch.linalg.norm(P.sum(0) - b) ** 2)
        assert float(err) <= 1e-8, (k, s)
    print("iterations saved by the gauge correction:", saved)
