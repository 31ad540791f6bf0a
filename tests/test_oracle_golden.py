"""The CPU oracle against the reference tests' own expected values.

Fixtures in tests/golden/ are produced by tests/golden/make_golden.py with
the reference tests' NumPy/SciPy logic (test/test_csr.py,
test/test_sparse_cholesky.py).  Tolerances are the reference tests' (1e-8).
"""
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_csr_known_answer():
    g = np.load(os.path.join(GOLD, "csr_n6_m3.npz"))
    r = oracle.t_sparsify(g["alpha"], g["beta"], g["M"], g["a"], g["b"], float(g["reg"]),
                          float(g["shift"]), int(g["K"]))
    for k in ("Trowsums", "Tcolsums", "grad", "csr_val"):
        assert np.linalg.norm(r[k] - g[k]) < 1e-8, k
    assert np.array_equal(r["csr_colind"], g["csr_colind"])
    assert np.array_equal(r["csr_rowptr"], g["csr_rowptr"])
    assert abs(r["objfn"] - g["objfn"]) < 1e-8
    assert abs(r["gnorm"] - g["gnorm"]) < 1e-8
    assert r["K_actual"] == 10


@pytest.mark.parametrize("n", [10, 100, 1000])
def test_spd_solve_known_answer(n):
    s = np.load(os.path.join(GOLD, f"spd_n{n}.npz"))
    for kind in ("full", "lower"):
        x = oracle.csr_spd_solve(s[f"{kind}_val"], s[f"{kind}_col"], s[f"{kind}_rowptr"],
                                 s["rhs"])
        assert np.linalg.norm(x - s["x"]) < 1e-8


def _problem(n, m, seed, reg_scale=1.0):
    rng = np.random.default_rng(seed)
    M = rng.uniform(size=(n, m)) * reg_scale
    a = rng.uniform(size=n); a /= a.sum()
    b = rng.uniform(size=m); b /= b.sum()
    return M, a, b


def test_bcd_oracle_niter_truncation():
    # reference test/test_sinkhorn_bcd.py:172-177: niter == max_iter when truncated
    M, a, b = _problem(50, 40, 456)
    r = oracle.bcd(M, a, b, 0.01, tol=1e-12, max_iter=10)
    assert r["niter"] == 10


def test_bcd_oracle_marginals_and_warm_start():
    # reference test/test_sinkhorn_bcd.py:201 (marginal error <= 10 tol) and
    # :330-340 (warm start from the dual: no more iterations, plan diff <= 1e-8)
    M, a, b = _problem(50, 40, 789)
    tol = 1e-8
    r = oracle.bcd(M, a, b, 0.01, tol=tol, max_iter=5000)
    P = r["plan"]
    assert np.linalg.norm(P.sum(1) - a) <= 10 * tol
    assert np.linalg.norm(P.sum(0) - b) <= 10 * tol
    r2 = oracle.bcd(M, a, b, 0.01, tol=tol, max_iter=5000, x0=r["dual"])
    assert r2["niter"] <= r["niter"]
    assert np.abs(r2["plan"] - P).max() <= 1e-8


@pytest.mark.parametrize("n,m,reg", [(80, 60, 0.01), (60, 80, 0.001)])
def test_splr_oracle_matches_bcd(n, m, reg):
    # reference test/test_sinkhorn_splr.py:45-120: SPLR vs BCD plans < 1e-3
    rng = np.random.default_rng(123)
    M = rng.uniform(size=(n, m))
    a = rng.uniform(size=n); a /= a.sum()
    b = rng.uniform(size=m); b /= b.sum()
    s = oracle.splr(M, a, b, reg, tol=1e-6, max_iter=5000)
    c = oracle.bcd(M, a, b, reg, tol=1e-6, max_iter=200000)
    rel = np.linalg.norm(s["plan"] - c["plan"]) / np.linalg.norm(c["plan"])
    assert rel < 1e-3
    assert np.linalg.norm(s["plan"].sum(1) - a) < 1e-4
    assert np.linalg.norm(s["plan"].sum(0) - b) < 1e-4


def test_backward_oracle_dense_ladder():
    # reference stage3b_validate.py:409-461 (L2): PCG lambda vs dense Q solve
    rng = np.random.default_rng(42)
    n, m, eta = 30, 36, 0.05
    M = rng.uniform(size=(n, m))
    a = np.full(n, 1.0 / n); b = np.full(m, 1.0 / m)
    s = oracle.splr(M, a, b, eta, tol=1e-10, max_iter=500)
    T = s["plan"]
    G = rng.normal(size=(n, m))
    ctx = s["context"]
    inv = oracle.inv_diag_from_csr(ctx["csr_values"], ctx["csr_colind"], ctx["csr_rowptr"])
    res = oracle.solve_backward(T, G, inv, eta)
    assert res["converged"]
    H = n + m - 1
    Q = np.stack([oracle.q_matvec(T, e, n, m) for e in np.eye(H)], axis=1)
    mu = oracle.rhs_Q_scale(G, T, n, m)
    lam = np.linalg.solve(Q, mu)
    assert np.linalg.norm(res["lambda"] - lam) / np.linalg.norm(lam) < 1e-8
