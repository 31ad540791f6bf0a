"""Precision form: FP32 cost matrix, FP64 duals, FP64-confirmed stopping.

The problem follows the precision-form configuration (X, Y ~ N(0, I_32),
M = |x - y|^2 / median stored in FP32, Dirichlet(1) marginals floored at
1e-7 and renormalised, eta = 1e-3) at n = m = 2048; the full 16384 x 16384
case runs through ``profile_cases precision``.  The marginal errors of the
mixed-precision duals are evaluated by the FP64 oracle on the same
FP32-valued M (upcast exactly)."""
import numpy as np
import pytest
import torch

import oracle
from curegot_backward_b200 import _solvers, synthetic
from profile_cases import fp64_marginal_errors

pytestmark = pytest.mark.gpu

N = 2048


@pytest.fixture(scope="module")
def problem():
    M, a, b, eta = synthetic.config2(device="cuda", n=N, m=N)
    return M, a, b, eta


def _oracle_errors(M, a, b, dual, eta):
    n = M.shape[0]
    d = dual.double().cpu().numpy()
    al, be = d[:n], d[n:]
    gamma = np.concatenate([al + be[-1], be[:-1] - be[-1]])
    an, bn = a.cpu().numpy(), b.cpu().numpy()
    ck = oracle.t_objfn_grad(gamma, M.double().cpu().numpy(), an, bn, eta)
    return (float(np.linalg.norm(ck["Trowsums"] - an)), float(np.linalg.norm(ck["Tcolsums"] - bn)),
            float(ck["gnorm"]))


def test_marginals_are_exact_cast(problem):
    M, a, b, eta = problem
    assert M.dtype == torch.float32 and a.dtype == torch.float64
    assert float(a.min()) >= 1e-7 * 0.999 and abs(float(a.sum()) - 1.0) < 1e-12
    assert abs(float(b.sum()) - 1.0) < 1e-12


def test_bcd_mixed_fp64_errors(problem):
    M, a, b, eta = problem
    niter, _, dual = _solvers._bcd_device(M, a, b, eta, 1e-8, 100000, None, "mixed",
                                          want_plan=False)
    assert niter < 100000
    row, col, _ = _oracle_errors(M, a, b, dual, eta)
    # the stopping rule: FP64 row-marginal error of the returned iterate
    assert row <= 1e-8, (niter, row, col)
    assert col <= 1e-12, (niter, row, col)
    # the torch FP64 evaluation used by the profiling case agrees with the oracle
    r2, c2 = fp64_marginal_errors(M, a, b, dual, eta)
    assert abs(r2 - row) <= 1e-12 and abs(c2 - col) <= 1e-12


def test_splr_mixed_fp64_errors(problem):
    M, a, b, eta = problem
    out = _solvers._splr_device(M, a, b, eta, 1e-8, 1000, 0, None, "mixed", 0.01, 1e-3, 30, 3,
                                want_plan=False)
    assert out["niter"] < 1000
    row, col, gnorm = _oracle_errors(M, a, b, out["dual"], eta)
    # mixed SPLR stops on the full marginal error: rows and all m columns
    # (the reference's test covers the first n + m - 1 dual entries only)
    assert gnorm <= 1e-8
    assert (row ** 2 + col ** 2) ** 0.5 <= 1e-8
