"""Parity at the full sizes of the SPLR and differentiation configurations,
against committed fixtures (tests/golden/make_parity_fixtures.py).

C1 -- plain FP64 SPLR, n = m = 4096, ~1% Hessian density (density_max 0.1),
eta 0.01, tol 1e-8, against the CPU oracle: identical niter, identical trace
columns K / low-rank / recompute / candidate / line-search trials, identical
final CSR pattern, duals within 1e-10 relative, plan within 1e-12 absolute
(the plan is recomputed here from the oracle's duals).

C3 -- n = 2048, m = 2560, d = 32, eta 0.05, loss = sum(T^2), forward tol
1e-9 (at 1e-10 the reference's SPLR iteration does not converge on this
problem: the oracle stops at its 2000-iteration cap, the line search being
at the FP64 resolution of the objective; 1e-9 is reached in one step):
  * forward duals against the oracle (1e-10 relative);
  * lambda and dL/dM against the reference's own curegot/_backward_core.py +
    curegot/backward.py run on CPU torch (tolerance 1e-8 relative: the two
    PCG runs stop at the same 1e-12 relative residual with different
    summation orders);
  * the autograd gradient against central finite differences, h = 1e-6, on
    64 seeded entries of M: normalised error ||fd - g|| / ||g|| <= 1e-3, the
    reference validator's bar (validate_stage4_autograd.py:314-362).
"""
import os
import sys

import numpy as np
import pytest
import torch

import curegot_backward_b200 as cg

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_parity_fixtures as fx  # noqa: E402

pytestmark = pytest.mark.gpu


def _load(name):
    return np.load(os.path.join(HERE, "golden", name))


@pytest.fixture(scope="module")
def c1():
    M, a, b, eta = fx.c1_problem()
    g = _load("splr_c1_4096.npz")
    assert fx.sha(M) == str(g["M_sha"]), "regenerated C1 cost matrix differs from the fixture's"
    return M, a, b, eta, g


def test_c1_splr_4096_matches_oracle(cuda_dev, c1):
    M, a, b, eta, g = c1
    Mt = torch.tensor(M, device=cuda_dev)
    at, bt = torch.tensor(a, device=cuda_dev), torch.tensor(b, device=cuda_dev)
    out = cg.torch.sinkhorn_splr_bwd(Mt, at, bt, eta, 1e-8, 1000, 0, density=0.1,
                                     return_trace=True)
    assert out["niter"] == int(g["niter"])
    assert out["converged"] == bool(g["converged"])
    tr, rt = out["trace"], g["trace"]
    np.testing.assert_array_equal(tr[:, [3, 4, 5, 6, 7]], rt[:, [3, 4, 5, 6, 7]])
    assert np.allclose(tr[:, 0], rt[:, 0], rtol=1e-10, atol=0)
    dual = out["dual"].cpu().numpy()
    ref = g["dual"]
    assert np.abs(dual - ref).max() <= 1e-10 * np.abs(ref).max()
    n = M.shape[0]
    P_ref = np.exp((ref[:n, None] + ref[None, n:] - M) / eta)
    assert np.abs(out["plan"].cpu().numpy() - P_ref).max() <= 1e-12
    ctx = out["context"]
    rp = ctx.csr_rowptr().cpu().numpy()
    ci = ctx.csr_colind().cpu().numpy().astype(np.int32)
    assert np.array_equal(rp, g["csr_rowptr"])
    assert len(ci) == int(g["csr_nnz"]) and fx.sha(ci) == str(g["csr_colind_sha"])


@pytest.fixture(scope="module")
def c3(cuda_dev):
    M, a, b, eta = fx.c3_problem()
    g = _load("backward_c3_2048x2560.npz")
    assert fx.sha(M) == str(g["M_sha"]), "regenerated C3 cost matrix differs from the fixture's"
    Mt = torch.tensor(M, device=cuda_dev)
    at, bt = torch.tensor(a, device=cuda_dev), torch.tensor(b, device=cuda_dev)
    return Mt, at, bt, eta, g


def test_c3_forward_and_backward_match_reference(cuda_dev, c3):
    Mt, at, bt, eta, g = c3
    out = cg.torch.sinkhorn_splr_bwd(Mt, at, bt, eta, float(g["tol"]), 2000, 0,
                                     return_trace=True)
    assert out["niter"] == int(g["niter"]) and out["converged"]
    np.testing.assert_array_equal(out["trace"][:, [3, 4, 5, 6, 7]], g["trace"][:, [3, 4, 5, 6, 7]])
    ref = g["dual"]
    assert np.abs(out["dual"].cpu().numpy() - ref).max() <= 1e-10 * np.abs(ref).max()
    T = out["plan"]
    res = cg.torch.solve_backward(T, 2.0 * T, out["context"], eta, preconditioner="diag")
    assert res["converged"]
    lam = res["lambda"].cpu().numpy()
    assert np.abs(lam - g["lam"]).max() <= 1e-8 * np.abs(g["lam"]).max()
    assert abs(int(res["iterations"]) - int(g["pcg_iterations"])) <= 2
    grad = res["grad"]
    ent = g["fd_entries"]
    ge = grad[ent[:, 0], ent[:, 1]].cpu().numpy()
    scale = np.abs(g["grad_at_entries"]).max()
    assert np.abs(ge - g["grad_at_entries"]).max() <= 1e-8 * scale
    assert abs(float(grad.abs().sum()) - float(g["grad_abs_sum"])) <= 1e-8 * float(g["grad_abs_sum"])
    assert abs(float((grad * grad).sum()) - float(g["grad_sq_sum"])) <= 1e-7 * float(g["grad_sq_sum"])


def test_c3_autograd_matches_finite_differences(cuda_dev, c3):
    Mt, at, bt, eta, g = c3
    tol, h = float(g["tol"]), 1e-6
    M = Mt.clone().requires_grad_(True)
    T = cg.torch.splr_ot(M, at, bt, eta=eta, tol=tol, max_iter=2000)
    (T * T).sum().backward()
    ent = g["fd_entries"]
    gv = M.grad[ent[:, 0], ent[:, 1]].cpu().numpy()
    # autograd (native adjoint) against the reference's backward
    scale = np.abs(g["grad_at_entries"]).max()
    assert np.abs(gv - g["grad_at_entries"]).max() <= 1e-8 * scale

    def loss(Mp):
        Tp = cg.torch.splr_ot(Mp, at, bt, eta=eta, tol=tol, max_iter=2000)
        return float((Tp * Tp).sum())

    fd = np.empty(len(ent))
    for k, (i, j) in enumerate(ent):
        Mp = Mt.clone()
        Mp[i, j] += h
        Mm = Mt.clone()
        Mm[i, j] -= h
        fd[k] = (loss(Mp) - loss(Mm)) / (2.0 * h)
    err = np.linalg.norm(fd - gv) / np.linalg.norm(gv)
    assert err <= 1e-3, err
