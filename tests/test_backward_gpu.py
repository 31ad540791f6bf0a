"""GPU checks of the implicit backward: native PCG vs the oracle's restatement
of the reference PCG, dense-oracle ladder, autograd semantics and central
finite differences (reference validate_stage4_autograd.py protocol)."""
import numpy as np
import pytest
import torch

import curegot_backward_b200 as cg
import oracle

pytestmark = pytest.mark.gpu


def make(n, m, seed, d=8):
    rng = np.random.default_rng(seed)
    X, Y = rng.uniform(size=(n, d)), rng.uniform(size=(m, d))
    M = ((X[:, None, :] - Y[None, :, :]) ** 2).mean(-1)
    return M, np.full(n, 1.0 / n), np.full(m, 1.0 / m)


@pytest.mark.parametrize("precond", ["diag", "none", "splr"])
def test_solve_backward_matches_oracle(cuda_dev, precond):
    n, m, eta = 60, 72, 0.05
    M, a, b = make(n, m, 42)
    dev = cuda_dev
    out = cg.torch.sinkhorn_splr_bwd(torch.tensor(M, device=dev), torch.tensor(a, device=dev),
                                     torch.tensor(b, device=dev), eta, 1e-10, 500, 0)
    T = out["plan"]
    G = torch.tensor(np.random.default_rng(1).normal(size=(n, m)), device=dev)
    res = cg.torch.solve_backward(T, G, out["context"], eta, preconditioner=precond)
    assert res["converged"]
    Tn, Gn = T.cpu().numpy(), G.cpu().numpy()
    H = n + m - 1
    Q = np.stack([oracle.q_matvec(Tn, e, n, m) for e in np.eye(H)], axis=1)
    lam = np.linalg.solve(Q, oracle.rhs_Q_scale(Gn, Tn, n, m))
    got = res["lambda"].cpu().numpy()
    assert np.linalg.norm(got - lam) / np.linalg.norm(lam) < 1e-8
    g_ref = oracle.assemble_grad(Tn, Gn, lam, eta, n, m)
    assert np.abs(res["grad"].cpu().numpy() - g_ref).max() <= 1e-8 * np.abs(g_ref).max()
    if precond == "diag":
        ctx = out["context"]
        inv = ctx.inv_diag().cpu().numpy()
        ref = oracle.solve_backward(Tn, Gn, inv, eta)
        assert abs(res["iterations"] - ref["iterations"]) <= 2


def test_zero_upstream_gradient_short_circuit(cuda_dev):
    n, m, eta = 20, 25, 0.05
    M, a, b = make(n, m, 3)
    out = cg.torch.sinkhorn_splr_bwd(torch.tensor(M, device=cuda_dev),
                                     torch.tensor(a, device=cuda_dev),
                                     torch.tensor(b, device=cuda_dev), eta, 1e-10, 500, 0)
    G = torch.zeros(n, m, dtype=torch.float64, device=cuda_dev)
    res = cg.torch.solve_backward(out["plan"], G, out["context"], eta)
    assert res["iterations"] == 0 and res["converged"]
    assert torch.count_nonzero(res["lambda"]) == 0


def test_autograd_central_fd(cuda_dev):
    # validate_stage4_autograd.py:314-362 protocol: n=5, m=6, 8 random entries,
    # accept <= 1e-3.  The forward uses the validator's tol (1e-8); the finite
    # differences use a tightly converged BCD forward (the FD target is the OT
    # map itself, independent of the solver).
    n, m, eta = 5, 6, 0.05
    M, a, b = make(n, m, 7)
    dev = cuda_dev
    Mt = torch.tensor(M, device=dev, requires_grad=True)
    at, bt = torch.tensor(a, device=dev), torch.tensor(b, device=dev)
    W = torch.tensor(np.random.default_rng(2).normal(size=(n, m)), device=dev)
    loss = (cg.torch.splr_ot(Mt, at, bt, eta=eta, tol=1e-8, max_iter=200) * W).sum()
    loss.backward()
    g = Mt.grad.cpu().numpy()

    def f(Mv):
        P = cg.torch.sinkhorn_bcd(torch.tensor(Mv, device=dev), at, bt, eta, tol=1e-14,
                                  max_iter=100000)["plan"]
        return float((P * W).sum())

    rng = np.random.default_rng(3)
    scale = np.abs(g).max()
    for _ in range(8):
        i, j = rng.integers(n), rng.integers(m)
        h = 1e-5
        Mp, Mm = M.copy(), M.copy()
        Mp[i, j] += h
        Mm[i, j] -= h
        fd = (f(Mp) - f(Mm)) / (2 * h)
        assert abs(fd - g[i, j]) <= 1e-3 * max(scale, 1e-12), (i, j, fd, g[i, j])


def test_autograd_error_contract(cuda_dev):
    n, m = 8, 9
    M, a, b = make(n, m, 1)
    dev = cuda_dev
    Mt, at, bt = (torch.tensor(x, device=dev) for x in (M, a, b))
    with pytest.raises(RuntimeError):
        cg.torch.splr_ot(Mt.float(), at, bt, eta=0.05)
    with pytest.raises(RuntimeError):
        cg.torch.splr_ot(Mt.cpu(), at, bt, eta=0.05)
    with pytest.raises(ValueError):
        cg.torch.splr_ot(Mt, at, bt, eta=-1.0)
    with pytest.raises(ValueError):
        cg.torch.splr_ot(Mt, at, bt, eta=0.05, backward_preconditioner="bogus")
    with pytest.raises(NotImplementedError):
        cg.torch.splr_ot(Mt, at.clone().requires_grad_(True), bt, eta=0.05)
    with pytest.raises(RuntimeError):  # forward non-convergence
        cg.torch.splr_ot(Mt, at, bt, eta=0.05, tol=1e-14, max_iter=1)
    info = cg.torch.splr_ot_with_info(Mt, at, bt, eta=0.05, tol=1e-14, max_iter=1)
    assert not info["converged"] and info["niter"] == 1
    layer = cg.torch.SPLROT(0.05, tol=1e-7)
    T1 = layer(Mt, at, bt)
    T2 = cg.torch.splr_ot(Mt, at, bt, eta=0.05, tol=1e-7)
    assert torch.equal(T1, T2)
    Tb = cg.torch.splr_ot_batch(torch.stack([Mt, Mt]), torch.stack([at, at]),
                                torch.stack([bt, bt]), eta=0.05, tol=1e-7)
    assert torch.equal(Tb[0], T1) and torch.equal(Tb[1], T1)


@pytest.mark.parametrize("B", [3, 11])
def test_batch_concurrent_matches_sequential(B):
    """splr_ot_batch runs its solves concurrently on worker streams; plans and
    gradients must be bitwise those of one splr_ot call per problem."""
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(100 + B)
    n, m = 160, 120
    X = torch.rand(B, n, 8, generator=g, device=dev, dtype=torch.float64)
    Y = torch.rand(B, m, 8, generator=g, device=dev, dtype=torch.float64)
    M = ((X[:, :, None, :] - Y[:, None, :, :]) ** 2).mean(-1)
    a = torch.rand(B, n, generator=g, device=dev, dtype=torch.float64) + 0.5
    b = torch.rand(B, m, generator=g, device=dev, dtype=torch.float64) + 0.5
    a, b = a / a.sum(1, keepdim=True), b / b.sum(1, keepdim=True)
    W = torch.rand(B, n, m, generator=g, device=dev, dtype=torch.float64)

    Mb = M.clone().requires_grad_(True)
    Tb = cg.torch.splr_ot_batch(Mb, a, b, eta=0.05, tol=1e-8)
    (Tb * W).sum().backward()

    Ms = M.clone().requires_grad_(True)
    Ts = torch.stack([cg.torch.splr_ot(Ms[i], a[i], b[i], eta=0.05, tol=1e-8) for i in range(B)])
    (Ts * W).sum().backward()

    assert torch.equal(Tb, Ts)
    assert torch.equal(Mb.grad, Ms.grad)
    with torch.no_grad():
        Tn = cg.torch.splr_ot_batch(M, a, b, eta=0.05, tol=1e-8)
    assert Tn.grad_fn is None and torch.equal(Tn, Ts.detach())


@pytest.mark.parametrize("precond", ["diag", "none"])
def test_batched_adjoint_matches_per_problem(precond):
    """cg_backward_batch_f64 (one launch per PCG iteration over all problems)
    gives each problem exactly the lambda, gradient and iteration count of
    cg_backward_f64."""
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(7)
    B, n, m, eta = 5, 90, 70, 0.05
    X = torch.rand(B, n, 8, generator=g, device=dev, dtype=torch.float64)
    Y = torch.rand(B, m, 8, generator=g, device=dev, dtype=torch.float64)
    M = ((X[:, :, None, :] - Y[:, None, :, :]) ** 2).mean(-1)
    a = torch.full((n,), 1.0 / n, dtype=torch.float64, device=dev)
    b = torch.full((m,), 1.0 / m, dtype=torch.float64, device=dev)
    outs = [cg.torch.sinkhorn_splr_bwd(M[i], a, b, eta, 1e-9, 500, 0) for i in range(B)]
    T = torch.stack([o["plan"] for o in outs])
    G = torch.randn(B, n, m, generator=g, device=dev, dtype=torch.float64)
    ctxs = [o["context"] for o in outs]
    res = cg.backward.solve_backward_batch(T, G, ctxs, eta, preconditioner=precond)
    for i in range(B):
        one = cg.torch.solve_backward(T[i], G[i], ctxs[i], eta, preconditioner=precond)
        assert torch.equal(res["lambda"][i], one["lambda"])
        assert torch.equal(res["grad"][i], one["grad"])
        assert res["iterations"][i] == one["iterations"] and res["converged"][i]
