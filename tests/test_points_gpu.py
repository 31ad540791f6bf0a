"""Cost recomputed from BF16 point clouds on the tensor cores (tcgen05).

Checks, in order: the cost tiles against an FP64 evaluation of the same
formula on the same BF16 values; that swapping the operand roles gives the
bitwise transpose (row and column passes see the same M); the fused solver
against the stored-M FP64 solver for a fixed number of iterations; and a
converged mixed-precision solve on the differentiation configuration's
shapes (n = 2048, m = 2560, d = 32, eta = 0.05, M the mean over features)
against the FP64 oracle's marginals."""
import numpy as np
import pytest
import torch

import oracle
from curegot_backward_b200 import _solvers
from curegot_backward_b200.points import cost_from_points, sinkhorn_bcd_points

pytestmark = pytest.mark.gpu


def _clouds(n, m, d, seed, dist="uniform"):
    g = torch.Generator(device="cuda").manual_seed(seed)
    if dist == "uniform":
        X = torch.rand(n, d, generator=g, device="cuda")
        Y = torch.rand(m, d, generator=g, device="cuda")
    else:
        X = torch.randn(n, d, generator=g, device="cuda")
        Y = torch.randn(m, d, generator=g, device="cuda")
    return X.bfloat16(), Y.bfloat16()


def _cost_fp64(X, Y, s):
    x, y = X.double(), Y.double()
    nx, ny = (x * x).sum(1), (y * y).sum(1)
    return torch.clamp(s * (nx[:, None] + ny[None, :] - 2.0 * x @ y.T), min=0.0), nx, ny


@pytest.mark.parametrize("n,m,d,dist", [(128, 128, 32, "uniform"), (300, 200, 32, "uniform"),
                                        (257, 383, 8, "normal"), (130, 70, 64, "normal"),
                                        (1000, 900, 20, "uniform")])
def test_cost_tiles_match_fp64(n, m, d, dist):
    X, Y = _clouds(n, m, d, 11 + n, dist)
    s = 1.0 / d
    M = cost_from_points(X, Y)
    ref, nx, ny = _cost_fp64(X, Y, s)
    # FP32 norms and FP32 accumulation of d exact BF16 products
    bound = 4e-7 * s * (nx[:, None] + ny[None, :]) * max(d, 8) ** 0.5 + 1e-30
    assert M.dtype == torch.float32 and M.shape == (n, m)
    assert bool(((M.double() - ref).abs() <= bound).all())


def test_operand_roles_give_the_transpose_bitwise():
    X, Y = _clouds(300, 200, 32, 5)
    M = cost_from_points(X, Y)
    Mt = cost_from_points(Y, X)
    assert torch.equal(M, Mt.T.contiguous())


@pytest.mark.parametrize("n,m,d", [(300, 200, 32), (129, 517, 16)])
def test_fixed_iterations_match_stored_cost_solver(n, m, d):
    X, Y = _clouds(n, m, d, 21)
    a = torch.full((n,), 1.0 / n, dtype=torch.float64, device="cuda")
    b = torch.full((m,), 1.0 / m, dtype=torch.float64, device="cuda")
    eta, iters = 0.05, 25
    r = sinkhorn_bcd_points(X, Y, a, b, eta, tol=0.0, max_iter=iters, precision="fp64")
    assert r["niter"] == iters
    M = cost_from_points(X, Y).double()
    niter, _, dual = _solvers._bcd_device(M, a, b, eta, 0.0, iters, None, "fp64", want_plan=False)
    assert niter == iters
    scale = dual.abs().max()
    assert float((r["dual"] - dual).abs().max() / scale) <= 1e-12


def test_converged_mixed_solve_marginals():
    n, m, d, eta = 2048, 2560, 32, 0.05
    X, Y = _clouds(n, m, d, 3)
    a = torch.full((n,), 1.0 / n, dtype=torch.float64, device="cuda")
    b = torch.full((m,), 1.0 / m, dtype=torch.float64, device="cuda")
    r = sinkhorn_bcd_points(X, Y, a, b, eta, tol=1e-8, max_iter=20000, precision="mixed")
    assert 0 < r["niter"] < 20000
    assert r["fast_iters"] >= 1
    M = cost_from_points(X, Y).double().cpu().numpy()
    dual = r["dual"].cpu().numpy()
    al, be = dual[:n], dual[n:]
    gamma = np.concatenate([al + be[-1], be[:-1] - be[-1]])
    ck = oracle.t_objfn_grad(gamma, M, a.cpu().numpy(), b.cpu().numpy(), eta)
    assert np.linalg.norm(ck["Trowsums"] - a.cpu().numpy()) <= 1e-8
    assert np.linalg.norm(ck["Tcolsums"] - b.cpu().numpy()) <= 1e-12


def test_invalid_arguments():
    X, Y = _clouds(16, 16, 8, 1)
    with pytest.raises(TypeError):
        cost_from_points(X.float(), Y)
    with pytest.raises(ValueError):
        cost_from_points(X, Y[:, :4])
    Z = torch.zeros(4, 65, dtype=torch.bfloat16, device="cuda")
    with pytest.raises(ValueError):
        cost_from_points(Z, Z)


@pytest.mark.parametrize("n,m,d", [(300, 260, 32), (1000, 777, 8), (129, 4000, 16)])
def test_cost_normalisers_on_the_tiles(cuda_dev, n, m, d):
    """max and lower median of the unscaled cost, computed on the tensor-core
    tiles by radix histograms, equal torch's max / kthvalue of the same FP32
    values written out by cost_from_points (scale 1)."""
    from curegot_backward_b200 import points
    g = torch.Generator(device=cuda_dev).manual_seed(n * 7 + m)
    X = torch.randn(n, d, generator=g, device=cuda_dev).to(torch.bfloat16)
    Y = torch.randn(m, d, generator=g, device=cuda_dev).to(torch.bfloat16)
    mx, med = points.cost_normalisers(X, Y)
    C = points.cost_from_points(X, Y, scale=1.0).flatten()
    assert mx == float(C.max())
    k = (C.numel() + 1) // 2
    assert med == float(torch.kthvalue(C.cpu(), k).values)
