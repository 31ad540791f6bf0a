"""A learning loop through the OT layer under the reference's import names:
embeddings X are trained so that point i of X is transported to point i of
Y (the workflow of the reference's examples/differentiable_splr_ot.py:
n = m = 48, d = 8, eta = 0.05, SPLROT(tol 1e-8, max_iter 1000,
density 0.1), Adam lr 0.05, 60 steps, cost = mean squared distance).  The
matched mass must grow and the gradients reaching X must stay finite."""
import pytest
import torch

import curegot_backward_b200 as cgb

pytestmark = pytest.mark.gpu


def test_embeddings_learn_through_splrot(cuda_dev):
    cgb.install_reference_names()
    import curegot
    n = m = 48
    d, eta = 8, 0.05
    g = torch.Generator(device="cpu").manual_seed(0)
    Y = torch.rand((m, d), generator=g, dtype=torch.float64).to(cuda_dev)
    X = torch.nn.Parameter(torch.rand((n, d), generator=g, dtype=torch.float64).to(cuda_dev))
    a = torch.full((n,), 1.0 / n, dtype=torch.float64, device=cuda_dev)
    b = torch.full((m,), 1.0 / m, dtype=torch.float64, device=cuda_dev)
    target = torch.eye(n, dtype=torch.float64, device=cuda_dev)
    layer = curegot.torch.SPLROT(eta=eta, tol=1e-8, max_iter=1000, density=0.10)
    opt = torch.optim.Adam([X], lr=0.05)
    losses = []
    for _ in range(60):
        opt.zero_grad()
        M = ((X[:, None, :] - Y[None, :, :]) ** 2).sum(dim=-1) / d
        loss = -(layer(M, a, b) * target).sum()
        loss.backward()
        assert bool(torch.isfinite(X.grad).all())
        opt.step()
        losses.append(float(loss.detach()))
    assert losses[-1] < losses[0]
