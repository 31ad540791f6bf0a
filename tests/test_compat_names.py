"""The reference's import names served by this package (CPU checks).

Mirrors the API checks of the reference's own validator
(validate_stage5_api.py checks 1-4): the public autograd API and the legacy
solvers sit on ``curegot.torch``; the repo-root modules re-export the
package objects (identity, not copies); ``curegot._backward_core`` computes
the reference's reduced-Hessian helpers, checked here against the NumPy
oracle on CPU tensors."""
import numpy as np
import torch

import curegot_backward_b200 as cgb
import oracle

cgb.install_reference_names()

import backward_core  # noqa: E402
import curegot  # noqa: E402
import splr_autograd  # noqa: E402
import splr_backward  # noqa: E402
from curegot.torch import SPLROT, splr_ot  # noqa: E402


def test_public_and_legacy_names():
    for sym in ("splr_ot", "splr_ot_with_info", "splr_ot_batch", "SPLROT", "solve_backward",
                "sinkhorn_bcd", "sinkhorn_splr", "sinkhorn_splr_bwd", "SPLRBackwardContext"):
        assert hasattr(curegot.torch, sym), sym
    assert hasattr(curegot.numpy, "sinkhorn_bcd") and hasattr(curegot.numpy, "sinkhorn_splr")
    assert hasattr(curegot.tests, "test_T_computation_sparsify")
    assert hasattr(curegot.tests, "test_sparse_cholesky_solve")
    assert splr_ot is curegot.autograd.splr_ot and SPLROT is curegot.autograd.SPLROT


def test_repo_root_modules_reexport_package_objects():
    assert splr_autograd.splr_ot is curegot.autograd.splr_ot
    assert splr_autograd.SPLROTFunction is curegot.autograd.SPLROTFunction
    assert splr_backward.solve_backward is curegot.backward.solve_backward
    assert splr_backward.select_preconditioner is curegot.backward.select_preconditioner
    assert backward_core.pcg is curegot._backward_core.pcg
    assert set(splr_backward._VALID_PRECONDITIONERS) == {"diag", "splr", "none"}


def test_backward_core_matches_oracle():
    rng = np.random.default_rng(3)
    n, m, eta = 9, 7, 0.05
    T = rng.uniform(0.01, 0.2, size=(n, m))
    G = rng.normal(size=(n, m))
    z = rng.normal(size=n + m - 1)
    bc = curegot._backward_core
    Tt, Gt, zt = (torch.from_numpy(x) for x in (T, G, z))
    assert np.allclose(bc.q_matvec(Tt, zt, n, m).numpy(), oracle.q_matvec(T, z, n, m),
                       rtol=1e-14, atol=1e-15)
    mu = bc.rhs_Q_scale(Gt, Tt, n, m)
    assert np.allclose(mu.numpy(), oracle.rhs_Q_scale(G, T, n, m), rtol=1e-14, atol=1e-15)
    lam, it, conv = bc.pcg(lambda v: bc.q_matvec(Tt, v, n, m), None, mu, tol=1e-12)
    ref = oracle.pcg(lambda v: oracle.q_matvec(T, v, n, m), None, mu.numpy(), tol=1e-12)
    assert conv and ref[2]
    assert np.allclose(lam.numpy(), ref[0], rtol=1e-9, atol=1e-12)
    g = bc.assemble_grad(Tt, Gt, lam, eta, n, m).numpy()
    assert np.allclose(g, oracle.assemble_grad(T, G, lam.numpy(), eta, n, m), rtol=1e-14,
                       atol=1e-15)
