"""Regenerates the full-size parity fixtures of the SPLR and backward
configurations (run from the repository root; takes minutes on the CPU).

``splr_c1_4096.npz`` -- plain FP64 SPLR, n = m = 4096: X, Y ~ N(0, I_16),
M = squared distance / max, marginals U[0.5, 1.5] normalised, eta = 0.01,
tol = 1e-8, density_max = 0.1 (the reference's kwarg; the first pattern holds
1% of the entries).  Expected values from the CPU oracle's restatement of
cuda_sinkhorn_splr_bwd (src/sinkhorn_splr.cu:1305-1611): niter, the trace
(objective, ||g||, step, K, low-rank flag, recompute flag, candidate
accepted, line-search trials), the duals, and the final sparsified Hessian's
row pointers with a SHA-256 of its column indices.

``backward_c3_2048x2560.npz`` -- differentiation configuration, n = 2048,
m = 2560: X, Y ~ U[0, 1]^{32}, M_ij = mean over the 32 features of
(x_i - y_j)^2, uniform marginals, eta = 0.05, loss = sum(T^2) so
G = dL/dT = 2T, forward tol = 1e-9.  (At tol = 1e-10 the SPLR iteration of
the reference does not converge on this problem: its first Newton step
reaches ||g|| = 7.8e-10, and the oracle then ran to its 2000-iteration cap,
because below that the Wolfe line search compares objective decreases at
the FP64 resolution of f ~ 0.67.  1e-9 is the tightest tolerance reached;
the reference's own finite-difference harness runs at 1e-8 for the same
reason, validate_stage4_autograd.py:314-330.)  The forward is the oracle's SPLR; the backward is the
reference's own curegot/_backward_core.py and curegot/backward.py, loaded
unmodified from the reference checkout and run on CPU torch, with its
diagonal preconditioner D_A^{-1} taken from the oracle's context CSR (the
native part of SPLRBackwardContext, backward_context.cu:616-655).  Stored:
the forward duals and niter, lambda, PCG iterations, 64 seeded entries of
dL/dM (the finite-difference entries of the test) and sums of dL/dM.

Both cost matrices are built with elementwise NumPy operations in a fixed
order (no BLAS), so the tests rebuild the identical M on any machine; the
SHA-256 of M is stored and checked.

Usage: python tests/golden/make_parity_fixtures.py [c1] [c3]
       (c3 reads the reference checkout: $REFERENCE_ROOT, else a `reference`
       directory beside this repository)
"""

import hashlib
import importlib.util
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

C1_SEED, C3_SEED = 101, 303
C3_TOL = 1e-9
FD_SEED, FD_ENTRIES = 7, 64


def sqdist_fixed(X, Y):
    """sum_k (x_ik - y_jk)^2 accumulated feature by feature (fixed order)."""
    D = np.zeros((X.shape[0], Y.shape[0]))
    for k in range(X.shape[1]):
        diff = X[:, k, None] - Y[None, :, k]
        D += diff * diff
    return D


def c1_problem():
    rng = np.random.default_rng(C1_SEED)
    n = m = 4096
    X = rng.standard_normal((n, 16))
    Y = rng.standard_normal((m, 16))
    M = sqdist_fixed(X, Y)
    M /= M.max()
    a = rng.uniform(0.5, 1.5, size=n)
    b = rng.uniform(0.5, 1.5, size=m)
    return M, a / a.sum(), b / b.sum(), 0.01


def c3_problem():
    rng = np.random.default_rng(C3_SEED)
    n, m, d = 2048, 2560, 32
    X = rng.uniform(size=(n, d))
    Y = rng.uniform(size=(m, d))
    M = sqdist_fixed(X, Y) / d
    return M, np.full(n, 1.0 / n), np.full(m, 1.0 / m), 0.05


def fd_entries(n, m):
    rng = np.random.default_rng(FD_SEED)
    flat = rng.choice(n * m, size=FD_ENTRIES, replace=False)
    return np.stack([flat // m, flat % m], axis=1)


def sha(x):
    return hashlib.sha256(np.ascontiguousarray(x).tobytes()).hexdigest()


def make_c1():
    import oracle
    M, a, b, eta = c1_problem()
    t = time.time()
    r = oracle.splr(M, a, b, eta, tol=1e-8, max_iter=1000, density=0.1, want_plan=False)
    print(f"c1: oracle SPLR niter {r['niter']} in {time.time() - t:.0f} s", flush=True)
    ctx = r["context"]
    np.savez_compressed(os.path.join(HERE, "splr_c1_4096.npz"), M_sha=sha(M), eta=eta,
                        tol=1e-8, density=0.1, niter=r["niter"], converged=r["converged"],
                        trace=r["trace"], dual=r["dual"], csr_rowptr=ctx["csr_rowptr"],
                        csr_colind_sha=sha(ctx["csr_colind"].astype(np.int32)),
                        csr_nnz=len(ctx["csr_colind"]))


def load_reference_backward(root):
    """curegot/_backward_core.py and curegot/backward.py from the reference
    checkout, as a package of their own (the reference package's __init__
    loads its compiled extension, which is not built here)."""
    pkg = types.ModuleType("curegot_refpkg")
    pkg.__path__ = [os.path.join(root, "curegot")]
    sys.modules["curegot_refpkg"] = pkg
    mods = {}
    for name in ("_backward_core", "backward"):
        spec = importlib.util.spec_from_file_location(
            f"curegot_refpkg.{name}", os.path.join(root, "curegot", f"{name}.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[spec.name] = mod
        spec.loader.exec_module(mod)
        mods[name] = mod
    return mods["backward"]


class DiagContext:
    """The two members of SPLRBackwardContext that the reference's
    solve_backward uses with preconditioner="diag"."""

    def __init__(self, inv_diag):
        import torch
        self.inv = torch.from_numpy(inv_diag)
        self.has_diagonal_preconditioner = True

    def apply_diagonal_preconditioner(self, r):
        return self.inv * r


def make_c3():
    import torch
    import oracle
    root = oracle.reference_root()
    if root is None:
        raise SystemExit("c3 needs the reference checkout (set REFERENCE_ROOT)")
    backward = load_reference_backward(root)
    M, a, b, eta = c3_problem()
    n, m = M.shape
    t = time.time()
    r = oracle.splr(M, a, b, eta, tol=C3_TOL, max_iter=2000, want_plan=True)
    print(f"c3: oracle SPLR niter {r['niter']} in {time.time() - t:.0f} s", flush=True)
    T = torch.from_numpy(r["plan"])
    G = 2.0 * T
    ctx = r["context"]
    inv = oracle.inv_diag_from_csr(ctx["csr_values"], ctx["csr_colind"], ctx["csr_rowptr"])
    t = time.time()
    out = backward.solve_backward(T, G, DiagContext(inv), eta, preconditioner="diag")
    print(f"c3: reference solve_backward {out['iterations']} PCG iterations in "
          f"{time.time() - t:.0f} s", flush=True)
    grad = out["grad"].numpy()
    ent = fd_entries(n, m)
    assert r["converged"], "the C3 forward must converge for the fixture"
    np.savez_compressed(os.path.join(HERE, "backward_c3_2048x2560.npz"), M_sha=sha(M), eta=eta,
                        tol=C3_TOL, niter=r["niter"], converged=r["converged"], dual=r["dual"],
                        trace=r["trace"],
                        lam=out["lambda"].numpy(), pcg_iterations=out["iterations"],
                        fd_entries=ent, grad_at_entries=grad[ent[:, 0], ent[:, 1]],
                        grad_sum=grad.sum(), grad_abs_sum=np.abs(grad).sum(),
                        grad_sq_sum=(grad * grad).sum())


if __name__ == "__main__":
    which = sys.argv[1:] or ["c1", "c3"]
    if "c3" in which:
        make_c3()
    if "c1" in which:
        make_c1()
    print("fixtures written to", HERE)
