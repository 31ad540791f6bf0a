"""Regenerates the golden fixtures in this directory.

The expected values are produced exactly the way the reference's own tests
produce them, with NumPy and SciPy and the same seeds and draw order:

* ``csr_n6_m3.npz`` follows test/test_csr.py:16-79 (seed 123, n=6, m=3,
  K=10, reg=0.1, shift=0.01): T row/column sums, objective, gradient, its
  norm, and the CSR triple of the sparsified lower Hessian built from a dense
  matrix with ``np.argpartition`` top-K and ``scipy.sparse.csr_matrix``.
* ``spd_n{10,100,1000,10000}.npz`` follow test/test_sparse_cholesky.py:24-88
  (seed 123, sequence n = 10, 100, 1000, 10000 with densities 0.1, 0.01,
  0.001, 0.0001): an SPD CSR matrix ``L L^T + 0.1 I``, its lower triangle, a
  right-hand side and the ``scipy.sparse.linalg.spsolve`` solution.

Run from the repository root: ``python tests/golden/make_golden.py``.
"""

import os

import numpy as np
import scipy.sparse as sparse
import scipy.sparse.linalg  # noqa: F401  (spsolve)
from scipy.sparse import csr_matrix

HERE = os.path.dirname(os.path.abspath(__file__))


def make_csr_case():
    np.random.seed(123)
    n, m, K = 6, 3, 10
    reg, shift = 0.1, 0.01
    alpha = np.random.normal(scale=0.1, size=n)
    beta = np.random.normal(scale=0.1, size=m)
    M = np.abs(np.random.normal(scale=0.1, size=(n, m)))
    a = np.random.uniform(size=n)
    b = np.random.uniform(size=m)
    a = a / np.sum(a)
    b = b / np.sum(b)
    T = np.exp((alpha.reshape(n, 1) + beta.reshape(1, m) - M) / reg)
    Trowsums = np.sum(T, axis=1)
    Tcolsums = np.sum(T, axis=0)
    objfn = reg * np.sum(T) - alpha.dot(a) - beta.dot(b)
    grad = np.concatenate((Trowsums - a, Tcolsums[:-1] - b[:-1]))
    gnorm = np.linalg.norm(grad)
    T[:, -1] = 0
    topk = np.argpartition(-T.flatten(), K)[:K]
    Tsp = np.zeros(n * m)
    Tsp[topk] = T.flatten()[topk]
    Tsp = Tsp.reshape(n, m)
    Hsl = np.diag(np.concatenate((Trowsums, Tcolsums[:-1])) + shift)
    Hsl[n:, :n] = Tsp[:, :-1].transpose()
    H = csr_matrix(Hsl)
    np.savez(os.path.join(HERE, "csr_n6_m3.npz"), alpha=alpha, beta=beta, M=M, a=a, b=b,
             reg=reg, shift=shift, K=K, Trowsums=Trowsums, Tcolsums=Tcolsums, objfn=objfn,
             grad=grad, gnorm=gnorm, csr_val=H.data, csr_colind=H.indices,
             csr_rowptr=H.indptr)


def make_spd_cases():
    np.random.seed(123)
    for n, density in ((10, 0.1), (100, 0.01), (1000, 0.001), (10000, 0.0001)):
        spmat = sparse.random(n, n, density=density, format="coo")
        L = sparse.tril(spmat)
        Mfull = sparse.csr_array(L.dot(L.T) + 0.1 * sparse.eye(n))
        Mlower = sparse.csr_array(sparse.tril(Mfull))
        rhs = np.random.normal(size=n)
        x = sparse.linalg.spsolve(Mfull, rhs)
        np.savez(os.path.join(HERE, f"spd_n{n}.npz"), n=n,
                 full_val=Mfull.data, full_col=Mfull.indices.astype(np.int32),
                 full_rowptr=Mfull.indptr.astype(np.int32),
                 lower_val=Mlower.data, lower_col=Mlower.indices.astype(np.int32),
                 lower_rowptr=Mlower.indptr.astype(np.int32), rhs=rhs, x=x)


if __name__ == "__main__":
    make_csr_case()
    make_spd_cases()
    print("golden fixtures written to", HERE)
