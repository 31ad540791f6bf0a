"""CPU oracle for the entropic-OT hot path (TEST INFRASTRUCTURE ONLY).

The C++ library built from ``ot_oracle.cpp`` restates the reference solver's
algorithms (benben-cd/curegot_backward: src/sinkhorn_bcd_kernel.cu,
src/sinkhorn_splr.cu, src/sinkhorn_splr_kernel*.cu, src/utils.h) in FP64 on
the host.  The NumPy functions below restate the reference's implicit
backward (curegot/_backward_core.py, curegot/backward.py).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and ``--impl reference`` legs may import this package; it is the checker,
never the thing measured as the product.

Pinning: ``tests/test_oracle_golden.py`` checks this oracle against the
reference's own known-answer tests (test/test_csr.py semantics,
test/test_sparse_cholesky.py vs SciPy) through committed fixtures under
``tests/golden/``; the GPU tests additionally compare it with the
reference's own GPU BCD solver built into ``oracle/_ref``.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libot_oracle.so")
_REF_PATH = os.path.join(_HERE, "_ref", "libref_bcd.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_long)


def build() -> str:
    """Compile the oracle library (make in this directory)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def reference_root() -> str | None:
    """The reference checkout: $REFERENCE_ROOT, else a `reference` directory
    beside this repository; None when neither holds its sources."""
    cand = os.environ.get("REFERENCE_ROOT") or os.path.join(os.path.dirname(_HERE), os.pardir,
                                                            "reference")
    cand = os.path.abspath(cand)
    return cand if os.path.isfile(os.path.join(cand, "src", "sinkhorn_bcd_kernel.cu")) else None


def build_ref(root: str | None = None) -> str | None:
    """Compile the reference's GPU BCD into oracle/_ref when its sources exist."""
    root = root or reference_root()
    script = os.path.join(_HERE, "build_ref.sh")
    subprocess.run(["bash", script] + ([root] if root else []), check=True)
    return _REF_PATH if os.path.exists(_REF_PATH) else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_bcd.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int, _dp, _dp, _dp, _ip, _dp,
                                 ctypes.c_int]
        L.oracle_bcd_half_steps.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_double, _dp, _dp, ctypes.c_int]
        L.oracle_t_objfn_grad.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, _dp, _dp, _dp, _dp]
        L.oracle_t_sparsify.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp,
                                        _dp, _dp, _dp, _dp, _ip, _ip, _lp]
        L.oracle_csr_spd_solve.argtypes = [_dp, _ip, _ip, ctypes.c_int, _dp, _dp]
        L.oracle_splr.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
                                  _ip, _ip, _dp, _ip, _ip, ctypes.c_long, _dp, _dp, _dp, _dp,
                                  ctypes.c_int]
        L.oracle_set_num_threads.argtypes = [ctypes.c_int]
        L.oracle_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(x, t=_dp):
    return None if x is None else x.ctypes.data_as(t)


def _f64(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def set_num_threads(t: int) -> None:
    lib().oracle_set_num_threads(int(t))


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def bcd(M, a, b, reg, tol=1e-6, max_iter=1000, x0=None, want_plan=True):
    """Restatement of cuda_sinkhorn_bcd (reference src/sinkhorn_bcd_kernel.cu:429-634)."""
    M, a, b = _f64(M), _f64(a), _f64(b)
    n, m = M.shape
    P = np.empty((n, m)) if want_plan else None
    dual = np.empty(n + m)
    niter = ctypes.c_int(0)
    trace = np.zeros(max(max_iter, 1))
    x0 = None if x0 is None else _f64(x0)
    lib().oracle_bcd(_p(M), _p(a), _p(b), n, m, float(reg), float(tol), int(max_iter),
                     _p(x0), _p(P), _p(dual), ctypes.byref(niter), _p(trace), int(max_iter))
    return {"niter": int(niter.value), "plan": P, "dual": dual, "trace": trace[:niter.value]}


def half_step(M, a, b, reg, alpha, beta, which):
    """One LSE half-step: which=0 updates alpha, which=1 updates beta."""
    M, a, b = _f64(M), _f64(a), _f64(b)
    alpha, beta = _f64(alpha).copy(), _f64(beta).copy()
    n, m = M.shape
    lib().oracle_bcd_half_steps(_p(M), _p(a), _p(b), n, m, float(reg), _p(alpha), _p(beta),
                                int(which))
    return alpha, beta


def t_objfn_grad(gamma, M, a, b, reg):
    M, a, b, gamma = _f64(M), _f64(a), _f64(b), _f64(gamma)
    n, m = M.shape
    rows, cols, grad, out = np.empty(n), np.empty(m), np.empty(n + m - 1), np.empty(2)
    lib().oracle_t_objfn_grad(_p(gamma), _p(M), _p(a), _p(b), n, m, float(reg), _p(rows),
                              _p(cols), _p(grad), _p(out))
    return {"Trowsums": rows, "Tcolsums": cols, "grad": grad, "objfn": out[0], "gnorm": out[1]}


def t_sparsify(alpha, beta, M, a, b, reg, shift, K):
    """Restatement of T_computation_sparsify_host (sinkhorn_splr_kernel.cu:909-1032)."""
    alpha, beta, M, a, b = map(_f64, (alpha, beta, M, a, b))
    n, m = M.shape
    H = n + m - 1
    Te = n * (m - 1)
    Ks = min(max(int(K), 1), Te)
    rows, cols, grad, out = np.empty(n), np.empty(m), np.empty(H), np.empty(2)
    val = np.empty(Ks + H)
    col = np.empty(Ks + H, dtype=np.int32)
    rowptr = np.empty(H + 1, dtype=np.int32)
    ka = ctypes.c_long(0)
    lib().oracle_t_sparsify(_p(alpha), _p(beta), _p(M), _p(a), _p(b), n, m, float(reg),
                            float(shift), int(K), _p(rows), _p(cols), _p(grad), _p(out),
                            _p(val), _p(col, _ip), _p(rowptr, _ip), ctypes.byref(ka))
    return {"Trowsums": rows, "Tcolsums": cols, "objfn": out[0], "grad": grad,
            "gnorm": out[1], "csr_val": val, "csr_colind": col, "csr_rowptr": rowptr,
            "K_actual": int(ka.value)}


def csr_spd_solve(values, colind, rowptr, rhs):
    values = _f64(values)
    colind = np.ascontiguousarray(colind, dtype=np.int32)
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
    rhs = _f64(rhs)
    n = rowptr.shape[0] - 1
    x = np.empty(n)
    rc = lib().oracle_csr_spd_solve(_p(values), _p(colind, _ip), _p(rowptr, _ip), n, _p(rhs),
                                    _p(x))
    if rc != 0:
        raise RuntimeError("oracle: matrix is not SPD")
    return x


def splr(M, a, b, reg, tol=1e-6, max_iter=1000, density=None, shift=1e-3,
         sparsity_pattern_cycle=30, candidate_sinkhorn_iter=3, x0=None, want_plan=True):
    """Restatement of cuda_sinkhorn_splr_bwd (reference src/sinkhorn_splr.cu:1305-1611).

    Keyword defaults follow the reference bindings (solvers_numpy.cpp:170-201):
    density_max = min(10 / min(n, m), 1), shift_max = 1e-3, cycle 30, 3
    candidate Sinkhorn iterations.
    """
    M, a, b = _f64(M), _f64(a), _f64(b)
    n, m = M.shape
    H = n + m - 1
    if density is None:
        density = min(10.0 / min(n, m), 1.0)
    density = min(max(float(density), 0.0), 1.0)
    shift = max(float(shift), 0.0)
    kmax = max(int(density * n * (m - 1)), 1)
    cap = kmax + H
    P = np.empty((n, m)) if want_plan else None
    dual = np.empty(n + m)
    niter, conv = ctypes.c_int(0), ctypes.c_int(0)
    cval = np.empty(cap)
    ccol = np.empty(cap, dtype=np.int32)
    crow = np.empty(H + 1, dtype=np.int32)
    cs, cy, csc = np.empty(H), np.empty(H), np.empty(5)
    trace = np.zeros((max(max_iter, 1), 8))
    x0 = None if x0 is None else _f64(x0)
    lib().oracle_splr(_p(M), _p(a), _p(b), n, m, float(reg), float(tol), int(max_iter),
                      density, shift, int(sparsity_pattern_cycle), int(candidate_sinkhorn_iter),
                      _p(x0), _p(P), _p(dual), ctypes.byref(niter), ctypes.byref(conv),
                      _p(cval), _p(ccol, _ip), _p(crow, _ip), cap, _p(cs), _p(cy), _p(csc),
                      _p(trace), int(max_iter))
    nnz = int(csc[4])
    ctx = {"csr_values": cval[:nnz].copy(), "csr_colind": ccol[:nnz].copy(),
           "csr_rowptr": crow.copy(), "s": cs, "y": cy, "ys": float(csc[0]),
           "low_rank": bool(csc[1]), "fallback": bool(csc[2]), "valid": bool(csc[3]),
           "reg": float(reg), "dim": H}
    k = int(niter.value)
    return {"niter": k, "converged": bool(conv.value), "plan": P, "dual": dual,
            "context": ctx, "trace": trace[:k]}


# ---------------------------------------------------------------------------
# Implicit backward, restated in NumPy from curegot/_backward_core.py:31-83
# and curegot/backward.py:72-144.
# ---------------------------------------------------------------------------

def q_matvec(T, z, n, m):
    """Q(T) z in the reduced gauge (_backward_core.py:31-38)."""
    Tred = T[:, : m - 1]
    za, zb = z[:n], z[n:]
    out_a = T.sum(axis=1) * za + Tred @ zb
    out_b = Tred.T @ za + T.sum(axis=0)[: m - 1] * zb
    return np.concatenate([out_a, out_b])


def rhs_Q_scale(G, T, n, m):
    """mu = [(G*T) 1, ((G*T)^T 1)_{:m-1}] (_backward_core.py:41-44)."""
    GT = G * T
    return np.concatenate([GT.sum(axis=1), GT.sum(axis=0)[: m - 1]])


def assemble_grad(T, G, lam, eta, n, m):
    """dL/dM = T * (lam_a 1^T + 1 lam_b^T - G) / eta (_backward_core.py:47-52)."""
    lb = np.zeros(m)
    lb[: m - 1] = lam[n:]
    return (T * (lam[:n, None] + lb[None, :] - G)) / eta


def pcg(matvec, precond, b, tol=1e-12, max_iter=2000):
    """Preconditioned CG (_backward_core.py:55-83); returns (x, iters, converged)."""
    x = np.zeros_like(b)
    r = b - matvec(x)
    bnorm = np.linalg.norm(r) if np.linalg.norm(b) == 0 else np.linalg.norm(b)
    z = r.copy() if precond is None else precond(r)
    p = z.copy()
    rz = r @ z
    for k in range(max_iter):
        w = matvec(p)
        pw = p @ w
        if pw <= 0:
            raise RuntimeError("PCG breakdown: p^T A p <= 0 (matrix not SPD?)")
        alpha = rz / pw
        x = x + alpha * p
        r = r - alpha * w
        if np.linalg.norm(r) < tol * bnorm:
            return x, k + 1, True
        z = r.copy() if precond is None else precond(r)
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, max_iter, False


def inv_diag_from_csr(values, colind, rowptr):
    """D_A^{-1} of a CSR matrix (sinkhorn_splr_kernel_low_rank.cu:404-452)."""
    H = len(rowptr) - 1
    out = np.zeros(H)
    for r in range(H):
        for q in range(rowptr[r], rowptr[r + 1]):
            if colind[q] == r:
                out[r] = 1.0 / values[q]
    return out


def solve_backward(T, G, inv_diag, eta, preconditioner="diag", tol=1e-12, max_iter=2000):
    """solve_backward (curegot/backward.py:72-144) with the diagonal preconditioner."""
    T, G = _f64(T), _f64(G)
    n, m = T.shape
    mu = rhs_Q_scale(G, T, n, m)
    if not np.any(mu):
        lam = np.zeros_like(mu)
        return {"lambda": lam, "grad": assemble_grad(T, G, lam, eta, n, m), "iterations": 0,
                "converged": True}
    precond = (lambda r: inv_diag * r) if preconditioner == "diag" else None
    lam, it, conv = pcg(lambda v: q_matvec(T, v, n, m), precond, mu, tol=tol,
                        max_iter=max_iter)
    return {"lambda": lam, "grad": assemble_grad(T, G, lam, eta, n, m), "iterations": it,
            "converged": conv}


# ---------------------------------------------------------------------------
# The reference's own GPU BCD (oracle/_ref, built from reference sources).
# ---------------------------------------------------------------------------

def ref_bcd_available() -> bool:
    return os.path.exists(_REF_PATH)


def ref_bcd(M, a, b, reg, tol=1e-6, max_iter=1000, x0=None):
    """Run the reference's cuda_sinkhorn_bcd (host-pointer path) from oracle/_ref."""
    L = ctypes.CDLL(_REF_PATH)
    f = L.ref_sinkhorn_bcd_host
    f.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                  ctypes.c_int, ctypes.c_int, _ip, _dp, _dp]
    M, a, b = _f64(M), _f64(a), _f64(b)
    n, m = M.shape
    P = np.empty((n, m))
    dual = np.empty(n + m)
    niter = ctypes.c_int(0)
    x0 = None if x0 is None else _f64(x0)
    f(_p(M), _p(a), _p(b), _p(P), float(reg), int(max_iter), float(tol), n, m,
      ctypes.byref(niter), _p(x0), _p(dual))
    return {"niter": int(niter.value), "plan": P, "dual": dual}


def ref_bcd_device(M_ptr, a_ptr, b_ptr, P_ptr, reg, tol, max_iter, n, m, dual_ptr):
    """The reference's cuda_sinkhorn_bcd on device pointers (input and output
    on the device), from oracle/_ref; returns niter.  For timing its GPU path
    beside ours on data already in HBM."""
    L = ctypes.CDLL(_REF_PATH)
    f = L.ref_sinkhorn_bcd_device
    vp = ctypes.c_void_p
    f.argtypes = [vp, vp, vp, vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                  ctypes.c_int, _ip, vp, vp]
    niter = ctypes.c_int(0)
    f(M_ptr, a_ptr, b_ptr, P_ptr, float(reg), int(max_iter), float(tol), n, m,
      ctypes.byref(niter), None, dual_ptr)
    return int(niter.value)
