"""``curegot._backward_core``: the reduced-Hessian backward helpers of the
reference (curegot/_backward_core.py:31-83) as PyTorch functions on the
caller's device, for code that drives its own PCG.  The library's backward
(``curegot.backward.solve_backward``) does not use them: it runs the whole
PCG in one native call (cg_backward_f64).

Definitions (reduced gauge, beta_{m-1} = 0; T is n x m, z has n + m - 1
entries):
    q_matvec(T, z)       = [ rowsum(T) * z_a + T[:, :m-1] z_b ;
                             T[:, :m-1]^T z_a + colsum(T)[:m-1] * z_b ]
    rhs_Q_scale(G, T)    = [ rowsum(G * T) ; colsum(G * T)[:m-1] ]
    assemble_grad(...)   = T * (lam_a 1^T + 1 lam_b^T - G) / eta, lam_b[m-1] = 0
    pcg(matvec, precond, b, tol, max_iter) -> (x, iterations, converged):
        conjugate gradients from x = 0, stopping when ||r|| < tol * ||b||,
        raising RuntimeError when p^T A p <= 0.
"""
import torch

__all__ = ["q_matvec", "rhs_Q_scale", "assemble_grad", "pcg"]


def q_matvec(T, z, n, m):
    za, zb = z[:n], z[n:]
    head = T[:, : m - 1]
    top = torch.addmv(T.sum(dim=1) * za, head, zb)
    bottom = torch.addmv(T.sum(dim=0)[: m - 1] * zb, head.t(), za)
    return torch.cat([top, bottom])


def rhs_Q_scale(G, T, n, m):
    W = G * T
    return torch.cat([W.sum(dim=1), W.sum(dim=0)[: m - 1]])


def assemble_grad(T, G, lam, eta, n, m):
    lb = torch.cat([lam[n:], lam.new_zeros(1)])
    return T * (lam[:n, None] + lb[None, :] - G) / eta


def pcg(matvec, precond, b, tol=1e-12, max_iter=2000):
    x = torch.zeros_like(b)
    r = b.clone()
    bnorm = torch.linalg.norm(b)
    if bnorm == 0:
        bnorm = torch.linalg.norm(r)
    z = r.clone() if precond is None else precond(r)
    p = z.clone()
    rz = torch.dot(r, z)
    for k in range(max_iter):
        w = matvec(p)
        curv = torch.dot(p, w)
        if curv <= 0:
            raise RuntimeError("PCG breakdown: p^T A p <= 0 (matrix not SPD?)")
        step = rz / curv
        x = x + step * p
        r = r - step * w
        if torch.linalg.norm(r) < tol * bnorm:
            return x, k + 1, True
        z = r.clone() if precond is None else precond(r)
        rz_next = torch.dot(r, z)
        p = z + (rz_next / rz) * p
        rz = rz_next
    return x, max_iter, False
