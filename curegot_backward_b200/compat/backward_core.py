"""Reference repo-root name ``backward_core`` (re-exports curegot._backward_core)."""
from curegot._backward_core import assemble_grad, pcg, q_matvec, rhs_Q_scale  # noqa: F401

__all__ = ["q_matvec", "rhs_Q_scale", "assemble_grad", "pcg"]
