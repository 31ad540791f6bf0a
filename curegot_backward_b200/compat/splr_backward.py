"""Reference repo-root name ``splr_backward`` (re-exports curegot.backward)."""
from curegot.backward import _VALID_PRECONDITIONERS, select_preconditioner, solve_backward  # noqa: F401

__all__ = ["solve_backward", "select_preconditioner", "_VALID_PRECONDITIONERS"]
