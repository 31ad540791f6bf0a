"""Reference repo-root name ``splr_autograd`` (re-exports curegot.autograd)."""
from curegot.autograd import SPLROT, SPLROTFunction, splr_ot, splr_ot_batch, splr_ot_with_info  # noqa: F401

__all__ = ["splr_ot", "splr_ot_with_info", "splr_ot_batch", "SPLROT", "SPLROTFunction"]
