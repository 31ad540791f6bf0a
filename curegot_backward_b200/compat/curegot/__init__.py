"""The reference's import name, ``curegot``, served by curegot_backward_b200.

With ``curegot_backward_b200/compat`` on ``sys.path`` (PYTHONPATH, or
``curegot_backward_b200.install_reference_names()``), code written against
the reference runs unchanged:

    import curegot
    r = curegot.numpy.sinkhorn_bcd(M, a, b, reg)
    from curegot.torch import splr_ot, SPLROT
    from curegot.backward import solve_backward

The submodules are the package's own objects, registered under the
reference's names (curegot/__init__.py:1-43 of the reference attaches the
autograd API onto ``curegot.torch`` the same way), so identity holds:
``curegot.torch.splr_ot is curegot.autograd.splr_ot``.
"""
import sys as _sys

import curegot_backward_b200 as _impl
from curegot_backward_b200 import autograd, backward, numpy, tests, torch  # noqa: F401
from curegot_backward_b200.autograd import SPLROT, splr_ot, splr_ot_batch, splr_ot_with_info  # noqa: F401
from curegot_backward_b200.backward import solve_backward  # noqa: F401

from . import _backward_core  # noqa: F401

for _name, _mod in (("numpy", numpy), ("torch", torch), ("tests", tests),
                    ("autograd", autograd), ("backward", backward)):
    _sys.modules[f"{__name__}.{_name}"] = _mod

__version__ = _impl.__version__
