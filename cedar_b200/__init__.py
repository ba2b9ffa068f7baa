"""cedar_b200 -- Cedar's BoxMG setup and V-cycle solve as sm_100a CUDA kernels.

The compute lives in ``libcdrgpu.so`` (C ABI: include/cdr_gpu.h).  This package
is the host side: the ctypes binding (``_lib``), Cedar's configuration keys
(``config``), the ``cdr2::solver`` and ``cdr3::solver`` mirrors
(``solver.Solver2D``, ``solver.Solver3D``) and the test
problem generators (``gallery``, ``problems``).
"""
from . import gallery  # noqa: F401
from .config import Config, MLSettings  # noqa: F401


def __getattr__(name):
    if name in ("Solver2D", "Solver3D"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
