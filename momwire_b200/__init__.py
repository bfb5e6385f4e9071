"""momwire_b200: B200-native (sm_100a) dense-solve path for momwire's
B-spline Galerkin thin-wire solver.

The public surface mirrors the reference package for this path:
``BSplineSolver`` (same constructor keywords), ``PortSolution``,
``CancelToken`` and ``SolveAborted``.  The heavy lifting runs in the native
library ``libmomwire_b200.so`` (see ``include/momwire_b200.h``).  Importing
the package does not load that library; the first solve (or reading
``accelerated``) does.
"""

from ._port_solution import PortSolution
from .bspline import BSplineSolver, CancelToken, SolveAborted
from .loading import insulation_inductance, wire_internal_impedance


def _native_loaded() -> bool:
    """The reference's ``momwire.accelerated``: whether the native library
    (here the sm_100a one) loads in this process."""
    try:
        from . import _lib

        _lib.load()
        return True
    except (OSError, RuntimeError, ImportError):
        return False


def __getattr__(name):
    # ``accelerated`` is evaluated on first access, so that importing the
    # package (for its workloads or tables) maps no native code.
    if name == "accelerated":
        value = _native_loaded()
        globals()["accelerated"] = value
        return value
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


__all__ = ["BSplineSolver", "PortSolution", "CancelToken", "SolveAborted", "wire_internal_impedance",
           "insulation_inductance", "accelerated"]
__version__ = "0.1.0"
