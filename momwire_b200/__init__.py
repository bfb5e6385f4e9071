"""momwire_b200: B200-native (sm_100a) dense-solve path for momwire's
B-spline Galerkin thin-wire solver.

The public surface mirrors the reference package for this path:
``BSplineSolver`` (same constructor keywords), ``PortSolution``,
``CancelToken`` and ``SolveAborted``.  The heavy lifting runs in the native
library ``libmomwire_b200.so`` (see ``include/momwire_b200.h``).
"""

from ._port_solution import PortSolution
from .bspline import BSplineSolver, CancelToken, SolveAborted

__all__ = ["BSplineSolver", "PortSolution", "CancelToken", "SolveAborted"]
__version__ = "0.1.0"
