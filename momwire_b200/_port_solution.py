"""The multi-port solve result, same surface as momwire's ``PortSolution``
(``_port_solution.py:22-73`` of the reference)."""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np


@dataclass(frozen=True)
class PortSolution:
    """Everything one multi-port solve produced, from one fill and one
    factorisation.

    y : (n_ports, n_ports) complex short-circuit admittance matrix.
    coeffs : (n_basis, n_ports) complex; column j is the B-spline amplitude
        vector for a 1 V drive at port j with every other port shorted.
    port_currents : the same object as ``y``.
    basis : opaque per-solve handle (stable across the ports of one
        solution, not across solves).

    Ports run [gap feeds..., junction_ports..., node_gaps...].
    """

    y: np.ndarray
    coeffs: np.ndarray
    port_currents: np.ndarray
    basis: Any

    @property
    def n_ports(self) -> int:
        return int(self.y.shape[0])
