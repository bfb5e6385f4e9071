"""What this solver serves, in the declaration form momwire's consumers
read from a solver class (``_capabilities.py`` of the reference,
``bspline.py:495-509``): one named tuple of axes plus the refusal text for
each unserved cell or "a+b" combination.  The field names and the
``refusal`` lookup are the reference's interface; the values are this
package's own."""

from __future__ import annotations

from typing import Mapping, NamedTuple

GROUNDS = ("pec", "refl-coef", "sommerfeld")
AXES = ("wire_loading", "extended_kernel", "junction_ports", "node_gaps", "per_wire_radius", "singular_enrichment")


def combination_key(cells) -> str:
    """Canonical "a+b" spelling: declared axes first in their order, then
    any other token alphabetically."""
    rank = {a: i for i, a in enumerate(AXES)}
    return "+".join(sorted(cells, key=lambda c: (c not in rank, rank.get(c, 0), c)))


class Capabilities(NamedTuple):
    grounds: frozenset
    wire_loading: bool
    extended_kernel: bool
    junction_ports: bool
    node_gaps: bool
    per_wire_radius: bool
    singular_enrichment: bool
    refusals: Mapping[str, str]

    def _served(self, cell: str) -> bool:
        if cell in GROUNDS:
            return cell in self.grounds
        if cell in AXES:
            return bool(getattr(self, cell))
        return True  # a condition token only means something inside a combination key

    def refusal(self, *cells: str):
        """Why ``cells`` (one cell, or two naming a combination) is refused,
        or None when served: the combination's declared text first, then the
        first unserved cell's declared text or a one-line default."""
        if len(cells) > 1:
            hit = self.refusals.get(combination_key(cells))
            if hit is not None:
                return hit
        for cell in cells:
            if not self._served(cell):
                return self.refusals.get(cell, f"{cell} is not supported by this solver")
        return None
