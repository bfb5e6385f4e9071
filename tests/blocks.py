"""The off-edge block fixtures of ``tests/golden/make_offedge_blocks.py``:
per case, the reference's arguments and its block, decoded."""

from pathlib import Path

import numpy as np

_F = np.load(Path(__file__).resolve().parent / "golden" / "offedge_blocks.npz")
CASES = sorted({k.split("/")[0] for k in _F.files})


def case(name):
    """(args dict, reference Z)."""
    g = {k.split("/", 1)[1]: _F[k] for k in _F.files if k.startswith(name + "/")}
    a2, k, om, eps, mu, d = g["params"]
    args = dict(supp_I=g["supp_I"], polys_I=g["polys_I"], segl_I=g["segl_I"], segr_I=g["segr_I"], tan_I=g["tan_I"],
                supp_J=g["supp_J"], polys_J=g["polys_J"], segl_J=g["segl_J"], segr_J=g["segr_J"], tan_J=g["tan_J"],
                a2=float(a2), k=float(k), omega=float(om), eps_=float(eps), mu_=float(mu), degree=int(d),
                t=g["gl_t"], w=g["gl_w"], group=(g["group_I"], g["group_J"]) if "group_I" in g else None,
                a_ek=float(g["a_ek"]) if "a_ek" in g else 0.0,
                refl=tuple(complex(x) for x in g["refl"]) if "refl" in g else None)
    return args, g["Z"]
