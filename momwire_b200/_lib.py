"""ctypes binding of ``libmomwire_b200.so`` (the C ABI in include/momwire_b200.h).

The library is loaded from ``momwire_b200/lib/`` (built in-tree by
``python -m momwire_b200.build``).  Loading fails loudly: there is no CPU
fallback behind this module.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libmomwire_b200.so"

MW_OK = 0
MW_ERR_INVALID = -1
MW_ERR_CUDA = -2
MW_ERR_CANCELLED = -3
MW_ERR_TIMEOUT = -4
MW_ERR_SINGULAR = -5
MW_ERR_WORKSPACE = -6

MW_GROUND_NONE = 0
MW_GROUND_PEC = 1
MW_GROUND_REFL = 2
MW_GROUND_SOMM_IMAGE = 3

PHI_MODES = {"rho_v": 0, "image": 1, "normal": 2, "blend": 3}

vp = C.c_void_p
i32, i64, f64, sz = C.c_int32, C.c_int64, C.c_double, C.c_size_t


class Segments(C.Structure):
    _fields_ = [
        ("n_seg", i32),
        ("seg_l", vp),
        ("seg_r", vp),
        ("tangent", vp),
        ("radius", vp),
        ("edge", vp),
        ("pos_in_edge", vp),
        ("ek_group", vp),
        ("ek_group_img", vp),
    ]


class Edges(C.Structure):
    _fields_ = [
        ("n_edge", i32),
        ("n_in_edge", vp),
        ("table_off", vp),
        ("h", vp),
        ("radius", vp),
        ("table_rows", i64),
        ("max_n", i32),
    ]


class BasisT(C.Structure):
    _fields_ = [
        ("degree", i32),
        ("n_basis", i32),
        ("supp", vp),
        ("polys", vp),
        ("n_tile", i32),
        ("max_tile_basis", i32),
        ("max_tile_seg", i32),
        ("tile_first", vp),
        ("tile_nb", vp),
        ("tile_ns", vp),
        ("tile_seg", vp),
        ("loc", vp),
    ]


class Freq(C.Structure):
    _fields_ = [("k", f64), ("omega", f64), ("eps0", f64), ("mu0", f64)]


class Ground(C.Structure):
    _fields_ = [
        ("model", i32),
        ("phi_mode", i32),
        ("ground_z", f64),
        ("eps_re", f64),
        ("eps_im", f64),
    ]


class BlockSide(C.Structure):
    _fields_ = [
        ("n_basis", i32),
        ("supp", vp),
        ("polys", vp),
        ("n_seg", i32),
        ("seg_l", vp),
        ("seg_r", vp),
        ("tangent", vp),
        ("ek_group", vp),
    ]


class BlockRefl(C.Structure):
    _fields_ = [(n, f64) for n in ("eps_re", "eps_im", "phi_c0_re", "phi_c0_im", "phi_c1_re", "phi_c1_im")]


class Enrich(C.Structure):
    _fields_ = [
        ("n_enrich", i32),
        ("seg", vp),
        ("origin", vp),
        ("n_qp", i32),
        ("t01", vp),
        ("w01", vp),
        ("proj", f64 * 4),
        ("radius", f64),
    ]


class SommGrid(C.Structure):
    _fields_ = [
        ("n_region", i32),
        ("n_r", i32 * 6),
        ("n_th", i32 * 6),
        ("offset", i64 * 6),
        ("r0", f64 * 6),
        ("dr", f64 * 6),
        ("th0", f64 * 6),
        ("dth", f64 * 6),
        ("r1_max", f64),
        ("r_break", f64),
        ("th_split", f64),
        ("r_near", f64),
        ("value_scale", f64),
        ("vals", vp),
    ]


# name -> (restype, argtypes)
_SIGS = {
    "mw_version": (i32, []),
    "mw_last_error": (C.c_char_p, []),
    "mw_launch_count": (i64, []),
    "mw_profile_enable": (None, [i32]),
    "mw_profile_read": (i32, [i32, C.POINTER(i64), C.POINTER(f64), C.POINTER(f64), C.POINTER(f64)]),
    "mw_selftest_wait_timeout": (i32, [i32, i64, vp, vp]),
    "mw_set_mixed_pivoting": (i32, [i32]),
    "mw_last_mixed_pivoting": (i32, []),
    "mw_last_mixed_growth": (f64, []),
    "mw_last_mixed_history": (i32, [C.POINTER(f64), i32]),
    "mw_same_edge_table": (i32, [C.POINTER(Edges), i32, i32, i32, f64, vp, vp]),
    "mw_offedge_moments": (i32, [C.POINTER(Segments), C.POINTER(Segments), i32, i32, f64, i32, f64, vp, vp, vp, vp]),
    "mw_fill_z": (i32, [C.POINTER(Segments), C.POINTER(BasisT), vp, C.POINTER(Edges), C.POINTER(Freq), i32, vp, i64, vp, i64, vp]),
    "mw_fill_z_image": (i32, [C.POINTER(Segments), C.POINTER(BasisT), C.POINTER(Ground), C.POINTER(Freq), i32, vp, i64, vp, i64, vp]),
    "mw_offedge_block": (i32, [i32, C.POINTER(BlockSide), C.POINTER(BlockSide), f64, C.POINTER(Freq), i32, vp, vp,
                               C.POINTER(BlockRefl), f64, vp, i64, vp]),
    "mw_enrich_blocks": (i32, [C.POINTER(Segments), C.POINTER(BasisT), C.POINTER(Enrich), C.POINTER(Freq),
                               C.POINTER(Ground), vp, i64, vp, i64, vp]),
    "mw_fill_z_noalloc": (i32, [C.POINTER(Segments), C.POINTER(BasisT), C.POINTER(Edges), C.POINTER(Freq), i32, i32, vp, i64, vp]),
    "mw_fill_z_noalloc_capacity": (sz, [i32]),
    "mw_cgemm_tc_workspace_size": (sz, [i64, i64, i64]),
    "mw_cgemm_tc_sub": (i32, [i64, i64, i64, vp, i64, vp, i64, vp, i64, vp, sz, vp, vp]),
    "mw_cgetrf_workspace_size": (sz, [i64, i64]),
    "mw_cgetrf": (i32, [i64, vp, i64, vp, vp, vp, sz, i64, vp, vp]),
    "mw_cgetrs": (i32, [i64, i64, vp, i64, vp, vp, i64, vp, sz, vp]),
    "mw_zgesv_mixed_workspace_size": (sz, [i64, i64]),
    "mw_zgesv_mixed": (i32, [i64, i64, vp, i64, vp, i64, vp, vp, i64, vp, i64, f64, i32, vp, sz, vp,
                             C.POINTER(i32), C.POINTER(f64), vp, vp]),
    "mw_fill_z_batch": (i32, [C.POINTER(Segments), C.POINTER(BasisT), C.POINTER(Edges), i32, vp, vp, f64, f64, i32,
                              i32, f64, i32, vp, vp, i64, i64, vp, i64, i64, vp]),
    "mw_zgesv_mixed_batched_workspace_size": (sz, [i32, i32, i32]),
    "mw_zgesv_mixed_batched": (i32, [i32, i32, i32, i32, vp, i64, i64, vp, i64, i64, vp, vp, vp, i64, i64, vp, f64,
                                     i32, vp, sz, C.POINTER(i32), C.POINTER(f64), vp]),
    "mw_getrf_workspace_size": (sz, [i64]),
    "mw_zgetrf": (i32, [i64, vp, i64, vp, vp, vp, sz, vp, vp]),
    "mw_zgetrs": (i32, [i64, i64, vp, i64, vp, vp, i64, vp]),
    "mw_scatter_c128": (i32, [i64, i64, i64, vp, vp, vp, vp, vp]),
    "mw_add_loading": (i32, [i64, i32, i64, vp, vp, vp, vp, vp, i32, vp, i64, i64, vp, i64, i64, vp, vp]),
    "mw_pad_identity": (i32, [i64, i64, i32, vp, i64, i64, vp, i64, i64, vp]),
    "mw_csr_mm_c128": (i32, [i64, i64, vp, vp, vp, vp, i64, vp, i64, vp]),
    "mw_build_tiles": (i32, [vp, i64, i32, i32, i32, vp, vp, vp, vp, vp, C.POINTER(i64)]),
    "mw_basis_polys": (i32, [vp, vp, vp, vp, i64, i32, vp, vp, i64, vp, vp]),
    "mw_zgemm": (i32, [i32, i32, i64, i64, i64, f64, f64, vp, i64, vp, i64, f64, f64, vp, i64, vp]),
    "mw_somm_surfaces_workspace_size": (sz, []),
    "mw_somm_surfaces": (i32, [i64, vp, vp, vp, vp, f64, f64, f64, f64, f64, f64, vp, vp, vp]),
    "mw_somm_surfaces_eps": (i32, [i64, vp, vp, vp, vp, vp, vp, f64, f64, f64, f64, vp, vp, vp]),
    "mw_somm_field_proj": (i32, [i64, vp, vp, i64, vp, vp, f64, f64, C.POINTER(SommGrid), vp, vp]),
    "mw_somm_remainder_q": (i32, [C.POINTER(Segments), C.POINTER(BasisT), C.POINTER(SommGrid), i32, f64, f64, vp,
                                  i64, vp, i64, vp]),
    "mw_max_image_distance": (i32, [i32, vp, vp, f64, vp, vp]),
    "mw_mlp_param_count": (i32, []),
    "mw_mlp_train_workspace_size": (sz, [i32]),
    "mw_mlp_to_bf16": (i32, [vp, vp, vp]),
    "mw_mlp_forward": (i32, [i32, vp, vp, vp, vp, vp, sz, vp]),
    "mw_mlp_grad": (i32, [i32, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
    "mw_mlp_train_step": (i32, [i32, vp, vp, vp, vp, vp, vp, vp, i32, C.c_float, C.c_float, C.c_float, C.c_float,
                                vp, vp, sz, vp]),
    "mw_mlp_infer": (i32, [i64, vp, vp, vp, vp, vp, vp]),
    "mw_somm_remainder_q_mlp": (i32, [C.POINTER(Segments), C.POINTER(BasisT), vp, vp, vp, f64, f64, i32, f64, f64, vp,
                                      i64, vp, i64, vp, vp]),
}

EXPORTED = tuple(_SIGS)

PROFILE_CLASSES = ("same_edge_table", "fill", "fill_image", "lu_panel", "laswp", "trsm", "zgemm",
                   "cgemm_tc", "refine", "misc", "somm_grid", "somm_q", "factor_wall", "solve_wall", "lu_l21")


def profile_enable(on=True):
    load().mw_profile_enable(1 if on else 0)


def profile_read():
    """{class name: (launches, total_ms, flops, bytes)} since profile_enable."""
    lib = load()
    out = {}
    for i, name in enumerate(PROFILE_CLASSES):
        n, ms, fl, by = i64(), f64(), f64(), f64()
        lib.mw_profile_read(i, C.byref(n), C.byref(ms), C.byref(fl), C.byref(by))
        if n.value:
            out[name] = (int(n.value), float(ms.value), float(fl.value), float(by.value))
    return out

_lib = None


class NativeError(RuntimeError):
    """A call into libmomwire_b200 returned a non-zero status."""

    def __init__(self, name, status, text):
        super().__init__(f"{name} failed with status {status}: {text}")
        self.status = status


def load():
    """Load (once) and return the native library; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("MOMWIRE_B200_LIB", str(LIB_PATH))
    if not Path(path).exists():
        raise ImportError(
            f"momwire_b200 native library not found at {path}; build it with "
            "`python -m momwire_b200.build` (there is no CPU fallback)"
        )
    lib = C.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def call(name, *args):
    """Invoke an mw_* entry point and raise NativeError on a bad status."""
    lib = load()
    st = getattr(lib, name)(*args)
    if st != MW_OK:
        raise NativeError(name, st, lib.mw_last_error().decode(errors="replace"))
    return st
