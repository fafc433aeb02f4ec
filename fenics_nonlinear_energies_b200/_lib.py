"""ctypes binding of ``libfne_asm.so`` (declared in ``include/fne_asm.h``).

The library is the product's only compute path: if it cannot be loaded the
import fails loudly -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libfne_asm.so"

FNE_OK, FNE_EINVAL, FNE_ECUDA, FNE_EBOUNDS, FNE_ETIMEOUT, FNE_ENOMEM, FNE_ELAYOUT = range(7)
FNE_PLAPLACE, FNE_GINZBURG_LANDAU, FNE_NEOHOOKEAN, FNE_MOHR_COULOMB, FNE_MOHR_COULOMB_3D = 1, 2, 3, 4, 5
FNE_FP64, FNE_FP32 = 0, 1
FNE_REORDER_NONE, FNE_REORDER_BLOCK_XYZ = 0, 1
FNE_ENERGY, FNE_GRAD, FNE_HESS = 1, 2, 4

_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)


class FneError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fne error {code}: {msg}")
        self.code = code


class LayoutDesc(C.Structure):
    _fields_ = [
        ("n_total", C.c_int64), ("n_free", C.c_int64), ("freedofs", _i64p),
        ("n_elem", C.c_int64), ("ndof_e", C.c_int32), ("elems", _i64p),
        ("block_size", C.c_int32), ("reorder", C.c_int32),
        ("n_nodes", C.c_int64), ("dim", C.c_int32), ("coords", _f64p),
        ("perm_override", _i64p), ("adj_indptr", _i64p), ("adj_indices", _i64p),
        ("comm_rank", C.c_int32), ("comm_size", C.c_int32),
    ]


class Desc(C.Structure):
    _fields_ = [
        ("family", C.c_int32), ("precision", C.c_int32), ("hess_fp32", C.c_int32),
        ("n_elem", C.c_int64), ("npe", C.c_int32), ("block_size", C.c_int32),
        ("elems", _i64p), ("n_total", C.c_int64), ("total_to_free_reord", _i64p),
        ("n_free", C.c_int64), ("lo", C.c_int64), ("hi", C.c_int64), ("nnz", C.c_int64),
        ("owned_rows", _i64p), ("owned_cols", _i64p), ("energy_weights", _f64p),
        ("nq", C.c_int32),
        ("e0", _f64p), ("e1", _f64p), ("e2", _f64p), ("e3", _f64p),
        ("s", C.c_double * 16),
        ("dirichlet", _f64p), ("rhs_owned", _f64p), ("dirichlet_only_energy", C.c_int32),
        ("kernel_variant", C.c_int32),
    ]


class Info(C.Structure):
    _fields_ = [
        ("n_rows", C.c_int64), ("nnz", C.c_int64), ("n_elem", C.c_int64),
        ("n_incidences", C.c_int64), ("device_bytes", C.c_int64),
        ("max_row_len", C.c_int32), ("kernel_variant", C.c_int32), ("row_lanes", C.c_int32),
    ]


def _load():
    if not LIB_PATH.exists():
        if os.environ.get("FNE_NO_AUTOBUILD"):
            raise ImportError(f"{LIB_PATH} is missing; run python -m fenics_nonlinear_energies_b200.build")
        from fenics_nonlinear_energies_b200 import build as _b

        _b.build()
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    sig = {
        "fne_layout_build": (C.c_int, [C.POINTER(LayoutDesc), C.POINTER(vp)]),
        "fne_layout_build_device": (C.c_int, [C.POINTER(LayoutDesc), C.POINTER(vp)]),
        "fne_layout_sizes": (C.c_int, [vp, _i64p, _i64p, _i64p, _i64p, _i64p, _i64p]),
        "fne_layout_copy": (C.c_int, [vp] + [_i64p] * 8),
        "fne_layout_free": (None, [vp]),
        "fne_create": (C.c_int, [C.POINTER(Desc), C.POINTER(vp)]),
        "fne_info_get": (C.c_int, [vp, C.POINTER(Info)]),
        "fne_set_dirichlet": (C.c_int, [vp, _f64p]),
        "fne_eval": (C.c_int, [vp, vp, C.c_int, vp, vp, vp, vp]),
        "fne_eval_host": (C.c_int, [vp, _f64p, C.c_int, _f64p, _f64p, vp]),
        "fne_destroy": (C.c_int, [vp]),
        "fne_check_device_status": (C.c_int, [vp]),
        "fne_poll_device_status": (C.c_int, [vp]),
        "fne_set_wait_limit": (C.c_int, [vp, C.c_int64]),
        "fne_hvp_prepare": (C.c_int, [vp, vp, vp]),
        "fne_hvp": (C.c_int, [vp, vp, vp, vp]),
        "fne_hvp_diagonal": (C.c_int, [vp, vp, vp]),
        "fne_cg_create": (C.c_int, [C.c_int32, C.c_int64, _i64p, _i64p, C.c_int32, C.c_int32, C.POINTER(vp)]),
        "fne_cg_set_matrix": (C.c_int, [vp, vp, vp]),
        "fne_cg_solve": (C.c_int, [vp, vp, vp, C.c_double, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   vp]),
        "fne_cg_destroy": (C.c_int, [vp]),
        "fne_energy_p1tri_noalloc": (C.c_int, [C.c_int32, C.c_int64, vp, vp, vp, vp, vp, vp, vp, _f64p, vp,
                                               C.c_int64, C.c_int64, vp, vp]),
        "fne_gemm_bf16": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, C.c_int64, C.c_int64, vp, C.c_int64, C.c_int64,
                                    vp, C.c_int64, C.c_float, vp]),
        "fne_gemm_check_status": (C.c_int, []),
        "fne_gemm_set_wait_limit": (C.c_int, [C.c_int64]),
        "fne_mlp_bias_act": (C.c_int, [C.c_int64, C.c_int, vp, vp, C.c_int, vp, vp, vp]),
        "fne_mlp_act_bwd": (C.c_int, [C.c_int64, vp, vp, C.c_int, vp, vp, vp]),
        "fne_mlp_colsum": (C.c_int, [C.c_int64, C.c_int, vp, vp, vp]),
        "fne_mlp_adam": (C.c_int, [C.c_int64, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                   vp, vp]),
        "fne_mlp_cast_bf16": (C.c_int, [C.c_int64, vp, vp, vp]),
        "fne_last_error": (C.c_char_p, []),
        "fne_version": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(code):
    if code != FNE_OK:
        raise FneError(code, lib.fne_last_error().decode())


def i64(a):
    """Contiguous int64 copy/view and its ctypes pointer (keep the array alive!)."""
    arr = np.ascontiguousarray(a, dtype=np.int64)
    return arr, arr.ctypes.data_as(_i64p)


def f64(a):
    arr = np.ascontiguousarray(a, dtype=np.float64)
    return arr, arr.ctypes.data_as(_f64p)


def build_layout(*, freedofs, elems, n_total, block_size, reorder="block_xyz", coords=None,
                 perm_override=None, adjacency=None, rank=0, size=1, device=False):
    """``build_global_layout``; returns a dict of int64 arrays + lo/hi.

    ``device=False``: the host C++ build (``fne_layout_build``);
    ``device=True``: the same arrays built on the current CUDA device
    (``fne_layout_build_device``) and copied back.
    """
    keep = []
    d = LayoutDesc()
    fd, d.freedofs = i64(freedofs)
    el, d.elems = i64(elems)
    if el.ndim != 2:
        raise ValueError("elems must be a 2-D (n_elem, ndof_e) array")
    keep += [fd, el]
    d.n_total, d.n_free = int(n_total), int(fd.size)
    d.n_elem, d.ndof_e = int(el.shape[0]), int(el.shape[1])
    d.block_size = int(block_size)
    d.reorder = {"none": FNE_REORDER_NONE, "block_xyz": FNE_REORDER_BLOCK_XYZ}[reorder]
    if coords is not None:
        co, d.coords = f64(coords)
        keep.append(co)
        d.n_nodes, d.dim = int(co.shape[0]), int(co.shape[1])
    if perm_override is not None:
        po, d.perm_override = i64(perm_override)
        keep.append(po)
    if adjacency is not None:
        csr = adjacency.tocsr()
        ip, d.adj_indptr = i64(csr.indptr)
        ix, d.adj_indices = i64(csr.indices)
        keep += [ip, ix]
    d.comm_rank, d.comm_size = int(rank), int(size)
    h = C.c_void_p()
    check((lib.fne_layout_build_device if device else lib.fne_layout_build)(C.byref(d), C.byref(h)))
    try:
        nf, lo, hi, nnz_t, nnz_o, ne = (C.c_int64() for _ in range(6))
        check(lib.fne_layout_sizes(h, C.byref(nf), C.byref(lo), C.byref(hi), C.byref(nnz_t),
                                   C.byref(nnz_o), C.byref(ne)))
        # one rank owns every row: the owned COO arrays are the COO arrays
        # (copied once, the same read-only NumPy arrays under both names)
        shared = int(size) == 1 and nnz_t.value == nnz_o.value
        out = {
            "perm": np.empty(nf.value, np.int64), "iperm": np.empty(nf.value, np.int64),
            "total_to_free_reord": np.empty(int(n_total), np.int64),
            "owned_rows": np.empty(nnz_o.value, np.int64), "owned_cols": np.empty(nnz_o.value, np.int64),
            "elem_owner": np.empty(ne.value, np.int64),
        }
        if shared:
            out["coo_rows"], out["coo_cols"] = out["owned_rows"], out["owned_cols"]
        else:
            out["coo_rows"] = np.empty(nnz_t.value, np.int64)
            out["coo_cols"] = np.empty(nnz_t.value, np.int64)
        ptr = lambda k: out[k].ctypes.data_as(_i64p)  # noqa: E731
        check(lib.fne_layout_copy(h, ptr("perm"), ptr("iperm"), ptr("total_to_free_reord"),
                                  None if shared else ptr("coo_rows"), None if shared else ptr("coo_cols"),
                                  ptr("owned_rows"), ptr("owned_cols"), ptr("elem_owner")))
        if shared:
            for k in ("owned_rows", "owned_cols"):
                out[k].flags.writeable = False
        out["lo"], out["hi"], out["n_free"] = lo.value, hi.value, nf.value
        return out
    finally:
        lib.fne_layout_free(h)
