"""ctypes binding of libpqi.so (C ABI in include/pqi.h).

The library is the only compute path of this package: there is no CPU
fallback. Loading fails loudly (``PQIUnavailable``) when the in-tree build is
missing; every entry point's status is turned into ``PQIError``.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpqi.so")

PQI_OK = 0
PQI_EINVAL = 1
PQI_ECUDA = 2
PQI_ETIMEOUT = 3
PQI_ENOTSUP = 4
_NAMES = {1: "PQI_EINVAL", 2: "PQI_ECUDA", 3: "PQI_ETIMEOUT", 4: "PQI_ENOTSUP"}

PQI_W_F32 = 0
PQI_W_I8 = 1

PQI_NOALLOC_MAX_N = 65536  # include/pqi.h


class PQIUnavailable(ImportError):
    pass


class PQIError(RuntimeError):
    def __init__(self, status, func, detail=""):
        self.status = status
        super().__init__(f"{func} returned {_NAMES.get(status, status)}" + (f": {detail}" if detail else ""))


class PqiWeights(ctypes.Structure):
    """Mirror of ``pqi_weights`` (include/pqi.h)."""

    _fields_ = [
        ("W", ctypes.c_void_p),
        ("W_i8", ctypes.c_void_p),
        ("W_hi", ctypes.c_void_p),
        ("W_lo", ctypes.c_void_p),
        ("W_f32z", ctypes.c_void_p),
        ("n", ctypes.c_int),
        ("ld", ctypes.c_int),
        ("kind", ctypes.c_int),
        ("upper_sum", ctypes.c_double),
        ("W_d", ctypes.c_void_p),
        ("wscale", ctypes.c_double),
    ]


class PqiWeightStats(ctypes.Structure):
    """Mirror of ``pqi_weight_stats`` (include/pqi.h)."""

    _fields_ = [
        ("nonfinite", ctypes.c_ulonglong),
        ("nonint", ctypes.c_ulonglong),
        ("asym", ctypes.c_ulonglong),
        ("maxabs", ctypes.c_float),
        ("kind", ctypes.c_int),
        ("upper_sum", ctypes.c_double),
    ]


class PqiCsr(ctypes.Structure):
    """Mirror of ``pqi_csr`` (include/pqi.h)."""

    _fields_ = [
        ("ptr", ctypes.c_void_p),
        ("col", ctypes.c_void_p),
        ("val", ctypes.c_void_p),
        ("n", ctypes.c_int),
        ("pad", ctypes.c_int),
        ("nnz", ctypes.c_longlong),
        ("upper_sum", ctypes.c_double),
    ]


_vp = ctypes.c_void_p
_i = ctypes.c_int
_l = ctypes.c_long
_sz = ctypes.c_size_t
_WP = ctypes.POINTER(PqiWeights)
_CP = ctypes.POINTER(PqiCsr)

# name -> (restype, argtypes); every function of include/pqi.h
SIGNATURES = {
    "pqi_version": (ctypes.c_char_p, []),
    "pqi_last_error": (ctypes.c_char_p, []),
    "pqi_check_device": (_i, [_i]),
    "pqi_workspace_bytes": (_sz, [_i, _l]),
    "pqi_padded_ld": (_i, [_i]),
    "pqi_scan_weights": (_i, [_vp, _i, _vp, _sz, ctypes.POINTER(PqiWeightStats), _vp]),
    "pqi_prepare_weights": (_i, [_vp, _i, ctypes.POINTER(PqiWeightStats), _vp, _vp, _vp, _vp, _WP, _vp]),
    "pqi_prepare_digits": (_i, [_WP, ctypes.c_float, _vp, _vp]),
    "pqi_score_set_path": (_i, [_i]),
    "pqi_score_set_events": (_i, [_vp, _vp]),
    "pqi_score_set_grid": (_i, [_i]),
    "pqi_calculate_cut": (_i, [_WP, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _sz, _vp]),
    "pqi_gains": (_i, [_WP, _vp, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_select": (_i, [_vp, _l, _i, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_select_host": (_i, [_vp, _l, _i, _i, _vp, _vp]),
    "pqi_single_bit_flips": (_i, [_WP, _vp, _i, _i, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_single_bit_flips_noalloc": (_i, [_WP, _vp, _i, _i, _i, _vp, _vp, _vp]),
    "pqi_double_bit_flips": (_i, [_WP, _vp, _vp, _i, _i, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_gray": (_i, [_WP, _vp, _vp, _i, _i, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_single_descent": (_i, [_WP, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _sz, _vp]),
    "pqi_apply_flip": (_i, [_WP, _vp, _vp, _i, _i, _vp]),
    "pqi_batch_graph_desc_bytes": (_sz, []),
    "pqi_batch_search": (_i, [_vp, _i, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, ctypes.c_uint64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pqi_mpnn_transpose64": (_i, [_vp, _i, _i, _vp, _i, _vp]),
    "pqi_mpnn_adj_gemm": (_i, [_vp, _i, _i, _vp, _i, ctypes.c_float, _vp, _vp, _i, _vp]),
    "pqi_batch_search_f32": (_i, [_vp, _i, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, ctypes.c_uint64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pqi_batch_search_cta": (_i, [_vp, _i, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, ctypes.c_uint64, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp]),
    "pqi_batch_search_warp": (_i, [_vp, _i, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, ctypes.c_uint64, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "pqi_cluster_ascent": (_i, [_vp, _i, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, ctypes.c_double, _vp, _vp]),
    "pqi_mpnn_gemm": (_i, [_i, _i, _i, _i, _i, ctypes.c_float, _vp, _i, _vp, _i, ctypes.c_float, _vp, _vp, _i, _vp, _i, _vp]),
    "pqi_mpnn_norm_adj": (_i, [_vp, _i, _vp, _i, _vp, _vp]),
    "pqi_mpnn_features": (_i, [_vp, _vp, _vp, ctypes.c_float, _i, _vp, _vp]),
    "pqi_mpnn_softmax_xent": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _vp]),
    "pqi_mpnn_kick_cdf": (_i, [_vp, _i, _i, ctypes.c_float, ctypes.c_float, _vp, _vp]),
    "pqi_mpnn_grad_clip": (_i, [_vp, _sz, ctypes.c_float, _vp, _vp]),
    "pqi_mpnn_sum": (_i, [_vp, _sz, _vp, _vp]),
    "pqi_mpnn_relu_bwd": (_i, [_vp, _vp, _sz, _vp, _vp, _vp]),
    "pqi_mpnn_colsum": (_i, [_vp, _i, _i, _i, _vp, _i, _vp]),
    "pqi_mpnn_to_bf16": (_i, [_vp, _sz, _vp, _vp]),
    "pqi_mpnn_adam": (_i, [_vp, _vp, _vp, _vp, _vp, _sz, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _i, _vp]),
    "pqi_tfim_jz": (_i, [_vp, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_tfim_jz_f32": (_i, [_vp, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_batch_set_staging": (_i, [_i]),
    "pqi_batch_set_tmem_fields": (_i, [_i]),
    "pqi_batch_set_start_pass": (_i, [_i]),
    "pqi_bnb_eval": (_i, [_vp, _i, _vp, _i, ctypes.c_double, _i, _vp, _vp, _vp, _vp, _vp]),
    "pqi_coo_to_dense": (_i, [_vp, _vp, _vp, ctypes.c_longlong, _i, _vp, _vp, _vp, _vp]),
    "pqi_tfim_cdf_workspace_bytes": (_sz, [_i, _i]),
    "pqi_tfim_cdf": (_i, [_vp, _vp, _i, _i, ctypes.c_double, ctypes.c_double, _vp, _vp, _vp, _sz, _vp]),
    "pqi_tfim_sample_workspace_bytes": (_sz, [_i]),
    "pqi_tfim_sample": (_i, [_vp, _i, _vp, ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64, _i, _vp, _vp, _sz, _vp]),
    "pqi_tfim_sample_adj": (_i, [_vp, _i, _vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64, _i, _vp, _vp, _sz, _vp]),
    "pqi_tfim_adj_count": (_i, [_vp, _i, _vp, _vp]),
    "pqi_tfim_adj_fill": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "pqi_exact_search": (_i, [_vp, _i, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_rescore_fp64": (_i, [_WP, _vp, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_pack_bits": (_i, [_vp, _i, _i, _vp, _vp]),
    "pqi_unpack_bits": (_i, [_vp, _i, _i, _vp, _vp]),
    "pqi_csr_gains": (_i, [_CP, _vp, _i, _vp, _vp, _vp]),
    "pqi_csr_single_bit_flips": (_i, [_CP, _vp, _i, _i, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_csr_apply_flip": (_i, [_CP, _vp, _vp, _i, _i, _vp]),
    "pqi_csr_single_descent": (_i, [_CP, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _sz, _vp]),
    "pqi_csr_double_bit_flips": (_i, [_CP, _vp, _vp, _i, _i, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_csr_improving_double_flip": (_i, [_CP, _vp, _vp, _i, _i, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_csr_gray": (_i, [_CP, _vp, _vp, _i, ctypes.c_longlong, _i, _vp, _vp, _vp, _sz, _vp]),
    "pqi_csr_rescore_fp64": (_i, [_CP, _vp, _i, _vp, _vp, _vp]),
    "pqi_csr_calculate_cut": (_i, [_CP, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _sz, _vp]),
    "pqi_csr_tfim_jz": (_i, [_vp, _vp, _vp, _i, ctypes.c_float, _vp, _vp, _vp]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libpqi.so and bind every entry point; raises PQIUnavailable."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise PQIUnavailable(
            f"{path} is missing: build it with `python -m pyqrackising_b200.build` (nvcc, sm_100a). "
            "This package has no CPU fallback."
        )
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def call(name, *args):
    """Call an entry point and raise PQIError on a non-zero status."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != PQI_OK:
        detail = lib.pqi_last_error().decode() if rc == PQI_ECUDA else ""
        raise PQIError(rc, name, detail)
    return rc


def status(name, *args) -> int:
    """Call an entry point and return its status without raising."""
    return getattr(load(), name)(*args)
