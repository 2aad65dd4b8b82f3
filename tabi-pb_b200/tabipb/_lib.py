"""ctypes binding of libtabi_gpu.so (include/tabi_gpu.h).

The shared library is built in-tree by tabi-pb_b200/build_lib.py.  There is no
CPU fallback: if the library is missing or no GPU is present the calls fail
with TabiError.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "_build", "libtabi_gpu.so")

TABI_ERRORS = {
    -1: "TABI_ERR_ARG",
    -2: "TABI_ERR_CUDA",
    -3: "TABI_ERR_NOMEM",
    -4: "TABI_ERR_STATE",
    -5: "TABI_ERR_SINGULAR",
    -6: "TABI_ERR_LIMIT",
}

SYMBOLS = [
    "tabi_default_params", "tabi_kappa", "tabi_create", "tabi_destroy", "tabi_last_error",
    "tabi_form_matrix", "tabi_set_surface", "tabi_rhs", "tabi_build_tree", "tabi_matvec",
    "tabi_matvec_dev", "tabi_msolve", "tabi_msolve_dev", "tabi_solve", "tabi_solve_dev",
    "tabi_energy", "tabi_energy_dev", "tabi_run_dev", "tabi_counts", "tabi_tree_nodes",
    "tabi_probe_fp64_peak", "tabi_profile_enable", "tabi_profile_read", "tabi_profile_nclasses",
    "tabi_profile_class_name", "tabi_energy_noalloc",
    "tabi_ws_create", "tabi_ws_destroy", "tabi_ws_nparams", "tabi_ws_get_params",
    "tabi_ws_set_params", "tabi_ws_predict_dev", "tabi_ws_loss_grad_dev",
    "tabi_ws_train_step_dev", "tabi_ws_graph_dev", "tabi_set_warmstart", "tabi_batch_run_dev",
    "tabi_output_potential", "tabi_output_potential_dev", "tabi_set_target_range",
    "tabi_direct_targets", "tabi_pivoted_leaves", "tabi_probe_fp32_peak",
    "tabi_face_filter_dev", "tabi_set_exchange",
]

# tabi_exchange_fn: int (*)(void* user, double* v_dev, int n2, int t0, int t1, void* stream)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                          C.c_void_p)


PREC_FP64 = 0   # TABI_PREC_FP64: the reference's FP64 arithmetic
PREC_MIXED = 1  # TABI_PREC_MIXED: FP32 treecode operator, FP64 refinement
FLAG_PIVOTED_LU = 1  # TABI_FLAG_PIVOTED_LU: partial pivoting for every leaf block


class TabiError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{TABI_ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    """tabi_params (include/tabi_gpu.h)."""
    _fields_ = [("order", C.c_int), ("maxparnode", C.c_int), ("theta", C.c_double),
                ("kappa", C.c_double), ("eps0", C.c_double), ("eps1", C.c_double),
                ("iprcd", C.c_int), ("tol", C.c_double), ("maxl", C.c_int), ("nrmax", C.c_int),
                ("precision", C.c_int), ("flags", C.c_int)]


class MolDev(C.Structure):
    """tabi_mol_dev (include/tabi_gpu.h): one molecule of a batch."""
    _fields_ = [("nspt", C.c_int), ("sptpos", C.c_void_p), ("sptnrm", C.c_void_p),
                ("nface", C.c_int), ("nvert", C.c_void_p), ("nchr", C.c_int),
                ("chrpos", C.c_void_p), ("atmchr", C.c_void_p), ("maxparnode", C.c_int),
                ("order", C.c_int)]


BATCH_STATS = 12

_lib = None
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


def load(path: str = LIB_PATH):
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise TabiError(-2, f"{path} not built (run tabi-pb_b200/build_lib.py)")
    L = C.CDLL(path)
    L.tabi_default_params.argtypes = [C.POINTER(Params)]
    L.tabi_default_params.restype = None
    L.tabi_kappa.argtypes = [C.c_double, C.c_double]
    L.tabi_kappa.restype = C.c_double
    L.tabi_create.argtypes = [C.POINTER(_vp), C.POINTER(Params)]
    L.tabi_destroy.argtypes = [_vp]
    L.tabi_last_error.argtypes = [_vp]
    L.tabi_last_error.restype = C.c_char_p
    L.tabi_form_matrix.argtypes = [_vp, C.c_int, _dp, _dp, C.c_int, _ip, C.c_int, _dp, _dp,
                                   _dp, _dp, _dp, _dp]
    L.tabi_set_surface.argtypes = [_vp, C.c_int, _dp, _dp, _dp]
    L.tabi_rhs.argtypes = [_vp, C.c_int, _dp, _dp, _dp]
    L.tabi_build_tree.argtypes = [_vp, _ip, _ip]
    L.tabi_matvec.argtypes = [_vp, C.c_int, _dp, _dp]
    L.tabi_matvec_dev.argtypes = [_vp, C.c_int, _vp, _vp, _vp]
    L.tabi_msolve.argtypes = [_vp, C.c_int, _dp, _dp]
    L.tabi_msolve_dev.argtypes = [_vp, C.c_int, _vp, _vp, _vp]
    L.tabi_solve.argtypes = [_vp, C.c_int, _dp, _dp, _ip, _dp, _ip, _dp, _ip]
    L.tabi_solve_dev.argtypes = [_vp, C.c_int, _vp, _vp, _ip, _dp, _ip, _dp, _ip, _vp]
    L.tabi_energy.argtypes = [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp]
    L.tabi_energy_dev.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _dp, _dp, _vp]
    L.tabi_run_dev.argtypes = [_vp, C.c_int, _vp, _vp, C.c_int, _vp, C.c_int, _vp, _vp, _vp,
                               _dp, _vp]
    L.tabi_counts.argtypes = [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.tabi_tree_nodes.argtypes = [_vp, _ip, _ip, _ip, _ip, _ip, _dp]
    L.tabi_probe_fp64_peak.argtypes = [C.c_double, _dp]
    L.tabi_probe_fp32_peak.argtypes = [C.c_double, _dp]
    L.tabi_face_filter_dev.argtypes = [_vp, C.c_int, _vp, C.c_int, _vp, _vp, _ip, _dp, _vp]
    L.tabi_profile_enable.argtypes = [_vp, C.c_int]
    L.tabi_profile_read.argtypes = [_vp, C.c_int, _dp, C.POINTER(C.c_int64)]
    L.tabi_profile_nclasses.argtypes = []
    L.tabi_profile_class_name.argtypes = [C.c_int]
    L.tabi_profile_class_name.restype = C.c_char_p
    L.tabi_energy_noalloc.argtypes = [C.c_int, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp, C.c_double,
                                      C.c_double, C.c_double, _vp, _vp]
    _fp = C.POINTER(C.c_float)
    L.tabi_ws_create.argtypes = [C.POINTER(_vp), C.c_int, C.c_int, C.c_ulonglong]
    L.tabi_ws_destroy.argtypes = [_vp]
    L.tabi_ws_nparams.argtypes = [_vp]
    L.tabi_ws_get_params.argtypes = [_vp, _fp, C.c_longlong]
    L.tabi_ws_set_params.argtypes = [_vp, _fp, C.c_longlong]
    L.tabi_ws_predict_dev.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.tabi_ws_loss_grad_dev.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _dp, _fp,
                                        _vp]
    L.tabi_ws_train_step_dev.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, C.c_double,
                                         _dp, _vp]
    L.tabi_ws_graph_dev.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _ip, _fp, _vp]
    L.tabi_set_warmstart.argtypes = [_vp, _vp]
    L.tabi_set_target_range.argtypes = [_vp, C.c_int, C.c_int]
    L.tabi_set_exchange.argtypes = [_vp, EXCHANGE_FN, _vp]
    L.tabi_direct_targets.argtypes = [_vp, C.c_int, _ip, _dp, _dp]
    L.tabi_pivoted_leaves.argtypes = [_vp, _ip]
    L.tabi_output_potential.argtypes = [_vp, C.c_int, _dp, C.c_int, _ip, _dp, _dp, _dp]
    L.tabi_output_potential_dev.argtypes = [_vp, C.c_int, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp]
    L.tabi_batch_run_dev.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(MolDev), _vp, C.c_int,
                                     _dp]
    for s in SYMBOLS:
        if s not in ("tabi_default_params", "tabi_kappa", "tabi_last_error",
                     "tabi_profile_class_name", "tabi_ws_nparams"):
            getattr(L, s).restype = C.c_int
    L.tabi_ws_nparams.restype = C.c_longlong
    _lib = L
    return L


def dptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def check(h, rc):
    if rc != 0:
        msg = load().tabi_last_error(h)
        raise TabiError(rc, msg.decode() if msg else "")
    return rc


def f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if shape is None else a.reshape(shape)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)
