"""ctypes binding of lib/libdgbgk.so (the C ABI declared in include/dgbgk.h).

The shared library is the product: every compute call goes to its sm_100a
kernels.  There is no CPU fallback; loading fails loudly when the library is
missing.
"""
import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_void_p

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libdgbgk.so")

DGBGK_OK = 0
DGBGK_EINVAL = -1
DGBGK_EMESH = -2
DGBGK_ECUDA = -3
DGBGK_ENONFINITE = -4
DGBGK_EUNSUP = -5


class DgbgkError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dgbgk error {code}: {msg}")
        self.code = code


class Mesh(ctypes.Structure):
    _fields_ = [
        ("nelem", c_int), ("npoin", c_int), ("nboun", c_int), ("nside", c_int),
        ("intma", POINTER(c_int)), ("coord", POINTER(c_double)), ("bsido", POINTER(c_int)),
        ("iside", POINTER(c_int)), ("nx", POINTER(c_double)), ("ny", POINTER(c_double)),
        ("el", POINTER(c_double)), ("geome", POINTER(c_double)), ("relen", POINTER(c_double)),
        ("mmat", POINTER(c_double)), ("cmmat", POINTER(c_double)), ("rsido", POINTER(c_double)),
    ]


class VSpace(ctypes.Structure):
    _fields_ = [("rorder", c_int), ("torder", c_int), ("vcord", POINTER(c_double)),
                ("sumweight", c_double), ("rv", c_double)]


class Params(ctypes.Structure):
    _fields_ = [
        ("immat", c_int), ("csafm", c_double), ("alpha", c_double), ("rgas", c_double),
        ("molar_mass", c_double), ("diameter", c_double), ("cinf", c_double * 4),
        ("precision", c_int), ("wall_velocity", POINTER(c_double)),
        ("tile_elems", c_int), ("moment_rows", c_int), ("device", c_int), ("shard", c_int),
    ]


class BatchParams(ctypes.Structure):
    _fields_ = [("tile_elems", c_int), ("units_per_cta", c_int), ("tune_steps", c_int), ("moment_rows", c_int)]


# name -> (restype, argtypes); mirrors include/dgbgk.h
_PD = POINTER(c_double)
_PI = POINTER(c_int)
SIGNATURES = {
    "dgbgk_default_params": (None, [POINTER(Params)]),
    "dgbgk_setup_mesh": (c_int, [c_int, c_int, c_int, _PI, _PD, _PI, _PI, _PI, _PD, _PD, _PD, _PD, _PD,
                                 _PD, _PD, _PD]),
    "dgbgk_vspace_build": (c_int, [c_int, c_int, _PD, _PD, _PD, _PD]),
    "dgbgk_create": (c_int, [POINTER(Mesh), POINTER(VSpace), POINTER(Params), POINTER(c_void_p)]),
    "dgbgk_set_state": (c_int, [c_void_p, _PD]),
    "dgbgk_get_state": (c_int, [c_void_p, _PD]),
    "dgbgk_set_state_f32": (c_int, [c_void_p, POINTER(c_float)]),
    "dgbgk_get_state_f32": (c_int, [c_void_p, POINTER(c_float)]),
    "dgbgk_init_uniform": (c_int, [c_void_p, c_double, c_double, c_double, c_double, _PD]),
    "dgbgk_init_maxwellian": (c_int, [c_void_p, _PD, _PD, _PD, _PD]),
    "dgbgk_advance": (c_int, [c_void_p, c_int, c_double, _PI, _PD, _PD, _PD]),
    "dgbgk_set_residual_reference": (c_int, [c_void_p, c_double]),
    "dgbgk_get_residual_reference": (c_int, [c_void_p, _PD]),
    "dgbgk_copy_state": (c_int, [c_void_p, c_void_p]),
    "dgbgk_snapshot": (c_int, [c_void_p, c_int]),
    "dgbgk_extrapolate": (c_int, [c_void_p, c_int, _PD]),
    "dgbgk_get_macros": (c_int, [c_void_p, _PD, _PD, _PD, _PD, _PD, _PD]),
    "dgbgk_get_macros_noalloc": (c_int, [c_void_p, _PD, _PD, _PD, _PD, _PD, _PD]),
    "dgbgk_get_forces": (c_int, [c_void_p, _PD, _PD]),
    "dgbgk_set_output": (c_int, [c_void_p, c_int, c_int]),
    "dgbgk_output_count": (c_int, [c_void_p, _PI]),
    "dgbgk_get_output": (c_int, [c_void_p, c_int, _PI, _PD, _PD, _PD, _PD, _PD, _PD, _PD, _PD]),
    "dgbgk_get_node_fields": (c_int, [c_void_p, _PD, _PD, _PD, _PD, _PD]),
    "dgbgk_shard_stream": (c_int, [c_void_p, POINTER(c_void_p)]),
    "dgbgk_shard_sizes": (c_int, [c_void_p, POINTER(ctypes.c_longlong), POINTER(ctypes.c_longlong)]),
    "dgbgk_shard_begin": (c_int, [c_void_p, c_int, c_double]),
    "dgbgk_shard_phase": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "dgbgk_shard_poll": (c_int, [c_void_p, _PI]),
    "dgbgk_shard_end": (c_int, [c_void_p, _PI, _PD, _PD, _PD, _PI]),
    "dgbgk_get_wall_eta": (c_int, [c_void_p, _PD]),
    "dgbgk_info": (c_int, [c_void_p, _PI]),
    "dgbgk_last_timing": (c_int, [c_void_p, _PD]),
    "dgbgk_profile_steps": (c_int, [c_void_p, c_int, _PD]),
    "dgbgk_destroy": (None, [c_void_p]),
    "dgbgk_last_error": (ctypes.c_char_p, []),
    "dgbgk_batch_default_params": (None, [POINTER(BatchParams)]),
    "dgbgk_batch_create": (c_int, [POINTER(c_void_p), c_int, POINTER(BatchParams), POINTER(c_void_p)]),
    "dgbgk_batch_advance": (c_int, [c_void_p, c_int, c_double, _PI, _PD]),
    "dgbgk_batch_set_active": (c_int, [c_void_p, _PI]),
    "dgbgk_batch_snapshot": (c_int, [c_void_p, c_int, _PI]),
    "dgbgk_batch_extrapolate": (c_int, [c_void_p, c_int, _PI, _PI, _PD]),
    "dgbgk_batch_status": (c_int, [c_void_p, _PI]),
    "dgbgk_batch_info": (c_int, [c_void_p, _PI]),
    "dgbgk_batch_tuning": (c_int, [c_void_p, c_int, _PD]),
    "dgbgk_batch_last_timing": (c_int, [c_void_p, _PD]),
    "dgbgk_batch_destroy": (None, [c_void_p]),
    "dgbgk_mlp_create": (c_int, [c_int, c_int, c_int, c_int, c_int, ctypes.c_ulonglong, c_int, POINTER(c_void_p)]),
    "dgbgk_mlp_param_count": (ctypes.c_longlong, [c_void_p]),
    "dgbgk_mlp_get_params": (c_int, [c_void_p, POINTER(c_float)]),
    "dgbgk_mlp_set_params": (c_int, [c_void_p, POINTER(c_float)]),
    "dgbgk_mlp_forward": (c_int, [c_void_p, POINTER(c_float), c_int, POINTER(c_float)]),
    "dgbgk_mlp_gradient": (c_int, [c_void_p, POINTER(c_float), POINTER(c_float), c_int, _PD, POINTER(c_float)]),
    "dgbgk_mlp_set_data": (c_int, [c_void_p, POINTER(c_float), POINTER(c_float), c_int]),
    "dgbgk_mlp_train": (c_int, [c_void_p, c_int, c_float, ctypes.c_ulonglong, _PD]),
    "dgbgk_mlp_destroy": (None, [c_void_p]),
}

_lib = None


def use_library(path):
    """Loads the library from `path` (another build of the same ABI, e.g. a
    build kept for an A/B timing) instead of lib/libdgbgk.so; call before the first
    use."""
    global LIB_PATH
    if _lib is not None:
        raise RuntimeError("the library is already loaded from " + LIB_PATH)
    LIB_PATH = os.path.abspath(path)


def lib():
    """Loads libdgbgk.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `make -C dg-bgk_b200` (or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise DgbgkError(rc, lib().dgbgk_last_error().decode(errors="replace"))
    return rc


def ptr(a, ctype=c_double):
    """Pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be contiguous"
    return a.ctypes.data_as(POINTER(ctype))
