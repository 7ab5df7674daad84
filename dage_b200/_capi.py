"""ctypes bindings of libdagegpu.so (declarations in include/dage_gpu.h)."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdagegpu.so")

DAGE_DEVICE_PTRS = 1
DAGE_ENERGY = 2
DAGE_NO_CODA = 4
DAGE_ACCUMULATE = 8
DAGE_NO_GRAPH = 16
DAGE_PRODUCT_COMPLETE = 32
DAGE_TAYLOR_EXACT = 64
DAGE_TAYLOR_IGNORE_BUBBLES = 128

DAGE_FP64 = 0
DAGE_MIXED_BF16X3 = 1
DAGE_MIXED_BF16X6 = 2
DAGE_MIXED_FP16X3 = 3


class DageGrid1D(ctypes.Structure):
    _fields_ = [
        ("ncell", ctypes.c_int),
        ("nlip", ctypes.c_int),
        ("grid_type", ctypes.c_int),
        ("qmin", ctypes.c_double),
        ("cell_scales", ctypes.POINTER(ctypes.c_double)),
    ]


class DageQuad(ctypes.Structure):
    _fields_ = [
        ("nlin", ctypes.c_int),
        ("nlog", ctypes.c_int),
        ("tstart", ctypes.c_double),
        ("tlin", ctypes.c_double),
        ("tlog", ctypes.c_double),
    ]


class DageError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dage error {code}: {msg}")
        self.code = code


_D = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p

# name -> (restype, argtypes); the complete list of exported entry points
SIGNATURES = {
    "dage_op3d_create": (ctypes.c_int, [ctypes.POINTER(DageGrid1D), ctypes.POINTER(DageGrid1D),
                                        ctypes.POINTER(DageQuad), ctypes.c_int,
                                        ctypes.POINTER(_VP)]),
    "dage_op3d_apply": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_uint, _D]),
    "dage_op3d_apply_batched": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_VP), ctypes.POINTER(_VP),
                                               ctypes.POINTER(_VP), ctypes.c_uint, _D]),
    "dage_op3d_set_weights": (ctypes.c_int, [_VP, ctypes.c_int, _D]),
    "dage_op3d_set_energy": (ctypes.c_int, [_VP, ctypes.c_double]),
    "dage_op3d_set_coda": (ctypes.c_int, [_VP, ctypes.c_double]),
    "dage_op3d_set_stream": (ctypes.c_int, [_VP, _VP]),
    "dage_op3d_get_quadrature": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int), _D, _D]),
    "dage_op3d_get_matrix": (ctypes.c_int, [_VP, ctypes.c_int, _D]),
    "dage_op3d_last_time_ms": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_float)]),
    "dage_op3d_set_timing": (ctypes.c_int, [_VP, ctypes.c_int]),
    "dage_op3d_get_timing": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), _D]),
    "dage_op3d_destroy": (ctypes.c_int, [_VP]),
    "dage_op3d_tiles": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int)]),
    "dage_op3d_mixed_schedule": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_int)]),
    "dage_op3d_create_cached": (ctypes.c_int, [ctypes.POINTER(DageGrid1D), ctypes.POINTER(DageGrid1D),
                                               ctypes.POINTER(DageQuad), ctypes.c_int, ctypes.c_char_p,
                                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_VP)]),
    "dage_gbfmm_create": (ctypes.c_int, [ctypes.POINTER(DageGrid1D), ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(DageQuad), ctypes.c_int,
                                         ctypes.POINTER(_VP)]),
    "dage_gbfmm_create_adaptive": (ctypes.c_int, [ctypes.POINTER(DageGrid1D), ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(DageQuad), ctypes.c_int,
                                         ctypes.POINTER(_VP)]),
    "dage_gbfmm_apply": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_uint, _D]),
    "dage_gbfmm_multipole_moments": (ctypes.c_int, [_VP, _VP, ctypes.c_uint, _D]),
    "dage_gbfmm_local_expansions": (ctypes.c_int, [_VP, _D]),
    "dage_gbfmm_evaluate_le": (ctypes.c_int, [_VP, _D, _VP, ctypes.c_uint]),
    "dage_gbfmm_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(DageGrid1D), ctypes.c_int,
                                               ctypes.c_int, _VP, ctypes.c_int, ctypes.c_size_t, _VP]),
    "dage_gbfmm_batch_apply": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_uint, _D]),
    "dage_gbfmm_batch_set_energies": (ctypes.c_int, [_VP, _D]),
    "dage_gbfmm_batch_set_bubbles": (ctypes.c_int, [_VP, _VP, _D, ctypes.c_int]),
    "dage_gbfmm_batch_info": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_longlong)]),
    "dage_gbfmm_batch_set_stream": (ctypes.c_int, [_VP, _VP]),
    "dage_gbfmm_batch_last_time_ms": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_float)]),
    "dage_gbfmm_batch_destroy": (ctypes.c_int, [_VP]),
    "dage_gbfmm_set_energy": (ctypes.c_int, [_VP, ctypes.c_double]),
    "dage_gbfmm_tiles": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int)]),
    "dage_gbfmm_box_count": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]),
    "dage_gbfmm_set_stream": (ctypes.c_int, [_VP, _VP]),
    "dage_gbfmm_last_time_ms": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_float)]),
    "dage_gbfmm_destroy": (ctypes.c_int, [_VP]),
    "dage_bubbles_create": (ctypes.c_int, [ctypes.c_int, _D, ctypes.POINTER(DageGrid1D), ctypes.c_int,
                                           ctypes.c_int, _D, ctypes.POINTER(_VP)]),
    "dage_bubbles_inject": (ctypes.c_int, [_VP, ctypes.POINTER(DageGrid1D), ctypes.c_int,
                                           ctypes.c_double, _VP, ctypes.c_uint]),
    "dage_bubbles_coulomb_potential": (ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    "dage_bubbles_get_f": (ctypes.c_int, [_VP, _D]),
    "dage_bubbles_integrate": (ctypes.c_int, [_VP, _D]),
    "dage_bubbles_helmholtz_potential": (ctypes.c_int, [_VP, ctypes.c_double, ctypes.POINTER(_VP)]),
    "dage_bubbles_multiply": (ctypes.c_int, [_VP, _VP, ctypes.c_uint, ctypes.POINTER(_VP)]),
    "dage_product_table": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int), _D,
                                          ctypes.POINTER(ctypes.c_int)]),
    "dage_function3d_multiply": (ctypes.c_int, [ctypes.POINTER(DageGrid1D), _VP, _VP, _VP, _VP,
                                                _VP, _VP, ctypes.c_uint]),
    "dage_bubbles_destroy": (ctypes.c_int, [_VP]),
    "dage_bubbles_contaminants": (ctypes.c_int, [_VP, ctypes.c_int, _D]),
    "dage_cube_contaminants": (ctypes.c_int, [ctypes.POINTER(DageGrid1D), _VP, ctypes.c_int, _D,
                                              ctypes.c_int, ctypes.c_uint, _D]),
    "dage_bubbles_make_taylor": (ctypes.c_int, [_VP, _D, _D, ctypes.c_int, ctypes.c_uint,
                                                ctypes.POINTER(_VP)]),
    "dage_bubbles_taylor": (ctypes.c_int, [_VP, ctypes.POINTER(DageGrid1D), _VP, ctypes.c_int,
                                           ctypes.c_uint, ctypes.POINTER(_VP)]),
    "dage_bubbles_multiply_taylor": (ctypes.c_int, [_VP, _VP, _VP, _VP, ctypes.c_uint,
                                                    ctypes.POINTER(_VP)]),
    "dage_cart2sph_table": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                           _D, ctypes.POINTER(ctypes.c_int)]),
    "dage_integrate": (ctypes.c_int, [ctypes.POINTER(DageGrid1D), _VP, _VP, ctypes.c_uint, _D]),
    "dage_op3d_apply_fp64_noalloc": (ctypes.c_int, [ctypes.c_int] * 7 + [_VP, _VP, _VP, _D, _VP,
                                                                       _VP, _VP]),
    "dage_last_error": (ctypes.c_char_p, []),
    "dage_abi_version": (ctypes.c_int, []),
    "dage_set_wait_limit": (ctypes.c_int, [ctypes.c_longlong]),
    "dage_set_tune_cache": (ctypes.c_int, [ctypes.c_char_p]),
}

_lib = None


def load():
    """Loads libdagegpu.so.  Raises ImportError when the library has not been
    built: there is no fallback implementation."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing; build it with `python -m dage_b200.build` "
            "(the operator path has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != 0:
        msg = load().dage_last_error()
        raise DageError(rc, msg.decode() if msg else "")
