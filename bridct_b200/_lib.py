"""ctypes binding of libbridct_b200.so (the C-ABI declared in include/bridct.h and
include/bridct_b200.h).  Importing this module fails loudly when the library is missing:
there is no CPU fallback."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libbridct_b200.so"

FORWARD, INVERSE, ROUNDTRIP = 0, 1, 2
OK, INVALID_ARGUMENT, WORKSPACE_TOO_SMALL, BAD_ALIGNMENT, OVERLAPPING_BUFFERS = 0, -1, -2, -3, -4
DEVICE_ERROR, TIMEOUT = -5, -6
FORM_SJ, FORM_TC_BF16X3, FORM_TC_TF32X3, FORM_TC_FP8 = 0, 1, 2, 3
RAGGED_QUEUE, RAGGED_CLASS_LAUNCH, RAGGED_CLASS_LAUNCH_SMALL, RAGGED_MERGED = 0, 1, 2, 3
VERSION = "0.2.0-dev.7"

_FP = C.POINTER(C.c_float)
_lib = None


class RaggedItem(C.Structure):
    _fields_ = [("height", C.c_int), ("width", C.c_int), ("mode", C.c_int), ("reserved", C.c_int),
                ("offset", C.c_size_t)]


class RaggedTuning(C.Structure):
    _fields_ = [("tile_floats", C.c_int), ("strip_floats", C.c_int), ("row_floats", C.c_int),
                ("lookahead", C.c_int)]


def _sig(lib, name, restype, argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = argtypes
    return f


def lib() -> C.CDLL:
    """Loads the library once; raises ImportError if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m bridct_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    _sig(L, "bridct_supported", C.c_int, [C.c_int, C.c_int])
    _sig(L, "bridct_plan_create", vp, [C.c_int, C.c_int])
    _sig(L, "bridct_plan_destroy", None, [vp])
    _sig(L, "bridct_plan_route", C.c_char_p, [vp])
    _sig(L, "bridct_plan_apply", C.c_int, [vp, C.c_int, vp, vp])
    _sig(L, "bridct_workspace_floats", C.c_size_t, [C.c_int])
    _sig(L, "bridct_apply", C.c_int, [C.c_int, C.c_int, vp, vp, vp, C.c_size_t])
    _sig(L, "bridct_last_error", C.c_char_p, [])
    _sig(L, "bridct_plan_gpu_route", C.c_char_p, [vp])
    _sig(L, "bridct_plan_apply_batch", C.c_int, [vp, C.c_int, vp, vp, C.c_size_t])
    _sig(L, "bridct_plan_roundtrip_batch", C.c_int, [vp, vp, vp, C.c_size_t])
    _sig(L, "bridct_plan_apply_device", C.c_int, [vp, C.c_int, vp, vp, C.c_size_t, vp])
    _sig(L, "bridct_plan_apply_form_device", C.c_int, [vp, C.c_int, C.c_int, vp, vp, C.c_size_t, vp])
    _sig(L, "bridct_plan_apply_strided_device", C.c_int, [vp, C.c_int, vp, C.c_size_t, C.c_size_t, vp,
                                                          C.c_size_t, C.c_size_t, C.c_size_t, vp])
    _sig(L, "bridct_plan_synchronize", C.c_int, [vp])
    for name, res, args in EXTRA_SIGNATURES:
        if hasattr(L, name):
            _sig(L, name, res, args)
    _lib = L
    return L


# Entry points added by later translation units (bound when present).
EXTRA_SIGNATURES = [
    ("bridct_ragged_default_tuning", None, [C.POINTER(RaggedTuning)]),
    ("bridct_ragged_create", C.c_void_p, [C.POINTER(RaggedItem), C.c_size_t]),
    ("bridct_ragged_create_tuned", C.c_void_p, [C.POINTER(RaggedItem), C.c_size_t, C.POINTER(RaggedTuning)]),
    ("bridct_ragged_destroy", None, [C.c_void_p]),
    ("bridct_ragged_units", C.c_size_t, [C.c_void_p]),
    ("bridct_ragged_apply_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("bridct_ragged_apply_loop_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("bridct_ragged_timeout_flag", C.c_int, [C.c_void_p]),
    ("bridct_ragged_set_wait_limit", C.c_int, [C.c_void_p, C.c_uint]),
    ("bridct_ragged_class_count", C.c_size_t, [C.c_void_p]),
    ("bridct_ragged_launch_count", C.c_size_t, [C.c_void_p]),
    ("bridct_ragged_class_info", C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                           C.POINTER(C.c_int), C.POINTER(C.c_size_t), C.POINTER(C.c_int)]),
    ("bridct_ragged_set_schedule", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_size_t, C.c_int]),
    ("bridct_ragged_apply_class_device", C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_void_p, C.c_void_p,
                                                   C.c_void_p]),
    ("bridct_device_timeout_flag", C.c_int, [C.c_int]),
    ("bridct_ragged_apply_noalloc", C.c_int, [C.POINTER(RaggedItem), C.c_size_t, C.c_void_p, C.c_void_p,
                                              C.c_void_p]),
    ("bridct_plan_form_workspace_bytes", C.c_size_t, [C.c_void_p, C.c_int, C.c_size_t]),
    ("bridct_plan_apply_form_device_ws", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                                   C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("bridct_image_blocks8_device", C.c_int, [C.c_int, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int,
                                              C.c_int, C.c_void_p, C.c_void_p]),
]


def last_error() -> str:
    return (lib().bridct_last_error() or b"").decode()


def check(status: int, what: str = "bridct") -> None:
    if status != OK:
        raise RuntimeError(f"{what} failed with status {status}: {last_error()}")
