"""ctypes binding of libspectral_gpu.so (the C ABI declared in include/spectral_gpu.h).

The shared library is built in-tree (``spectral_rs_b200/libspectral_gpu.so``) by
``spectral_rs_b200/build.py``.  There is no CPU fallback: if the library is
missing or cannot be loaded, importing a GPU entry point raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# SPX_LIB_PATH selects another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("SPX_LIB_PATH") or os.path.join(HERE, "libspectral_gpu.so")

SPX_OK = 0
ERRORS = {1: "SPX_ERR_ARG", 2: "SPX_ERR_CUDA", 3: "SPX_ERR_BOUNDS", 4: "SPX_ERR_WALL",
          5: "SPX_ERR_NOMEM", 6: "SPX_ERR_STATE", 7: "SPX_ERR_GAMMA", 8: "SPX_ERR_TIMEOUT"}

FIELD_IDS = {"Ex": 0, "Ey": 1, "Ez": 2, "Bx": 3, "By": 4, "Bz": 5, "Jx": 6, "Jy": 7, "Jz": 8,
             "Rho": 9, "Dens": 10}
PATH_SPLIT, PATH_PLAIN = 0, 1

# Every exported symbol of the C ABI; tests check the library exports exactly these.
EXPORTS = [
    "spx_create", "spx_destroy", "spx_last_error", "spx_version", "spx_add_species",
    "spx_init_species", "spx_species_count", "spx_num_species", "spx_get_species",
    "spx_set_tags", "spx_get_tags", "spx_get_tracked",
    "spx_zero_sources", "spx_move_and_deposit", "spx_deposit_ghosts", "spx_fields_update",
    "spx_boris_push", "spx_prepare", "spx_step", "spx_flush", "spx_synchronize",
    "spx_get_field", "spx_set_field", "spx_get_bwrk", "spx_set_bwrk", "spx_diag",
    "spx_field_op", "spx_fft2d", "spx_set_timing", "spx_get_timing", "spx_last_launch_count",
    "spx_get_stream", "spx_get_counters", "spx_filter_noalloc", "spx_noalloc_last_error",
    "spx_batch_create", "spx_batch_destroy", "spx_batch_last_error", "spx_batch_sim", "spx_batch_prepare",
    "spx_batch_step", "spx_batch_set_timing", "spx_batch_get_timing", "spx_batch_get_field", "spx_batch_get_stream",
    "spx_batch_last_launch_count",
]


class SpxParams(ctypes.Structure):
    """Mirror of ``spx_params``."""
    _fields_ = [
        ("size_x", ctypes.c_uint64), ("size_y", ctypes.c_uint64), ("delta", ctypes.c_uint64),
        ("dt", ctypes.c_float), ("c", ctypes.c_float), ("dens", ctypes.c_uint32),
        ("gamma_inj", ctypes.c_float), ("n_pass", ctypes.c_uint32), ("periodic_x", ctypes.c_int32),
        ("left_wall", ctypes.c_int32),
        ("path", ctypes.c_int32), ("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32),
        ("slot_capacity", ctypes.c_int32), ("device", ctypes.c_int32), ("compensated", ctypes.c_int32),
        ("slot_headroom", ctypes.c_float), ("arrival_slots", ctypes.c_int32),
    ]


class SpxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None

P = ctypes.c_void_p
F32P = ctypes.POINTER(ctypes.c_float)
U64P = ctypes.POINTER(ctypes.c_uint64)


def load():
    """Load libspectral_gpu.so once; raises if it is absent (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python spectral_rs_b200/build.py` "
                          "(the GPU path has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    sig = {
        "spx_create": (ctypes.c_int, [ctypes.POINTER(SpxParams), ctypes.POINTER(P)]),
        "spx_destroy": (ctypes.c_int, [P]),
        "spx_last_error": (ctypes.c_char_p, [P]),
        "spx_version": (ctypes.c_char_p, []),
        "spx_add_species": (ctypes.c_int, [P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint64,
                                            P, P, P, P, P, P, P, P, ctypes.POINTER(ctypes.c_int32)]),
        "spx_init_species": (ctypes.c_int, [P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint32,
                                             ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float, ctypes.c_float,
                                             ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32)]),
        "spx_species_count": (ctypes.c_uint64, [P, ctypes.c_int32]),
        "spx_num_species": (ctypes.c_int32, [P]),
        "spx_get_species": (ctypes.c_int, [P, ctypes.c_int32, ctypes.c_uint64, P, P, P, P, P, P, P, P]),
        "spx_set_tags": (ctypes.c_int, [P, ctypes.c_int32, P, P]),
        "spx_get_tags": (ctypes.c_int, [P, ctypes.c_int32, ctypes.c_uint64, P, P]),
        "spx_get_tracked": (ctypes.c_int, [P, ctypes.c_int32, ctypes.c_uint64, P, P, P,
                                            ctypes.POINTER(ctypes.c_uint64)]),
        "spx_zero_sources": (ctypes.c_int, [P]),
        "spx_move_and_deposit": (ctypes.c_int, [P, ctypes.c_int32]),
        "spx_deposit_ghosts": (ctypes.c_int, [P, ctypes.c_int32]),
        "spx_fields_update": (ctypes.c_int, [P]),
        "spx_boris_push": (ctypes.c_int, [P, ctypes.c_int32]),
        "spx_prepare": (ctypes.c_int, [P]),
        "spx_step": (ctypes.c_int, [P, ctypes.c_uint32]),
        "spx_flush": (ctypes.c_int, [P]),
        "spx_synchronize": (ctypes.c_int, [P]),
        "spx_get_field": (ctypes.c_int, [P, ctypes.c_int32, ctypes.c_int32, P]),
        "spx_set_field": (ctypes.c_int, [P, ctypes.c_int32, P]),
        "spx_get_bwrk": (ctypes.c_int, [P, ctypes.c_int32, P]),
        "spx_set_bwrk": (ctypes.c_int, [P, ctypes.c_int32, P]),
        "spx_diag": (ctypes.c_int, [P, P]),
        "spx_field_op": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint32, P]),
        "spx_fft2d": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32, P]),
        "spx_set_timing": (ctypes.c_int, [P, ctypes.c_int32]),
        "spx_get_timing": (ctypes.c_int, [P, P]),
        "spx_last_launch_count": (ctypes.c_uint64, [P]),
        "spx_get_stream": (ctypes.c_void_p, [P]),
        "spx_get_counters": (ctypes.c_int, [P, P]),
        "spx_filter_noalloc": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, P, P, P]),
        "spx_noalloc_last_error": (ctypes.c_char_p, []),
        "spx_batch_create": (ctypes.c_int, [ctypes.c_int32, P, ctypes.POINTER(P)]),
        "spx_batch_destroy": (ctypes.c_int, [P]),
        "spx_batch_last_error": (ctypes.c_char_p, [P]),
        "spx_batch_sim": (ctypes.c_void_p, [P, ctypes.c_int32]),
        "spx_batch_prepare": (ctypes.c_int, [P]),
        "spx_batch_step": (ctypes.c_int, [P, ctypes.c_uint32]),
        "spx_batch_set_timing": (ctypes.c_int, [P, ctypes.c_int32]),
        "spx_batch_get_timing": (ctypes.c_int, [P, P]),
        "spx_batch_get_field": (ctypes.c_int, [P, ctypes.c_int32, ctypes.c_int32, P]),
        "spx_batch_get_stream": (ctypes.c_void_p, [P]),
        "spx_batch_last_launch_count": (ctypes.c_uint64, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def ptr(a):
    """Pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return ctypes.c_void_p(a.ctypes.data)


def check(code, ctx=None):
    if code != SPX_OK:
        lib = load()
        msg = lib.spx_last_error(ctx).decode(errors="replace")
        raise SpxError(code, msg)
    return code


def field_op(size_x, size_y, op, spatial, n_pass=0):
    """Standalone Field op on the GPU: 0 deposit_ghosts, 1 update_ghosts, 2 binomial filter
    (one kernel per pass), 3 binomial filter (the fused n-pass kernel)."""
    lib = load()
    a = np.ascontiguousarray(spatial, dtype=np.float32).copy()
    check(lib.spx_field_op(size_x, size_y, op, n_pass, ptr(a)))
    return a


def fft2d(data, inverse=False):
    """Fft2D::fft / inv_fft of a (size_y, size_x) complex64 array on the GPU."""
    lib = load()
    a = np.ascontiguousarray(data, dtype=np.complex64).copy()
    ny, nx = a.shape
    check(lib.spx_fft2d(nx, ny, 1 if inverse else 0, ptr(a)))
    return a
