"""ctypes binding of libpyfwi_b200.so (include/pyfwi_b200.h).

The library is the only compute path: if it is missing or fails to load the
import raises, there is no fallback."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpyfwi_b200.so")

_i32 = ctypes.c_int32
_P = ctypes.c_void_p

PYFWI_OK = 0
CKPT_EXACT, CKPT_REVERSE = 0, 1
SNAP_FP32, SNAP_BF16, SNAP_FP24 = 0, 1, 2
ADJOINT_REFERENCE, ADJOINT_EXACT = 0, 1
PARAM_LMD, PARAM_DV = 0, 1


class RecLine(ctypes.Structure):
    _fields_ = [("row0", _i32), ("col0", _i32), ("drow", _i32), ("dcol", _i32), ("count", _i32), ("slot0", _i32),
                ("vz_from_vx", _i32)]


class Geometry(ctypes.Structure):
    _fields_ = [("nz", _i32), ("nx", _i32), ("npml", _i32), ("half_order", _i32), ("nt", _i32), ("nt_ext", _i32),
                ("dt_scale", _i32), ("dt", ctypes.c_float), ("dh", ctypes.c_float), ("c", ctypes.c_float * 4),
                ("ns", _i32), ("nr", _i32), ("n_lines", _i32), ("lines", RecLine * 3),
                ("mask_row0", _i32), ("mask_row1", _i32), ("mask_col0", _i32), ("mask_col1", _i32)]


ABI_VERSION = 8  # PYFWI_ABI_VERSION of include/pyfwi_b200.h
REDUCE_SLOTS = 2368  # PYFWI_REDUCE_SLOTS


class Options(ctypes.Structure):
    _fields_ = [("checkpoint", _i32), ("segment", _i32), ("snapshot", _i32), ("shot_batch", _i32), ("energy", _i32),
                ("nchp", _i32), ("chp", ctypes.POINTER(_i32)), ("tile", _i32), ("graph", _i32), ("chunk", _i32),
                ("adj_tile", _i32), ("adjoint", _i32), ("persist", _i32), ("overlap", _i32),
                ("store_diffs", _i32)]


class NativeError(RuntimeError):
    pass


_lib = None


def lib():
    """The loaded library (raises ImportError when it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libpyfwi_b200.so is not built; run `python -m pyfwi_b200.build` "
                          "(the CUDA library is the only compute path)")
    L = ctypes.CDLL(LIB_PATH)
    L.pyfwi_plan_create.argtypes = [ctypes.POINTER(Geometry), ctypes.POINTER(_i32), ctypes.POINTER(_i32),
                                    ctypes.POINTER(Options), ctypes.POINTER(_P)]
    L.pyfwi_plan_destroy.argtypes = [_P]
    L.pyfwi_workspace_size.argtypes = [_P, ctypes.POINTER(ctypes.c_size_t)]
    L.pyfwi_set_model.argtypes = [_P, _P, ctypes.c_size_t, _P, _P, _P, _P, _P, _P]
    L.pyfwi_forward.argtypes = [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_float), _i32, _P, _P]
    L.pyfwi_gradient.argtypes = [_P, _P, ctypes.c_size_t, ctypes.POINTER(_P), _i32, _P, _P, _P]
    L.pyfwi_l2_residual.argtypes = [_P, _P, _P, ctypes.c_int64, _P, _P, _P]
    L.pyfwi_mean2.argtypes = [_P, _P, _P, ctypes.c_int64, _P]
    L.pyfwi_misfit_gradient.argtypes = [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_float), _i32,
                                        ctypes.POINTER(_P), _i32, ctypes.POINTER(_P), _i32, _P, _P, _P, _P]
    L.pyfwi_lowpass.argtypes = [_P, _i32, _P, _P, _i32, ctypes.c_int64, _i32, _P]
    L.pyfwi_smooth.argtypes = [_P, _P, _P, _i32, _i32, _i32, ctypes.POINTER(ctypes.c_double), _i32, _P]
    L.pyfwi_tile_count.argtypes = [_i32]
    L.pyfwi_launch_count.argtypes = [_P, ctypes.POINTER(ctypes.c_int64)]
    L.pyfwi_plan_flags.argtypes = [_P, ctypes.POINTER(_i32)]
    L.pyfwi_device_error.argtypes = [_P, _P, ctypes.c_size_t, ctypes.POINTER(_i32), _P]
    L.pyfwi_wait_selftest.argtypes = [_P, _P, ctypes.c_size_t, ctypes.c_int64, _P]
    L.pyfwi_barrier_selftest.argtypes = [_P, _P, ctypes.c_size_t, ctypes.c_int64, _P]
    L.pyfwi_frame_check.argtypes = [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64), _P]
    L.pyfwi_checkpoint_states.argtypes = [_P, _P, ctypes.c_size_t, _P, _P]
    L.pyfwi_profile_enable.argtypes = [_P, _i32]
    L.pyfwi_profile_read.argtypes = [_P, _i32, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_double)]
    L.pyfwi_last_error.restype = ctypes.c_char_p
    L.pyfwi_abi_version.restype = ctypes.c_int
    if L.pyfwi_abi_version() != ABI_VERSION:
        raise ImportError("libpyfwi_b200.so has ABI %d, this package needs %d: rebuild with "
                          "`python -m pyfwi_b200.build`" % (L.pyfwi_abi_version(), ABI_VERSION))
    for name in ("pyfwi_plan_create", "pyfwi_plan_destroy", "pyfwi_workspace_size", "pyfwi_set_model",
                 "pyfwi_forward", "pyfwi_gradient", "pyfwi_l2_residual", "pyfwi_mean2", "pyfwi_tile_count",
                 "pyfwi_launch_count", "pyfwi_plan_flags", "pyfwi_profile_enable", "pyfwi_profile_read", "pyfwi_device_error",
                 "pyfwi_smooth", "pyfwi_misfit_gradient", "pyfwi_lowpass", "pyfwi_wait_selftest", "pyfwi_barrier_selftest",
                 "pyfwi_frame_check", "pyfwi_checkpoint_states"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def check(status):
    if status != PYFWI_OK:
        msg = lib().pyfwi_last_error().decode(errors="replace")
        raise NativeError("pyfwi_b200 error %d: %s" % (status, msg))
    return status
