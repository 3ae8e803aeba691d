"""ctypes binding of libfomo_b200.so (declarations in include/fomo_b200.h).

There is no fallback: if the library is missing or fails to load, every entry
point raises.  Build it with ``python -m fomo_julia_b200.build``.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libfomo_b200.so")

FOMO_OK = 0
ERRORS = {
    -1: "FOMO_EINVAL", -2: "FOMO_ENOMEM", -3: "FOMO_ECUDA", -4: "FOMO_ETIMEOUT",
    -5: "FOMO_ECANCELLED", -6: "FOMO_ENOTREADY", -7: "FOMO_ENOINIT",
}


class FomoError(RuntimeError):
    def __init__(self, code: int, func: str, msg: str):
        self.code = code
        super().__init__(f"{func}: {ERRORS.get(code, code)}: {msg}")


class FomoHabc(ctypes.Structure):
    _fields_ = [
        ("nbc", ctypes.c_int32),
        ("qx", ctypes.c_float), ("qz", ctypes.c_float), ("qt_x", ctypes.c_float),
        ("qt_z", ctypes.c_float), ("qxt", ctypes.c_float),
        ("w_vx", ctypes.c_void_p), ("w_vz", ctypes.c_void_p), ("w_tau", ctypes.c_void_p),
    ]


class FomoShot(ctypes.Structure):
    _fields_ = [
        ("a", ctypes.c_void_p), ("M", ctypes.c_int32),
        ("dt", ctypes.c_float), ("dtx", ctypes.c_float), ("dtz", ctypes.c_float),
        ("nt", ctypes.c_int32),
        ("src_i", ctypes.c_int32), ("src_j", ctypes.c_int32),
        ("wavelet", ctypes.c_void_p), ("n_wavelet", ctypes.c_int32),
        ("n_rec", ctypes.c_int32),
        ("rec_i", ctypes.c_void_p), ("rec_j", ctypes.c_void_p),
        ("rec_kind", ctypes.c_int32),
    ]


class FomoRunStats(ctypes.Structure):
    _fields_ = [
        ("device_ms", ctypes.c_double), ("steps", ctypes.c_int64),
        ("kernel_launches", ctypes.c_int64), ("h2d_bytes", ctypes.c_int64),
        ("d2h_bytes", ctypes.c_int64),
    ]


class FomoKernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_int64), ("total_ms", ctypes.c_double),
                ("bytes_per_launch", ctypes.c_double)]


class FomoServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("max_shots", ctypes.c_int32),
                ("steps_per_launch", ctypes.c_int32)]


class FomoRequestStats(ctypes.Structure):
    _fields_ = [("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("steps", ctypes.c_int32), ("batch_peak", ctypes.c_int32)]


class FomoServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("cancelled", ctypes.c_int64), ("batch_steps", ctypes.c_int64),
                ("kernel_launches", ctypes.c_int64), ("graph_replays", ctypes.c_int64),
                ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
                ("peak_shots", ctypes.c_int32), ("steps_per_launch", ctypes.c_int32),
                ("peak_bytes", ctypes.c_uint64)]


# Every symbol include/fomo_b200.h declares, with its ctypes signature.
_U64 = ctypes.c_uint64
_P = ctypes.c_void_p
_I32 = ctypes.c_int32
SIGNATURES = {
    "fomo_b200_init": [ctypes.c_int],
    "fomo_b200_shutdown": [],
    "fomo_b200_last_error": None,
    "fomo_b200_version": [],
    "fomo_b200_alloc": [ctypes.c_size_t, ctypes.POINTER(_U64)],
    "fomo_b200_upload": [_U64, _P, ctypes.c_size_t],
    "fomo_b200_download": [_U64, _P, ctypes.c_size_t],
    "fomo_b200_memset": [_U64, ctypes.c_float],
    "fomo_b200_free": [_U64],
    "fomo_b200_synchronize": [],
    "fomo_b200_get_stream": [ctypes.POINTER(ctypes.c_void_p)],
    "fomo_b200_medium_create": [_I32, _I32, _I32, _I32, _I32, ctypes.c_float, ctypes.c_float,
                                _P, _P, _P, _P, _P, ctypes.POINTER(_U64)],
    "fomo_b200_medium_destroy": [_U64],
    "fomo_b200_medium_create_from_model": [_I32, _I32, _P, _P, _P, ctypes.c_float, ctypes.c_float, _I32, _I32, _I32,
                                           ctypes.POINTER(_U64)],
    "fomo_b200_medium_download": [_U64, _I32, _P],
    "fomo_b200_wavefield_create": [_I32, _I32, ctypes.POINTER(_U64)],
    "fomo_b200_wavefield_destroy": [_U64],
    "fomo_b200_wavefield_reset": [_U64],
    "fomo_b200_wavefield_download": [_U64, _I32, _P],
    "fomo_b200_wavefield_upload": [_U64, _I32, _P],
    "fomo_b200_wavefield_snapshot": [_U64, _I32, _I32, _P],
    "fomo_b200_run_shot": [_U64, _U64, ctypes.POINTER(FomoHabc), ctypes.POINTER(FomoShot), _P,
                           ctypes.POINTER(FomoRunStats)],
    "fomo_b200_shot_begin": [_U64, _U64, ctypes.POINTER(FomoHabc), ctypes.POINTER(FomoShot),
                             ctypes.POINTER(_U64)],
    "fomo_b200_shot_advance": [_U64, _I32, ctypes.POINTER(_I32)],
    "fomo_b200_shot_finish": [_U64, _P, ctypes.POINTER(FomoRunStats)],
    "fomo_b200_shot_profile": [_U64, _I32, ctypes.POINTER(FomoKernelTime), _I32, ctypes.POINTER(_I32)],
    "fomo_b200_selftest_wait": [_I32, ctypes.POINTER(_I32)],
    "fomo_b200_set_step_kernel": [_I32, _I32],
    "fomo_b200_shot_save_gather": [_U64, ctypes.c_char_p],
    "fomo_b200_run_shot_noalloc": [_I32, _I32, _I32, _I32, _I32, _P, _P, _P, _P, _P, _I32,
                                   ctypes.POINTER(FomoHabc), ctypes.POINTER(FomoShot), _P, _P],
    "fomo_b200_run_batch": [_U64, ctypes.POINTER(FomoHabc), ctypes.POINTER(FomoShot), _I32,
                            ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(FomoRunStats)],
    "fomo_b200_server_create": [ctypes.POINTER(FomoServerConfig), ctypes.POINTER(_U64)],
    "fomo_b200_server_submit": [_U64, _U64, ctypes.POINTER(FomoHabc), ctypes.POINTER(FomoShot), _P,
                                ctypes.POINTER(_U64)],
    "fomo_b200_server_poll": [_U64, _U64, ctypes.POINTER(_I32)],
    "fomo_b200_server_wait": [_U64, _U64, ctypes.c_double, ctypes.POINTER(FomoRequestStats)],
    "fomo_b200_server_cancel": [_U64, _U64],
    "fomo_b200_server_stats": [_U64, ctypes.POINTER(FomoServerStats)],
    "fomo_b200_server_destroy": [_U64],
}

_lib = None
_lock = threading.Lock()


def load(path: str | None = None) -> ctypes.CDLL:
    """Loads libfomo_b200.so (raises OSError if it is absent: no fallback)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise OSError(f"libfomo_b200.so not found at {p}; build it with "
                          f"`python -m fomo_julia_b200.build` (there is no CPU fallback)")
        L = ctypes.CDLL(p)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            if name == "fomo_b200_last_error":
                f.restype = ctypes.c_char_p
                f.argtypes = []
            else:
                f.restype = ctypes.c_int
                f.argtypes = args
        _lib = L
        return L


def call(name: str, *args) -> None:
    """Calls a C-ABI entry point and raises FomoError on a negative status."""
    L = load()
    rc = getattr(L, name)(*args)
    if rc != FOMO_OK:
        raise FomoError(rc, name, L.fomo_b200_last_error().decode(errors="replace"))


_inited_device: int | None = None


def ensure_init(device: int = 0) -> None:
    global _inited_device
    if _inited_device is None:
        call("fomo_b200_init", int(device))
        _inited_device = int(device)
    elif _inited_device != int(device):
        raise FomoError(-1, "fomo_b200_init", f"library already bound to device {_inited_device}")
