"""CPU oracle for the Elastic2D time-stepping path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  The product (``fomo_julia_b200`` and
``libfomo_b200.so``) never imports, links or runs it.

The C++ restatement lives in ``oracle/fomo_oracle.cpp`` and is built by
``oracle/Makefile`` into ``oracle/_build/libfomo_oracle.so``.  Every function
here cites the reference file it restates (paths inside Wuheng10086/Fomo_julia).

Grid arrays use the reference's layout: numpy shape ``(nx, nz)`` stored
column-major (x fastest), so ``a[i-1, j-1]`` is the reference's ``a[i, j]``.  Gathers are returned with shape
``(nt, n_rec)`` in Fortran order, the reference's ``[nt x n_rec]`` layout.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libfomo_oracle.so")
_lib = None

REC_KIND = {"vz": 0, "vx": 1, "p": 2}
HABC_MODE = {"jacobi": 0, "sequential": 1, "simd8": 2}


class OrcShot(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("M", ctypes.c_int32), ("pad", ctypes.c_int32), ("nbc", ctypes.c_int32),
        ("free_surface", ctypes.c_int32),
        ("rho_vx", ctypes.c_void_p), ("rho_vz", ctypes.c_void_p), ("lam", ctypes.c_void_p),
        ("mu_txx", ctypes.c_void_p), ("mu_txz", ctypes.c_void_p),
        ("qx", ctypes.c_double), ("qz", ctypes.c_double), ("qt_x", ctypes.c_double),
        ("qt_z", ctypes.c_double), ("qxt", ctypes.c_double),
        ("w_vx_table", ctypes.c_void_p), ("w_vz_table", ctypes.c_void_p),
        ("w_tau_table", ctypes.c_void_p),
        ("a", ctypes.c_void_p),
        ("dt", ctypes.c_double), ("dtx", ctypes.c_double), ("dtz", ctypes.c_double),
        ("nt", ctypes.c_int32),
        ("src_i", ctypes.c_int32), ("src_j", ctypes.c_int32),
        ("wavelet", ctypes.c_void_p), ("n_wavelet", ctypes.c_int32),
        ("n_rec", ctypes.c_int32),
        ("rec_i", ctypes.c_void_p), ("rec_j", ctypes.c_void_p),
        ("rec_kind", ctypes.c_int32),
        ("habc_mode", ctypes.c_int32), ("contract", ctypes.c_int32),
        ("n_threads", ctypes.c_int32),
    ]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (``make -C oracle``)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        L.orc_fd_coefficients_f32.argtypes = [ctypes.c_int, P]
        L.orc_fd_coefficients_f64.argtypes = [ctypes.c_int, P]
        L.orc_ricker_f32.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_int, P]
        L.orc_ricker_f64.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, P]
        L.orc_init_medium_f32.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [P] * 5
        L.orc_init_medium_f64.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [P] * 5
        L.orc_habc_coefficients_f32.argtypes = [ctypes.c_float] * 4 + [P]
        L.orc_habc_coefficients_f64.argtypes = [ctypes.c_double] * 4 + [P]
        L.orc_habc_weight_table_f32.argtypes = [ctypes.c_int, ctypes.c_double, P]
        L.orc_habc_weight_table_f64.argtypes = [ctypes.c_int, ctypes.c_double, P]
        L.orc_habc_weights_full_f32.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, P]
        L.orc_coord_to_index.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_int]
        L.orc_coord_to_index.restype = ctypes.c_int
        L.orc_run_shot_f32.argtypes = [ctypes.POINTER(OrcShot), P, P, ctypes.c_int]
        L.orc_run_shot_f64.argtypes = [ctypes.POINTER(OrcShot), P, P, ctypes.c_int]
        L.orc_max_threads.restype = ctypes.c_int
        L.orc_create_geometry.argtypes = ([ctypes.c_int] * 3 + [P, P, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                           ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [P] * 6)
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def max_threads() -> int:
    return lib().orc_max_threads()


# --------------------------------------------------------------------------
# init.jl restatements (src/utils/init.jl)
# --------------------------------------------------------------------------

def fd_coefficients(order: int, dtype=np.float32) -> np.ndarray:
    """get_fd_coefficients (src/utils/init.jl:13-29); order 12 from the Taylor system."""
    out = np.zeros(8, dtype=dtype)
    f = lib().orc_fd_coefficients_f32 if dtype == np.float32 else lib().orc_fd_coefficients_f64
    m = f(int(order), _p(out))
    if m < 0:
        raise ValueError(f"Unsupported FD order: {order}")
    return out[:m].copy()


def ricker(f0: float, dt: float, nt: int, dtype=np.float32) -> np.ndarray:
    """ricker_wavelet (src/utils/init.jl:40-49)."""
    out = np.zeros(nt, dtype=dtype)
    if dtype == np.float32:
        lib().orc_ricker_f32(float(np.float32(f0)), float(np.float32(dt)), nt, _p(out))
    else:
        lib().orc_ricker_f64(float(f0), float(dt), nt, _p(out))
    return out


@dataclass
class OMedium:
    nx: int
    nz: int
    M: int
    pad: int
    nbc: int
    dx: float
    dz: float
    free_surface: bool
    rho_vx: np.ndarray
    rho_vz: np.ndarray
    lam: np.ndarray
    mu_txx: np.ndarray
    mu_txz: np.ndarray


def init_medium(vp, vs, rho, dx, dz, nbc, fd_order, free_surface=True, dtype=np.float32) -> OMedium:
    """init_medium (src/utils/init.jl:68-99).  vp/vs/rho: (nx_in, nz_in)."""
    vp = np.asfortranarray(vp, dtype=np.float32)
    vs = np.asfortranarray(vs, dtype=np.float32)
    rho = np.asfortranarray(rho, dtype=np.float32)
    nx_in, nz_in = vp.shape
    M = fd_order // 2
    pad = nbc + M
    nx, nz = nx_in + 2 * pad, nz_in + 2 * pad
    outs = [np.zeros((nx, nz), dtype=dtype, order="F") for _ in range(5)]
    f = lib().orc_init_medium_f32 if dtype == np.float32 else lib().orc_init_medium_f64
    f(_p(vp), _p(vs), _p(rho), nx_in, nz_in, pad, *[_p(o) for o in outs])
    return OMedium(nx, nz, M, pad, nbc, float(np.float32(dx)), float(np.float32(dz)), bool(free_surface), *outs)


@dataclass
class OHabc:
    nbc: int
    q: np.ndarray          # qx, qz, qt_x, qt_z, qxt
    w_vx: np.ndarray       # tables by dist, nbc+2 entries
    w_vz: np.ndarray
    w_tau: np.ndarray


def init_habc(nbc, dt, dx, dz, v_ref, dtype=np.float32) -> OHabc:
    """init_habc (src/utils/init.jl:171-203), weights as tables by dist."""
    L = lib()
    q = np.zeros(5, dtype=dtype)
    tabs = [np.zeros(nbc + 2, dtype=dtype) for _ in range(3)]
    if dtype == np.float32:
        L.orc_habc_coefficients_f32(float(np.float32(v_ref)), float(np.float32(dt)),
                                    float(np.float32(dx)), float(np.float32(dz)), _p(q))
        for t, off in zip(tabs, (0.0, 0.5, 0.75)):
            L.orc_habc_weight_table_f32(nbc, off, _p(t))
    else:
        L.orc_habc_coefficients_f64(float(v_ref), float(dt), float(dx), float(dz), _p(q))
        for t, off in zip(tabs, (0.0, 0.5, 0.75)):
            L.orc_habc_weight_table_f64(nbc, off, _p(t))
    return OHabc(nbc, q, *tabs)


def habc_weights_full(nx, nz, nbc, off) -> np.ndarray:
    """The reference's full (nz, nx) weight matrix, w[j-1, i-1], column-major."""
    w = np.zeros((nz, nx), dtype=np.float32, order="F")
    lib().orc_habc_weights_full_f32(nx, nz, nbc, float(off), _p(w))
    return w


def coord_to_index(x: float, dx: float, pad: int) -> int:
    """round(Int, x/dx) + pad + 1, Float32 division, ties to even
    (src/utils/init.jl:220-221, src/simulation/shot_manager.jl:189-191)."""
    return int(lib().orc_coord_to_index(float(np.float32(x)), float(np.float32(dx)), int(pad)))


def create_geometry(src_i, src_j, rec_i, rec_j, pad, dx, dz, dt, nt, nx, nz) -> dict:
    """create_geometry (src/io/geometry_io.jl:85-130) for one shot's 1-based
    padded-grid indices: discretised coordinates, indices relative to the
    physical domain, t_max and the physical grid size."""
    ri = np.ascontiguousarray(rec_i, dtype=np.int32)
    rj = np.ascontiguousarray(rec_j, dtype=np.int32)
    n = ri.size
    gf = np.zeros(3, np.float32)
    gi = np.zeros(4, np.int32)
    rx, rz = np.zeros(n, np.float32), np.zeros(n, np.float32)
    rip, rjp = np.zeros(n, np.int32), np.zeros(n, np.int32)
    lib().orc_create_geometry(int(src_i), int(src_j), n, _p(ri), _p(rj), int(pad), float(np.float32(dx)),
                              float(np.float32(dz)), float(np.float32(dt)), int(nt), int(nx), int(nz),
                              _p(gf), _p(gi), _p(rx), _p(rz), _p(rip), _p(rjp))
    return dict(src_x=gf[0], src_z=gf[1], t_max=gf[2], src_i=int(gi[0]), src_j=int(gi[1]), nx=int(gi[2]),
                nz=int(gi[3]), rec_x=rx, rec_z=rz, rec_i=rip, rec_j=rjp)


# --------------------------------------------------------------------------
# run_shot! (src/simulation/shot_manager.jl:46-68) over time_step!
# (src/simulation/time_stepper.jl:39-63)
# --------------------------------------------------------------------------

def run_shot(med: OMedium, habc: OHabc, a, dt, nt, src_i, src_j, wavelet, rec_i, rec_j,
             rec_kind="vz", habc_mode="simd8", contract=0, dtype=np.float32,
             dtx=None, dtz=None, final_fields=False, n_steps=None, n_threads=0):
    """Run one shot; returns the gather (nt, n_rec) [and the final fields
    vx, vz, txx, tzz, txz as an (nx, nz, 5) array]."""
    T = dtype
    arrs = [np.asfortranarray(x, dtype=T) for x in
            (med.rho_vx, med.rho_vz, med.lam, med.mu_txx, med.mu_txz)]
    a = np.ascontiguousarray(a, dtype=T)
    wav = np.ascontiguousarray(wavelet, dtype=T)
    tabs = [np.ascontiguousarray(t, dtype=T) for t in (habc.w_vx, habc.w_vz, habc.w_tau)]
    ri = np.ascontiguousarray(rec_i, dtype=np.int32)
    rj = np.ascontiguousarray(rec_j, dtype=np.int32)
    if T == np.float32:
        dt_ = np.float32(dt)
        dtx = np.float32(dt_ / np.float32(med.dx)) if dtx is None else np.float32(dtx)
        dtz = np.float32(dt_ / np.float32(med.dz)) if dtz is None else np.float32(dtz)
    else:
        dt_ = float(dt)
        dtx = dt_ / med.dx if dtx is None else float(dtx)
        dtz = dt_ / med.dz if dtz is None else float(dtz)
    s = OrcShot()
    s.nx, s.nz, s.M, s.pad, s.nbc = med.nx, med.nz, med.M, med.pad, med.nbc
    s.free_surface = int(med.free_surface)
    s.rho_vx, s.rho_vz, s.lam, s.mu_txx, s.mu_txz = [x.ctypes.data for x in arrs]
    s.qx, s.qz, s.qt_x, s.qt_z, s.qxt = [float(v) for v in habc.q]
    s.w_vx_table, s.w_vz_table, s.w_tau_table = [t.ctypes.data for t in tabs]
    s.a = a.ctypes.data
    s.dt, s.dtx, s.dtz = float(dt_), float(dtx), float(dtz)
    s.nt = int(nt)
    s.src_i, s.src_j = int(src_i), int(src_j)
    s.wavelet, s.n_wavelet = wav.ctypes.data, int(wav.size)
    s.n_rec = int(ri.size)
    s.rec_i, s.rec_j = ri.ctypes.data, rj.ctypes.data
    s.rec_kind = REC_KIND[rec_kind] if isinstance(rec_kind, str) else int(rec_kind)
    s.habc_mode = HABC_MODE[habc_mode] if isinstance(habc_mode, str) else int(habc_mode)
    s.contract = int(contract)
    s.n_threads = int(n_threads)
    gather = np.zeros((nt, ri.size), dtype=T, order="F")
    fin = np.zeros((med.nx, med.nz, 5), dtype=T, order="F") if final_fields else None
    f = lib().orc_run_shot_f32 if T == np.float32 else lib().orc_run_shot_f64
    rc = f(ctypes.byref(s), _p(gather), _p(fin) if fin is not None else None,
           -1 if n_steps is None else int(n_steps))
    if rc != 0:
        raise RuntimeError(f"oracle run_shot failed ({rc})")
    return (gather, fin) if final_fields else gather
