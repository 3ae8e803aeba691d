"""Host-side mirror of the reference's Elastic2D API for ``backend(:b200)``.

Same names, argument meaning and error behaviour as Wuheng10086/Fomo_julia's
``src/Elastic2D.jl`` exports for the time-stepping path, with Julia's ``!``
dropped (``run_shots!`` -> ``run_shots``).  Set-up (``init_medium``,
``init_habc``, ``ricker_wavelet``, ``setup_receivers``) runs on the host in
Float32 arithmetic, as the reference's does, and uploads through the C ABI;
every time step runs in libfomo_b200.so on the GPU.  There is no CPU backend
and no fallback.

Arrays follow the reference's layout: a grid is a numpy array of shape
``(nx, nz)`` stored column-major (x fastest), so ``a[i-1, j-1]`` is the
reference's ``a[i, j]``; a gather is ``(nt, n_rec)`` column-major.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field
from fractions import Fraction
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import FomoHabc, FomoRunStats, FomoShot, call

f32 = np.float32

# ---------------------------------------------------------------------------
# Backends  (src/backends/backend.jl:10-79)
# ---------------------------------------------------------------------------


class AbstractBackend:
    pass


@dataclass(frozen=True)
class B200Backend(AbstractBackend):
    """The B200 backend: every kernel runs in libfomo_b200.so on ``device``."""
    device: int = 0


B200_BACKEND = B200Backend(0)


def backend(name) -> B200Backend:
    """backend(name) (backend.jl:39-53).  Only :b200 exists in this package."""
    key = str(name).lstrip(":").lower()
    if key in ("b200",):
        _lib.ensure_init(B200_BACKEND.device)
        return B200_BACKEND
    raise ValueError(f"Unknown backend: {name}. This package provides :b200 only "
                     f"(the reference's :cpu and :cuda backends live in its Julia package)")


@dataclass
class DeviceArray:
    """A Float32 device buffer owned by the library (to_device result)."""
    handle: int
    shape: tuple
    nbytes: int

    def to_host(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=f32, order="F")
        call("fomo_b200_download", self.handle, out.ctypes.data, self.nbytes)
        return out

    def fill(self, value: float) -> None:
        call("fomo_b200_memset", self.handle, float(value))

    def free(self) -> None:
        if self.handle:
            call("fomo_b200_free", self.handle)
            self.handle = 0


def to_device(data, b: B200Backend = B200_BACKEND) -> DeviceArray:
    """to_device(data, backend) (backend.jl:68-71)."""
    _lib.ensure_init(b.device)
    a = np.asfortranarray(data, dtype=f32)
    h = ctypes.c_uint64(0)
    call("fomo_b200_alloc", a.nbytes, ctypes.byref(h))
    call("fomo_b200_upload", h.value, a.ctypes.data, a.nbytes)
    return DeviceArray(h.value, a.shape, a.nbytes)


def synchronize(b: B200Backend = B200_BACKEND) -> None:
    """synchronize(backend) (backend.jl:78-79)."""
    call("fomo_b200_synchronize")


STEP_KERNELS = {"auto": 0, "split": 1, "fused": 2}


def set_step_kernel(mode: str = "auto", n_segs: int = 0) -> None:
    """Time-step kernels of single shots (no reference counterpart).  "split":
    four launches per step (velocity tiles, velocity band pass, stress
    tiles, stress band pass); "fused": one launch per step computing velocity
    and stress in column strips (fails a shot it cannot run); "auto": times
    both on the first long enough shot of a grid and keeps the faster.
    n_segs > 0 fixes the fused step's row segments per column strip.  Results
    are the same bit for bit."""
    call("fomo_b200_set_step_kernel", STEP_KERNELS[mode], int(n_segs))


# ---------------------------------------------------------------------------
# Initialisation  (src/utils/init.jl)
# ---------------------------------------------------------------------------

FD_COEFFICIENTS = {
    2: np.array([1.0], dtype=f32),
    4: np.array([1.125, -0.041666667], dtype=f32),
    6: np.array([1.171875, -0.065104167, 0.0046875], dtype=f32),
    8: np.array([1.1962890625, -0.079752604167, 0.0095703125, -0.000697544643], dtype=f32),
    10: np.array([1.2115478515625, -0.089721679687, 0.0138427734375, -0.00176565987723,
                  0.0001186795166], dtype=f32),
}


def taylor_coefficients(M: int) -> List[Fraction]:
    """Exact staggered-grid Taylor coefficients: sum_l a_l (2l-1)^(2k-1) = [k == 1]."""
    A = [[Fraction((2 * l + 1) ** (2 * k + 1)) for l in range(M)] for k in range(M)]
    b = [Fraction(1 if k == 0 else 0) for k in range(M)]
    for c in range(M):
        p = next(r for r in range(c, M) if A[r][c] != 0)
        A[c], A[p] = A[p], A[c]
        b[c], b[p] = b[p], b[c]
        for r in range(M):
            if r != c and A[r][c] != 0:
                f = A[r][c] / A[c][c]
                A[r] = [x - f * y for x, y in zip(A[r], A[c])]
                b[r] -= f * b[c]
    return [b[r] / A[r][r] for r in range(M)]


def get_fd_coefficients(order: int) -> np.ndarray:
    """get_fd_coefficients (init.jl:13-29).  Order 12 (beyond the reference's
    table) comes from the same Taylor system that gives orders 2-10."""
    if order in FD_COEFFICIENTS:
        return FD_COEFFICIENTS[order].copy()
    if order == 12:
        return np.array([float(c) for c in taylor_coefficients(6)], dtype=f32)
    raise ValueError(f"Unsupported FD order: {order}")


def ricker_wavelet(f0, dt, nt: int) -> np.ndarray:
    """ricker_wavelet (init.jl:40-49) with Julia's promotion rules for Float32
    f0 and dt: (i-1)*dt and pi*f0 are Float32 products, the rest Float64."""
    f0 = f32(f0)
    dt = f32(dt)
    t0 = 1.0 / float(f0)
    pif0 = float(f32(f32(math.pi) * f0))
    out = np.zeros(nt, dtype=f32)
    for i in range(1, nt + 1):
        tau = float(f32(f32(i - 1) * dt)) - t0
        x = pif0 * tau
        arg = x * x
        out[i - 1] = f32((1.0 - 2.0 * arg) * math.exp(-arg))
    return out


def julia_mean(a) -> np.float32:
    """Statistics.mean of a Float32 array as Julia computes it -- the v_ref of
    run.jl:57: Base's pairwise mapreduce (split at the midpoint until a block
    holds fewer than 1024 elements), then one Float32 division by the length.

    Each block is summed strictly in order here (np.cumsum accumulates in
    Float32, one element after the other).  Julia's block loop carries
    ``@simd``, which lets LLVM reassociate it into vector partial sums whose
    shape depends on the host's vector width; that shape cannot be pinned
    without Julia, so this order is exact only where the block sums are
    (every constant-valued model, including the run.jl golden case)."""
    v = np.asfortranarray(a, dtype=f32).ravel(order="F")
    if v.size == 0:
        return f32(np.nan)

    def rec(i0: int, i1: int) -> np.float32:
        if i0 == i1:
            return v[i0]
        if i1 - i0 < 1024:
            return np.cumsum(v[i0:i1 + 1], dtype=f32)[-1]
        im = i0 + ((i1 - i0) >> 1)
        return f32(rec(i0, im) + rec(im + 1, i1))

    return f32(rec(0, v.size - 1) / f32(v.size))


@dataclass
class Medium:
    """Medium{T} (Structures.jl:66-83).  Host copies of the staggered arrays
    are kept; `handle` is the library's device copy."""
    nx: int
    nz: int
    dx: float
    dz: float
    x_max: float
    z_max: float
    M: int
    pad: int
    is_free_surface: bool
    rho_vx: np.ndarray
    rho_vz: np.ndarray
    lam: np.ndarray
    mu_txx: np.ndarray
    mu_txz: np.ndarray
    handle: int = 0
    device: int = 0

    def upload(self) -> int:
        if not self.handle:
            _lib.ensure_init(self.device)
            h = ctypes.c_uint64(0)
            arrs = [np.asfortranarray(x, dtype=f32) for x in
                    (self.rho_vx, self.rho_vz, self.lam, self.mu_txx, self.mu_txz)]
            call("fomo_b200_medium_create", self.nx, self.nz, self.M, self.pad,
                 int(self.is_free_surface), float(self.dx), float(self.dz),
                 *[x.ctypes.data for x in arrs], ctypes.byref(h))
            self.handle = h.value
        return self.handle

    def array(self, q: int) -> np.ndarray:
        """Array q (0 rho_vx, 1 rho_vz, 2 lam, 3 mu_txx, 4 mu_txz) as the device holds it."""
        out = np.zeros((self.nx, self.nz), dtype=f32, order="F")
        call("fomo_b200_medium_download", self.upload(), int(q), out.ctypes.data)
        return out

    def release(self) -> None:
        if self.handle:
            call("fomo_b200_medium_destroy", self.handle)
            self.handle = 0


def pad_array(data, pad: int) -> np.ndarray:
    """_pad_array (init.jl:119-134): edge replication by `pad` cells."""
    return np.asfortranarray(np.pad(np.asarray(data, dtype=f32), pad, mode="edge"))


def compute_staggered_params(vp, vs, rho):
    """_compute_staggered_params (init.jl:136-158), Float32 arithmetic."""
    vp = np.asarray(vp, dtype=f32)
    vs = np.asarray(vs, dtype=f32)
    rho = np.asarray(rho, dtype=f32)
    mu = rho * (vs * vs)
    lam = rho * (vp * vp) - f32(2.0) * mu
    rho_vx = rho.copy()
    rho_vz = np.zeros_like(rho)
    rho_vz[:-1, :-1] = f32(0.25) * (((rho[:-1, :-1] + rho[1:, :-1]) + rho[:-1, 1:]) + rho[1:, 1:])
    rho_vz[-1, :] = rho_vz[-2, :]
    rho_vz[:, -1] = rho_vz[:, -2]
    mu_txz = np.zeros_like(mu)
    with np.errstate(divide="ignore"):
        mu_txz[:, :-1] = f32(2.0) / ((f32(1.0) / mu[:, :-1]) + (f32(1.0) / mu[:, 1:]))
    mu_txz[:, -1] = mu_txz[:, -2]
    F = np.asfortranarray
    return F(lam), F(mu), F(mu_txz), F(rho_vx), F(rho_vz)


def init_medium(vp, vs, rho, dx, dz, nbc: int, fd_order: int, b: B200Backend = B200_BACKEND,
                free_surface: bool = True) -> Medium:
    """init_medium (init.jl:68-99).  vp, vs, rho: (nx_in, nz_in) arrays."""
    if fd_order % 2 or not 2 <= fd_order <= 12:
        raise ValueError(f"Unsupported FD order: {fd_order}")
    M = fd_order // 2
    pad = nbc + M
    vp = np.asarray(vp)
    if vp.ndim != 2 or np.shape(vs) != vp.shape or np.shape(rho) != vp.shape:
        raise ValueError("vp, vs and rho must be matrices of the same size")
    nx_in, nz_in = vp.shape
    nx, nz = nx_in + 2 * pad, nz_in + 2 * pad
    x_max = float(f32((nx_in - 1) * float(f32(dx))))
    z_max = float(f32((nz_in - 1) * float(f32(dz))))
    lam, mu, mu_txz, rho_vx, rho_vz = compute_staggered_params(
        pad_array(vp, pad), pad_array(vs, pad), pad_array(rho, pad))
    m = Medium(nx, nz, float(f32(dx)), float(f32(dz)), x_max, z_max, M, pad, bool(free_surface),
               rho_vx, rho_vz, lam, mu, mu_txz, device=b.device)
    m.upload()
    return m


def init_medium_device(vp, vs, rho, dx, dz, nbc: int, fd_order: int, b: B200Backend = B200_BACKEND,
                       free_surface: bool = True) -> Medium:
    """init_medium with the padding and staggered parameters computed on the
    GPU (fomo_b200_medium_create_from_model): the same medium bit for bit,
    without the host-side set-up.  The returned Medium holds no host copies
    (download them with Medium.array)."""
    if fd_order % 2 or not 2 <= fd_order <= 12:
        raise ValueError(f"Unsupported FD order: {fd_order}")
    M = fd_order // 2
    pad = nbc + M
    arrs = [np.asfortranarray(a, dtype=f32) for a in (vp, vs, rho)]
    if arrs[0].ndim != 2 or arrs[1].shape != arrs[0].shape or arrs[2].shape != arrs[0].shape:
        raise ValueError("vp, vs and rho must be matrices of the same size")
    nx_in, nz_in = arrs[0].shape
    _lib.ensure_init(b.device)
    h = ctypes.c_uint64(0)
    call("fomo_b200_medium_create_from_model", nx_in, nz_in, *[a.ctypes.data for a in arrs], float(f32(dx)),
         float(f32(dz)), int(nbc), M, int(free_surface), ctypes.byref(h))
    x_max = float(f32((nx_in - 1) * float(f32(dx))))
    z_max = float(f32((nz_in - 1) * float(f32(dz))))
    return Medium(nx_in + 2 * pad, nz_in + 2 * pad, float(f32(dx)), float(f32(dz)), x_max, z_max, M, pad,
                  bool(free_surface), None, None, None, None, None, handle=h.value, device=b.device)


@dataclass
class HABCConfig:
    """HABCConfig{T} (Structures.jl:94-105).  The weight matrices of the
    reference depend on dist = min(i-1, nx-i, j-1, nz-j) only; they are kept
    as tables over dist = 0..nbc+1."""
    nbc: int
    qx: np.float32
    qz: np.float32
    qt_x: np.float32
    qt_z: np.float32
    qxt: np.float32
    w_vx: np.ndarray
    w_vz: np.ndarray
    w_tau: np.ndarray

    def weight_matrix(self, which: str, nx: int, nz: int) -> np.ndarray:
        """The reference's full (nz, nx) weight matrix for 'vx', 'vz' or 'tau'."""
        tab = {"vx": self.w_vx, "vz": self.w_vz, "tau": self.w_tau}[which]
        i = np.arange(1, nx + 1)[None, :]
        j = np.arange(1, nz + 1)[:, None]
        d = np.minimum(np.minimum(i - 1, nx - i), np.minimum(j - 1, nz - j))
        return tab[np.minimum(d, self.nbc + 1)]


def habc_weight_table(nbc: int, off: float) -> np.ndarray:
    d = np.arange(nbc + 2, dtype=np.float64)
    return np.clip((d - off) / nbc, 0.0, 1.0).astype(f32)


def init_habc(nx: int, nz: int, nbc: int, dt, dx, dz, v_ref, b: B200Backend = B200_BACKEND) -> HABCConfig:
    """init_habc (init.jl:171-203), Float32 arithmetic as the reference's."""
    if nbc < 1:
        raise ValueError(f"nbc must be >= 1, got {nbc}")
    dt, dx, dz, v_ref = f32(dt), f32(dx), f32(dz), f32(v_ref)
    rx = f32(f32(v_ref * dt) / dx)
    rz = f32(f32(v_ref * dt) / dz)
    b_p, beta, one = f32(0.45), f32(1.0), f32(1.0)
    omb = f32(one - b_p)

    def q(r, num_sub):
        return f32(f32(f32(b_p * f32(beta + r)) - num_sub) / f32(f32(beta + r) * omb))

    qx = q(rx, rx)
    qz = q(rz, rz)
    qt_x = q(rx, beta)
    qt_z = q(rz, beta)
    qxt = f32(b_p / f32(b_p - one))
    return HABCConfig(nbc, qx, qz, qt_x, qt_z, qxt, habc_weight_table(nbc, 0.0),
                      habc_weight_table(nbc, 0.5), habc_weight_table(nbc, 0.75))


# ---------------------------------------------------------------------------
# Structures  (src/core/Structures.jl)
# ---------------------------------------------------------------------------

@dataclass
class SimParams:
    dt: np.float32
    nt: int
    dtx: np.float32
    dtz: np.float32
    fd_order: int
    M: int

    @classmethod
    def make(cls, dt, nt: int, dx, dz, fd_order: int) -> "SimParams":
        """SimParams(dt, nt, dx, dz, fd_order) (Structures.jl:152-155)."""
        dt = f32(dt)
        return cls(dt, int(nt), f32(dt / f32(dx)), f32(dt / f32(dz)), int(fd_order), int(fd_order) // 2)


def sim_params(dt, nt: int, dx, dz, fd_order: int) -> SimParams:
    return SimParams.make(dt, nt, dx, dz, fd_order)


class Wavefield:
    """Wavefield(nx, nz, backend) (Structures.jl:39-55): the library's
    device state of one shot.  Field properties download the current value."""

    FIELDS = ("vx", "vz", "txx", "tzz", "txz")

    def __init__(self, nx: int, nz: int, b: B200Backend = B200_BACKEND):
        _lib.ensure_init(b.device)
        self.nx, self.nz = int(nx), int(nz)
        h = ctypes.c_uint64(0)
        call("fomo_b200_wavefield_create", self.nx, self.nz, ctypes.byref(h))
        self.handle = h.value

    def field(self, name: str) -> np.ndarray:
        out = np.empty((self.nx, self.nz), dtype=f32, order="F")
        call("fomo_b200_wavefield_download", self.handle, self.FIELDS.index(name), out.ctypes.data)
        return out

    def set_field(self, name: str, value) -> None:
        a = np.asfortranarray(value, dtype=f32)
        if a.shape != (self.nx, self.nz):
            raise ValueError(f"field shape {a.shape} != {(self.nx, self.nz)}")
        call("fomo_b200_wavefield_upload", self.handle, self.FIELDS.index(name), a.ctypes.data)

    vx = property(lambda self: self.field("vx"))
    vz = property(lambda self: self.field("vz"))
    txx = property(lambda self: self.field("txx"))
    tzz = property(lambda self: self.field("tzz"))
    txz = property(lambda self: self.field("txz"))

    def snapshot(self, field: str = "p", downsample: int = 1) -> np.ndarray:
        """One frame of the current state (fomo_b200_wavefield_snapshot):
        field p, vel, vx or vz, every downsample-th cell; (cld(nx, ds),
        cld(nz, ds)) Float32, column major."""
        kinds = {"p": 0, "vel": 1, "vx": 2, "vz": 3}
        if field not in kinds:
            raise ValueError(f"Unknown field: {field}. Use p, vel, vx, or vz")
        ds = int(downsample)
        if ds < 1:
            raise ValueError("downsample must be >= 1")
        out = np.zeros((-(-self.nx // ds), -(-self.nz // ds)), dtype=f32, order="F")
        call("fomo_b200_wavefield_snapshot", self.handle, kinds[field], ds, out.ctypes.data)
        return out

    def release(self) -> None:
        if self.handle:
            call("fomo_b200_wavefield_destroy", self.handle)
            self.handle = 0


def reset(b: B200Backend, W: Wavefield) -> None:
    """reset!(backend, W) (source_receiver.jl:115-133)."""
    call("fomo_b200_wavefield_reset", W.handle)


@dataclass
class Source:
    """Source{V,I} (Structures.jl:116-120): 1-based grid indices."""
    i: int
    j: int
    wavelet: np.ndarray


@dataclass
class Receivers:
    """Receivers{T,I} (Structures.jl:127-132): 1-based indices, data [nt x n_rec]."""
    i: np.ndarray
    j: np.ndarray
    data: np.ndarray
    type: str = "vz"


@dataclass
class TimeStepInfo:
    """TimeStepInfo (time_stepper.jl:17-21)."""
    k: int
    t: np.float32
    nt: int


@dataclass
class ShotResult:
    """ShotResult (shot_manager.jl:17-28)."""
    gather: np.ndarray
    shot_id: int
    src_i: int
    src_j: int
    rec_i: np.ndarray
    rec_j: np.ndarray
    stats: Optional[dict] = None


@dataclass
class ShotConfig:
    source_x: np.float32
    source_z: np.float32
    shot_id: int


@dataclass
class MultiShotConfig:
    """MultiShotConfig (shot_manager.jl:110-119)."""
    shots: List[ShotConfig]
    wavelet: np.ndarray
    source_type: str = "pressure"

    @classmethod
    def make(cls, x_positions: Sequence, z_positions: Sequence, wavelet, source_type: str = "pressure"):
        if len(x_positions) != len(z_positions):
            raise ValueError("x and z must have same length")
        shots = [ShotConfig(f32(x), f32(z), k + 1) for k, (x, z) in enumerate(zip(x_positions, z_positions))]
        return cls(shots, np.asarray(wavelet, dtype=f32), source_type)


def multi_shot_config(x_positions, z_positions, wavelet, source_type: str = "pressure") -> MultiShotConfig:
    return MultiShotConfig.make(x_positions, z_positions, wavelet, source_type)


REC_KIND = {"vz": 0, "vx": 1, "p": 2}


def coord_to_index(x, dx, pad: int) -> int:
    """round(Int32, x/dx) + pad + 1 with Float32 division, ties to even
    (shot_manager.jl:189-191)."""
    return int(np.rint(f32(f32(x) / f32(dx)))) + int(pad) + 1


def setup_receivers(x, z, M: Medium, type: str = "vz") -> Receivers:
    """setup_receivers (init.jl:214-227)."""
    x = np.asarray(x)
    z = np.asarray(z)
    if x.shape != z.shape:
        raise ValueError("x and z must have same length")
    if type not in REC_KIND:
        raise ValueError(f"unknown receiver type {type!r}")
    # Julia promotes Float32/Float32 and Int/Float32 to Float32, Float64/Float32 to Float64.
    xi = x / float(M.dx) if x.dtype == np.float64 else x.astype(f32) / f32(M.dx)
    zi = z / float(M.dz) if z.dtype == np.float64 else z.astype(f32) / f32(M.dz)
    i_rec = np.rint(xi).astype(np.int64) + M.pad + 1
    j_rec = np.rint(zi).astype(np.int64) + M.pad + 1
    return Receivers(i_rec, j_rec, np.zeros((1, len(x)), dtype=f32, order="F"), type)


# ---------------------------------------------------------------------------
# Shots  (src/simulation/shot_manager.jl, time_stepper.jl)
# ---------------------------------------------------------------------------

def _ctypes_shot(a, params: SimParams, src: Source, rec: Receivers, keep: list) -> FomoShot:
    a = np.ascontiguousarray(a, dtype=f32)
    wav = np.ascontiguousarray(src.wavelet, dtype=f32)
    ri = np.ascontiguousarray(rec.i, dtype=np.int32)
    rj = np.ascontiguousarray(rec.j, dtype=np.int32)
    keep += [a, wav, ri, rj]
    s = FomoShot()
    s.a, s.M = a.ctypes.data, a.size
    s.dt, s.dtx, s.dtz = float(params.dt), float(params.dtx), float(params.dtz)
    s.nt = int(params.nt)
    s.src_i, s.src_j = int(src.i), int(src.j)
    s.wavelet, s.n_wavelet = wav.ctypes.data, wav.size
    s.n_rec = ri.size
    s.rec_i, s.rec_j = (ri.ctypes.data if ri.size else None), (rj.ctypes.data if rj.size else None)
    s.rec_kind = REC_KIND[rec.type]
    return s


def _ctypes_habc(H: HABCConfig, keep: list) -> FomoHabc:
    tabs = [np.ascontiguousarray(t, dtype=f32) for t in (H.w_vx, H.w_vz, H.w_tau)]
    keep += tabs
    h = FomoHabc()
    h.nbc = H.nbc
    h.qx, h.qz, h.qt_x, h.qt_z, h.qxt = (float(H.qx), float(H.qz), float(H.qt_x), float(H.qt_z), float(H.qxt))
    h.w_vx, h.w_vz, h.w_tau = [t.ctypes.data for t in tabs]
    return h


def _stats_dict(st: FomoRunStats) -> dict:
    return {"device_ms": st.device_ms, "steps": st.steps, "kernel_launches": st.kernel_launches,
            "h2d_bytes": st.h2d_bytes, "d2h_bytes": st.d2h_bytes}


def run_shot(b: B200Backend, W: Wavefield, M: Medium, H: HABCConfig, a, src: Source, rec: Receivers,
             params: SimParams, shot_id: int = 1, progress: bool = False,
             on_step: Optional[Callable] = None, step_chunk: int = 1,
             gather_path: Optional[str] = None) -> ShotResult:
    """run_shot! (shot_manager.jl:46-68): reset, run nt steps, return the
    gather on the host.  With `on_step` the loop runs in chunks of
    `step_chunk` steps and calls on_step(W, TimeStepInfo) after each chunk;
    a False return stops the shot early (time_stepper.jl:112-119).  With
    `gather_path` the gather is also written there as save_gather's raw
    .bin (output.jl:28-33), straight from the device seismogram."""
    if gather_path is not None and on_step is None:
        on_step, step_chunk = (lambda W_, info: None), params.nt
    keep: list = []
    hs = _ctypes_habc(H, keep)
    ss = _ctypes_shot(a, params, src, rec, keep)
    n_rec = ss.n_rec
    gather = np.zeros((params.nt, n_rec), dtype=f32, order="F")
    st = FomoRunStats()
    mh = M.upload()
    if on_step is None:
        call("fomo_b200_run_shot", mh, W.handle, ctypes.byref(hs), ctypes.byref(ss),
             gather.ctypes.data if gather.size else None, ctypes.byref(st))
    else:
        sh = ctypes.c_uint64(0)
        call("fomo_b200_shot_begin", mh, W.handle, ctypes.byref(hs), ctypes.byref(ss), ctypes.byref(sh))
        k = ctypes.c_int32(0)
        try:
            while k.value < params.nt:
                call("fomo_b200_shot_advance", sh.value, max(1, int(step_chunk)), ctypes.byref(k))
                info = TimeStepInfo(k.value, f32(k.value * params.dt), params.nt)
                if on_step(W, info) is False:
                    break
            if gather_path is not None:
                call("fomo_b200_shot_save_gather", sh.value, os.fsencode(gather_path))
        finally:
            call("fomo_b200_shot_finish", sh.value, gather.ctypes.data if gather.size else None,
                 ctypes.byref(st))
    return ShotResult(gather, int(shot_id), int(src.i), int(src.j), np.asarray(rec.i, dtype=np.int64).copy(),
                      np.asarray(rec.j, dtype=np.int64).copy(), _stats_dict(st))


def create_source(M: Medium, shot: ShotConfig, wavelet) -> Source:
    """_create_source (shot_manager.jl:196-206)."""
    return Source(coord_to_index(shot.source_x, M.dx, M.pad), coord_to_index(shot.source_z, M.dz, M.pad),
                  np.asarray(wavelet, dtype=f32))


def run_shots(b: B200Backend, W: Wavefield, M: Medium, H: HABCConfig, a, rec_template: Receivers,
              shot_config: MultiShotConfig, params: SimParams,
              on_shot_complete: Optional[Callable] = None, on_step: Optional[Callable] = None,
              progress: bool = False, step_chunk: int = 1, batched: bool = False) -> List[ShotResult]:
    """run_shots! (shot_manager.jl:145-180): the shots in order, one after
    another, each with a fresh gather.

    batched=True runs all shots side by side instead (fomo_b200_run_batch:
    every time-step launch covers every shot in flight); the gathers are the
    same bit for bit, and `W` is not used.  on_step needs the sequential loop."""
    if batched:
        if on_step is not None:
            raise ValueError("on_step needs the sequential loop (batched=False)")
        results = run_batch(b, M, H, a, rec_template, shot_config, params)
        if on_shot_complete is not None:
            for r in results:
                on_shot_complete(r)
        return results
    results = []
    for shot in shot_config.shots:
        src = create_source(M, shot, shot_config.wavelet)
        rec = Receivers(np.asarray(rec_template.i).copy(), np.asarray(rec_template.j).copy(),
                        np.zeros((params.nt, len(rec_template.i)), dtype=f32, order="F"), rec_template.type)
        r = run_shot(b, W, M, H, a, src, rec, params, shot_id=shot.shot_id, progress=progress,
                     on_step=on_step, step_chunk=step_chunk)
        results.append(r)
        if on_shot_complete is not None:
            on_shot_complete(r)
    return results


def run_batch(b: B200Backend, M: Medium, H: HABCConfig, a, rec_template: Receivers,
              shot_config: MultiShotConfig, params: SimParams) -> List[ShotResult]:
    """The shots of `shot_config` on one medium, run side by side
    (fomo_b200_run_batch).  Returns one ShotResult per shot, in order; the
    first result's stats cover the whole batch."""
    keep: list = []
    hs = _ctypes_habc(H, keep)
    n = len(shot_config.shots)
    shots = (FomoShot * max(n, 1))()
    gathers, srcs = [], []
    for k, shot in enumerate(shot_config.shots):
        src = create_source(M, shot, shot_config.wavelet)
        srcs.append(src)
        shots[k] = _ctypes_shot(a, params, src, rec_template, keep)
        gathers.append(np.zeros((params.nt, len(rec_template.i)), dtype=f32, order="F"))
    ptrs = (ctypes.c_void_p * max(n, 1))(*[g.ctypes.data if g.size else None for g in gathers])
    st = FomoRunStats()
    mh = M.upload()
    call("fomo_b200_run_batch", mh, ctypes.byref(hs), shots, n, ptrs, ctypes.byref(st))
    return [ShotResult(gathers[k], int(shot.shot_id), int(srcs[k].i), int(srcs[k].j),
                       np.asarray(rec_template.i, dtype=np.int64).copy(),
                       np.asarray(rec_template.j, dtype=np.int64).copy(),
                       _stats_dict(st) if k == 0 else None)
            for k, shot in enumerate(shot_config.shots)]


# ---------------------------------------------------------------------------
# Gather output  (src/io/output.jl)
# ---------------------------------------------------------------------------

def save_gather(result: ShotResult, path: str, format: str = "bin") -> None:
    """save_gather (output.jl:18-33): raw little-endian Float32, column
    major [nt x n_rec], no header."""
    if format != "bin":
        raise ValueError(f"Unknown format: {format}")
    np.asfortranarray(result.gather, dtype="<f4").ravel(order="F").tofile(path)


def load_gather(path: str, nt: int, n_rec: int) -> np.ndarray:
    """load_gather (output.jl:61-67)."""
    d = np.fromfile(path, dtype="<f4", count=nt * n_rec)
    return np.asfortranarray(d.reshape((nt, n_rec), order="F").astype(f32))
