"""Velocity-model loaders feeding init_medium (src/io/model_loader.jl).

``load_model`` dispatches on the extension as the reference does
(model_loader.jl:88-106).  Here:
* ``.bin``: raw binary (model_loader.jl:141-189).  nx and nz are required.
  dtype Float32 by default; order column-major (x fastest) or row-major.
  vs and rho come from files, from arrays, or are estimated from vp.
* ``.npy``: NumPy arrays (model_loader.jl:288-320).
* ``.segy``/``.sgy``: SEG-Y (model_loader.jl:199-248, which reads through
  SegyIO.jl's segy_read and takes its data matrix, samples x traces, as vp).
  Read here without SegyIO: ``read_segy`` below.
* ``.mat``: MATLAB v4/v5 files through scipy.io.loadmat (model_loader.jl:
  254-283: vp under vp_key, "Vp" or "VP"; vs under vs_key or "Vs"; rho under
  rho_key, "Rho" or "density"; missing vs and rho estimated).  v7.3 files are
  HDF5 and need a reader absent here.
* ``.jld2``, ``.h5``/``.hdf5`` need Julia or libraries not present here.
  They raise NotImplementedError naming the format; convert such models to
  .bin, .npy, SEG-Y or MAT v5 first.

Estimates as in the reference: vs = vp / 1.73 and rho = 310 vp^0.25 (Gardner),
in Float32.  numpy's float32 power may differ from Julia's in the last bit;
these estimates are set-up data, off the time-stepping path.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import Optional, Union

import numpy as np

f32 = np.float32


@dataclass
class VelocityModel:
    """VelocityModel (model_loader.jl:27-38)."""
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    dx: np.float32
    dz: np.float32
    nx: int
    nz: int
    x_origin: np.float32 = f32(0)
    z_origin: np.float32 = f32(0)
    name: str = "unnamed"

    @classmethod
    def make(cls, vp, vs, rho, dx, dz, x_origin=0.0, z_origin=0.0, name="unnamed") -> "VelocityModel":
        vp, vs, rho = (np.asfortranarray(a, dtype=f32) for a in (vp, vs, rho))
        if vs.shape != vp.shape:
            raise ValueError("vs size mismatch")
        if rho.shape != vp.shape:
            raise ValueError("rho size mismatch")
        nx, nz = vp.shape
        return cls(vp, vs, rho, f32(dx), f32(dz), int(nx), int(nz), f32(x_origin), f32(z_origin), name)


def estimate_vs(vp) -> np.ndarray:
    """vp ./ 1.73f0 (model_loader.jl:163)."""
    vp = np.asarray(vp)
    return vp / (f32(1.73) if vp.dtype == np.float32 else 1.73)


def gardner_rho(vp) -> np.ndarray:
    """310.0f0 .* (vp .^ 0.25f0) (model_loader.jl:173)."""
    vp = np.asarray(vp)
    if vp.dtype == np.float32:
        return f32(310.0) * np.power(vp, f32(0.25))
    return 310.0 * np.power(vp, 0.25)


def _read_bin(path, nx, nz, dtype, order):
    data = np.fromfile(path, dtype=np.dtype(dtype).newbyteorder("<"), count=nx * nz)
    if data.size != nx * nz:
        raise ValueError(f"{path}: {data.size} values, expected nx*nz = {nx * nz}")
    if order == "row_major":
        return np.asfortranarray(data.reshape((nz, nx)).T)
    if order != "column_major":
        raise ValueError(f"order must be column_major or row_major, got {order!r}")
    return np.asfortranarray(data.reshape((nx, nz), order="F"))


def _other(v, reader, vp, estimate):
    if isinstance(v, (str, os.PathLike)):
        return reader(v)
    if v is None:
        return estimate(vp)
    return np.asarray(v)


# ---------------------------------------------------------------- SEG-Y
# Layout (SEG-Y rev 0/1, big-endian): a 3200-byte textual header, a 400-byte
# binary header (samples per trace at byte 20, sample format code at byte 24,
# count of extended 3200-byte textual headers at byte 304), then traces of a
# 240-byte trace header and the samples.  Format codes: 1 IBM 4-byte float,
# 2 int32, 3 int16, 5 IEEE 4-byte float, 8 int8.
_SEGY_TEXT, _SEGY_BIN, _SEGY_TRACE_HDR = 3200, 400, 240
_SEGY_FORMATS = {1: ">u4", 2: ">i4", 3: ">i2", 5: ">f4", 8: "i1"}


def ibm_to_float32(words) -> np.ndarray:
    """IBM System/360 single-precision floats (32-bit words) to float32.

    An IBM float is sign s, 7-bit excess-64 exponent e and 24-bit fraction f:
    (-1)^s * (f / 2^24) * 16^(e - 64).  That value is exact in float64 and
    rounded once to float32 (values beyond float32's range become inf or
    round to zero or a subnormal)."""
    w = np.asarray(words, dtype=np.uint32)
    sign = np.where(w >> 31, -1.0, 1.0)
    expo = ((w >> 24) & 0x7F).astype(np.int64) - 64
    frac = (w & 0x00FFFFFF).astype(np.float64) / float(1 << 24)
    with np.errstate(over="ignore", under="ignore"):
        return (sign * np.ldexp(frac, 4 * expo)).astype(np.float32)


def float32_to_ibm(values) -> np.ndarray:
    """float32 to IBM single-precision words (the inverse of ibm_to_float32
    for values IBM can hold; the 24-bit fraction truncates, as IBM
    arithmetic does).  Zero maps to 0."""
    v = np.asarray(values, dtype=np.float64)
    out = np.zeros(v.shape, dtype=np.uint32)
    nz = v != 0
    a = np.abs(v[nz])
    expo = np.floor(np.log2(a) / 4).astype(np.int64) + 1  # a = frac * 16^expo with frac in [1/16, 1)
    frac = a / np.ldexp(1.0, 4 * expo)
    hi = frac >= 1.0                                      # guard the log2 rounding at powers of 16
    expo[hi] += 1
    frac[hi] /= 16.0
    lo = frac < 1.0 / 16
    expo[lo] -= 1
    frac[lo] *= 16.0
    f24 = np.floor(frac * (1 << 24)).astype(np.uint64)
    words = (np.where(v[nz] < 0, 1, 0).astype(np.uint64) << 31) | (((expo + 64) & 0x7F).astype(np.uint64) << 24) | f24
    out[nz] = words.astype(np.uint32)
    return out


def read_segy(path: str) -> np.ndarray:
    """The data matrix of a SEG-Y file as float32, samples x traces (the
    orientation of SegyIO's SeisBlock.data), for fixed-length traces."""
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size < _SEGY_TEXT + _SEGY_BIN:
        raise ValueError(f"{path}: {raw.size} bytes, too short for a SEG-Y file")
    bh = raw[_SEGY_TEXT:_SEGY_TEXT + _SEGY_BIN]
    ns = int(bh[20:22].view(">u2")[0])
    fmt = int(bh[24:26].view(">u2")[0])
    n_ext = int(bh[304:306].view(">i2")[0])
    if fmt not in _SEGY_FORMATS:
        raise ValueError(f"{path}: sample format code {fmt} not supported (1, 2, 3, 5, 8)")
    if ns <= 0:
        raise ValueError(f"{path}: {ns} samples per trace in the binary header")
    dt = np.dtype(_SEGY_FORMATS[fmt])
    start = _SEGY_TEXT + _SEGY_BIN + max(n_ext, 0) * _SEGY_TEXT
    trace_bytes = _SEGY_TRACE_HDR + ns * dt.itemsize
    body = raw.size - start
    if body < 0 or body % trace_bytes:
        raise ValueError(f"{path}: {body} bytes of traces is not a whole number of "
                         f"{trace_bytes}-byte traces (variable-length traces are not supported)")
    n_tr = body // trace_bytes
    traces = raw[start:].reshape(n_tr, trace_bytes)[:, _SEGY_TRACE_HDR:]
    samples = np.ascontiguousarray(traces).view(dt).reshape(n_tr, ns)
    data = ibm_to_float32(samples) if fmt == 1 else samples.astype(np.float32)
    return np.asfortranarray(data.T)


def write_segy(path: str, data, fmt: int = 5, sample_interval_us: int = 0) -> None:
    """Writes `data` (samples x traces) as a SEG-Y rev 1 file with IEEE
    (fmt 5) or IBM (fmt 1) 4-byte floats: blank EBCDIC textual header,
    binary header with the sample count and format, minimal trace headers."""
    if fmt not in (1, 5):
        raise ValueError("fmt must be 1 (IBM) or 5 (IEEE)")
    d = np.asarray(data, dtype=np.float32)
    if d.ndim != 2:
        raise ValueError("data must be a 2-D samples x traces array")
    ns, n_tr = d.shape
    text = np.full(_SEGY_TEXT, 0x40, dtype=np.uint8)  # EBCDIC spaces
    bh = np.zeros(_SEGY_BIN, dtype=np.uint8)
    bh[16:18] = np.array([sample_interval_us], dtype=">u2").view(np.uint8)
    bh[20:22] = np.array([ns], dtype=">u2").view(np.uint8)
    bh[24:26] = np.array([fmt], dtype=">u2").view(np.uint8)
    bh[300:302] = np.array([0x0100], dtype=">u2").view(np.uint8)  # revision 1
    bh[302:304] = np.array([1], dtype=">u2").view(np.uint8)       # fixed-length traces
    hdr = np.zeros((n_tr, _SEGY_TRACE_HDR), dtype=np.uint8)
    hdr[:, 0:4] = np.arange(1, n_tr + 1, dtype=">i4").view(np.uint8).reshape(n_tr, 4)  # trace sequence number
    hdr[:, 114:116] = np.array([ns], dtype=">u2").view(np.uint8)
    hdr[:, 116:118] = np.array([sample_interval_us], dtype=">u2").view(np.uint8)
    cols = d.T  # traces x samples
    body = float32_to_ibm(cols).astype(">u4") if fmt == 1 else cols.astype(">f4")
    traces = np.concatenate([hdr, np.ascontiguousarray(body).view(np.uint8).reshape(n_tr, 4 * ns)], axis=1)
    with open(path, "wb") as f:
        f.write(text.tobytes())
        f.write(bh.tobytes())
        f.write(traces.tobytes())


def _load_mat(path: str, vp_key: str, vs_key: str, rho_key: str, dx, dz) -> VelocityModel:
    """_load_mat (model_loader.jl:254-283) for MATLAB v4/v5 files."""
    from scipy.io import loadmat
    try:
        data = loadmat(path)
    except NotImplementedError as e:  # scipy's answer to v7.3 (HDF5) files
        raise NotImplementedError(f"{path}: MATLAB v7.3 files are HDF5, and no HDF5 reader is present here; "
                                  f"save the model with -v7 or convert it to .bin, .npy or SEG-Y") from e

    def pick(*keys):
        for k in keys:
            if k in data:
                return data[k]
        return None

    vp = pick(vp_key, "Vp", "VP")
    if vp is None:
        raise ValueError(f"Cannot find vp field. Available keys: {sorted(k for k in data if not k.startswith('__'))}")
    vp = np.asfortranarray(np.asarray(vp).astype(f32))
    vs = pick(vs_key, "Vs")
    rho = pick(rho_key, "Rho", "density")
    vs = estimate_vs(vp) if vs is None else np.asarray(vs).astype(f32)
    rho = gardner_rho(vp) if rho is None else np.asarray(rho).astype(f32)
    return VelocityModel.make(vp, vs, rho, dx, dz, name=os.path.basename(path))


def load_model(path: str, nx: Optional[int] = None, nz: Optional[int] = None, dx=1.0, dz=None,
               dtype=np.float32, order: str = "column_major", vs=None, rho=None, single: bool = False,
               vp_key: str = "vp", vs_key: str = "vs", rho_key: str = "rho") -> Union[VelocityModel, np.ndarray]:
    """load_model (model_loader.jl:88-106) for .bin, .npy, SEG-Y and MAT v4/v5 files."""
    ext = os.path.splitext(path)[1].lower()
    dz = dx if dz is None else dz
    if ext == ".mat":
        m = _load_mat(path, vp_key, vs_key, rho_key, dx, dz)
        return m.vp if single else m
    if ext == ".bin":
        if nx is None or nz is None:
            raise ValueError("Binary files require nx and nz parameters")
        read = lambda p: _read_bin(p, int(nx), int(nz), dtype, order)  # noqa: E731
    elif ext == ".npy":
        read = lambda p: np.asfortranarray(np.load(p).astype(f32))  # noqa: E731
    elif ext in (".segy", ".sgy"):
        def read(p):
            if not str(p).lower().endswith((".segy", ".sgy")):  # model_loader.jl:229-245 reads only SEG-Y paths
                raise ValueError(f"{p}: vs and rho of a SEG-Y model must be SEG-Y files or arrays")
            return read_segy(p)
    elif ext in (".jld2", ".h5", ".hdf5"):
        raise NotImplementedError(f"{ext} models need Julia or a library absent here; "
                                  f"convert to .bin, .npy, SEG-Y or MAT v5")
    else:
        raise ValueError(f"Unsupported format: {ext}\nSupported: .jld2, .segy, .sgy, .bin, .mat, .npy, .h5, .hdf5")
    vp = read(path)
    if single:
        return vp
    vs_d = _other(vs, read, vp, estimate_vs)
    rho_d = _other(rho, read, vp, gardner_rho)
    return VelocityModel.make(vp, vs_d, rho_d, dx, dz, name=os.path.basename(path))


def save_model_bin(prefix: str, model: VelocityModel) -> dict:
    """Writes vp, vs, rho as <prefix>_{vp,vs,rho}.bin (Float32, column
    major) and returns the load_model keyword arguments that read them back."""
    paths = {}
    for name in ("vp", "vs", "rho"):
        p = f"{prefix}_{name}.bin"
        np.asfortranarray(getattr(model, name), dtype="<f4").ravel(order="F").tofile(p)
        paths[name] = p
    return dict(nx=model.nx, nz=model.nz, dx=float(model.dx), dz=float(model.dz), vs=paths["vs"], rho=paths["rho"],
                path=paths["vp"])
