"""Velocity-model loaders feeding init_medium (src/io/model_loader.jl).

``load_model`` dispatches on the extension as the reference does
(model_loader.jl:88-106).  Here:
* ``.bin``: raw binary (model_loader.jl:141-189).  nx and nz are required.
  dtype Float32 by default; order column-major (x fastest) or row-major.
  vs and rho come from files, from arrays, or are estimated from vp.
* ``.npy``: NumPy arrays (model_loader.jl:288-320).
* ``.jld2``, ``.segy``/``.sgy``, ``.mat``, ``.h5``/``.hdf5`` need Julia or
  libraries not present here.  They raise NotImplementedError naming the
  format; convert such models to .bin or .npy first.

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


def load_model(path: str, nx: Optional[int] = None, nz: Optional[int] = None, dx=1.0, dz=None,
               dtype=np.float32, order: str = "column_major", vs=None, rho=None, single: bool = False
               ) -> Union[VelocityModel, np.ndarray]:
    """load_model (model_loader.jl:88-106) for .bin and .npy files."""
    ext = os.path.splitext(path)[1].lower()
    dz = dx if dz is None else dz
    if ext == ".bin":
        if nx is None or nz is None:
            raise ValueError("Binary files require nx and nz parameters")
        read = lambda p: _read_bin(p, int(nx), int(nz), dtype, order)  # noqa: E731
    elif ext == ".npy":
        read = lambda p: np.asfortranarray(np.load(p).astype(f32))  # noqa: E731
    elif ext in (".jld2", ".segy", ".sgy", ".mat", ".h5", ".hdf5"):
        raise NotImplementedError(f"{ext} models need Julia or a library absent here; convert to .bin or .npy")
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
