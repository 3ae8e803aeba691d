"""Seeded synthetic media and shot layouts for the benchmark workloads.

The reference publishes one timing, on the proprietary SEAM model
(README.md:93-102: 4444 x 3819 cells, nt = 11520).  No model files are
available here, so the workloads use seeded layered media of the same shape:

* ``homogeneous``  -- vp 3000, vs 1732, rho 2000 (the small CPU-runnable case).
* ``layered``      -- 40 equal-thickness layers, vp rising linearly
  1500 -> 4500 m/s with depth, times (1 + 0.05 p) where p is N(0,1) white
  noise (numpy PCG64, seeded) smoothed by a Gaussian of sigma 200 m / dx and
  scaled to max |p| = 1; the top 150 m is water (vp 1500, vs 0, no
  perturbation); elsewhere vs = vp / 1.73; rho = 310 vp^0.25 (Gardner).

Grids are (nx, nz) float32 arrays in column-major (x fastest) order.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

f32 = np.float32


def homogeneous(nx: int, nz: int, vp=3000.0, vs=1732.0, rho=2000.0):
    shape = (nx, nz)
    return (np.full(shape, vp, dtype=f32, order="F"), np.full(shape, vs, dtype=f32, order="F"),
            np.full(shape, rho, dtype=f32, order="F"))


def _gaussian_smooth(p: np.ndarray, sigma: float) -> np.ndarray:
    """Separable Gaussian filter (truncated at 4 sigma, reflecting edges)."""
    from scipy.ndimage import gaussian_filter1d
    out = gaussian_filter1d(p, sigma, axis=0, mode="reflect", truncate=4.0)
    return gaussian_filter1d(out, sigma, axis=1, mode="reflect", truncate=4.0)


def layered(nx: int, nz: int, dx: float, seed: int, n_layers: int = 40, vp_top: float = 1500.0,
            vp_bottom: float = 4500.0, water_depth: float = 150.0, perturbation: float = 0.05,
            corr_length: float = 200.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    j = np.arange(nz)
    layer = np.minimum(j * n_layers // nz, n_layers - 1)
    vp_layer = vp_top + (vp_bottom - vp_top) * layer / (n_layers - 1)
    p = rng.standard_normal((nx, nz), dtype=np.float32)
    p = _gaussian_smooth(p, corr_length / dx)
    p /= np.abs(p).max()
    vp = vp_layer[None, :] * (1.0 + perturbation * p)
    vs = vp / 1.73
    water = j * dx < water_depth
    vp[:, water] = 1500.0
    vs[:, water] = 0.0
    rho = 310.0 * vp ** 0.25
    F = lambda a: np.asfortranarray(a, dtype=f32)  # noqa: E731
    return F(vp), F(vs), F(rho)


@dataclass
class Workload:
    """One benchmark configuration: medium, time axis, sources and receivers."""
    name: str
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    dx: float
    dz: float
    nbc: int
    fd_order: int
    free_surface: bool
    dt: float
    nt: int
    f0: float
    src_x: List[float]
    src_z: List[float]
    rec_x: np.ndarray
    rec_z: np.ndarray
    rec_types: List[str] = field(default_factory=lambda: ["vz"])
    extra: dict = field(default_factory=dict)

    @property
    def nx_in(self) -> int:
        return self.vp.shape[0]

    @property
    def nz_in(self) -> int:
        return self.vp.shape[1]

    def padded_cells(self) -> int:
        pad = self.nbc + self.fd_order // 2
        return (self.nx_in + 2 * pad) * (self.nz_in + 2 * pad)


def small_homogeneous() -> Workload:
    """400 x 200 homogeneous medium, 8th order, nbc 50, free surface, dt 1 ms,
    nt 1500, 10 Hz Ricker at (2000, 20) m, 199 receivers every 20 m at z = 10 m
    recording vx and vz."""
    vp, vs, rho = homogeneous(400, 200)
    rec_x = np.arange(1, 200, dtype=np.float64) * 20.0
    return Workload("homogeneous_400x200_o8_nt1500", vp, vs, rho, 10.0, 10.0, 50, 8, True, 0.001, 1500, 10.0,
                    [2000.0], [20.0], rec_x.astype(f32), np.full(rec_x.size, 10.0, dtype=f32), ["vx", "vz"])


def large_layered(seed: int = 1, nt: Optional[int] = None) -> Workload:
    """4444 x 3819 layered medium (dx = dz = 10 m), 8th order, nbc 50, free
    surface, dt 0.8 ms, nt 11520, 12 Hz Ricker at the surface centre
    (z = 10 m: a source on the zeroed free-surface rows would have its tzz
    injection erased), 1000 receivers evenly spread across x at z = 10 m."""
    nx, nz, dx = 4444, 3819, 10.0
    vp, vs, rho = layered(nx, nz, dx, seed)
    rec_x = np.linspace(0.0, (nx - 1) * dx, 1000)
    return Workload("layered_4444x3819_o8_nt11520", vp, vs, rho, dx, dx, 50, 8, True, 0.0008,
                    11520 if nt is None else nt, 12.0, [float((nx - 1) * dx / 2)], [10.0],
                    rec_x.astype(f32), np.full(1000, 10.0, dtype=f32), ["vz"])


def batched_layered(seed: int = 2) -> Workload:
    """64 shots on one 2000 x 800 medium (dx = dz = 12.5 m), 8th order, nbc 50,
    dt 1 ms, nt 4000, 12 Hz sources every 31 grid points along z = 12.5 m,
    400 receivers (every 5 grid points)."""
    nx, nz, dx = 2000, 800, 12.5
    vp, vs, rho = layered(nx, nz, dx, seed)
    src_x = [31 * s * dx for s in range(64)]
    rec_x = np.arange(400) * 5 * dx
    return Workload("layered_2000x800_o8_nt4000_64shots", vp, vs, rho, dx, dx, 50, 8, True, 0.001, 4000, 12.0,
                    src_x, [12.5] * 64, rec_x.astype(f32), np.full(400, 12.5, dtype=f32), ["vz"])


@dataclass
class Request:
    """One shot request of an uneven batch or a serving stream."""
    medium: int          # index into the media list
    src_x: float         # metres
    src_z: float
    nt: int
    n_rec: int
    f0: float
    fd_order: int
    arrival_s: float = 0.0


UNEVEN_GRIDS = [(600, 300, 3), (1200, 500, 4), (2400, 1000, 5), (3200, 1400, 6)]  # (nx, nz, seed), dx = 10 m


def uneven_media():
    """The four layered media of the uneven batch: 600x300, 1200x500,
    2400x1000 and 3200x1400 cells, dx = dz = 10 m, seeds 3..6."""
    return [(layered(nx, nz, 10.0, seed), 10.0) for nx, nz, seed in UNEVEN_GRIDS]


def uneven_requests(n: int = 48, seed: int = 7) -> List[Request]:
    """48 shots over the uneven media: FD order 4, 8 or 12, nt ~ U[1500, 6000]
    (dt 0.8 ms), 100..800 receivers, f0 ~ U[8, 15] Hz, source x uniform at
    the surface (z = 10 m)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        m = int(rng.integers(0, len(UNEVEN_GRIDS)))
        nx = UNEVEN_GRIDS[m][0]
        out.append(Request(m, float(rng.uniform(0, (nx - 1) * 10.0)), 10.0, int(rng.integers(1500, 6001)),
                           int(rng.integers(100, 801)), float(rng.uniform(8.0, 15.0)),
                           int(rng.choice([4, 8, 12]))))
    return out


def serving_requests(n: int, media_nx: List[int], media_dx: List[float], rate_per_s: float,
                     seed: int = 8) -> List[Request]:
    """A Poisson stream of shot requests over resident media: medium uniform,
    source x uniform at z = 10 m, nt ~ U[1500, 6000], 100..1000 receivers,
    order 8, 12 Hz; arrivals with exponential gaps of mean 1/rate_per_s."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for _ in range(n):
        m = int(rng.integers(0, len(media_nx)))
        out.append(Request(m, float(rng.uniform(0, (media_nx[m] - 1) * media_dx[m])), 10.0,
                           int(rng.integers(1500, 6001)), int(rng.integers(100, 1001)), 12.0, 8, t))
        t += float(rng.exponential(1.0 / rate_per_s))
    return out
