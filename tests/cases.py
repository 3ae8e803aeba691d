"""Shared inputs for the parity tests (test helpers, not product code)."""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
f32 = np.float32


@dataclass
class Case:
    name: str
    vp: np.ndarray            # (nx_in, nz_in) float32
    vs: np.ndarray
    rho: np.ndarray
    dx: float
    dz: float
    nbc: int
    fd_order: int
    free_surface: bool
    dt: np.float32
    nt: int
    f0: float
    v_ref: np.float32
    src_x: float
    src_z: float
    rec_x: np.ndarray
    rec_z: np.ndarray
    rec_type: str = "vz"
    extra: dict = field(default_factory=dict)


def runjl_case() -> Case:
    """The run.jl synthetic single shot that produced shot_1.bin (run.jl:36-61, 90-131)."""
    from fomo_julia_b200 import julia_mean
    r = json.load(open(os.path.join(GOLDEN, "runjl_case.json")))
    nx, nz = r["nx"], r["nz"]
    vp = np.full((nx, nz), r["vp"], dtype=f32, order="F")
    vs = np.full((nx, nz), r["vs"], dtype=f32, order="F")
    rho = np.full((nx, nz), r["rho"], dtype=f32, order="F")
    vp[:, r["layer_from_row"] - 1:] = r["vp_layer"]
    vs[:, r["layer_from_row"] - 1:] = r["vs_layer"]
    dx = f32(r["dx"])
    dt = f32(f32(f32(r["cfl"]) * min(f32(r["dx"]), f32(r["dz"]))) / vp.max())
    nt = int(np.ceil(f32(f32(r["total_time"]) / dt)))
    # Float32.(range(500, 3500, length=100)): exact rational points, rounded once.
    xs = np.array([float(Fraction(r["rec_x_start"]) + Fraction(r["rec_x_stop"] - r["rec_x_start"], r["n_rec"] - 1) * k)
                   for k in range(r["n_rec"])], dtype=f32)
    x_max = f32((nx - 1) * dx)
    return Case("runjl", vp, vs, rho, float(dx), float(r["dz"]), r["nbc"], r["fd_order"], r["free_surface"],
                dt, nt, r["f0"], julia_mean(vp), float(f32(x_max / f32(2))), r["src_z"], xs,
                np.full(r["n_rec"], r["rec_z"], dtype=f32), r["rec_type"])


def golden_gather() -> np.ndarray:
    d = np.fromfile(os.path.join(GOLDEN, "shot_1.bin"), dtype="<f4")
    return np.asfortranarray(d.reshape((800, 100), order="F"))


def layered(nx_in, nz_in, seed, dx=10.0, nbc=8, fd_order=8, free_surface=True, nt=120, water_rows=0,
            rec_type="vz", n_rec=17, src=None, f0=None) -> Case:
    """A small random layered elastic model (seeded), for oracle-vs-GPU parity."""
    rng = np.random.default_rng(seed)
    n_layers = max(2, nz_in // 6)
    z = np.arange(nz_in)
    layer = np.minimum(z * n_layers // nz_in, n_layers - 1)
    vp_l = 1800.0 + 2400.0 * layer / max(n_layers - 1, 1)
    vp = np.repeat(vp_l[None, :], nx_in, axis=0) * (1.0 + 0.05 * rng.uniform(-1, 1, (nx_in, nz_in)))
    vs = vp / 1.73
    if water_rows:
        vp[:, :water_rows] = 1500.0
        vs[:, :water_rows] = 0.0
    rho = 310.0 * vp ** 0.25
    vp, vs, rho = (np.asfortranarray(a, dtype=f32) for a in (vp, vs, rho))
    dt = f32(0.5 * dx / vp.max())
    f0 = f0 if f0 is not None else float(vp.min() / (8.0 * dx))
    from fomo_julia_b200 import julia_mean
    if src is None:
        src = (float(dx * (nx_in // 2) + 0.5 * dx), float(dx * 3))
    rec_x = np.linspace(0.0, dx * (nx_in - 1), n_rec).astype(f32)
    rec_z = np.full(n_rec, dx * 2, dtype=f32)
    return Case(f"layered{nx_in}x{nz_in}s{seed}o{fd_order}b{nbc}{'fs' if free_surface else 'nofs'}{rec_type}",
                vp, vs, rho, dx, dx, nbc, fd_order, free_surface, dt, nt, f0, julia_mean(vp),
                src[0], src[1], rec_x, rec_z, rec_type)


def per_trace_rel_l2(g, ref) -> np.ndarray:
    g = np.asarray(g, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    num = np.linalg.norm(g - ref, axis=0)
    den = np.linalg.norm(ref, axis=0)
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)


def oracle_inputs(c: Case, oracle):
    """Medium, HABC, coefficients, wavelet and indices from the oracle's restatement."""
    med = oracle.init_medium(c.vp, c.vs, c.rho, c.dx, c.dz, c.nbc, c.fd_order, c.free_surface)
    h = oracle.init_habc(c.nbc, c.dt, c.dx, c.dz, c.v_ref)
    a = oracle.fd_coefficients(c.fd_order)
    wav = oracle.ricker(c.f0, c.dt, c.nt)
    si = oracle.coord_to_index(c.src_x, c.dx, med.pad)
    sj = oracle.coord_to_index(c.src_z, c.dz, med.pad)
    ri = [oracle.coord_to_index(x, c.dx, med.pad) for x in c.rec_x]
    rj = [oracle.coord_to_index(z, c.dz, med.pad) for z in c.rec_z]
    return med, h, a, wav, si, sj, np.array(ri, np.int32), np.array(rj, np.int32)


def case_from_workload(w, rec_type=None, shot=0, nt=None) -> Case:
    """A parity Case for one shot of a benchmark workload
    (fomo_julia_b200.synthetic): the same medium, time axis, source and
    receivers, with v_ref = mean(vp) as run.jl:57 computes it."""
    from fomo_julia_b200 import julia_mean
    rt = rec_type or w.rec_types[0]
    return Case(f"{w.name}_shot{shot}_{rt}" + ("" if nt is None else f"_nt{nt}"), w.vp, w.vs, w.rho,
                float(w.dx), float(w.dz), w.nbc, w.fd_order, w.free_surface, f32(w.dt),
                w.nt if nt is None else nt, w.f0, julia_mean(w.vp), float(w.src_x[shot]), float(w.src_z[shot]),
                np.asarray(w.rec_x, dtype=f32), np.asarray(w.rec_z, dtype=f32), rt)
