"""Survey geometry of shot results and its JSON / TXT writers.

Restates src/io/geometry_io.jl of the reference: ``create_geometry``
(:85-130) turns a ShotResult's grid indices into the actual discretised
coordinates, and ``save_geometry`` (:152-178) writes them as JSON (:230-283)
or text (:289-368), byte for byte as the reference prints them:

* Float32 values interpolated into strings print as Julia prints them: the
  shortest decimal string that reads back to the same Float32, in plain
  notation when the decimal point falls within -4 < p <= 6 digits of the first
  digit, else as ``d.ddde<exp>`` (``1.0e6``, ``1.0e-5``);
* ``@printf`` fields (``%.4f``, ``%.6f``, ``%12.4f``, ``%6d``) format the exact
  binary value, correctly rounded (ties to even on exact binary ties).

The ``.jld2`` format of the reference needs Julia's JLD2 package and is not
written here.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass
from typing import List, Sequence, Union

import numpy as np

f32 = np.float32


# ---------------------------------------------------------------- Julia's Float32 printing
def _shortest_digits(x: np.float32):
    """(digits, e10) of the shortest decimal that rounds back to x (> 0):
    x ~= 0.digits * 10^(e10 + 1), i.e. the first digit has exponent e10."""
    s = np.format_float_scientific(x, unique=True, trim="-")
    mant, exp = s.split("e")
    digits = mant.replace(".", "").lstrip("-")
    digits = digits.rstrip("0") or "0"
    return digits, int(exp)


def julia_str(x) -> str:
    """print(x::Float32) in Julia (Base.Ryu.writeshortest with default
    arguments): the form ``"$(x)"`` gives in the reference's writers."""
    x = f32(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "Inf" if x > 0 else "-Inf"
    neg = bool(np.signbit(x))
    if x == 0:
        return "-0.0" if neg else "0.0"
    ax = f32(-x) if neg else x
    digits, e10 = _shortest_digits(ax)
    olength = len(digits)
    pt = e10 + 1  # digits before the decimal point
    plain = -4 < pt <= 6
    if plain and pt >= olength:
        # the writer falls back to the exponent form when the value is not
        # (close to) a multiple of the trailing power of ten
        plain = not (abs(math.fmod(float(ax) + 0.05, 10.0 ** (pt - olength)) - 0.05) > 0.05)
    if plain:
        if pt <= 0:
            body = "0." + "0" * (-pt) + digits
        elif pt >= olength:
            body = digits + "0" * (pt - olength) + ".0"
        else:
            body = digits[:pt] + "." + digits[pt:]
    else:
        body = digits[0] + "." + (digits[1:] or "0") + "e" + str(e10)
    return ("-" if neg else "") + body


def _jvec(v) -> str:
    return ", ".join(julia_str(a) for a in v)


def _ivec(v) -> str:
    return ", ".join(str(int(a)) for a in v)


# ---------------------------------------------------------------- geometry
@dataclass
class SurveyGeometry:
    """SurveyGeometry (geometry_io.jl:26-54)."""
    shot_id: int
    src_x: np.float32
    src_z: np.float32
    src_i: int
    src_j: int
    n_rec: int
    rec_x: np.ndarray
    rec_z: np.ndarray
    rec_i_idx: np.ndarray
    rec_j_idx: np.ndarray
    dt: np.float32
    nt: int
    t_max: np.float32
    dx: np.float32
    dz: np.float32
    nx: int
    nz: int


@dataclass
class MultiShotGeometry:
    """MultiShotGeometry (geometry_io.jl:61-72)."""
    n_shots: int
    shots: List[SurveyGeometry]
    dt: np.float32
    nt: int
    dx: np.float32
    dz: np.float32
    nx: int
    nz: int


def _one(result, medium, params) -> SurveyGeometry:
    pad = int(medium.pad)
    dx, dz = f32(medium.dx), f32(medium.dz)
    # (Int - pad - 1) * Float32: the Int converts to Float32, one Float32 product
    src_x = f32(f32(int(result.src_i) - pad - 1) * dx)
    src_z = f32(f32(int(result.src_j) - pad - 1) * dz)
    ri = np.asarray(result.rec_i, dtype=np.int64)
    rj = np.asarray(result.rec_j, dtype=np.int64)
    rec_x = ((ri - pad - 1).astype(f32) * dx).astype(f32)
    rec_z = ((rj - pad - 1).astype(f32) * dz).astype(f32)
    dt = f32(params.dt)
    return SurveyGeometry(int(result.shot_id), src_x, src_z, int(result.src_i) - pad, int(result.src_j) - pad,
                          int(ri.size), rec_x, rec_z, ri - pad, rj - pad, dt, int(params.nt),
                          f32(dt * f32(int(params.nt))), dx, dz, int(medium.nx) - 2 * pad, int(medium.nz) - 2 * pad)


def create_geometry(results, medium, params) -> Union[SurveyGeometry, MultiShotGeometry]:
    """create_geometry (geometry_io.jl:85-130): one ShotResult gives a
    SurveyGeometry, a list gives a MultiShotGeometry.  Coordinates are the
    discretised ones, (index - pad - 1) * dx; indices are index - pad (the
    reference's "0-based" comment notwithstanding, these are 1-based)."""
    if isinstance(results, (list, tuple)):
        shots = [_one(r, medium, params) for r in results]
        pad = int(medium.pad)
        return MultiShotGeometry(len(shots), shots, f32(params.dt), int(params.nt), f32(medium.dx), f32(medium.dz),
                                 int(medium.nx) - 2 * pad, int(medium.nz) - 2 * pad)
    return _one(results, medium, params)


# ---------------------------------------------------------------- writers
NOTE = "All coordinates are ACTUAL discretized grid positions"


def geometry_json(g: Union[SurveyGeometry, MultiShotGeometry]) -> str:
    """The text _save_geometry_json / _save_multigeom_json write."""
    L = ["{", f'  "_note": "{NOTE}",']
    if isinstance(g, SurveyGeometry):
        L += [f'  "shot_id": {g.shot_id},',
              '  "source": {',
              f'    "x": {julia_str(g.src_x)}, "z": {julia_str(g.src_z)},',
              f'    "i": {g.src_i}, "j": {g.src_j}',
              '  },',
              '  "receivers": {',
              f'    "n": {g.n_rec},',
              f'    "x": [{_jvec(g.rec_x)}],',
              f'    "z": [{_jvec(g.rec_z)}],',
              f'    "i": [{_ivec(g.rec_i_idx)}],',
              f'    "j": [{_ivec(g.rec_j_idx)}]',
              '  },',
              f'  "time": {{"dt": {julia_str(g.dt)}, "nt": {g.nt}, "t_max": {julia_str(g.t_max)}}},',
              f'  "grid": {{"dx": {julia_str(g.dx)}, "dz": {julia_str(g.dz)}, "nx": {g.nx}, "nz": {g.nz}}}',
              "}"]
    else:
        L += [f'  "n_shots": {g.n_shots},',
              '  "common": {',
              f'    "dt": {julia_str(g.dt)}, "nt": {g.nt},',
              f'    "dx": {julia_str(g.dx)}, "dz": {julia_str(g.dz)},',
              f'    "nx": {g.nx}, "nz": {g.nz}',
              '  },',
              '  "shots": [']
        for k, s in enumerate(g.shots):
            comma = "," if k + 1 < g.n_shots else ""
            L += ['    {',
                  f'      "id": {s.shot_id},',
                  f'      "src_x": {julia_str(s.src_x)}, "src_z": {julia_str(s.src_z)},',
                  f'      "src_i": {s.src_i}, "src_j": {s.src_j},',
                  f'      "n_rec": {s.n_rec},',
                  f'      "rec_x": [{_jvec(s.rec_x)}],',
                  f'      "rec_z": [{_jvec(s.rec_z)}],',
                  f'      "rec_i": [{_ivec(s.rec_i_idx)}],',
                  f'      "rec_j": [{_ivec(s.rec_j_idx)}]',
                  f'    }}{comma}']
        L += ['  ]', "}"]
    return "\n".join(L) + "\n"


def _f(fmt: str, x) -> str:
    return fmt % float(x)


def _rec_lines(s: SurveyGeometry) -> List[str]:
    return ["%6d  %12.4f  %12.4f  %6d  %6d" % (r + 1, float(s.rec_x[r]), float(s.rec_z[r]), int(s.rec_i_idx[r]),
                                               int(s.rec_j_idx[r])) for r in range(s.n_rec)]


def geometry_txt(g: Union[SurveyGeometry, MultiShotGeometry]) -> str:
    """The text _save_geometry_txt / _save_multigeom_txt write."""
    rule = "#" + "=" * 60
    if isinstance(g, SurveyGeometry):
        L = ["# Survey Geometry - Single Shot", "# Generated by Elastic2D",
             "# NOTE: All coordinates are ACTUAL DISCRETIZED grid positions!", rule, "",
             "# Shot Info", f"shot_id      {g.shot_id}", "",
             "# Source (actual discretized position)",
             _f("src_x        %.4f    # meters", g.src_x),
             _f("src_z        %.4f    # meters", g.src_z),
             f"src_i        {g.src_i}        # grid index (0-based)",
             f"src_j        {g.src_j}        # grid index (0-based)", "",
             "# Time Info",
             _f("dt           %.6f  # seconds", g.dt),
             f"nt           {g.nt}",
             _f("t_max        %.4f    # seconds", g.t_max), "",
             "# Grid Info (physical domain)",
             _f("dx           %.4f    # meters", g.dx),
             _f("dz           %.4f    # meters", g.dz),
             f"nx           {g.nx}", f"nz           {g.nz}", "",
             f"# Receivers: {g.n_rec} total (actual discretized positions)",
             "# Format: rec_id  x(m)  z(m)  i_idx  j_idx",
             f"n_rec        {g.n_rec}", "receivers"] + _rec_lines(g)
    else:
        L = ["# Survey Geometry - Multi Shot", "# Generated by Elastic2D",
             "# NOTE: All coordinates are ACTUAL DISCRETIZED grid positions!", rule, "",
             "# Common Parameters", f"n_shots      {g.n_shots}",
             _f("dt           %.6f  # seconds", g.dt),
             f"nt           {g.nt}",
             _f("dx           %.4f    # meters", g.dx),
             _f("dz           %.4f    # meters", g.dz),
             f"nx           {g.nx}", f"nz           {g.nz}", "",
             "# Shot List (actual discretized positions)",
             "# Format: shot_id  src_x(m)  src_z(m)  src_i  src_j  n_rec", "shots"]
        L += ["%6d  %12.4f  %12.4f  %6d  %6d  %6d" % (s.shot_id, float(s.src_x), float(s.src_z), s.src_i, s.src_j,
                                                      s.n_rec) for s in g.shots]
        L += ["", "# Receiver Coordinates per Shot (actual discretized positions)",
              "# Format: rec_id  x(m)  z(m)  i_idx  j_idx"]
        for s in g.shots:
            L += ["", f"# Shot {s.shot_id} receivers", f"shot_{s.shot_id}_receivers  {s.n_rec}"] + _rec_lines(s)
    return "\n".join(L) + "\n"


def save_geometry(path: str, geom: Union[SurveyGeometry, MultiShotGeometry]) -> None:
    """save_geometry (geometry_io.jl:152-178): .json, or .txt / .dat / .geo."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".json":
        text = geometry_json(geom)
    elif ext in (".txt", ".dat", ".geo"):
        text = geometry_txt(geom)
    elif ext == ".jld2":
        raise NotImplementedError("JLD2 is Julia's own format; write .json or .txt")
    else:
        raise ValueError(f"Unsupported format: {ext}. Use .jld2, .json, or .txt")
    with open(path, "w", newline="\n") as f:
        f.write(text)


def load_gather_geom(path: str, geom: SurveyGeometry) -> np.ndarray:
    """load_gather(path, geom) (geometry_io.jl:466-472): [nt x n_rec] Float32."""
    d = np.fromfile(path, dtype="<f4", count=geom.nt * geom.n_rec)
    return np.asfortranarray(d.reshape((geom.nt, geom.n_rec), order="F"))
