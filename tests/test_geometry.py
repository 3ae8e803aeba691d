"""Geometry writers against the reference's formats (src/io/geometry_io.jl).

The expected texts below are written out from the reference's println and
@printf statements for a small two-shot survey; Float32 fields interpolated
into strings follow Julia's shortest round-trip printing.
"""
import json

import numpy as np
import pytest

import fomo_julia_b200 as F
from fomo_julia_b200 import geometry as G
from fomo_julia_b200.elastic2d import ShotResult

f32 = np.float32


@pytest.mark.parametrize("x,s", [
    (1995.0, "1995.0"), (0.00125, "0.00125"), (0.001, "0.001"), (1e-5, "1.0e-5"), (0.0001, "0.0001"),
    (1e6, "1.0e6"), (100000.0, "100000.0"), (123456.0, "123456.0"), (1234567.0, "1.234567e6"),
    (-2.5, "-2.5"), (0.0, "0.0"), (-0.0, "-0.0"), (0.1, "0.1"), (16777216.0, "1.6777216e7"),
    (3.4028235e38, "3.4028235e38"), (1.0e-45, "1.0e-45"), (44430.0, "44430.0"), (12.5, "12.5"),
    (5.0, "5.0"), (0.0008, "0.0008"), (2.0e-5, "2.0e-5"), (1.2e-4, "0.00012"), (9.2, "9.2"),
])
def test_julia_float32_printing(x, s):
    assert G.julia_str(f32(x)) == s


def test_julia_printing_round_trips():
    rng = np.random.default_rng(0)
    vals = np.concatenate([rng.uniform(-1e4, 1e4, 2000), 10.0 ** rng.uniform(-8, 9, 2000)]).astype(f32)
    for v in vals:
        s = G.julia_str(v)
        assert f32(float(s.replace("e", "e"))) == v, (v, s)


class _Med:
    nx, nz, pad, dx, dz = 200 + 108, 100 + 108, 54, f32(12.5), f32(12.5)


class _Par:
    dt, nt = f32(0.001), 4000


def _results():
    r1 = ShotResult(np.zeros((4000, 3), f32), 1, 55, 56, np.array([55, 60, 254]), np.array([56, 56, 56]))
    r2 = ShotResult(np.zeros((4000, 3), f32), 2, 86, 56, np.array([55, 60, 254]), np.array([56, 56, 56]))
    return [r1, r2]


def test_create_geometry_values():
    g = G.create_geometry(_results()[1], _Med, _Par)
    assert g.src_x == f32(31 * 12.5) and g.src_z == f32(12.5)
    assert (g.src_i, g.src_j) == (32, 2)  # index - pad: 1-based
    assert list(g.rec_x) == [0.0, 62.5, 2487.5] and list(g.rec_i_idx) == [1, 6, 200]
    assert g.t_max == f32(f32(0.001) * f32(4000)) and (g.nx, g.nz) == (200, 100)


def test_single_shot_json_and_txt():
    g = G.create_geometry(_results()[0], _Med, _Par)
    want_json = """{
  "_note": "All coordinates are ACTUAL discretized grid positions",
  "shot_id": 1,
  "source": {
    "x": 0.0, "z": 12.5,
    "i": 1, "j": 2
  },
  "receivers": {
    "n": 3,
    "x": [0.0, 62.5, 2487.5],
    "z": [12.5, 12.5, 12.5],
    "i": [1, 6, 200],
    "j": [2, 2, 2]
  },
  "time": {"dt": 0.001, "nt": 4000, "t_max": 4.0},
  "grid": {"dx": 12.5, "dz": 12.5, "nx": 200, "nz": 100}
}
"""
    assert G.geometry_json(g) == want_json
    json.loads(want_json)
    want_txt = """# Survey Geometry - Single Shot
# Generated by Elastic2D
# NOTE: All coordinates are ACTUAL DISCRETIZED grid positions!
#============================================================

# Shot Info
shot_id      1

# Source (actual discretized position)
src_x        0.0000    # meters
src_z        12.5000    # meters
src_i        1        # grid index (0-based)
src_j        2        # grid index (0-based)

# Time Info
dt           0.001000  # seconds
nt           4000
t_max        4.0000    # seconds

# Grid Info (physical domain)
dx           12.5000    # meters
dz           12.5000    # meters
nx           200
nz           100

# Receivers: 3 total (actual discretized positions)
# Format: rec_id  x(m)  z(m)  i_idx  j_idx
n_rec        3
receivers
     1        0.0000       12.5000       1       2
     2       62.5000       12.5000       6       2
     3     2487.5000       12.5000     200       2
"""
    assert G.geometry_txt(g) == want_txt


def test_multi_shot_json_and_txt(tmp_path):
    mg = G.create_geometry(_results(), _Med, _Par)
    G.save_geometry(str(tmp_path / "s.json"), mg)
    G.save_geometry(str(tmp_path / "s.txt"), mg)
    text = (tmp_path / "s.json").read_text()
    d = json.loads(text)
    assert d["n_shots"] == 2 and d["shots"][1]["src_x"] == 387.5 and d["shots"][0]["rec_i"] == [1, 6, 200]
    assert '    "dt": 0.001, "nt": 4000,\n' in text and '    },\n    {\n      "id": 2,' in text
    assert text.endswith("    }\n  ]\n}\n")
    txt = (tmp_path / "s.txt").read_text()
    assert "shots\n     1        0.0000       12.5000       1       2       3\n" \
           "     2      387.5000       12.5000      32       2       3\n" in txt
    assert "\n# Shot 2 receivers\nshot_2_receivers  3\n     1        0.0000" in txt
    with pytest.raises(NotImplementedError):
        G.save_geometry(str(tmp_path / "s.jld2"), mg)
    with pytest.raises(ValueError):
        G.save_geometry(str(tmp_path / "s.xyz"), mg)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_create_geometry_matches_oracle(seed, oracle_lib):
    # geometry_io.jl:85-130 restated in the oracle: coordinates, indices, t_max, grid size
    rng = np.random.default_rng(seed)
    pad = int(rng.integers(5, 60))
    dx, dz = f32(rng.choice([10.0, 12.5, 7.3])), f32(rng.choice([10.0, 12.5, 3.1]))
    dt, nt = f32(rng.uniform(1e-4, 2e-3)), int(rng.integers(100, 20000))
    nx, nz = int(rng.integers(2 * pad + 10, 5000)), int(rng.integers(2 * pad + 10, 4000))
    n_rec = int(rng.integers(1, 500))
    ri = rng.integers(1, nx + 1, n_rec)
    rj = rng.integers(1, nz + 1, n_rec)
    si, sj = int(rng.integers(1, nx + 1)), int(rng.integers(1, nz + 1))
    med = F.Medium(nx, nz, float(dx), float(dz), 0.0, 0.0, 4, pad, True, *[None] * 5)
    par = F.sim_params(dt, nt, float(dx), float(dz), 8)
    g = G.create_geometry(ShotResult(np.zeros((1, n_rec), f32), 3, si, sj, ri, rj), med, par)
    o = oracle_lib.create_geometry(si, sj, ri, rj, pad, dx, dz, dt, nt, nx, nz)
    assert (g.src_x, g.src_z, g.t_max) == (o["src_x"], o["src_z"], o["t_max"])
    assert (g.src_i, g.src_j, g.nx, g.nz) == (o["src_i"], o["src_j"], o["nx"], o["nz"])
    assert np.array_equal(g.rec_x, o["rec_x"]) and np.array_equal(g.rec_z, o["rec_z"])
    assert np.array_equal(g.rec_i_idx, o["rec_i"]) and np.array_equal(g.rec_j_idx, o["rec_j"])
