"""Model loaders (fomo_julia_b200.models) for the formats available here."""
import numpy as np
import pytest

from fomo_julia_b200 import models

f32 = np.float32


def _model():
    rng = np.random.default_rng(3)
    vp = rng.uniform(1500, 4500, (17, 11)).astype(f32)
    return models.VelocityModel.make(vp, vp / f32(1.73), f32(310) * vp ** f32(0.25), 10.0, 12.5, name="m")


def test_bin_round_trip(tmp_path):
    m = _model()
    kw = models.save_model_bin(str(tmp_path / "m"), m)
    path = kw.pop("path")
    got = models.load_model(path, **kw)
    for n in ("vp", "vs", "rho"):
        assert np.array_equal(getattr(got, n), getattr(m, n))
    assert (got.nx, got.nz, got.dx, got.dz) == (17, 11, f32(10), f32(12.5))
    assert np.array_equal(models.load_model(path, nx=17, nz=11, single=True), m.vp)


def test_bin_row_major_and_estimates(tmp_path):
    m = _model()
    p = tmp_path / "vp_rows.bin"
    np.ascontiguousarray(m.vp.T, dtype="<f4").tofile(p)  # nz rows of nx values
    got = models.load_model(str(p), nx=17, nz=11, dx=5.0, order="row_major")
    assert np.array_equal(got.vp, m.vp) and got.dz == f32(5.0)
    assert np.array_equal(got.vs, m.vp / f32(1.73))
    assert got.rho.dtype == f32 and np.allclose(got.rho, 310 * m.vp.astype(np.float64) ** 0.25, rtol=1e-6)
    with pytest.raises(ValueError):
        models.load_model(str(p), nx=17)
    with pytest.raises(ValueError):
        models.load_model(str(p), nx=18, nz=11)


def test_npy_and_unsupported(tmp_path):
    m = _model()
    for n in ("vp", "vs", "rho"):
        np.save(tmp_path / f"{n}.npy", getattr(m, n))
    got = models.load_model(str(tmp_path / "vp.npy"), vs=str(tmp_path / "vs.npy"), rho=str(tmp_path / "rho.npy"),
                            dx=10.0, dz=12.5)
    assert np.array_equal(got.rho, m.rho) and got.name == "vp.npy"
    for ext in (".jld2", ".segy", ".mat", ".h5"):
        with pytest.raises(NotImplementedError):
            models.load_model(str(tmp_path / f"x{ext}"))
    with pytest.raises(ValueError):
        models.load_model(str(tmp_path / "x.xyz"))
