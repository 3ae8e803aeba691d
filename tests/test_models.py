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
    for ext in (".jld2", ".h5"):
        with pytest.raises(NotImplementedError):
            models.load_model(str(tmp_path / f"x{ext}"))
    with pytest.raises(ValueError):
        models.load_model(str(tmp_path / "x.xyz"))


# ---------------------------------------------------------------- SEG-Y
def test_ibm_float_known_words():
    # System/360 single precision: (-1)^s * 0.f * 16^(e-64)
    words = np.array([0x41100000, 0xC276A000, 0x40280000, 0x42640000, 0x00000000], dtype=np.uint32)
    assert np.array_equal(models.ibm_to_float32(words), np.array([1.0, -118.625, 0.15625, 100.0, 0.0], np.float32))
    assert [int(w) for w in models.float32_to_ibm(np.array([1.0, -118.625, 0.15625, 100.0, 0.0], np.float32))] == \
        [0x41100000, 0xC276A000, 0x40280000, 0x42640000, 0]


def test_segy_ieee_and_ibm_round_trips(tmp_path):
    rng = np.random.default_rng(3)
    data = rng.uniform(1500.0, 4500.0, (37, 23)).astype(np.float32)  # samples x traces
    p5 = tmp_path / "m5.segy"
    models.write_segy(str(p5), data, fmt=5)
    assert p5.stat().st_size == 3600 + 23 * (240 + 4 * 37)
    got = models.read_segy(str(p5))
    assert got.shape == (37, 23) and got.dtype == np.float32 and np.array_equal(got, data)
    exact = np.round(data * 16) / 16  # multiples of 1/16 below 2^12: exact in IBM's 24-bit fraction
    p1 = tmp_path / "m1.sgy"
    models.write_segy(str(p1), exact, fmt=1)
    assert np.array_equal(models.read_segy(str(p1)), exact)


def test_segy_extended_headers_and_integer_samples(tmp_path):
    data = np.arange(6 * 4, dtype=np.float32).reshape(6, 4) - 7
    p = tmp_path / "m.segy"
    models.write_segy(str(p), data, fmt=5)
    raw = bytearray(p.read_bytes())
    # one extended textual header after the binary header
    raw[3600 + 304 - 400:3600 + 306 - 400] = (1).to_bytes(2, "big")
    ext = bytes(raw[:3600]) + b"\x40" * 3200 + bytes(raw[3600:])
    (tmp_path / "ext.segy").write_bytes(ext)
    assert np.array_equal(models.read_segy(str(tmp_path / "ext.segy")), data)
    # the same samples as big-endian int16 (format code 3)
    hdr = bytearray(raw[:3600])
    hdr[3200 + 24:3200 + 26] = (3).to_bytes(2, "big")
    hdr[3200 + 304:3200 + 306] = (0).to_bytes(2, "big")
    body = b"".join(bytes(240) + data[:, t].astype(">i2").tobytes() for t in range(4))
    (tmp_path / "i16.segy").write_bytes(bytes(hdr) + body)
    assert np.array_equal(models.read_segy(str(tmp_path / "i16.segy")), data)
    (tmp_path / "bad.segy").write_bytes(bytes(hdr) + body[:-3])
    with pytest.raises(ValueError):
        models.read_segy(str(tmp_path / "bad.segy"))


def test_load_model_segy(tmp_path):
    rng = np.random.default_rng(4)
    vp = rng.uniform(1500.0, 4500.0, (30, 20)).astype(np.float32)
    vs = (vp / np.float32(1.8)).astype(np.float32)
    rho = np.full_like(vp, 2100.0)
    for n, a in (("vp", vp), ("vs", vs), ("rho", rho)):
        models.write_segy(str(tmp_path / f"{n}.segy"), a)
    m = models.load_model(str(tmp_path / "vp.segy"), vs=str(tmp_path / "vs.segy"), rho=str(tmp_path / "rho.segy"),
                          dx=12.5)
    assert (m.nx, m.nz) == (30, 20) and m.dx == m.dz == np.float32(12.5) and m.name == "vp.segy"
    assert np.array_equal(m.vp, vp) and np.array_equal(m.vs, vs) and np.array_equal(m.rho, rho)
    est = models.load_model(str(tmp_path / "vp.segy"))
    assert np.array_equal(est.vs, vp / np.float32(1.73)) and np.array_equal(est.rho, models.gardner_rho(vp))
    assert np.array_equal(models.load_model(str(tmp_path / "vp.segy"), single=True), vp)
    np.save(tmp_path / "vs.npy", vs)
    with pytest.raises(ValueError):
        models.load_model(str(tmp_path / "vp.segy"), vs=str(tmp_path / "vs.npy"))


# ---------------------------------------------------------------- MAT
def test_load_model_mat(tmp_path):
    from scipy.io import savemat
    rng = np.random.default_rng(5)
    vp = rng.uniform(1500.0, 4500.0, (12, 9))            # float64, as MATLAB saves
    vs = vp / 1.8
    rho = np.full_like(vp, 2150.25)
    savemat(str(tmp_path / "a.mat"), {"Vp": vp, "Vs": vs, "density": rho})
    m = models.load_model(str(tmp_path / "a.mat"), dx=5.0)
    assert (m.nx, m.nz) == (12, 9) and m.dx == m.dz == np.float32(5.0) and m.name == "a.mat"
    assert np.array_equal(m.vp, vp.astype(np.float32)) and np.array_equal(m.vs, vs.astype(np.float32))
    assert np.array_equal(m.rho, rho.astype(np.float32))
    # only vp, under a custom key: vs and rho estimated as for the other formats
    savemat(str(tmp_path / "b.mat"), {"velocity": vp})
    m2 = models.load_model(str(tmp_path / "b.mat"), vp_key="velocity")
    v32 = vp.astype(np.float32)
    assert np.array_equal(m2.vs, v32 / np.float32(1.73)) and np.array_equal(m2.rho, models.gardner_rho(v32))
    assert np.array_equal(models.load_model(str(tmp_path / "b.mat"), vp_key="velocity", single=True), v32)
    with pytest.raises(ValueError):
        models.load_model(str(tmp_path / "b.mat"))       # no vp, Vp or VP
