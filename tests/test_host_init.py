"""Host-side set-up of the package against the oracle's restatement: bit-exact."""
import numpy as np
import pytest

import fomo_julia_b200 as F
from cases import layered, runjl_case

f32 = np.float32


@pytest.mark.parametrize("order", [2, 4, 6, 8, 10, 12])
def test_fd_coefficients(order, oracle_lib):
    assert np.array_equal(F.get_fd_coefficients(order), oracle_lib.fd_coefficients(order))


def test_fd_order_unsupported():
    with pytest.raises(ValueError, match="Unsupported FD order"):
        F.get_fd_coefficients(14)


def test_taylor_matches_reference_table():
    # the reference's orders 2-8 are the Taylor coefficients rounded to Float32 (to its decimals)
    for order in (2, 4, 6, 8):
        exact = np.array([float(x) for x in F.taylor_coefficients(order // 2)])
        assert np.allclose(F.get_fd_coefficients(order), exact, rtol=2e-7, atol=1e-9)
    # order 10 keeps the reference's table verbatim, including its a_1 =
    # 1.2115478515625 = 19850/16384 where the Taylor value is 19845/16384
    a10 = F.get_fd_coefficients(10)
    exact = np.array([float(x) for x in F.taylor_coefficients(5)])
    assert float(F.taylor_coefficients(5)[0]) == 19845 / 16384
    assert a10[0] == np.float32(19850 / 16384)
    assert np.allclose(a10[1:], exact[1:], rtol=2e-7, atol=1e-9)


@pytest.mark.parametrize("f0,dt,nt", [(15.0, 0.00125, 800), (10.0, 0.001, 1500), (12.0, 0.0008, 3000),
                                      (8.3, 0.0007, 257)])
def test_ricker(f0, dt, nt, oracle_lib):
    assert np.array_equal(F.ricker_wavelet(f0, dt, nt), oracle_lib.ricker(f0, dt, nt))


@pytest.mark.parametrize("water", [0, 3])
@pytest.mark.parametrize("order,nbc", [(8, 6), (4, 5), (12, 7)])
def test_init_medium(order, nbc, water, oracle_lib):
    c = layered(23, 17, seed=5, nbc=nbc, fd_order=order, water_rows=water)
    m = F.Medium.__new__(F.Medium)
    lam, mu, mu_txz, rho_vx, rho_vz = F.compute_staggered_params(
        F.pad_array(c.vp, nbc + order // 2), F.pad_array(c.vs, nbc + order // 2), F.pad_array(c.rho, nbc + order // 2))
    o = oracle_lib.init_medium(c.vp, c.vs, c.rho, c.dx, c.dz, nbc, order, True)
    for mine, theirs in ((rho_vx, o.rho_vx), (rho_vz, o.rho_vz), (lam, o.lam), (mu, o.mu_txx), (mu_txz, o.mu_txz)):
        assert mine.shape == theirs.shape
        assert np.array_equal(mine.view(np.uint32), theirs.view(np.uint32))
    if water:
        assert (mu_txz[:, : nbc + order // 2 + water - 1] == 0).all()


def test_init_habc(oracle_lib):
    for (vref, dt, dx, dz, nbc) in ((3505.0, 0.00125, 10.0, 10.0, 50), (2750.5, 0.0008, 10.0, 12.5, 20),
                                    (1500.0, 0.001, 12.5, 12.5, 3)):
        h = F.init_habc(0, 0, nbc, dt, dx, dz, vref)
        o = oracle_lib.init_habc(nbc, dt, dx, dz, vref)
        assert np.array_equal(np.array([h.qx, h.qz, h.qt_x, h.qt_z, h.qxt], dtype=f32), o.q)
        for t1, t2 in ((h.w_vx, o.w_vx), (h.w_vz, o.w_vz), (h.w_tau, o.w_tau)):
            assert np.array_equal(t1, t2)


@pytest.mark.parametrize("off,which", [(0.0, "vx"), (0.5, "vz"), (0.75, "tau")])
def test_weight_tables_equal_full_matrices(off, which, oracle_lib):
    nx, nz, nbc = 37, 29, 6
    h = F.init_habc(nx, nz, nbc, 0.001, 10.0, 10.0, 3000.0)
    full = oracle_lib.habc_weights_full(nx, nz, nbc, off)   # the reference's (nz, nx) matrix
    assert np.array_equal(h.weight_matrix(which, nx, nz), full)


def test_coord_to_index_ties_to_even(oracle_lib):
    pad = 54
    for x, dx in ((1995.0, 10.0), (2005.0, 10.0), (15.0, 10.0), (25.0, 10.0), (12.5, 5.0), (31.25, 12.5),
                  (0.0, 10.0), (3.0e3, 12.5), (1234.56, 10.0)):
        assert F.coord_to_index(x, dx, pad) == oracle_lib.coord_to_index(x, dx, pad)
    assert F.coord_to_index(1995.0, 10.0, pad) == 200 + pad + 1
    assert F.coord_to_index(2005.0, 10.0, pad) == 200 + pad + 1


def test_setup_receivers_and_vref():
    c = runjl_case()
    assert float(c.v_ref) == 3505.0
    med = F.Medium(c.vp.shape[0] + 108, c.vp.shape[1] + 108, 10.0, 10.0, 0, 0, 4, 54, True, *[None] * 5)
    rec = F.setup_receivers(c.rec_x, c.rec_z, med, type="vz")
    assert rec.i[0] == 105 and rec.i[-1] == 405 and (rec.j == 65).all()
    rec64 = F.setup_receivers(c.rec_x.astype(np.float64), c.rec_z.astype(np.float64), med)
    assert np.array_equal(rec64.i, rec.i)
    with pytest.raises(ValueError):
        F.setup_receivers([1.0], [1.0, 2.0], med)


def _mean_scalar_loop(a):
    """Julia's pairwise Float32 sum (blocks under 1024 elements summed in
    order, one scalar add at a time), divided by the length."""
    f32 = np.float32
    v = np.asfortranarray(a, dtype=f32).ravel(order="F")

    def rec(i0, i1):
        if i0 == i1:
            return v[i0]
        if i1 - i0 < 1024:
            s = f32(v[i0] + v[i0 + 1])
            for x in v[i0 + 2:i1 + 1]:
                s = f32(s + x)
            return s
        im = i0 + ((i1 - i0) >> 1)
        return f32(rec(i0, im) + rec(im + 1, i1))

    return f32(rec(0, v.size - 1) / f32(v.size))


@pytest.mark.parametrize("n", [1, 2, 3, 1023, 1024, 1025, 4099, 65537])
def test_julia_mean_block_order(n):
    # the vectorised block sums equal the scalar loop, block boundaries included
    a = (np.random.default_rng(n).random(n) * 3000.0 + 1500.0).astype(np.float32)
    assert F.julia_mean(a) == _mean_scalar_loop(a)


def test_backend_names():
    with pytest.raises(ValueError, match="Unknown backend"):
        F.backend("cpu")
    with pytest.raises(ValueError, match="Unknown backend"):
        F.backend(":cuda")


def test_percentile_nearest_rank():
    from fomo_julia_b200.serving import percentile
    v = list(range(1, 101))
    assert percentile(v, 50) == 50
    assert percentile(v, 99) == 99
    assert percentile(v, 100) == 100
    assert percentile([7.0], 99) == 7.0
    with pytest.raises(ValueError):
        percentile([], 50)
