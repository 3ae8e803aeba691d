"""Batched shots and the shot server against single shots.

A batched or served shot runs the same per-block code as a single shot on
its own wavefield, so its gather must equal fomo_b200_run_shot's bit for bit,
whatever else runs in the same launches (other shots of the same medium,
other media, other FD orders, shots joining and leaving mid-run).  The single
path itself is checked against the oracle in test_gpu_parity.py; one batched
shot is also checked against the oracle directly here.
"""
import dataclasses
import time
from dataclasses import dataclass

import numpy as np
import pytest

import fomo_julia_b200 as F
from fomo_julia_b200._lib import FomoError
from cases import Case, layered, oracle_inputs

pytestmark = pytest.mark.gpu
WAIT_S = 300.0


@dataclass
class Setup:
    case: Case
    med: F.Medium
    H: F.HABCConfig
    a: np.ndarray
    rec: F.Receivers


def setup(c: Case, b200) -> Setup:
    med = F.init_medium(c.vp, c.vs, c.rho, c.dx, c.dz, c.nbc, c.fd_order, b200, free_surface=c.free_surface)
    H = F.init_habc(med.nx, med.nz, c.nbc, c.dt, c.dx, c.dz, c.v_ref, b200)
    rec = F.setup_receivers(c.rec_x, c.rec_z, med, type=c.rec_type)
    return Setup(c, med, H, F.get_fd_coefficients(c.fd_order), rec)


def params_of(S: Setup, nt=None):
    c = S.case
    return F.sim_params(c.dt, nt or c.nt, c.dx, c.dz, c.fd_order)


def source(S: Setup, x, z, nt=None):
    c = S.case
    wav = F.ricker_wavelet(c.f0, c.dt, nt or c.nt)
    return F.Source(F.coord_to_index(x, S.med.dx, S.med.pad), F.coord_to_index(z, S.med.dz, S.med.pad), wav)


def single(S: Setup, src, b200, nt=None):
    W = F.Wavefield(S.med.nx, S.med.nz, b200)
    r = F.run_shot(b200, W, S.med, S.H, S.a, src, S.rec, params_of(S, nt))
    W.release()
    return r.gather


def source_xs(c: Case, n):
    nx_in = c.vp.shape[0]
    return [float(c.dx) * v for v in np.linspace(-c.nbc // 2, nx_in + c.nbc // 2, n)]


MEDIUM_A = dict(nx_in=231, nz_in=90, seed=13, nbc=10, fd_order=8, nt=100, n_rec=41)


@pytest.fixture(params=["fused", "split"])
def step_mode(request):
    """Fused-step batch launches and the split launches ("auto" runs the split ones)."""
    F.set_step_kernel(request.param)
    yield request.param
    F.set_step_kernel("auto")


def test_batch_equals_single_shots_and_oracle(b200, oracle_lib, step_mode):
    c = layered(**MEDIUM_A)
    S = setup(c, b200)
    xs = source_xs(c, 6)
    cfg = F.multi_shot_config(xs, [float(c.dx) * 3] * len(xs), F.ricker_wavelet(c.f0, c.dt, c.nt))
    res = F.run_shots(b200, None, S.med, S.H, S.a, S.rec, cfg, params_of(S), batched=True)
    assert len(res) == len(xs)
    assert res[0].stats["steps"] == len(xs) * c.nt
    # one fused launch per batch step, or four split launches (tiles and band passes of both half steps)
    per_step = res[0].stats["kernel_launches"] / c.nt
    assert (per_step < 2.5) == (step_mode == "fused"), per_step
    for k, r in enumerate(res):
        src = F.create_source(S.med, cfg.shots[k], cfg.wavelet)
        assert (r.src_i, r.src_j) == (src.i, src.j)
        assert np.array_equal(r.gather, single(S, src, b200)), f"shot {k}: batched gather differs from the single shot"
    # shot 2 against the oracle directly
    c2 = layered(**MEDIUM_A)
    c2.src_x, c2.src_z = xs[2], float(c.dx) * 3
    med, h, a, wav, si, sj, ri, rj = oracle_inputs(c2, oracle_lib)
    g_orc = oracle_lib.run_shot(med, h, a, c2.dt, c2.nt, si, sj, wav, ri, rj, c2.rec_type, "simd8")
    assert np.array_equal(res[2].gather, g_orc)
    S.med.release()


@pytest.mark.parametrize("K", [1, 5, 8, 32])
def test_steps_per_launch_do_not_change_results(b200, K):
    c = layered(**MEDIUM_A)
    S = setup(c, b200)
    xs = source_xs(c, 3)
    nts = [100, 37, 64]
    refs = [single(S, source(S, x, 20.0, nt), b200, nt) for x, nt in zip(xs, nts)]
    with F.ShotServer(steps_per_launch=K) as srv:
        ts = [srv.submit(S.med, S.H, S.a, source(S, x, 20.0, nt), S.rec, params_of(S, nt), shot_id=i)
              for i, (x, nt) in enumerate(zip(xs, nts))]
        out = [srv.wait(t, timeout=WAIT_S) for t in ts]
        st = srv.stats()
    for r, g in zip(out, refs):
        assert np.array_equal(r.gather, g)
    assert st["completed"] == 3 and st["failed"] == 0
    S.med.release()


def test_batch_with_dz_not_dx(b200):
    """dz != dx: four buoyancy arrays per medium (the tiles load and prefetch
    all four); a batch of three shots equals the shots run alone."""
    c = dataclasses.replace(layered(**MEDIUM_A), dz=13.0)
    S = setup(c, b200)
    xs = source_xs(c, 3)
    nts = [100, 61, 80]
    refs = [single(S, source(S, x, 26.0, nt), b200, nt) for x, nt in zip(xs, nts)]
    with F.ShotServer(steps_per_launch=8) as srv:
        ts = [srv.submit(S.med, S.H, S.a, source(S, x, 26.0, nt), S.rec, params_of(S, nt), shot_id=i)
              for i, (x, nt) in enumerate(zip(xs, nts))]
        out = [srv.wait(t, timeout=WAIT_S) for t in ts]
    for r, g in zip(out, refs):
        assert np.array_equal(r.gather, g)
    assert max(r.stats["batch_peak"] for r in out) >= 2
    S.med.release()


def _mixed_setups(b200):
    return [
        setup(layered(**MEDIUM_A), b200),
        setup(layered(41, 27, seed=3, nbc=7, fd_order=12, nt=120, rec_type="p", water_rows=3), b200),
        setup(layered(37, 33, seed=2, nbc=5, fd_order=4, nt=150, rec_type="vx", free_surface=False), b200),
        setup(layered(150, 70, seed=15, nbc=60, fd_order=4, nt=90, rec_type="vx"), b200),
    ]


def test_server_mixed_media_orders_and_arrivals(b200):
    """Shots over four media (orders 4, 8, 12; with and without free
    surface; uneven nt and receivers) arrive in two waves; each result
    equals the shot run alone."""
    Ss = _mixed_setups(b200)
    jobs = []
    rng = np.random.default_rng(5)
    for w in range(2):
        for m, S in enumerate(Ss):
            c = S.case
            nt = int(c.nt - 20 * w - 7 * m)
            x = float(rng.uniform(0, c.dx * (c.vp.shape[0] - 1)))
            jobs.append((w, S, nt, x))
    refs = [single(S, source(S, x, float(S.case.dx) * 2, nt), b200, nt) for _, S, nt, x in jobs]
    with F.ShotServer() as srv:
        tickets = []
        for w in range(2):
            for k, (wj, S, nt, x) in enumerate(jobs):
                if wj == w:
                    tickets.append((k, srv.submit(S.med, S.H, S.a, source(S, x, float(S.case.dx) * 2, nt), S.rec,
                                                  params_of(S, nt), shot_id=k)))
            if w == 0:
                time.sleep(0.02)  # the second wave arrives while the first runs
        results = {k: srv.wait(t, timeout=WAIT_S) for k, t in tickets}
        st = srv.stats()
    for k, r in results.items():
        assert np.array_equal(r.gather, refs[k]), f"request {k} differs from its single run"
        assert r.stats["steps"] == jobs[k][2]
        assert r.stats["latency_ms"] >= r.stats["run_ms"] >= 0
    assert max(r.stats["batch_peak"] for r in results.values()) >= 2
    assert st["completed"] == len(jobs) and st["peak_shots"] >= 2
    for S in Ss:
        S.med.release()


def test_same_result_alone_and_in_the_mix(b200):
    Ss = _mixed_setups(b200)
    S = Ss[0]
    x = source_xs(S.case, 5)[1]
    with F.ShotServer() as srv:
        alone = srv.wait(srv.submit(S.med, S.H, S.a, source(S, x, 30.0), S.rec, params_of(S)), timeout=WAIT_S)
        mix = []
        for j, T in enumerate(Ss * 2):
            mix.append(srv.submit(T.med, T.H, T.a, source(T, source_xs(T.case, 8)[j % 8], 20.0), T.rec,
                                  params_of(T)))
        target = srv.submit(S.med, S.H, S.a, source(S, x, 30.0), S.rec, params_of(S))
        mix.append(srv.submit(S.med, S.H, S.a, source(S, x + 40.0, 30.0), S.rec, params_of(S)))
        in_mix = srv.wait(target, timeout=WAIT_S)
        srv.wait_all(mix, timeout=WAIT_S)
    assert alone.stats["batch_peak"] == 1
    assert in_mix.stats["batch_peak"] >= 2
    assert np.array_equal(alone.gather, in_mix.gather)
    for T in Ss:
        T.med.release()


def test_hbm_budget_admission(b200):
    c = layered(**MEDIUM_A)
    S = setup(c, b200)
    pitch = (S.med.nx + 31) // 32 * 32
    plane = pitch * S.med.nz * 4
    budget = 10 * plane + 2 * plane + (1 << 20)  # one shot and the buoyancy, not two shots
    xs = source_xs(c, 3)
    refs = [single(S, source(S, x, 20.0), b200) for x in xs]
    with F.ShotServer(hbm_budget_bytes=budget) as srv:
        ts = [srv.submit(S.med, S.H, S.a, source(S, x, 20.0), S.rec, params_of(S)) for x in xs]
        out = [srv.wait(t, timeout=WAIT_S) for t in ts]
        st = srv.stats()
        SB = setup(layered(500, 300, seed=21, nbc=10, fd_order=8, nt=10), b200)
        with pytest.raises(FomoError) as e:
            srv.submit(SB.med, SB.H, SB.a, source(SB, 500.0, 20.0), SB.rec, params_of(SB))
        assert e.value.code == -2
        SB.med.release()
    for r, g in zip(out, refs):
        assert np.array_equal(r.gather, g)
        assert r.stats["batch_peak"] == 1
    assert st["peak_shots"] == 1
    assert st["peak_bytes"] <= budget
    S.med.release()


def test_cancel_and_medium_in_use(b200):
    c = layered(41, 27, seed=3, nbc=7, fd_order=8, nt=400)
    S = setup(c, b200)
    with F.ShotServer(max_shots=1) as srv:
        ts = [srv.submit(S.med, S.H, S.a, source(S, 100.0 + 20 * k, 20.0), S.rec, params_of(S)) for k in range(4)]
        srv.cancel(ts[3])
        with pytest.raises(FomoError) as e:
            S.med.release()
        assert e.value.code == -1 and S.med.handle
        with pytest.raises(FomoError) as e:
            srv.wait(ts[3], timeout=WAIT_S)
        assert e.value.code == -5
        for t in ts[:3]:
            srv.wait(t, timeout=WAIT_S)
        st = srv.stats()
    assert st["cancelled"] == 1 and st["completed"] == 3 and st["peak_shots"] == 1
    S.med.release()
    assert S.med.handle == 0


def test_more_media_than_one_launch_holds(b200):
    """18 media of one order: the server splits them over two launch sets."""
    Ss = [setup(layered(30 + k, 24 + (k % 5), seed=40 + k, nbc=5, fd_order=8, nt=60), b200) for k in range(18)]
    refs = [single(S, source(S, 100.0, 20.0), b200) for S in Ss]
    with F.ShotServer() as srv:
        ts = [srv.submit(S.med, S.H, S.a, source(S, 100.0, 20.0), S.rec, params_of(S)) for S in Ss]
        out = [srv.wait(t, timeout=WAIT_S) for t in ts]
    for r, g in zip(out, refs):
        assert np.array_equal(r.gather, g)
    for S in Ss:
        S.med.release()


def test_bounded_device_wait_reports_timeout(b200):
    """The kernels' bounded wait, run on a barrier nothing completes, ends
    with FOMO_ETIMEOUT and leaves the context usable."""
    import ctypes
    from fomo_julia_b200._lib import call
    st = ctypes.c_int32(0)
    call("fomo_b200_selftest_wait", 1000, ctypes.byref(st))
    assert st.value == -4
    c = layered(41, 27, seed=3, nbc=7, fd_order=8, nt=50)
    S = setup(c, b200)
    g = single(S, source(S, 100.0, 20.0), b200)
    assert np.isfinite(g).all() and np.abs(g).max() > 0
    S.med.release()


def test_server_rejects_bad_requests(b200):
    import ctypes
    from fomo_julia_b200._lib import FomoHabc, FomoShot, call
    c = layered(41, 27, seed=3, nbc=7, fd_order=8, nt=50)
    S = setup(c, b200)
    with F.ShotServer() as srv:
        t = ctypes.c_uint64(0)
        with pytest.raises(FomoError) as e:  # a medium handle that does not exist
            call("fomo_b200_server_submit", srv.handle, 987654, ctypes.byref(FomoHabc()), ctypes.byref(FomoShot()),
                 None, ctypes.byref(t))
        assert e.value.code == -1
        bad = layered(41, 27, seed=3, nbc=7, fd_order=8, nt=50)
        bad.src_x = 1.0e6  # source outside the grid
        with pytest.raises(FomoError):
            srv.submit(S.med, S.H, S.a, source(S, bad.src_x, 20.0), S.rec, params_of(S))
        with pytest.raises(FomoError):
            srv.wait(F.Ticket(424242, 0, None, None, None))
        ok = srv.wait(srv.submit(S.med, S.H, S.a, source(S, 100.0, 20.0), S.rec, params_of(S)), timeout=WAIT_S)
        assert ok.stats["steps"] == 50
    with pytest.raises(FomoError):
        call("fomo_b200_server_destroy", 987654)
    S.med.release()


def test_tune_cache_file(b200, tmp_path, monkeypatch):
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("FOMO_B200_TUNE_CACHE", str(path))
    c = layered(97, 61, seed=8, nbc=6, fd_order=8, nt=400)
    S = setup(c, b200)
    with F.ShotServer() as srv:  # autotuned K: the candidates are timed on live chunks
        srv.wait_all([srv.submit(S.med, S.H, S.a, source(S, 100.0 + 30 * k, 20.0), S.rec, params_of(S))
                      for k in range(3)], timeout=WAIT_S)
    lines = path.read_text().split("\n")
    assert any(l.startswith(f"{S.med.nx} {S.med.nz} 4 1 ") for l in lines), lines
    S.med.release()


def test_step_kernel_choice_in_tune_cache_file(b200, tmp_path, monkeypatch):
    # a grid's first shot times the split launches and the fused step on live steps and
    # records the faster in the cache file; the shot is the same bits either way
    path = tmp_path / "tune.txt"
    path.write_text("101 67 4 0 8\n")  # a server line first: both readers skip the other's lines
    monkeypatch.setenv("FOMO_B200_TUNE_CACHE", str(path))
    c = layered(103, 59, seed=9, nbc=7, fd_order=8, nt=120)
    S = setup(c, b200)
    g = single(S, source(S, 300.0, 20.0), b200)
    F.set_step_kernel("split")
    try:
        ref = single(S, source(S, 300.0, 20.0), b200)
    finally:
        F.set_step_kernel("auto")
    assert np.array_equal(g, ref)
    lines = [l.split() for l in path.read_text().split("\n") if l.startswith("step ")]
    assert [l[1:7] for l in lines] == [[str(S.med.nx), str(S.med.nz), "4", "7", "1", "1"]], lines
    assert lines[0][7] in ("0", "1")
    S.med.release()
