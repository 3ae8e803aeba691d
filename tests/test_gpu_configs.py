"""Parity on the benchmark workloads themselves, at their full grid sizes.

* the small homogeneous shot exactly as specified (400 x 200, vp 3000 /
  vs 1732 / rho 2000, 8th order, nbc 50, free surface, dt 1 ms, nt 1500,
  10 Hz Ricker at (2000, 20) m, 199 receivers at z = 10 m), recording vx and
  vz, over all 1500 steps;
* the 4444 x 3819 layered shot (padded 4552 x 3927) over its first 60
  steps: every tile launch there overlaps the band pass before it, and the
  stress launch walks its tiles in reverse, as in the timed benchmark;
* the 2000 x 800 medium of the batched workload (padded 2108 x 908): single
  shots over 300 steps, and three of its shots run as one batch.

Gathers and all five final wavefields are compared with the CPU oracle bit
for bit (the kernels evaluate the reference's Float32 expressions in the
same order with IEEE rounding); relative L2 <= 1e-5 per trace is asserted
as well.
"""
import numpy as np
import pytest

import fomo_julia_b200 as F
from fomo_julia_b200 import synthetic
from cases import case_from_workload, oracle_inputs, per_trace_rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5
FIELDS = ("vx", "vz", "txx", "tzz", "txz")


def _gpu(c, b200, n_steps=None):
    """The shot through the C ABI, stopped after n_steps (all nt if None)."""
    med = F.init_medium(c.vp, c.vs, c.rho, c.dx, c.dz, c.nbc, c.fd_order, b200, free_surface=c.free_surface)
    H = F.init_habc(med.nx, med.nz, c.nbc, c.dt, c.dx, c.dz, c.v_ref, b200)
    params = F.sim_params(c.dt, c.nt, c.dx, c.dz, c.fd_order)
    rec = F.setup_receivers(c.rec_x, c.rec_z, med, type=c.rec_type)
    src = F.Source(F.coord_to_index(c.src_x, med.dx, med.pad), F.coord_to_index(c.src_z, med.dz, med.pad),
                   F.ricker_wavelet(c.f0, c.dt, c.nt))
    W = F.Wavefield(med.nx, med.nz, b200)
    stop = c.nt if n_steps is None else n_steps
    r = F.run_shot(b200, W, med, H, F.get_fd_coefficients(c.fd_order), src, rec, params,
                   on_step=lambda W_, info: info.k < stop, step_chunk=stop)
    fields = {f: W.field(f) for f in FIELDS}
    W.release()
    med.release()
    return r, fields


def _oracle(c, oracle, n_steps=None):
    med, h, a, wav, si, sj, ri, rj = oracle_inputs(c, oracle)
    g, fin = oracle.run_shot(med, h, a, c.dt, c.nt, si, sj, wav, ri, rj, c.rec_type, "simd8",
                             final_fields=True, n_steps=n_steps)
    return g, {f: fin[:, :, q] for q, f in enumerate(FIELDS)}


def _assert_bit_exact(g_gpu, g_orc, f_gpu=None, f_orc=None):
    assert g_gpu.shape == g_orc.shape
    rl = per_trace_rel_l2(g_gpu, g_orc)
    assert rl.max() <= TOL, f"gather: max per-trace rel L2 {rl.max():.3e}"
    assert np.array_equal(g_gpu, g_orc), f"gather not bit-identical (max abs {np.abs(g_gpu - g_orc).max():.3e})"
    for f in FIELDS if f_gpu is not None else ():
        assert np.array_equal(f_gpu[f], f_orc[f]), \
            f"field {f} not bit-identical (max abs {np.abs(f_gpu[f] - f_orc[f]).max():.3e})"


@pytest.mark.parametrize("rec_type", ["vx", "vz"])
def test_small_homogeneous_full_shot(rec_type, b200, oracle_lib):
    w = synthetic.small_homogeneous()
    assert (w.nx_in, w.nz_in, w.nt, len(w.rec_x)) == (400, 200, 1500, 199)
    c = case_from_workload(w, rec_type)
    assert float(c.v_ref) == 3000.0
    r, f_gpu = _gpu(c, b200)
    g_orc, f_orc = _oracle(c, oracle_lib)
    assert r.stats["steps"] == 1500 and np.abs(g_orc).max() > 0
    _assert_bit_exact(r.gather, g_orc, f_gpu, f_orc)


@pytest.fixture(params=["fused", "split"])
def step_mode(request):
    """The fused step and the split launches."""
    F.set_step_kernel(request.param)
    yield request.param
    F.set_step_kernel("auto")


def test_large_layered_first_steps(b200, oracle_lib, step_mode):
    n = 60
    w = synthetic.large_layered()
    c = case_from_workload(w)
    r, f_gpu = _gpu(c, b200, n_steps=n)
    assert (r.stats["kernel_launches"] <= n + 1) == (step_mode == "fused")
    assert r.stats["steps"] == n
    g_orc, f_orc = _oracle(c, oracle_lib, n_steps=n)
    assert (r.gather.shape, f_gpu["vx"].shape) == ((11520, 1000), (4552, 3927))
    assert np.abs(f_orc["vz"]).max() > 0
    _assert_bit_exact(r.gather, g_orc, f_gpu, f_orc)


@pytest.mark.parametrize("shot", [0, 33])
def test_batched_medium_single_shots(shot, b200, oracle_lib, step_mode):
    n = 300
    w = synthetic.batched_layered()
    c = case_from_workload(w, shot=shot, nt=n)
    r, f_gpu = _gpu(c, b200)
    g_orc, f_orc = _oracle(c, oracle_lib)
    assert f_gpu["vx"].shape == (2108, 908)
    _assert_bit_exact(r.gather, g_orc, f_gpu, f_orc)


def test_batched_medium_three_shots_as_one_batch(b200, oracle_lib):
    n = 300
    w = synthetic.batched_layered()
    shots = [0, 31, 63]
    med = F.init_medium(w.vp, w.vs, w.rho, w.dx, w.dz, w.nbc, w.fd_order, b200, free_surface=w.free_surface)
    c0 = case_from_workload(w, nt=n)
    H = F.init_habc(med.nx, med.nz, w.nbc, c0.dt, w.dx, w.dz, c0.v_ref, b200)
    wav = F.ricker_wavelet(w.f0, c0.dt, n)
    cfg = F.multi_shot_config([w.src_x[s] for s in shots], [w.src_z[s] for s in shots], wav)
    rec = F.setup_receivers(w.rec_x, w.rec_z, med, type="vz")
    res = F.run_batch(b200, med, H, F.get_fd_coefficients(w.fd_order), rec, cfg,
                      F.sim_params(c0.dt, n, w.dx, w.dz, w.fd_order))
    med.release()
    for k, s in enumerate(shots):
        g_orc, _ = _oracle(case_from_workload(w, shot=s, nt=n), oracle_lib)
        _assert_bit_exact(res[k].gather, g_orc)
