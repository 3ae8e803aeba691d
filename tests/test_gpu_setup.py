"""Device-side medium set-up (fomo_b200_medium_create_from_model) against
the host restatement of init_medium (init.jl:68-158), bit for bit, and a
shot on it against the same shot on the host-built medium."""
import numpy as np
import pytest

import fomo_julia_b200 as F
from cases import layered

pytestmark = pytest.mark.gpu

CASES = [
    dict(nx_in=40, nz_in=30, seed=1, nbc=6, fd_order=8),
    dict(nx_in=37, nz_in=33, seed=2, nbc=5, fd_order=4, water_rows=4),   # vs = 0: mu = 0, 1/mu = Inf
    dict(nx_in=231, nz_in=90, seed=13, nbc=10, fd_order=12, water_rows=6),
]


@pytest.mark.parametrize("kw", CASES)
def test_device_medium_equals_host_medium(b200, kw):
    c = layered(**kw)
    host = F.init_medium(c.vp, c.vs, c.rho, c.dx, c.dz, c.nbc, c.fd_order, b200, free_surface=c.free_surface)
    dev = F.init_medium_device(c.vp, c.vs, c.rho, c.dx, c.dz, c.nbc, c.fd_order, b200, free_surface=c.free_surface)
    assert (dev.nx, dev.nz, dev.pad, dev.M) == (host.nx, host.nz, host.pad, host.M)
    want = [host.rho_vx, host.rho_vz, host.lam, host.mu_txx, host.mu_txz]
    for q in range(5):
        got = dev.array(q)
        assert np.array_equal(got, want[q]), f"array {q}"
        assert np.array_equal(host.array(q), want[q]), f"host upload of array {q}"
    # a shot on either medium gives the same gather
    H = F.init_habc(host.nx, host.nz, c.nbc, c.dt, c.dx, c.dz, c.v_ref, b200)
    params = F.sim_params(c.dt, 80, c.dx, c.dz, c.fd_order)
    a = F.get_fd_coefficients(c.fd_order)
    wav = F.ricker_wavelet(c.f0, c.dt, 80)
    src = F.Source(host.nx // 2, host.pad + 3, wav)
    rec = F.setup_receivers(c.rec_x, c.rec_z, host, type=c.rec_type)
    W = F.Wavefield(host.nx, host.nz, b200)
    g1 = F.run_shot(b200, W, host, H, a, src, rec, params).gather
    g2 = F.run_shot(b200, W, dev, H, a, src, rec, params).gather
    W.release()
    assert np.array_equal(g1, g2)
    host.release()
    dev.release()


def test_snapshots_match_host_extraction(b200):
    """Device frames equal the reference's _extract_frame! of the downloaded fields."""
    c = layered(61, 43, seed=5, nbc=6, fd_order=8, nt=60)
    med = F.init_medium(c.vp, c.vs, c.rho, c.dx, c.dz, c.nbc, c.fd_order, b200, free_surface=c.free_surface)
    H = F.init_habc(med.nx, med.nz, c.nbc, c.dt, c.dx, c.dz, c.v_ref, b200)
    params = F.sim_params(c.dt, 60, c.dx, c.dz, c.fd_order)
    src = F.Source(med.nx // 2, med.pad + 3, F.ricker_wavelet(c.f0, c.dt, 60))
    rec = F.setup_receivers(c.rec_x, c.rec_z, med, type=c.rec_type)
    W = F.Wavefield(med.nx, med.nz, b200)
    recd = F.SnapshotRecorder(F.VideoConfig(fields=["p", "vel", "vx", "vz"], skip=20, downsample=3))
    seen = []

    def hook(Wh, info):
        recd(Wh, info)
        vx, vz, txx, tzz = (Wh.field(n) for n in ("vx", "vz", "txx", "tzz"))
        raw = {"p": (txx + tzz) * np.float32(0.5), "vel": np.sqrt(vx * vx + vz * vz), "vx": vx, "vz": vz}
        if info.k % 20 == 0:
            for f, a in raw.items():
                want = a[::3, ::3]
                assert np.array_equal(recd.frames[f][-1][2], want), (f, info.k)
            seen.append(info.k)
        return True

    F.run_shot(b200, W, med, H, F.get_fd_coefficients(c.fd_order), src, rec, params, on_step=hook, step_chunk=10)
    assert seen == [20, 40, 60]
    assert recd.stack("p").shape == (3, -(-med.nx // 3), -(-med.nz // 3))
    W.release()
    med.release()
