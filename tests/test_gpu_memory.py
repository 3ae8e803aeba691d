"""Device memory of media, wavefields and shots comes from the library's
stream-ordered pool.  An allocation that cannot fit must fail with
FOMO_ENOMEM and a message, leave no CUDA error behind for later calls, and
leave the pool usable: shots before and after the failure give the same
gather."""
import ctypes

import numpy as np
import pytest

import fomo_julia_b200 as F
from fomo_julia_b200 import _lib
from cases import layered

pytestmark = pytest.mark.gpu


def _shot(c, b200):
    med = F.init_medium(c.vp, c.vs, c.rho, c.dx, c.dz, c.nbc, c.fd_order, b200, free_surface=c.free_surface)
    H = F.init_habc(med.nx, med.nz, c.nbc, c.dt, c.dx, c.dz, c.v_ref, b200)
    params = F.sim_params(c.dt, c.nt, c.dx, c.dz, c.fd_order)
    a = F.get_fd_coefficients(c.fd_order)
    src = F.Source(med.nx // 2, med.pad + 3, F.ricker_wavelet(c.f0, c.dt, c.nt))
    rec = F.setup_receivers(c.rec_x, c.rec_z, med, type=c.rec_type)
    W = F.Wavefield(med.nx, med.nz, b200)
    g = F.run_shot(b200, W, med, H, a, src, rec, params).gather
    W.release()
    med.release()
    return g


def test_oversized_allocation_fails_cleanly(b200):
    c = layered(60, 40, seed=61, nbc=6, fd_order=8, nt=80)
    g0 = _shot(c, b200)
    lib = _lib.load()
    h = ctypes.c_uint64(0)
    # 10 fields of 200000 x 100000 floats: 800 GB, more than any GPU holds
    rc = lib.fomo_b200_wavefield_create(200000, 100000, ctypes.byref(h))
    assert rc == -2, f"expected FOMO_ENOMEM, got {rc}"
    assert b"allocation" in lib.fomo_b200_last_error()
    assert h.value == 0
    g1 = _shot(c, b200)
    assert np.array_equal(g0, g1)


def test_repeated_create_and_destroy_reuses_memory(b200):
    # media, wavefields and shots created and destroyed again and again: same results each time
    c = layered(60, 40, seed=62, nbc=6, fd_order=4, nt=60)
    first = _shot(c, b200)
    for _ in range(5):
        assert np.array_equal(_shot(c, b200), first)
