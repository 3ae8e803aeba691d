"""The allocation-free shot entry point, fomo_b200_run_shot_noalloc.

It serves callers that cannot allocate device memory while a shot runs (a
serving loop whose memory is carved from a fixed pool at start-up, a
framework that forbids cudaMalloc and cudaFree on its latency path): all of
its scratch comes from one static device array.  Here the caller's buffers (the
medium on the device and the output gather) are allocated by torch, as such
a caller would hand them over; the entry point itself allocates nothing.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes
import dataclasses

import numpy as np
import pytest

import fomo_julia_b200 as F
from fomo_julia_b200 import _lib
from cases import layered, per_trace_rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5  # relative L2 per trace, the tolerance of the other parity tests


def _inputs(c, b200):
    med = F.init_medium(c.vp, c.vs, c.rho, c.dx, c.dz, c.nbc, c.fd_order, b200, free_surface=c.free_surface)
    H = F.init_habc(med.nx, med.nz, c.nbc, c.dt, c.dx, c.dz, c.v_ref, b200)
    params = F.sim_params(c.dt, c.nt, c.dx, c.dz, c.fd_order)
    wav = F.ricker_wavelet(c.f0, c.dt, c.nt)
    rec = F.setup_receivers(c.rec_x, c.rec_z, med, type=c.rec_type)
    src = F.Source(F.coord_to_index(c.src_x, med.dx, med.pad), F.coord_to_index(c.src_z, med.dz, med.pad), wav)
    return med, H, params, F.get_fd_coefficients(c.fd_order), src, rec


SCRATCH_BYTES = 48 << 20  # the entry point's static array


def _scratch_need(nx, nz, pitch, nbc, n_rec, iso):
    """Bytes the entry point carves from its array: status word, three weight
    tables, receiver offsets, 2 or 4 buoyancy planes, 5 band planes of nbc
    rows, two wavefield copies of 5 fields (each piece 256-byte aligned)."""
    a = lambda n: (n + 255) // 256 * 256  # noqa: E731
    plane = pitch * nz * 4
    return (256 + a(3 * (nbc + 2) * 4) + a(n_rec * 4) + a((2 if iso else 4) * plane) + a(5 * nbc * pitch * 4)
            + 10 * plane)


def _caller_buffers(med, n_rec, nt, pitch):
    """Caller-owned device buffers, as such a caller hands them over: the
    medium rows padded to `pitch` floats and the gather."""
    import torch
    dev = torch.device("cuda", 0)
    arrays = []
    for host in (med.rho_vx, med.rho_vz, med.lam, med.mu_txx, med.mu_txz):
        t = torch.zeros((med.nz, pitch), dtype=torch.float32, device=dev)
        t[:, :med.nx] = torch.from_numpy(np.ascontiguousarray(np.asarray(host, dtype=np.float32).T)).to(dev)
        arrays.append(t)
    gather = torch.empty((n_rec, nt), dtype=torch.float32, device=dev)  # [nt x n_rec] column major
    return arrays, gather


def _noalloc_twice_vs_run_shot(c, b200, pitch_of=lambda nx: (nx + 3) // 4 * 4, expect_need=None):
    import torch
    med, H, params, a, src, rec = _inputs(c, b200)

    # the existing, allocating entry point
    W = F.Wavefield(med.nx, med.nz, b200)
    ref = F.run_shot(b200, W, med, H, a, src, rec, params).gather
    W.release()

    pitch = pitch_of(med.nx)
    if expect_need is not None:
        expect_need(_scratch_need(med.nx, med.nz, pitch, c.nbc, len(rec.i), float(c.dx) == float(c.dz)))
    arrays, gather = _caller_buffers(med, len(rec.i), c.nt, pitch)
    keep = []
    hs = F.elastic2d._ctypes_habc(H, keep)
    ss = F.elastic2d._ctypes_shot(a, params, src, rec, keep)
    stream = torch.cuda.current_stream(torch.device("cuda", 0))
    lib = _lib.load()
    for call in range(2):
        gather.fill_(float("nan"))  # every sample must be written by the call
        rc = lib.fomo_b200_run_shot_noalloc(med.nx, med.nz, med.M, med.pad, int(med.is_free_surface),
                                            *[t.data_ptr() for t in arrays], pitch, ctypes.byref(hs),
                                            ctypes.byref(ss), gather.data_ptr(), stream.cuda_stream)
        assert rc == 0, lib.fomo_b200_last_error().decode()
        g = gather.cpu().numpy().T
        assert np.isfinite(g).all(), f"call {call + 1}: gather samples left unwritten"
        rl = per_trace_rel_l2(g, ref)
        assert rl.max() <= TOL, f"call {call + 1}: max per-trace rel L2 {rl.max():.3e}"
        assert np.array_equal(g, ref), f"call {call + 1}: not bit-identical to fomo_b200_run_shot"
    med.release()


def test_noalloc_matches_run_shot_twice(b200):
    c = layered(61, 47, seed=51, nbc=8, fd_order=8, nt=160, rec_type="p", n_rec=29)
    _noalloc_twice_vs_run_shot(c, b200)


def test_noalloc_dz_ne_dx_without_free_surface(b200):
    # dtx != dtz: four buoyancy planes in the scratch; no free surface: a top
    # HABC band; vx receivers
    c = layered(83, 51, seed=53, nbc=9, fd_order=6, nt=140, free_surface=False, rec_type="vx", n_rec=21)
    c = dataclasses.replace(c, dz=13.0, name=c.name + "dz13")
    _noalloc_twice_vs_run_shot(c, b200)


def test_noalloc_grid_just_inside_the_limit(b200):
    # the tallest grid of this width whose scratch still fits the array
    nbc, order, n_rec = 50, 8, 31
    pad = nbc + order // 2
    nx = 1000
    pitch = (nx + 3) // 4 * 4
    nz = 2 * pad + 1
    while _scratch_need(nx, nz + 1, pitch, nbc, n_rec, True) <= SCRATCH_BYTES:
        nz += 1
    assert _scratch_need(nx, nz, pitch, nbc, n_rec, True) > SCRATCH_BYTES - 48 * pitch * 4
    c = layered(nx - 2 * pad, nz - 2 * pad, seed=54, nbc=nbc, fd_order=order, nt=40, n_rec=n_rec)
    _noalloc_twice_vs_run_shot(c, b200, expect_need=lambda need: need <= SCRATCH_BYTES)


def test_noalloc_rejects_grids_beyond_its_scratch(b200):
    import torch
    c = layered(30, 24, seed=52, nbc=5, fd_order=8, nt=10)
    med, H, params, a, src, rec = _inputs(c, b200)
    t = torch.zeros(1024, dtype=torch.float32, device="cuda")
    keep = []
    hs = F.elastic2d._ctypes_habc(H, keep)
    ss = F.elastic2d._ctypes_shot(a, params, src, rec, keep)
    lib = _lib.load()
    nx = nz = 4000  # 10 fields of 4000 x 4000 floats are far more than the static array
    rc = lib.fomo_b200_run_shot_noalloc(nx, nz, med.M, med.pad, 1, *[t.data_ptr()] * 5, nx, ctypes.byref(hs),
                                        ctypes.byref(ss), t.data_ptr(), None)
    assert rc == -1  # FOMO_EINVAL
    assert b"scratch" in lib.fomo_b200_last_error()
    # one row more than the tallest grid that fits (test_noalloc_grid_just_inside_the_limit)
    nx, pitch = 1000, 1000
    nz = 2 * med.pad + 1
    while _scratch_need(nx, nz, pitch, c.nbc, len(rec.i), True) <= SCRATCH_BYTES:
        nz += 1
    rc = lib.fomo_b200_run_shot_noalloc(nx, nz, med.M, med.pad, 1, *[t.data_ptr()] * 5, pitch, ctypes.byref(hs),
                                        ctypes.byref(ss), t.data_ptr(), None)
    assert rc == -1
    assert b"scratch" in lib.fomo_b200_last_error()
    med.release()
