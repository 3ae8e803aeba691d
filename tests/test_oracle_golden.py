"""The oracle against the reference's one known-answer artefact, shot_1.bin."""
import numpy as np
import pytest

from cases import golden_gather, oracle_inputs, per_trace_rel_l2, runjl_case

TOL = 1e-5  # relative L2 per trace


@pytest.fixture(scope="module")
def runjl(oracle_lib):
    c = runjl_case()
    return c, oracle_inputs(c, oracle_lib)


def test_runjl_recipe_indices(runjl):
    c, (med, h, a, wav, si, sj, ri, rj) = runjl
    assert c.nt == 800 and abs(float(c.dt) - 0.00125) < 1e-9
    assert float(c.v_ref) == 3505.0
    assert (med.nx, med.nz, med.pad) == (508, 308, 54)
    # x_src = 1995 m -> round(199.5) = 200 (ties to even) -> 200 + 54 + 1
    assert (si, sj) == (255, 60)
    assert ri[0] == 105 and ri[-1] == 405 and set(rj.tolist()) == {65}


def test_oracle_reproduces_shot_1(runjl, oracle_lib):
    c, (med, h, a, wav, si, sj, ri, rj) = runjl
    g = oracle_lib.run_shot(med, h, a, c.dt, c.nt, si, sj, wav, ri, rj, "vz", "simd8")
    ref = golden_gather()
    rl = per_trace_rel_l2(g, ref)
    assert g.shape == ref.shape == (800, 100)
    assert rl.max() <= TOL, f"max per-trace rel L2 {rl.max():.3e}"
    k, r = np.unravel_index(np.abs(ref).argmax(), ref.shape)
    assert (k, r) == np.unravel_index(np.abs(g).argmax(), g.shape)


def test_habc_order_pin(runjl, oracle_lib):
    """The HABC loop semantics are pinned by shot_1.bin: only the 8-lane
    chunked order keeps the right-edge traces within tolerance."""
    c, (med, h, a, wav, si, sj, ri, rj) = runjl
    ref = golden_gather()
    for mode in ("jacobi", "sequential"):
        g = oracle_lib.run_shot(med, h, a, c.dt, c.nt, si, sj, wav, ri, rj, "vz", mode)
        rl = per_trace_rel_l2(g, ref)
        assert rl.max() > 2 * TOL, mode
        assert rl[:50].max() <= TOL, mode  # left half unaffected


def test_float64_oracle_close(runjl, oracle_lib):
    c, (med, h, a, wav, si, sj, ri, rj) = runjl
    med64 = oracle_lib.init_medium(c.vp, c.vs, c.rho, c.dx, c.dz, c.nbc, c.fd_order, True, dtype=np.float64)
    h64 = oracle_lib.init_habc(c.nbc, float(c.dt), c.dx, c.dz, float(c.v_ref), dtype=np.float64)
    g64 = oracle_lib.run_shot(med64, h64, oracle_lib.fd_coefficients(8, np.float64), float(c.dt), c.nt, si, sj,
                              oracle_lib.ricker(c.f0, float(c.dt), c.nt, np.float64), ri, rj, "vz", "simd8",
                              dtype=np.float64)
    assert per_trace_rel_l2(g64, golden_gather()).max() <= TOL
