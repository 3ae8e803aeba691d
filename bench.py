#!/usr/bin/env python
"""Benchmark of the Elastic2D time-stepping path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step is one complete shot of the workload: the 4444 x 3819 layered
medium, 8th order, nbc 50, free surface, nt = 11520 (the shape of the
reference's only published timing, README.md:93-102).  Metric: Gcell-steps/s
over padded cells (4552 x 3927) x nt, whole job (all ranks).

Multi-GPU: one process per GPU (torchrun); shots are independent, so every
rank runs its own shot with no data-path collective (weak scaling).  The
timed region is bracketed by a barrier and a device synchronisation and
timed with CUDA events on the library's stream; the max over ranks is taken.

``--impl reference`` times the CPU restatement of the reference (the
oracle/ port; Julia is not available) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

PUBLISHED_CUDA_GCELLS = 1.14   # README.md:102: < 3 min on an RTX 3060 -> > 1.14 Gcell-steps/s
METRIC = "Gcell-steps/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--nt", type=int, default=None, help="override nt (development only: not the workload)")
    p.add_argument("--profile-steps", type=int, default=200)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-batched", action="store_true", help="skip the batched-shots section")
    p.add_argument("--no-serving", action="store_true", help="skip the serving section")
    p.add_argument("--batch-nt", type=int, default=None, help="override nt of the batched section (development)")
    p.add_argument("--serve-requests", type=int, default=400,
                   help="requests of the serving sample (the full stream of the serving workload is 2000)")
    p.add_argument("--serve-load", type=float, default=4.0,
                   help="offered load of the serving sample, as a multiple of the sequential plain capacity")
    p.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch section")
    p.add_argument("--step-kernel", choices=["auto", "split", "fused"], default="auto",
                   help="single-shot time-step kernels: the faster on the grid, timed on live steps (auto), "
                        "or one of the two")
    p.add_argument("--segs", type=int, default=0, help="fused step: row segments per column strip (0 = auto)")
    return p.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=10)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- workload
def make_workload(nt_override):
    from fomo_julia_b200 import synthetic
    return synthetic.large_layered(seed=1, nt=nt_override)


def host_inputs(w):
    """Host-side set-up exactly as the reference's init.jl does it."""
    import fomo_julia_b200 as F
    pad = w.nbc + w.fd_order // 2
    lam, mu, mu_txz, rho_vx, rho_vz = F.compute_staggered_params(
        F.pad_array(w.vp, pad), F.pad_array(w.vs, pad), F.pad_array(w.rho, pad))
    nx, nz = w.nx_in + 2 * pad, w.nz_in + 2 * pad
    v_ref = F.julia_mean(w.vp)  # mean(vp), run.jl:57
    habc = F.init_habc(nx, nz, w.nbc, w.dt, w.dx, w.dz, v_ref)
    habc_v_ref = v_ref
    params = F.sim_params(w.dt, w.nt, w.dx, w.dz, w.fd_order)
    a = F.get_fd_coefficients(w.fd_order)
    wav = F.ricker_wavelet(w.f0, w.dt, w.nt)
    si = F.coord_to_index(w.src_x[0], w.dx, pad)
    sj = F.coord_to_index(w.src_z[0], w.dz, pad)
    ri = np.rint(w.rec_x.astype(np.float32) / np.float32(w.dx)).astype(np.int32) + pad + 1
    rj = np.rint(w.rec_z.astype(np.float32) / np.float32(w.dz)).astype(np.int32) + pad + 1
    return dict(pad=pad, nx=nx, nz=nz, arrays=(rho_vx, rho_vz, lam, mu, mu_txz), habc=habc, habc_v_ref=habc_v_ref,
                params=params,
                a=a, wav=wav, si=si, sj=sj, ri=ri, rj=rj)


# ---------------------------------------------------------------- reference arm
def cpu_sample(w, hi, seconds: float, threads: int = 0, keep=False):
    """Times the oracle (CPU restatement of the reference) on the first time
    steps of the same shot; returns (Gcell-steps/s, steps, cores, seconds)
    and, with keep, also the oracle's gather and final fields (nx, nz, 5)."""
    import oracle
    oracle.build()
    med = oracle.OMedium(hi["nx"], hi["nz"], w.fd_order // 2, hi["pad"], w.nbc, w.dx, w.dz, w.free_surface,
                         *hi["arrays"])
    h = oracle.OHabc(w.nbc, np.array([hi["habc"].qx, hi["habc"].qz, hi["habc"].qt_x, hi["habc"].qt_z,
                                      hi["habc"].qxt], dtype=np.float32),
                     hi["habc"].w_vx, hi["habc"].w_vz, hi["habc"].w_tau)
    cells = hi["nx"] * hi["nz"]
    out = {}

    def run(n, final=False):
        t = time.perf_counter()
        r = oracle.run_shot(med, h, hi["a"], w.dt, w.nt, hi["si"], hi["sj"], hi["wav"], hi["ri"], hi["rj"], "vz",
                            "simd8", n_steps=n, n_threads=threads, final_fields=final)
        dt = time.perf_counter() - t
        if final:
            out["gather"], out["fields"] = r
        return dt

    t1 = run(2)
    n = max(2, min(w.nt, int(seconds / max(t1 / 2, 1e-6))))
    t = run(n, final=keep)
    cores = threads or oracle.max_threads()
    if keep:
        return cells * n / t / 1e9, n, cores, t, out
    return cells * n / t / 1e9, n, cores, t


def error_stats(g, ref):
    """Max abs error, relative L2 over the whole gather, and the largest
    per-trace relative L2 over the traces the wavefield has reached (trace
    norm above 1e-6 of the largest; earlier traces hold only round-off)."""
    g = np.asarray(g, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    num = np.linalg.norm(g - ref, axis=0)
    den = np.linalg.norm(ref, axis=0)
    live = den > 1e-6 * den.max() if den.size and den.max() > 0 else den > 0
    return {"max_abs": float(np.abs(g - ref).max()) if g.size else 0.0,
            "rel_l2": float(np.linalg.norm(g - ref) / max(np.linalg.norm(ref), 1e-300)),
            "max_trace_rel_l2": float((num[live] / den[live]).max()) if live.any() else 0.0,
            "traces_compared": int(live.sum())}


def float64_gather(w, n):
    """The same shot in Float64 through the oracle (init, HABC tables,
    coefficients, wavelet and time steps all in double), first n steps."""
    import oracle
    import fomo_julia_b200 as F
    med = oracle.init_medium(w.vp, w.vs, w.rho, w.dx, w.dz, w.nbc, w.fd_order, w.free_surface, dtype=np.float64)
    h = oracle.init_habc(w.nbc, w.dt, w.dx, w.dz, float(F.julia_mean(w.vp)), dtype=np.float64)
    a = oracle.fd_coefficients(w.fd_order, dtype=np.float64)
    wav = oracle.ricker(w.f0, w.dt, w.nt, dtype=np.float64)
    si = oracle.coord_to_index(w.src_x[0], w.dx, med.pad)
    sj = oracle.coord_to_index(w.src_z[0], w.dz, med.pad)
    ri = [oracle.coord_to_index(x, w.dx, med.pad) for x in w.rec_x]
    rj = [oracle.coord_to_index(z, w.dz, med.pad) for z in w.rec_z]
    return oracle.run_shot(med, h, a, w.dt, w.nt, si, sj, wav, ri, rj, "vz", "simd8", dtype=np.float64,
                           n_steps=n)


def reference_arm(args, rank, world):
    if rank != 0:
        return
    w = make_workload(args.nt)
    hi = host_inputs(w)
    import oracle
    oracle.build()
    per_step_s = args.cpu_seconds / 2
    vals = []
    for k in range(args.warmup + args.steps):
        v, n, cores, t = cpu_sample(w, hi, per_step_s)
        if k >= args.warmup:
            vals.append((v, n, t))
    value = float(np.mean([v for v, _, _ in vals]))
    n = vals[-1][1]
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(np.mean([t for _, _, t in vals]) * 1e3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": w.name, "cells_padded": hi["nx"] * hi["nz"], "nt": w.nt,
                   "step": f"first {n} time steps of the shot (bounded CPU sample)"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "port",
                         "sample": f"{n} time steps of {w.name} per step, OpenMP over {cores} threads "
                                   f"(C++ restatement of the reference's Float32 CPU path; Julia absent)"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- batched and served shots
def hbm_peak():
    """HBM bandwidth denominator: MEASURED_PEAKS.json hbm_gbs, else the fallback figure."""
    try:
        return float(json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def batched_section(args):
    """64 shots on one 2000 x 800 medium: sequential plain shots
    (fomo_b200_run_shot, one after another) against one fomo_b200_run_batch
    call.  Shots/hour from the host clock around each call (inputs resident,
    gathers copied to the host)."""
    import fomo_julia_b200 as F
    from fomo_julia_b200 import synthetic
    B = F.backend("b200")
    w = synthetic.batched_layered()
    nt = args.batch_nt or w.nt
    med = F.init_medium(w.vp, w.vs, w.rho, w.dx, w.dz, w.nbc, w.fd_order, B, free_surface=w.free_surface)
    H = F.init_habc(med.nx, med.nz, w.nbc, w.dt, w.dx, w.dz, F.julia_mean(w.vp), B)
    params = F.sim_params(w.dt, nt, w.dx, w.dz, w.fd_order)
    a = F.get_fd_coefficients(w.fd_order)
    wav = F.ricker_wavelet(w.f0, w.dt, nt)
    rec = F.setup_receivers(w.rec_x, w.rec_z, med, type="vz")
    cfg = F.multi_shot_config(w.src_x, w.src_z, wav)
    W = F.Wavefield(med.nx, med.nz, B)
    n_plain = 4
    src0 = F.create_source(med, cfg.shots[0], wav)
    F.run_shot(B, W, med, H, a, src0, rec, F.sim_params(w.dt, 64, w.dx, w.dz, w.fd_order))  # warm-up
    plain, plain_dev = [], []
    for k in range(n_plain):
        src = F.create_source(med, cfg.shots[k], wav)
        t0 = time.perf_counter()
        r = F.run_shot(B, W, med, H, a, src, rec, params)
        plain.append((time.perf_counter() - t0, r.gather))
        plain_dev.append(r.stats["device_ms"] / 1e3)
    W.release()
    warm = F.multi_shot_config(w.src_x[:8], w.src_z[:8], wav[:64])
    F.run_batch(B, med, H, a, rec, warm, F.sim_params(w.dt, 64, w.dx, w.dz, w.fd_order))  # warm-up
    t0 = time.perf_counter()
    res = F.run_batch(B, med, H, a, rec, cfg, params)
    t_batch = time.perf_counter() - t0
    med.release()
    same = all(np.array_equal(res[k].gather, plain[k][1]) for k in range(n_plain))
    t_plain = float(np.median([t for t, _ in plain]))  # host noise makes single calls spike
    cells = med.nx * med.nz
    n = len(cfg.shots)
    return {
        "workload": f"{w.name}" + ("" if nt == w.nt else f" (nt {nt})"), "shots": n, "nt": nt,
        "grid_padded": [med.nx, med.nz],
        "plain_s_per_shot": t_plain, "plain_device_s_per_shot": float(np.mean(plain_dev)),
        "plain_shots_per_hour": 3600.0 / t_plain, "plain_sample": f"first {n_plain} shots, one after another",
        "batched_s": t_batch, "batched_device_s": res[0].stats["device_ms"] / 1e3,
        "batched_shots_per_hour": n * 3600.0 / t_batch,
        "speedup_vs_plain": (n * 3600.0 / t_batch) / (3600.0 / t_plain),
        "batched_gcell_steps_s": n * cells * nt / t_batch / 1e9,
        "roofline": batched_roofline(n * cells * nt, res[0].stats["device_ms"] / 1e3),
        "batched_launches": res[0].stats["kernel_launches"],
        "gathers_identical_to_plain": bool(same),
    }


def step_kernel_used(roofline) -> str:
    """Which time-step form the profiled steps ran (the same the timed shots ran)."""
    names = {k["name"] for k in (roofline or {}).get("kernels", [])}
    return "fused" if "step" in names else "split"


def batched_roofline(shot_cell_steps, device_s, shots_per_pass=12):
    """Batched throughput against the one-pass byte minimum with S shots sharing a
    medium pass: 40 B per shot-cell-step of fields (read and write the five) plus
    20/S B of medium (read once per launch set of up to 12 shots)."""
    peak, src = hbm_peak()
    b = 40.0 + 20.0 / shots_per_pass
    gbs = shot_cell_steps * b / device_s / 1e9
    return {"bytes_per_shot_cell_step": b, "basis": f"one pass per step, medium read once per {shots_per_pass} shots",
            "achieved_gbs": gbs, "peak": peak, "peak_source": src, "frac": gbs / peak}


def uneven_section(args):
    """The uneven batch: 48 shots over four media (600x300, 1200x500,
    2400x1000, 3200x1400; dx 10 m) with FD orders 4, 8 and 12, nt ~
    U[1500, 6000] (dt 0.8 ms), 100..800 receivers, 8..15 Hz sources,
    submitted at once to one ShotServer.  Sequential plain time per shot is
    its (medium, order)'s measured single-shot device step time times nt."""
    import fomo_julia_b200 as F
    from fomo_julia_b200 import synthetic
    B = F.backend("b200")
    dt = 0.0008
    reqs = synthetic.uneven_requests()
    base = synthetic.uneven_media()
    med, hab = {}, {}
    for m, order in sorted({(q.medium, q.fd_order) for q in reqs}):
        (vp, vs, rho), dx = base[m]
        M = F.init_medium(vp, vs, rho, dx, dx, 50, order, B, free_surface=True)
        med[(m, order)] = M
        hab[(m, order)] = F.init_habc(M.nx, M.nz, 50, dt, dx, dx, F.julia_mean(vp), B)
    plain_step = {}
    for key, M in med.items():
        W = F.Wavefield(M.nx, M.nz, B)
        a = F.get_fd_coefficients(key[1])
        src = F.Source(M.nx // 2, M.pad + 2, F.ricker_wavelet(10.0, dt, 200))
        rec = F.setup_receivers(np.linspace(0, (M.nx - 2 * M.pad - 1) * M.dx, 400).astype(np.float32),
                                np.full(400, 10.0, np.float32), M)
        F.run_shot(B, W, M, hab[key], a, src, rec, F.sim_params(dt, 200, M.dx, M.dz, key[1]))
        r = F.run_shot(B, W, M, hab[key], a, src, rec, F.sim_params(dt, 200, M.dx, M.dz, key[1]))
        plain_step[key] = r.stats["device_ms"] / 1e3 / 200
        W.release()
    plain_total = sum(plain_step[(q.medium, q.fd_order)] * q.nt for q in reqs)
    with F.ShotServer() as srv:
        t0 = time.perf_counter()
        ts = []
        for k, q in enumerate(reqs):
            M = med[(q.medium, q.fd_order)]
            nx_in = M.nx - 2 * M.pad
            src = F.Source(F.coord_to_index(q.src_x, M.dx, M.pad), F.coord_to_index(q.src_z, M.dz, M.pad),
                           F.ricker_wavelet(q.f0, dt, q.nt))
            rec = F.setup_receivers(np.linspace(0, (nx_in - 1) * M.dx, q.n_rec).astype(np.float32),
                                    np.full(q.n_rec, 10.0, np.float32), M)
            ts.append(srv.submit(M, hab[(q.medium, q.fd_order)], F.get_fd_coefficients(q.fd_order), src, rec,
                                 F.sim_params(dt, q.nt, M.dx, M.dz, q.fd_order), k))
        srv.wait_all(ts)
        makespan = time.perf_counter() - t0
        st = srv.stats()
    for M in med.values():
        M.release()
    cell_steps = sum(med[(q.medium, q.fd_order)].nx * med[(q.medium, q.fd_order)].nz * q.nt for q in reqs)
    return {"shots": len(reqs), "media_orders": len(med), "makespan_s": makespan,
            "batched_shots_per_hour": len(reqs) * 3600.0 / makespan,
            "plain_shots_per_hour": len(reqs) * 3600.0 / plain_total,
            "speedup_vs_plain": plain_total / makespan, "batched_gcell_steps_s": cell_steps / makespan / 1e9,
            "plain": "device step time of one shot per (medium, order) x nt, shots one after another",
            "peak_shots": st["peak_shots"], "kernel_launches": st["kernel_launches"]}


def serving_section(args, c1):
    """A Poisson stream of shot requests over six resident media (600x300,
    1200x500, 2400x1000, 3200x1400, 2000x800 and the 4444x3819 medium),
    order 8, nt ~ U[1500, 6000], 100..1000 receivers, served by one
    ShotServer with a 150 GB budget.  Sequential plain time per request is
    its medium's measured single-shot step time times nt."""
    import threading
    import fomo_julia_b200 as F
    from fomo_julia_b200 import synthetic
    B = F.backend("b200")
    dt = 0.0008
    media = []
    for (vp, vs, rho), dx in synthetic.uneven_media():
        media.append((vp, vs, rho, dx))
    w2 = synthetic.batched_layered()
    media.append((w2.vp, w2.vs, w2.rho, w2.dx))
    M, Hs, recs_x = [], [], []
    for vp, vs, rho, dx in media:
        m = F.init_medium(vp, vs, rho, dx, dx, 50, 8, B, free_surface=True)
        M.append(m)
        Hs.append(F.init_habc(m.nx, m.nz, 50, dt, dx, dx, F.julia_mean(vp), B))
    M.append(c1["medium"])
    Hs.append(F.init_habc(c1["medium"].nx, c1["medium"].nz, 50, dt, 10.0, 10.0, c1["v_ref"], B))
    dxs = [m.dx for m in M]
    nx_in = [m.nx - 2 * m.pad for m in M]
    a = F.get_fd_coefficients(8)
    # plain step time per medium: one single shot of 200 steps
    plain_step = []
    for m, H in zip(M, Hs):
        W = F.Wavefield(m.nx, m.nz, B)
        wav = F.ricker_wavelet(12.0, dt, 200)
        src = F.Source(m.nx // 2, m.pad + 2, wav)
        rec = F.setup_receivers(np.linspace(0, (m.nx - 2 * m.pad - 1) * m.dx, 500).astype(np.float32),
                                np.full(500, 10.0, np.float32), m)
        F.run_shot(B, W, m, H, a, src, rec, F.sim_params(dt, 200, m.dx, m.dz, 8))
        r = F.run_shot(B, W, m, H, a, src, rec, F.sim_params(dt, 200, m.dx, m.dz, 8))
        plain_step.append(r.stats["device_ms"] / 1e3 / 200)
        W.release()
    n = args.serve_requests
    probe = synthetic.serving_requests(n, nx_in, dxs, 1.0)
    plain_total = sum(plain_step[q.medium] * q.nt for q in probe)
    rate = args.serve_load * n / plain_total  # offered load: a multiple of what sequential plain shots sustain
    reqs = synthetic.serving_requests(n, nx_in, dxs, rate)
    budget = 150 << 30
    try:
        import torch
        free, _ = torch.cuda.mem_get_info()
        budget = min(budget, int(0.85 * free))
    except Exception:
        pass
    results = [None] * n
    with F.ShotServer(hbm_budget_bytes=budget) as srv:
        tickets = [None] * n
        t_start = time.perf_counter()

        def submitter():
            for k, q in enumerate(reqs):
                d = q.arrival_s - (time.perf_counter() - t_start)
                if d > 0:
                    time.sleep(d)
                m = M[q.medium]
                wav = F.ricker_wavelet(q.f0, dt, q.nt)
                src = F.Source(F.coord_to_index(q.src_x, m.dx, m.pad), F.coord_to_index(q.src_z, m.dz, m.pad), wav)
                xs = np.linspace(0, (nx_in[q.medium] - 1) * m.dx, q.n_rec).astype(np.float32)
                rec = F.setup_receivers(xs, np.full(q.n_rec, 10.0, np.float32), m)
                tickets[k] = srv.submit(m, Hs[q.medium], a, src, rec, F.sim_params(dt, q.nt, m.dx, m.dz, 8), k)

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        for k in range(n):
            results[k] = srv.wait(tickets[k])
        makespan = time.perf_counter() - t_start
        st = srv.stats()
    for m in M[:-1]:
        m.release()
    lat = [r.stats["latency_ms"] for r in results]
    cell_steps = sum((M[q.medium].nx * M[q.medium].nz) * q.nt for q in reqs)
    from fomo_julia_b200.serving import percentile
    return {
        "requests": n, "media": [[m.nx, m.nz] for m in M], "arrival_rate_per_s": rate,
        "arrival": f"Poisson, rate = {args.serve_load:g} x the sequential plain capacity of this request mix",
        "offered_load_vs_plain_capacity": args.serve_load,
        "fraction_of_full_stream": n / 2000.0,
        "hbm_budget_bytes": budget, "makespan_s": makespan,
        "p50_latency_ms": percentile(lat, 50), "p99_latency_ms": percentile(lat, 99),
        "p50_run_ms": percentile([r.stats["run_ms"] for r in results], 50),
        "p99_run_ms": percentile([r.stats["run_ms"] for r in results], 99),
        "latency_note": "latency = submit to gather on the host; run = admission to completion (queueing excluded)",
        "served_shots_per_hour": n * 3600.0 / makespan,
        "plain_shots_per_hour": n * 3600.0 / plain_total,
        "speedup_vs_plain": plain_total / makespan,
        "served_gcell_steps_s": cell_steps / makespan / 1e9,
        "plain_us_per_step_by_medium": [round(t * 1e6, 2) for t in plain_step],
        "peak_shots": st["peak_shots"], "peak_bytes": st["peak_bytes"], "kernel_launches": st["kernel_launches"],
        "graph_replays": st["graph_replays"],
    }


# ---------------------------------------------------------------- B200 arm
def b200_arm(args, rank, world, local):
    import torch
    import torch.distributed as dist
    import fomo_julia_b200 as F
    from fomo_julia_b200 import _lib
    from fomo_julia_b200._lib import FomoKernelTime, FomoRunStats, call

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    _lib.ensure_init(local)
    F.set_step_kernel(args.step_kernel, args.segs)
    sp = ctypes.c_void_p(0)
    call("fomo_b200_get_stream", ctypes.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device("cuda", local))

    w = make_workload(args.nt)
    hi = host_inputs(w)
    nx, nz = hi["nx"], hi["nz"]
    cells = nx * nz
    # pinned host copies of the inputs (medium arrays) and the output gather
    pinned = []
    for arr in hi["arrays"]:
        t = torch.empty(arr.size, dtype=torch.float32, pin_memory=True)
        t.numpy()[:] = np.asfortranarray(arr).ravel(order="F")
        pinned.append(t)
    n_rec = hi["ri"].size
    gather = torch.zeros(w.nt * n_rec, dtype=torch.float32, pin_memory=True)

    keep = []
    H = F.elastic2d._ctypes_habc(hi["habc"], keep)
    src = F.Source(hi["si"], hi["sj"], hi["wav"])
    rec = F.Receivers(hi["ri"], hi["rj"], None, "vz")
    S = F.elastic2d._ctypes_shot(hi["a"], hi["params"], src, rec, keep)

    def medium_create():
        h = ctypes.c_uint64(0)
        call("fomo_b200_medium_create", nx, nz, w.fd_order // 2, hi["pad"], int(w.free_surface),
             float(w.dx), float(w.dz), *[t.data_ptr() for t in pinned], ctypes.byref(h))
        return h.value

    med = medium_create()
    wf = ctypes.c_uint64(0)
    call("fomo_b200_wavefield_create", nx, nz, ctypes.byref(wf))
    wf = wf.value

    def device_shot():
        """One shot with inputs resident: reset, nt steps, gather left on the device."""
        sh = ctypes.c_uint64(0)
        call("fomo_b200_shot_begin", med, wf, ctypes.byref(H), ctypes.byref(S), ctypes.byref(sh))
        k = ctypes.c_int32(0)
        call("fomo_b200_shot_advance", sh.value, w.nt, ctypes.byref(k))
        st = FomoRunStats()
        call("fomo_b200_shot_finish", sh.value, None, ctypes.byref(st))
        return st

    model = []
    for arr in (w.vp, w.vs, w.rho):
        t = torch.empty(arr.size, dtype=torch.float32, pin_memory=True)
        t.numpy()[:] = np.asfortranarray(arr).ravel(order="F")
        model.append(t)

    def e2e_shot():
        """The drop-in call sequence with host buffers: create the medium
        from the unpadded model (padding and staggered parameters on the
        device), run the shot, read the gather back, release the medium."""
        h = ctypes.c_uint64(0)
        call("fomo_b200_medium_create_from_model", w.nx_in, w.nz_in, *[t.data_ptr() for t in model], float(w.dx),
             float(w.dz), w.nbc, w.fd_order // 2, int(w.free_surface), ctypes.byref(h))
        m2 = h.value
        st = FomoRunStats()
        call("fomo_b200_run_shot", m2, wf, ctypes.byref(H), ctypes.byref(S), gather.data_ptr(), ctypes.byref(st))
        call("fomo_b200_medium_destroy", m2)
        return st

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(fn, k):
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launches = 0
        stats = []
        for _ in range(k):
            st = fn()
            launches += st.kernel_launches
            stats.append(st)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, launches, stats

    for _ in range(args.warmup):
        device_shot()
    with ClockSampler(local) as clk:
        ms, launches, st_v = timed(device_shot, args.steps)
    clocks = clk.summary()
    value = world * args.steps * cells * w.nt / (ms / 1e3) / 1e9

    e2e = None
    if not args.no_e2e:
        e2e_shot()
        with ClockSampler(local) as clk_e:
            ms_e, _, st_e = timed(e2e_shot, args.steps)
        h2d = sum(t.numel() * 4 for t in model) + st_e[0].h2d_bytes
        e2e = {"value": world * args.steps * cells * w.nt / (ms_e / 1e3) / 1e9, "unit": METRIC,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(st_e[0].d2h_bytes),
               "ms_per_step": ms_e / args.steps,
               "loop_ms_per_shot": [round(t.device_ms, 2) for t in st_e],
               "clocks": clk_e.summary(),
               "path": "fomo_b200_medium_create_from_model (unpadded vp/vs/rho from pinned host memory) + "
                       "fomo_b200_run_shot (gather to pinned host memory) + fomo_b200_medium_destroy"}

    # roofline of the dominant kernel: CUDA events around each launch
    sh = ctypes.c_uint64(0)
    call("fomo_b200_shot_begin", med, wf, ctypes.byref(H), ctypes.byref(S), ctypes.byref(sh))
    kt = (FomoKernelTime * 8)()
    nk = ctypes.c_int32(0)
    call("fomo_b200_shot_profile", sh.value, min(args.profile_steps, w.nt), kt, 5, ctypes.byref(nk))
    call("fomo_b200_shot_finish", sh.value, None, None)
    kernels = []
    for i in range(nk.value):
        k = kt[i]
        if k.launches:
            avg = k.total_ms / k.launches
            kernels.append({"name": k.name.decode(), "launches": k.launches, "avg_ms": avg,
                            "bytes_per_launch": k.bytes_per_launch, "gbs": k.bytes_per_launch / (avg / 1e3) / 1e9})
    peak, peak_src = hbm_peak()
    dom = max(kernels, key=lambda k: k["avg_ms"] * k["launches"]) if kernels else None
    # one time step of the timed shots (band passes overlap the tile launches there, so this
    # is below the sum of the separately timed launches)
    step_ms = ms / args.steps / w.nt
    roofline = None
    if dom:
        traffic = None
        tf = os.path.join(REPO, "profiles", "dram_traffic_per_launch.txt")
        if os.path.exists(tf):
            for line in open(tf):
                f = line.split()
                if len(f) >= 2 and not line.startswith("#") and f[0] == dom["name"]:
                    traffic = float(f[1])
        roofline = {"bound": "hbm", "kernel": dom["name"], "achieved": dom["gbs"], "peak": peak, "unit": "GB/s",
                    "frac": dom["gbs"] / peak, "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)",
                    "traffic": traffic,
                    "step_ms": step_ms,
                    "step_achieved": 60.0 * cells / (step_ms / 1e3) / 1e9,
                    "step_frac": (60.0 * cells / (step_ms / 1e3) / 1e9) / peak,
                    "launches_sum_ms": sum(k["avg_ms"] for k in kernels),
                    # perimeter work: the bottom-band passes, as a share of the launches timed one by one
                    "perimeter_frac": sum(k["avg_ms"] for k in kernels if k["name"].startswith("band"))
                    / sum(k["avg_ms"] for k in kernels),
                    "kernels": kernels}

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, n, cores, t, orc = cpu_sample(w, hi, args.cpu_seconds, keep=True)
        cpu = {"value": v, "unit": METRIC, "cores": cores, "kind": "port",
               "sample": f"first {n} time steps of the same shot ({t:.1f} s), C++ restatement of the "
                         f"reference's Float32 CPU path (oracle/), OpenMP"}
        # the same n steps on the GPU, against the oracle's answer (not timed)
        sh = ctypes.c_uint64(0)
        call("fomo_b200_shot_begin", med, wf, ctypes.byref(H), ctypes.byref(S), ctypes.byref(sh))
        kd = ctypes.c_int32(0)
        call("fomo_b200_shot_advance", sh.value, n, ctypes.byref(kd))
        g_gpu = np.zeros((w.nt, n_rec), dtype=np.float32, order="F")
        same_fields = True
        for q in range(5):
            f = np.zeros((nx, nz), dtype=np.float32, order="F")
            call("fomo_b200_wavefield_download", wf, q, f.ctypes.data)
            same_fields &= bool(np.array_equal(f, orc["fields"][:, :, q]))
        call("fomo_b200_shot_finish", sh.value, g_gpu.ctypes.data, None)
        g64 = float64_gather(w, n)
        parity = {"steps": n, "oracle": "Float32 CPU restatement of the reference (oracle/)",
                  "bit_exact": bool(np.array_equal(g_gpu, orc["gather"])) and same_fields,
                  "gather_bit_exact": bool(np.array_equal(g_gpu, orc["gather"])),
                  "final_fields_bit_exact": same_fields,
                  **{k: v for k, v in error_stats(g_gpu, orc["gather"]).items() if k != "traces_compared"},
                  "vs_float64": {"gpu": error_stats(g_gpu, g64), "oracle_f32": error_stats(orc["gather"], g64),
                                 "reference": "the oracle instantiated in double (Float64 init and steps)"}}
        del orc, g64

    batched = served = uneven = None
    if rank == 0 and world == 1:
        call("fomo_b200_wavefield_destroy", wf)
        wf = None
        if not args.no_batched:
            batched = batched_section(args)
        if not args.no_uneven:
            uneven = uneven_section(args)
        if not args.no_serving:
            pad = hi["pad"]
            c1_medium = F.Medium(nx, nz, float(w.dx), float(w.dz), 0.0, 0.0, w.fd_order // 2, pad,
                                 bool(w.free_surface), None, None, None, None, None, handle=med)
            served = serving_section(args, {"medium": c1_medium, "v_ref": hi["habc_v_ref"]})
    if wf is not None:
        call("fomo_b200_wavefield_destroy", wf)
    call("fomo_b200_medium_destroy", med)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / PUBLISHED_CUDA_GCELLS, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name, "cells_padded": cells, "grid_padded": [nx, nz], "nt": w.nt,
                       "shots_per_gpu_per_step": 1, "parallelism": f"shot-sharded x{world}",
                       "l2": "inputs larger than L2 (357 MB medium + 715 MB state per shot)",
                       "step_kernel": args.step_kernel,
                       "step_kernel_used": step_kernel_used(roofline),
                       "bytes_per_cell_step_algorithmic": 60},
            "physical_cells": {"cells": w.nx_in * w.nz_in,
                               "value": value * (w.nx_in * w.nz_in) / cells,
                               "note": "the same run counted on the unpadded model cells, as the reference's README counts"},
            "loop_ms_per_shot": [round(t.device_ms, 2) for t in st_v],
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks, "roofline": roofline,
            "cpu_baseline": cpu, "parity": parity,
            "batched": batched, "uneven": uneven, "serving": served,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    b200_arm(args, rank, world, local)


if __name__ == "__main__":
    main()
