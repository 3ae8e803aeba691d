"""Shot server: run_shot! requests served with continuous batching.

The reference runs shots one after another (``run_shots!``,
src/simulation/shot_manager.jl:145-180).  ``ShotServer`` wraps the library's
server (``fomo_b200_server_*`` in include/fomo_b200.h): requests are queued
from any thread, admitted in arrival order while their device memory fits the
HBM budget, and every admitted shot runs in the same time-step launches as
the others, joining and leaving the batch at step boundaries.  Each result is
the gather ``run_shot`` returns for that shot, bit for bit.

    with ShotServer(hbm_budget_bytes=150 << 30) as srv:
        t = srv.submit(M, H, a, src, rec, params, shot_id=7)
        result = srv.wait(t)           # ShotResult; stats hold the latency
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _lib
from ._lib import FomoRequestStats, FomoServerConfig, FomoServerStats, call
from .elastic2d import (HABCConfig, Medium, Receivers, ShotResult, SimParams, Source, _ctypes_habc,
                        _ctypes_shot)

f32 = np.float32


@dataclass
class Ticket:
    """A submitted request; holds the host buffers the server reads and writes."""
    id: int
    shot_id: int
    gather: np.ndarray
    src: Source
    rec: Receivers
    keep: list = field(default_factory=list, repr=False)


def percentile(values, q: float) -> float:
    """Nearest-rank percentile (q in [0, 100]) of a non-empty sequence."""
    v = sorted(float(x) for x in values)
    if not v:
        raise ValueError("percentile of an empty sequence")
    k = max(1, int(np.ceil(q / 100.0 * len(v))))
    return v[min(k, len(v)) - 1]


class ShotServer:
    """Continuous-batching shot server on one GPU (the library's device)."""

    def __init__(self, hbm_budget_bytes: int = 0, max_shots: int = 0, steps_per_launch: int = 0,
                 device: int = 0):
        _lib.ensure_init(device)
        cfg = FomoServerConfig()
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        cfg.max_shots = int(max_shots)
        cfg.steps_per_launch = int(steps_per_launch)
        h = ctypes.c_uint64(0)
        call("fomo_b200_server_create", ctypes.byref(cfg), ctypes.byref(h))
        self.handle = h.value

    def submit(self, M: Medium, H: HABCConfig, a, src: Source, rec: Receivers, params: SimParams,
               shot_id: int = 1) -> Ticket:
        """Queues one shot; returns at once."""
        keep: list = []
        hs = _ctypes_habc(H, keep)
        ss = _ctypes_shot(a, params, src, rec, keep)
        gather = np.zeros((params.nt, ss.n_rec), dtype=f32, order="F")
        t = ctypes.c_uint64(0)
        call("fomo_b200_server_submit", self.handle, M.upload(), ctypes.byref(hs), ctypes.byref(ss),
             gather.ctypes.data if gather.size else None, ctypes.byref(t))
        return Ticket(t.value, int(shot_id), gather, src, rec, keep)

    def poll(self, ticket: Ticket) -> bool:
        done = ctypes.c_int32(0)
        call("fomo_b200_server_poll", self.handle, ticket.id, ctypes.byref(done))
        return bool(done.value)

    def wait(self, ticket: Ticket, timeout: Optional[float] = None) -> ShotResult:
        """Blocks until the request is done (raises FomoError on failure,
        cancellation, or FOMO_ENOTREADY after `timeout` seconds)."""
        st = FomoRequestStats()
        call("fomo_b200_server_wait", self.handle, ticket.id, -1.0 if timeout is None else float(timeout),
             ctypes.byref(st))
        stats = {"queue_ms": st.queue_ms, "run_ms": st.run_ms, "latency_ms": st.latency_ms,
                 "steps": st.steps, "batch_peak": st.batch_peak}
        return ShotResult(ticket.gather, ticket.shot_id, int(ticket.src.i), int(ticket.src.j),
                          np.asarray(ticket.rec.i, dtype=np.int64).copy(),
                          np.asarray(ticket.rec.j, dtype=np.int64).copy(), stats)

    def wait_all(self, tickets: List[Ticket], timeout: Optional[float] = None) -> List[ShotResult]:
        return [self.wait(t, timeout) for t in tickets]

    def cancel(self, ticket: Ticket) -> None:
        call("fomo_b200_server_cancel", self.handle, ticket.id)

    def stats(self) -> dict:
        s = FomoServerStats()
        call("fomo_b200_server_stats", self.handle, ctypes.byref(s))
        return {name: getattr(s, name) for name, _ in FomoServerStats._fields_}

    def close(self) -> None:
        if self.handle:
            call("fomo_b200_server_destroy", self.handle)
            self.handle = 0

    def __enter__(self) -> "ShotServer":
        return self

    def __exit__(self, *exc) -> None:
        self.close()
