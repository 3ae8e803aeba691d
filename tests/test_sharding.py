"""Shot sharding over ranks (fomo_julia_b200.sharding), on CPU with gloo.

Shots are independent, so the multi-GPU path is a round-robin shard of the
shots per rank and one gather of the seismograms to rank 0.  These tests run
two real ranks (processes, gloo backend on 127.0.0.1) with the oracle as the
per-shot computation and check the gather against a single-process run, and
that a rank that fails before the gather makes the other rank fail within
the process-group timeout instead of hanging.
"""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from fomo_julia_b200 import sharding

HERE = os.path.dirname(os.path.abspath(__file__))
WORKER = os.path.join(HERE, "shard_worker.py")


def test_shard_round_robin():
    for n in (0, 1, 5, 64):
        for world in (1, 2, 3, 8):
            parts = [sharding.shard(n, world, r) for r in range(world)]
            flat = sorted(k for p in parts for k in p)
            assert flat == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        sharding.shard(4, 2, 2)


def test_single_process_needs_no_group():
    assert sharding.run_sharded(lambda idx: [k * k for k in idx], 4) == [0, 1, 4, 9]
    assert sharding.max_over_ranks(3.5) == 3.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(world, out, fail_rank=-1):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, WORKER, "--out", out, "--fail-rank", str(fail_rank)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    rcs, logs = [], []
    for p in procs:
        try:
            o, _ = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            p.kill()
            o, _ = p.communicate()
            o += "\n<killed after 240 s>"
        rcs.append(p.returncode)
        logs.append(o)
    return rcs, logs


def test_gloo_world2_gathers_in_shot_order(tmp_path, oracle_lib):
    sys.path.insert(0, HERE)
    import shard_worker
    out = str(tmp_path / "g.npz")
    rcs, logs = _launch(2, out)
    assert rcs == [0, 0], logs
    d = np.load(out)
    ref = shard_worker.run_oracle(range(shard_worker.N_SHOTS))
    for k in range(shard_worker.N_SHOTS):
        assert np.array_equal(d[f"g{k}"], ref[k]), f"shot {k}"
    assert float(d["slowest"]) == 2.0


def test_gloo_failed_rank_does_not_hang_the_others(tmp_path, oracle_lib):
    rcs, logs = _launch(2, str(tmp_path / "g.npz"), fail_rank=1)
    assert rcs[1] != 0 and "injected failure" in logs[1]
    assert rcs[0] != 0, "rank 0 should fail when its peer dies before the gather"
    assert "<killed" not in logs[0]
