"""One rank of the sharding tests (run as a script, gloo on CPU).

Environment: RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT.  Runs five small
shots sharded over the ranks with the oracle as the per-shot computation
(the GPU is not needed to test the distribution and the gather) and, on
rank 0, saves the gathered seismograms in shot order.
"""
import argparse
import datetime
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import torch.distributed as dist  # noqa: E402

from cases import layered, oracle_inputs  # noqa: E402
from fomo_julia_b200 import sharding  # noqa: E402

N_SHOTS = 5


def shot(k):
    c = layered(40, 30, seed=1, nbc=6, fd_order=8, nt=60)
    c.src_x = 30.0 + 70.0 * k
    return c


def run_oracle(idx):
    import oracle
    oracle.build()
    out = []
    for k in idx:
        c = shot(k)
        med, h, a, wav, si, sj, ri, rj = oracle_inputs(c, oracle)
        out.append(oracle.run_shot(med, h, a, c.dt, c.nt, si, sj, wav, ri, rj, c.rec_type, "simd8"))
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--out", required=True)
    p.add_argument("--fail-rank", type=int, default=-1)
    a = p.parse_args()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=20))
    rank = dist.get_rank()

    def run(idx):
        if rank == a.fail_rank:
            raise RuntimeError(f"rank {rank}: injected failure before the gather")
        return run_oracle(idx)

    res = sharding.run_sharded(run, N_SHOTS)
    slowest = sharding.max_over_ranks(float(rank + 1))
    if rank == 0:
        np.savez(a.out, slowest=slowest, **{f"g{k}": g for k, g in enumerate(res)})
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
