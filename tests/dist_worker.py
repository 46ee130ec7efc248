"""One rank of the two-process gloo tests of trackpad_b200.sharding (run by
tests/test_sharding.py with RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT set)."""
import json
import os
import sys
from datetime import timedelta

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def synthetic(n=1000, nparam=7, seed=5):
    """Per-particle loss terms q, gradients dq/dk, alive-at-start and survivor masks."""
    rng = np.random.Generator(np.random.Philox(seed))
    q = rng.uniform(0.0, 3.0, n)
    dq = rng.normal(size=(n, nparam))
    alive0 = rng.uniform(size=n) > 0.05
    surv = alive0 & (rng.uniform(size=n) > 0.2)
    return q, dq, alive0, surv


def rank_result(q, dq, alive0, surv, w):
    s = int(surv.sum())
    a = int(alive0.sum())
    loss = (q[surv].mean() if s else 0.0) + w * ((a - s) / a if a else 0.0)
    grad = dq[surv].mean(axis=0) if s else np.zeros(dq.shape[1])
    return loss, grad, s, a


def main():
    import __graft_entry__
    __graft_entry__.load_package()
    import torch.distributed as dist
    from trackpad_b200 import sharding
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    mode = sys.argv[1]
    if mode == "absent" and rank == 1:
        return  # this rank never joins
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=8))
    try:
        q, dq, alive0, surv = synthetic()
        w = 1e3
        lo, hi = sharding.particle_shard(len(q), rank, world)
        loss, grad, s, a = rank_result(q[lo:hi], dq[lo:hi], alive0[lo:hi], surv[lo:hi], w)
        terms = sharding.local_terms(loss, grad, s, a, w)
        gl, gg = sharding.combine_adjoint(terms, sharding.torch_all_reduce(), w)
        rl, rg, _, _ = rank_result(q, dq, alive0, surv, w)
        print(json.dumps({"rank": rank, "loss": gl, "ref_loss": rl, "grad_err": float(np.abs(gg - rg).max())}))
    except Exception as e:  # a peer that never joined: the collective ends with an error
        print(json.dumps({"rank": rank, "error": type(e).__name__}))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


if __name__ == "__main__":
    main()
