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


def fake_track(c, lf, lt, le, start):
    """A stand-in for tracking on CPU: a deterministic change of every particle
    that depends on its global index, plus a loss pattern."""
    idx = start + np.arange(c.shape[0])
    c[:, 0] += 1e-3 * idx
    c[:, 5] *= -1.0
    lost = idx % 7 == 3
    lf[lost] = 1
    if lt is not None:
        lt[lost] = (idx[lost] % 5).astype(np.int32)
    if le is not None:
        le[lost] = (idx[lost] % 11).astype(np.int32)


def forward_fake(rank, world):
    from trackpad_b200 import sharding
    n = 1001
    rng = np.random.Generator(np.random.Philox(9))
    c0 = np.asfortranarray(rng.normal(size=(n, 6)))
    c = c0.copy(order="F")
    lf = np.zeros(n, np.int64)
    lt = np.full(n, -1, np.int32)
    le = np.full(n, -1, np.int32)
    start = sharding.particle_shard(n, rank, world)[0]
    lo, hi = sharding.shard_and_gather(c, lf, rank, world, lambda a, b, x, y: fake_track(a, b, x, y, start),
                                       sharding.torch_all_gather(), lost_turn=lt, lost_elem=le)
    r = c0.copy(order="F")
    rl = np.zeros(n, np.int64)
    rlt = np.full(n, -1, np.int32)
    rle = np.full(n, -1, np.int32)
    fake_track(r, rl, rlt, rle, 0)
    ok = (np.array_equal(c, r) and np.array_equal(lf, rl) and np.array_equal(lt, rlt) and np.array_equal(le, rle))
    return {"rank": rank, "ok": bool(ok), "shard": [lo, hi]}


def forward_gpu(rank, world):
    """The DBA ring split over the ranks (both on this process's current GPU)
    against one process tracking the whole beam."""
    import trackpad_b200 as tp
    import trackpad_b200.workloads as W
    lat, beam = W.dba_ring(cells=4), W.dba_beam()
    c0 = np.asfortranarray(np.concatenate([W.gaussian(3000, seed=4), W.da_grid(20, 20)]))
    n = len(c0)
    c = c0.copy(order="F")
    lf = np.zeros(n, np.int64)
    lt = np.full(n, -1, np.int32)
    le = np.full(n, -1, np.int32)
    tp.sharding.distributed_ringpass_(c, lat, beam, lf, 12, aperture=0.02, lost_turn=lt, lost_elem=le)
    r = c0.copy(order="F")
    rl = np.zeros(n, np.int64)
    rlt = np.full(n, -1, np.int32)
    rle = np.full(n, -1, np.int32)
    tp.ringpass_(r, lat, beam, rl, 12, aperture=0.02, lost_turn=rlt, lost_elem=rle)
    ok = (np.array_equal(c, r) and np.array_equal(lf, rl) and np.array_equal(lt, rlt) and np.array_equal(le, rle))
    return {"rank": rank, "ok": bool(ok), "lost": int(lf.sum()), "n": n}


def adjoint_gpu(rank, world):
    """distributed_ringpass_adjoint on real DBA shards against one process
    differentiating the whole beam."""
    import trackpad_b200 as tp
    import trackpad_b200.workloads as W
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    params = W.magnet_indices(lat)
    c0 = np.asfortranarray(np.concatenate([W.gaussian(2000, seed=6), W.da_grid(8, 8, half=0.019)]))
    lo, hi = tp.sharding.particle_shard(len(c0), rank, world)
    loss, grad = tp.sharding.distributed_ringpass_adjoint(np.asfortranarray(c0[lo:hi]), lat, beam, None, 8, params,
                                                          checkpoint_every=1, sigma=1e-4, lost_weight=1e3, aperture=0.02)
    rloss, rgrad = tp.ringpass_adjoint(c0, lat, beam, None, 8, params, checkpoint_every=1, sigma=1e-4, lost_weight=1e3, aperture=0.02)[:2]
    return {"rank": rank, "loss": loss, "ref_loss": rloss,
            "grad_err": float(np.abs(grad - rgrad).max() / np.abs(rgrad).max())}


def main():
    import __graft_entry__
    __graft_entry__.load_package()
    import torch.distributed as dist
    from trackpad_b200 import sharding
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    mode = sys.argv[1]
    if mode == "absent" and rank == 1:
        return  # this rank never joins
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=8 if mode == "absent" else 120))
    if mode in ("forward_fake", "forward_gpu", "adjoint_gpu"):
        try:
            fn = {"forward_fake": forward_fake, "forward_gpu": forward_gpu, "adjoint_gpu": adjoint_gpu}[mode]
            print(json.dumps(fn(rank, world)))
        finally:
            dist.destroy_process_group()
        return
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
