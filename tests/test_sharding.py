"""Sharding of the tracking path over ranks (CPU, gloo): particle and variant
partitions, and the adjoint's one all-reduce combining per-rank loss terms,
run as two processes on 127.0.0.1."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import tp

HERE = os.path.dirname(os.path.abspath(__file__))


def test_particle_shard_covers_everything_once():
    for n in (0, 1, 31, 1000, 1048576 + 262144):
        for world in (1, 2, 3, 8):
            parts = [tp.sharding.particle_shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        tp.sharding.particle_shard(10, 2, 2)


def test_variant_shard_balances_work():
    rng = np.random.Generator(np.random.Philox(3))
    costs = rng.integers(81, 402, 256) * rng.integers(1024, 4097, 256)
    for world in (1, 2, 4, 8):
        parts = tp.sharding.variant_shard(costs, world)
        flat = sorted(v for p in parts for v in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[v] for v in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
        assert parts == tp.sharding.variant_shard(costs, world)  # deterministic on every rank


def test_local_terms_round_trip_single_rank():
    terms = tp.sharding.local_terms(2.5, [1.0, -2.0], 40, 50, 1e3)
    loss, grad = tp.sharding.combine_adjoint(terms, lambda v: v, 1e3)
    assert abs(loss - 2.5) < 1e-12 and np.allclose(grad, [1.0, -2.0], rtol=1e-15)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(mode, world=2, timeout=60, gpu=False):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        if not gpu:
            env["CUDA_VISIBLE_DEVICES"] = ""
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "dist_worker.py"), mode], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            o, e = p.communicate()
        outs.append((p.returncode, o, e))
    return outs


def test_two_rank_adjoint_combine_equals_single_process():
    outs = _run_ranks("combine")
    results = []
    for rc, o, e in outs:
        assert rc == 0, e[-2000:]
        results.append(json.loads(o.strip().splitlines()[-1]))
    for r in results:
        assert "error" not in r
        assert abs(r["loss"] - r["ref_loss"]) <= 1e-12 * abs(r["ref_loss"])
        assert r["grad_err"] < 1e-13
    assert results[0]["loss"] == results[1]["loss"]


def test_rank_that_never_joins_ends_with_an_error_not_a_hang():
    outs = _run_ranks("absent", timeout=90)
    rc, o, e = outs[0]
    # rank 0 either fails to rendezvous or its collective times out: an error, within the limit
    assert rc != 0 or '"error"' in o


def _results(outs):
    res = []
    for rc, o, e in outs:
        assert rc == 0, e[-3000:]
        res.append(json.loads(o.strip().splitlines()[-1]))
    return res


def test_two_rank_shard_and_gather_reassembles_every_particle():
    """The forward sharding with a stand-in for the tracking call: every rank
    ends with the full, correctly ordered result (coordinates, flags, turn and
    element of loss), shards of unequal size included (1001 particles)."""
    res = _results(_run_ranks("forward_fake"))
    assert all(r["ok"] for r in res)
    assert res[0]["shard"] == [0, 501] and res[1]["shard"] == [501, 1001]


@pytest.mark.gpu
def test_two_rank_forward_tracking_equals_single_process():
    """Two gloo ranks on the one GPU, each tracking its shard of the DBA ring's
    beam (no collective on the tracking path; the kernels do not wait on each
    other), gathered back: bit-identical to one process tracking it all."""
    res = _results(_run_ranks("forward_gpu", timeout=300, gpu=True))
    assert all(r["ok"] for r in res)
    assert 0 < res[0]["lost"] < res[0]["n"]


@pytest.mark.gpu
def test_two_rank_adjoint_on_tracked_shards_equals_single_process():
    """distributed_ringpass_adjoint with each rank's shard of a tracked DBA
    beam (losses included) against one process differentiating the whole beam."""
    res = _results(_run_ranks("adjoint_gpu", timeout=300, gpu=True))
    for r in res:
        assert abs(r["loss"] - r["ref_loss"]) <= 1e-12 * abs(r["ref_loss"])
        assert r["grad_err"] < 1e-12
    assert res[0]["loss"] == res[1]["loss"]
