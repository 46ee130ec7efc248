"""The batched launch's cached CUDA graph is replayed only with the arguments it
was captured with.

The graph of tp_ringpass_batched bakes in device pointers: the caller's
coordinate, flag and loss-record arrays, and the context's counters, error word
and staging buffers (which grow when a larger call needs them).  A later call
with other arrays, or after the context's buffers were reallocated, must give
the bits of the launch without a graph, and must not write into the arrays of
an earlier call.
"""
import numpy as np
import pytest

from conftest import tp

pytestmark = pytest.mark.gpu
W = __import__("trackpad_b200.workloads", fromlist=["x"])


def _setup():
    variants = W.dba_variants(nvar=4, seed=5, n_base=256, cells_range=(2, 4))
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([np.concatenate([W.gaussian(n // 2, seed=90 + i),
                                                               W.da_grid(1, n - n // 2, half=0.019)])
                                               for i, n in enumerate(counts)]))
    return tp.Batch([v for v, _ in variants]), poff, np.full(len(counts), tp.beti(W.dba_beam())), coords


def _run_host(batch, poff, betis, coords, use_graph):
    c = coords.copy(order="F")
    l = np.zeros(len(c), np.int64)
    lt = np.full(len(c), -1, np.int32)
    le = np.full(len(c), -1, np.int32)
    batch.ringpass_(c, poff, betis, l, 8, aperture=0.02, lost_turn=lt, lost_elem=le, use_graph=use_graph)
    return c, l, lt, le


def test_graph_replay_uses_each_calls_device_arrays():
    import torch
    batch, poff, betis, coords = _setup()
    ref = _run_host(batch, poff, betis, coords, use_graph=False)
    n = len(coords)
    init = torch.from_numpy(np.ascontiguousarray(coords.T)).cuda()
    outs = []
    for _call in range(3):  # three sets of device arrays, all kept alive
        c = init.clone()
        l = torch.zeros(n, dtype=torch.int64, device="cuda")
        lt = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        le = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        batch.ringpass_(c.T, poff, betis, l, 8, aperture=0.02, lost_turn=lt, lost_elem=le, use_graph=True)
        torch.cuda.synchronize()
        outs.append((c, l, lt, le))
    for c, l, lt, le in outs:
        assert np.array_equal(c.T.cpu().numpy(), ref[0]) and np.array_equal(l.cpu().numpy(), ref[1])
        # lanes that survive keep the caller's initial value; lost ones get the record
        lost = ref[1] == 1
        assert np.array_equal(lt.cpu().numpy()[lost], ref[2][lost])
        assert np.array_equal(le.cpu().numpy()[lost], ref[3][lost])
        assert (lt.cpu().numpy()[~lost] == -7).all() and (le.cpu().numpy()[~lost] == -7).all()


def test_graph_replay_after_the_context_buffers_grow():
    batch, poff, betis, coords = _setup()
    ref = _run_host(batch, poff, betis, coords, use_graph=False)
    first = _run_host(batch, poff, betis, coords, use_graph=True)
    # a larger host-array call on the same context reallocates its staging buffers
    lat, beam = W.dba_ring(cells=1), W.dba_beam()
    big = W.gaussian(4 * len(coords) + 4096, seed=3)
    tp.ringpass_(big, lat, beam, np.zeros(len(big), np.int64), 2, aperture=0.02)
    second = _run_host(batch, poff, betis, coords, use_graph=True)
    for out in (first, second):
        for a, b in zip(out, ref):
            assert np.array_equal(a, b)
