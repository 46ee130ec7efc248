"""The allocation-free entry point tp_ringpass_noalloc.

It exists for callers that cannot let the library allocate device memory (a
memory pool that owns the device, an allocation-free real-time loop, code that
must not let cudaMalloc/cudaFree synchronise the device).  Its scratch lives in
a fixed device array of the library, so the test checks that two calls in a row
-- which share that array -- each give what tp_ringpass gives on the same input.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import tp

abi = tp._abi
W = __import__("trackpad_b200.workloads", fromlist=["x"])


def _noalloc(lat, coords, lost, lt, le, beti, nturns, aperture, stream):
    return abi.lib().tp_ringpass_noalloc(lat.handle, C.c_void_p(coords.data_ptr()), coords.shape[1],
                                         C.c_void_p(lost.data_ptr()), C.c_void_p(lt.data_ptr()),
                                         C.c_void_p(le.data_ptr()), C.c_double(beti), nturns, 0,
                                         C.c_double(aperture), C.c_double(aperture), C.c_void_p(stream))


@pytest.mark.gpu
def test_noalloc_matches_ringpass_on_two_calls_in_a_row():
    import torch
    lat, beam = W.dba_ring(cells=4), W.dba_beam()
    host = np.concatenate([W.gaussian(3000, seed=21), W.da_grid(24, 24)])
    n = len(host)
    cols = torch.from_numpy(np.ascontiguousarray(host.T)).cuda()  # (6, N): the N x 6 column-major matrix
    # existing entry point (device pointers)
    ref = cols.clone()
    ref_lost = torch.zeros(n, dtype=torch.int64, device="cuda")
    ref_lt = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    ref_le = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    tp.ringpass_(ref.T, lat, beam, ref_lost, 5, aperture=0.02, lost_turn=ref_lt, lost_elem=ref_le)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    for _call in range(2):
        c = cols.clone()
        lost = torch.zeros(n, dtype=torch.int64, device="cuda")
        lt = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        le = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        st = _noalloc(lat, c, lost, lt, le, tp.beti(beam), 5, 0.02, stream)
        assert st == abi.TP_OK, abi.lib().tp_last_error_string().decode()
        torch.cuda.synchronize()
        # the tolerance of the default-build parity tests: identical bits
        assert torch.equal(lost, ref_lost) and torch.equal(lt, ref_lt) and torch.equal(le, ref_le)
        assert torch.equal(c, ref)
    assert 0 < int(ref_lost.sum()) < n


@pytest.mark.gpu
def test_noalloc_switches_lattices():
    """The array keeps the last call's element table: a call on another lattice
    replaces it, and a call back on the first lattice restores it."""
    import torch
    beam = W.dba_beam()
    lats = [W.dba_ring(cells=4), W.dba_ring(cells=3)]
    host = np.concatenate([W.gaussian(1000, seed=22), W.da_grid(12, 12)])
    n = len(host)
    cols = torch.from_numpy(np.ascontiguousarray(host.T)).cuda()
    refs = []
    for lat in lats:
        r = cols.clone()
        rl = torch.zeros(n, dtype=torch.int64, device="cuda")
        tp.ringpass_(r.T, lat, beam, rl, 3, aperture=0.02)
        refs.append((r, rl))
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    for k in (0, 1, 0, 1):
        c = cols.clone()
        lost = torch.zeros(n, dtype=torch.int64, device="cuda")
        lt = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        le = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        st = _noalloc(lats[k], c, lost, lt, le, tp.beti(beam), 3, 0.02, stream)
        assert st == abi.TP_OK, abi.lib().tp_last_error_string().decode()
        torch.cuda.synchronize()
        assert torch.equal(c, refs[k][0]) and torch.equal(lost, refs[k][1])


def test_noalloc_rejects_tables_beyond_its_limit():
    # 1500 exact bends need more than the 16384-word table of the fixed array.
    lat = tp.Lattice([tp.ExactSBend(1.0, 0.01)] * 1500)
    c = np.zeros((6, 1))
    lost = np.zeros(1, np.int64)
    st = abi.lib().tp_ringpass_noalloc(lat.handle, c.ctypes.data_as(C.c_void_p), 1, lost.ctypes.data_as(C.c_void_p),
                                       None, None, C.c_double(1.0), 1, 0, C.c_double(0.0), C.c_double(0.0), None)
    assert st == abi.TP_ERANGE
    assert b"16384" in abi.lib().tp_last_error_string()
