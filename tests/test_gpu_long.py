"""Long-track parity: 1000 turns of the DBA ring on regular orbits (the
Gaussian core), 1e-9 relative against the oracle; survival identical."""
import numpy as np
import pytest

import oracle_ref
from conftest import col_rel_err, tp

pytestmark = pytest.mark.gpu
W = __import__("trackpad_b200.workloads", fromlist=["x"])


def test_dba_1000_turns_regular_orbits():
    lat, beam = W.dba_ring(), W.dba_beam()
    c0 = W.gaussian(64, seed=11)
    a = c0.copy(order="F")
    la = np.zeros(64, np.int64)
    tp.ringpass_(a, lat, beam, la, 1000, aperture=0.02)
    r = c0.copy(order="F")
    rl = np.zeros(64, np.int64)
    oracle_ref.ringpass(lat, r, rl, tp.beti(beam), 1000, aperture=0.02)
    assert la.sum() == 0, f"{int(la.sum())} core particles lost on the GPU"
    assert np.array_equal(la, rl), "survival differs from the oracle"
    err = col_rel_err(a, r)
    assert err < 1e-9, f"relative error after 1000 turns {err}"
    assert np.array_equal(a, r), "not bit-identical to the oracle after 1000 turns"
