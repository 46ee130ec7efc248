"""Checkpoint and resume of long tracks (trackpad_b200.checkpoint).

CPU: the file round-trips every array bit for bit, and a checkpoint is tied to
its lattice.  GPU: tracking turns [0, 10), saving, loading and tracking
[10, 25) gives the bits of one 25-turn track, losses included.
"""
import numpy as np
import pytest

from conftest import tp

W = __import__("trackpad_b200.workloads", fromlist=["x"])


def test_save_load_round_trip(tmp_path):
    rng = np.random.Generator(np.random.Philox(5))
    c = np.asfortranarray(rng.normal(size=(37, 6)))
    lost = (rng.uniform(size=37) < 0.3).astype(np.int64)
    lt = np.where(lost == 1, 3, -1).astype(np.int32)
    le = np.where(lost == 1, 17, -1).astype(np.int32)
    lat = W.dba_ring(cells=1)
    p = tmp_path / "state.ckpt"
    tp.checkpoint.save(p, c, lost, 12, lat=lat, lost_turn=lt, lost_elem=le)
    st = tp.checkpoint.load(p)
    assert st["turn"] == 12 and st["lattice"] == tp.checkpoint.lattice_fingerprint(lat)
    assert np.array_equal(st["coords"], c) and st["coords"].flags.f_contiguous
    assert np.array_equal(st["lost_flags"], lost)
    assert np.array_equal(st["lost_turn"], lt) and np.array_equal(st["lost_elem"], le)


def test_checkpoint_is_tied_to_its_lattice(tmp_path):
    p = tmp_path / "state.ckpt"
    tp.checkpoint.save(p, np.zeros((4, 6)), np.zeros(4, np.int64), 5, lat=W.dba_ring(cells=1))
    assert tp.checkpoint.lattice_fingerprint(W.dba_ring(cells=2)) != tp.checkpoint.load(p)["lattice"]
    with pytest.raises(ValueError):
        tp.checkpoint.resume_ringpass_(p, W.dba_ring(cells=2), W.dba_beam(), 1)
    body = p.read_bytes()
    p.write_bytes(body[:-8])
    with pytest.raises(ValueError):
        tp.checkpoint.load(p)


def _mixed_beam(lat, beam):
    """Particles lost before, at and after turn 10 of 25, and survivors: the
    oracle picks them from a wide DA grid and a wide Gaussian beam."""
    import oracle_ref
    cand = np.asfortranarray(np.concatenate([W.da_grid(30, 30, half=0.02),
                                             W.gaussian(200, seed=61, sigma=(2e-3, 1e-4, 2e-3, 1e-4, 1e-2, 2e-3))]))
    r = cand.copy(order="F")
    rl = np.zeros(len(r), np.int64)
    rlt = np.full(len(r), -1, np.int32)
    oracle_ref.ringpass(lat, r, rl, tp.beti(beam), 25, aperture=(0.02, 0.02), lost_turn=rlt)
    late = np.flatnonzero((rl == 1) & (rlt >= 10))
    early = np.flatnonzero((rl == 1) & (rlt < 10))[:100]
    alive = np.flatnonzero(rl == 0)
    return np.asfortranarray(cand[np.sort(np.concatenate([late, early, alive]))]), len(late)


@pytest.mark.gpu
def test_resumed_track_equals_one_track(tmp_path):
    lat, beam = W.dba_ring(cells=3), W.dba_beam()
    c0, nlate = _mixed_beam(lat, beam)
    assert nlate >= 10
    n = len(c0)
    ref = c0.copy(order="F")
    rl = np.zeros(n, np.int64)
    rlt = np.full(n, -1, np.int32)
    rle = np.full(n, -1, np.int32)
    tp.ringpass_(ref, lat, beam, rl, 25, aperture=0.02, lost_turn=rlt, lost_elem=rle)
    c = c0.copy(order="F")
    l = np.zeros(n, np.int64)
    lt = np.full(n, -1, np.int32)
    le = np.full(n, -1, np.int32)
    tp.ringpass_(c, lat, beam, l, 10, aperture=0.02, lost_turn=lt, lost_elem=le)
    p = tmp_path / "state.ckpt"
    tp.checkpoint.save(p, c, l, 10, lat=lat, lost_turn=lt, lost_elem=le)
    st = tp.checkpoint.resume_ringpass_(p, lat, beam, 15, aperture=0.02)
    assert st["turn"] == 25
    assert np.array_equal(st["coords"], ref) and np.array_equal(st["lost_flags"], rl)
    assert np.array_equal(st["lost_turn"], rlt) and np.array_equal(st["lost_elem"], rle)
    assert 0 < rl.sum() < n and (rlt[rl == 1] >= 10).any()
