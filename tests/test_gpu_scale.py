"""Parity at the benchmarked configurations, against the oracle.

* DBA ring tracking: 8,192 particles drawn from the tracking benchmark's own
  input (4,096 from its 1,048,576-particle Gaussian beam, 4,096 from its
  512 x 512 dynamic-aperture grid), 1000 turns.  Gates: coordinates of the
  survivors within 1e-9 relative (per coordinate, scaled by the column's
  largest magnitude); loss flags, turn and element of loss identical except for
  particles that came within 1e-10 of an aperture or limit edge.  The default
  build is in fact bit-identical, which the test also checks.
* Batched tracking: 16 DBA variants in one launch, among them a 401-element
  and an 81-element ring, with losses, static tiles and pooled refill (and the
  CUDA graph), each variant compared with the oracle directly.
* Gradient: central differences (h = 1e-7 relative) of the loss at the full
  gradient configuration (65,536 particles, 256 turns) for two quadrupole and
  two sextupole strengths, against the adjoint: 1e-5 relative, plus the
  rounding error of the difference quotient.  The loss of 65,536 particles
  tracked 256 turns carries a rounding error of ~2e-11 relative (measured), so
  the quotient's rounding error is up to ~1e-10 |loss| / (2h); that term
  dominates for the sextupoles, whose gradients are ~1e-5 of the quadrupoles',
  so they are also checked at h = 1e-5 relative.
* Misalignment: the DBA ring with an offset and a roll on most magnets and
  drifts, exact bends included, and one general entrance matrix, bit-identical
  to the oracle.
"""
import numpy as np
import pytest

import oracle_ref
from conftest import col_rel_err, tp

pytestmark = pytest.mark.gpu
W = __import__("trackpad_b200.workloads", fromlist=["x"])

SIGMA = 1e-4
LW = 1e3


def _oracle(lat, beam, c0, nturns, aperture, turn0=0):
    n = c0.shape[0]
    r = c0.copy(order="F")
    rl = np.zeros(n, np.int64)
    rlt = np.full(n, -1, np.int32)
    rle = np.full(n, -1, np.int32)
    edge = np.full(n, np.inf)
    oracle_ref.ringpass(lat, r, rl, tp.beti(beam), nturns, turn0=turn0, aperture=(aperture, aperture),
                        lost_turn=rlt, lost_elem=rle, min_edge=edge)
    return r, rl, rlt, rle, edge


def _gates(c, lost, lt, le, ref, rtol=1e-9):
    r, rl, rlt, rle, edge = ref
    mism = (lost != rl) | (lt != rlt) | (le != rle)
    assert not (mism & (edge > 1e-10)).any(), f"{int(mism.sum())} loss records differ away from the edges"
    surv = (lost == 0) & (rl == 0)
    if surv.any():
        err = col_rel_err(c[surv], r[surv])
        assert err < rtol, f"survivors differ by {err:.3e} relative"
    return int(mism.sum())


def test_dba_1000_turns_on_the_benchmark_beam():
    lat, beam = W.dba_ring(), W.dba_beam()
    full = W.dba_particles(1 << 20, 512, seed=0)
    rng = np.random.Generator(np.random.Philox(2024))
    idx = np.concatenate([rng.choice(1 << 20, 4096, replace=False),
                          (1 << 20) + rng.choice(512 * 512, 4096, replace=False)])
    c0 = np.asfortranarray(full[np.sort(idx)])
    n = c0.shape[0]
    c = c0.copy(order="F")
    lost = np.zeros(n, np.int64)
    lt = np.full(n, -1, np.int32)
    le = np.full(n, -1, np.int32)
    tp.ringpass_(c, lat, beam, lost, 1000, aperture=0.02, lost_turn=lt, lost_elem=le)
    ref = _oracle(lat, beam, c0, 1000, 0.02)
    assert _gates(c, lost, lt, le, ref) == 0
    survivors = int((lost == 0).sum())
    assert 4096 <= survivors < n  # the Gaussian core survives, most of the grid does not
    # stronger than the gates: the default build evaluates the same operations
    assert np.array_equal(c, ref[0]) and np.array_equal(lost, ref[1])
    assert np.array_equal(lt, ref[2]) and np.array_equal(le, ref[3])


def _batched_inputs():
    variants = W.dba_variants(nvar=14, seed=31, n_base=384, cells_range=(5, 19))
    variants += W.dba_variants(nvar=1, seed=32, n_base=384, cells_range=(20, 20))
    variants += W.dba_variants(nvar=1, seed=33, n_base=384, cells_range=(4, 4))
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([np.concatenate([W.gaussian(n - n // 3, seed=300 + i),
                                                               W.da_grid(1, n // 3, half=0.019)])
                                               for i, n in enumerate(counts)]))
    return variants, counts, poff, coords


@pytest.mark.parametrize("schedule,use_graph", [(1, False), (2, True)])
def test_batched_variants_against_the_oracle(schedule, use_graph):
    variants, counts, poff, coords = _batched_inputs()
    assert {len(v) for v, _ in variants} >= {401, 81} and len(variants) >= 16
    beam = W.dba_beam()
    batch = tp.Batch([v for v, _ in variants])
    c = coords.copy(order="F")
    n = len(c)
    lost = np.zeros(n, np.int64)
    lt = np.full(n, -1, np.int32)
    le = np.full(n, -1, np.int32)
    nturns = 40
    batch.ringpass_(c, poff, np.full(len(counts), tp.beti(beam)), lost, nturns, aperture=0.02, lost_turn=lt,
                    lost_elem=le, schedule=schedule, use_graph=use_graph)
    assert tp.last_stats()["schedule"] == schedule
    assert 0 < lost.sum() < n
    for v, (lat, nv) in enumerate(variants):
        s = slice(int(poff[v]), int(poff[v + 1]))
        ref = _oracle(lat, beam, np.asfortranarray(coords[s]), nturns, 0.02)
        assert _gates(c[s], lost[s], lt[s], le[s], ref) == 0
        assert np.array_equal(c[s], ref[0]) and np.array_equal(lost[s], ref[1])
        assert np.array_equal(lt[s], ref[2]) and np.array_equal(le[s], ref[3])


def test_gradient_central_differences_at_full_size():
    """65,536 Gaussian particles, 256 turns, 120 k1 + 80 k2: the adjoint
    gradient against central differences of the loss for four strengths."""
    lat, beam = W.dba_ring(), W.dba_beam()
    params = W.magnet_indices(lat)
    assert len(params) == 200
    c0 = W.gaussian(65536, seed=0)
    loss, g = tp.ringpass_adjoint(c0, lat, beam, None, 256, params, sigma=SIGMA, lost_weight=LW, aperture=0.02)
    surv0 = tp.last_stats()["survivors"]
    elems = list(lat.elements)
    kinds = [elems[e].kind for e in params]
    picks = [0, 2, 104, 199]  # Q1 of cell 0, S1 of cell 0, S2 of cell 10, Q1 of cell 19
    assert [kinds[j] for j in picks] == ["QUADRUPOLE", "SEXTUPOLE", "SEXTUPOLE", "QUADRUPOLE"]
    for j in picks:
        e = params[j]
        k = elems[e].k
        for hrel in ((1e-7, 1e-5) if kinds[j] == "SEXTUPOLE" else (1e-7,)):
            h = hrel * abs(k)
            vals = []
            for sgn in (1, -1):
                var = list(elems)
                var[e] = type(elems[e])(elems[e].L, k + sgn * h, name=elems[e].name)
                l, _ = tp.ringpass_adjoint(c0, tp.Lattice(var), beam, None, 256, [], sigma=SIGMA, lost_weight=LW,
                                           aperture=0.02)
                assert tp.last_stats()["survivors"] == surv0  # the same survivor set on both sides
                vals.append(l)
            fd = (vals[0] - vals[1]) / (2 * h)
            rounding = 1e-10 * abs(loss) / (2 * h)
            assert abs(fd - g[j]) <= 1e-5 * abs(g[j]) + rounding, (j, hrel, fd, g[j], rounding)


def _roll(th):
    c, s = np.cos(th), np.sin(th)
    R = np.eye(6)
    R[0, 0] = R[1, 1] = R[2, 2] = R[3, 3] = c
    R[0, 2] = R[1, 3] = s
    R[2, 0] = R[3, 1] = -s
    return R


def test_misaligned_dba_ring_forward_against_the_oracle():
    lat = W.dba_ring()
    rng = np.random.Generator(np.random.Philox(77))
    els = list(lat.elements)
    first = True
    for e in els:
        if e.kind in ("QUADRUPOLE", "SEXTUPOLE", "EXACT_SBEND", "DRIFT") and rng.uniform() < 0.8:
            dx, dy = rng.normal(0, 3e-5, 2)
            th = rng.normal(0, 2e-4)
            r1 = _roll(th)
            if first:
                r1 = r1 @ (np.eye(6) + 1e-3 * rng.standard_normal((6, 6)))
                first = False
            e._misalign_init([-dx, 0, -dy, 0, 0, 0], [dx, 0, dy, 0, 0, 0], r1, np.linalg.inv(_roll(th)))
    mlat = tp.Lattice(els)
    assert mlat.pack()[3] > 250
    beam = W.dba_beam()
    c0 = np.asfortranarray(np.concatenate([W.gaussian(3072, seed=78), W.da_grid(32, 32, half=0.018)]))
    n = len(c0)
    c = c0.copy(order="F")
    lost = np.zeros(n, np.int64)
    lt = np.full(n, -1, np.int32)
    le = np.full(n, -1, np.int32)
    tp.ringpass_(c, mlat, beam, lost, 20, aperture=0.02, lost_turn=lt, lost_elem=le)
    ref = _oracle(mlat, beam, c0, 20, 0.02)
    assert np.array_equal(c, ref[0]) and np.array_equal(lost, ref[1])
    assert np.array_equal(lt, ref[2]) and np.array_equal(le, ref[3])
    assert 0 < lost.sum() < n
    # the misalignment changes the orbit: not the aligned ring's result
    a = c0.copy(order="F")
    tp.ringpass_(a, W.dba_ring(), beam, np.zeros(n, np.int64), 20, aperture=0.02)
    assert not np.array_equal(a, c)
