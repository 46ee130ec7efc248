"""Adjoint gradients and tangent maps on the GPU, through the C ABI.

Checkers:
  * the oracle in forward-mode dual numbers (oracle/tp_oracle.hpp run with a
    dual scalar): the exact derivative of the same maps, one parameter at a
    time, on the same survivor set;
  * central finite differences of the GPU's own loss (h = 1e-7 relative);
  * the oracle's dual-number Jacobian for the tangent maps.

Tolerances.  The loss is the forward pass of the default build (bit-identical
maps to the oracle) summed in another order: 1e-12 relative.  The gradient
differs from the dual-number oracle only by rounding, plus the reconstruction
of states by the time-reversed maps inside a checkpoint segment: 1e-8 of the
largest gradient component.  Finite differences: 1e-5 relative (their own
truncation and rounding error).  Tangent maps: 1e-9 of the largest entry.
"""
import math

import numpy as np
import pytest

import oracle_ref
from conftest import tp

pytestmark = pytest.mark.gpu
W = __import__("trackpad_b200.workloads", fromlist=["x"])

SIGMA = 1e-4
LW = 1e3


def oracle_grad(lat, coords0, beam, nturns, params, aperture, sched=None, turn0=0, exact=True, lost0=None):
    n = coords0.shape[0]
    l0 = np.zeros(n, np.int64) if lost0 is None else lost0
    grads = []
    loss = surv = None
    for e in params:
        loss, d, surv = oracle_ref.loss_and_dk(lat, coords0, l0, tp.beti(beam), nturns, e, SIGMA, LW,
                                               aperture=(aperture, aperture), turn0=turn0, exact=exact, sched=sched)
        grads.append(d)
    if not params:
        loss, _, surv = oracle_ref.loss_and_dk(lat, coords0, l0, tp.beti(beam), nturns, -1, SIGMA, LW,
                                               aperture=(aperture, aperture), turn0=turn0, exact=exact, sched=sched)
    return loss, np.array(grads), surv


def assert_grad_close(g, ref, tol=1e-8):
    scale = np.abs(ref).max()
    assert scale > 0
    err = np.abs(g - ref).max() / scale
    assert err < tol, f"gradient error {err:.3e} of the largest component (tolerance {tol})"


def test_adjoint_dba_cells_match_dual_oracle():
    """Two DBA cells + RF, 256 Gaussian particles, 8 turns, gradient with
    respect to every quadrupole k1 and sextupole k2."""
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    params = W.magnet_indices(lat)
    c0 = W.gaussian(256, seed=21)
    loss, g, cout, lout = tp.ringpass_adjoint(c0, lat, beam, None, 8, params, checkpoint_every=1, sigma=SIGMA, lost_weight=LW,
                                              aperture=0.02, return_state=True)
    st = tp.adjoint_stats()
    rloss, rg, rsurv = oracle_grad(lat, c0, beam, 8, params, 0.02)
    assert abs(loss - rloss) <= 1e-12 * abs(rloss)
    assert_grad_close(g, rg)
    # the forward state equals ringpass! (default build: bit-identical)
    c = c0.copy(order="F")
    l = np.zeros(len(c), np.int64)
    tp.ringpass_(c, lat, beam, l, 8, aperture=0.02)
    assert np.array_equal(cout, c) and np.array_equal(lout, l)
    assert int((lout == 0).sum()) == rsurv
    assert st["reconstruction_error"] < 1e-12
    assert st["units"] == 256 * len(lat) * 8


def test_checkpoint_interval_changes_nothing_but_memory():
    """K only moves where the reverse sweep restarts from a stored state: the
    gradients of K = 1, 3, 9 and the autotuned K agree to the reconstruction
    drift of a few turns (measured 2e-11 of the largest component)."""
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    params = W.magnet_indices(lat)
    c0 = W.gaussian(128, seed=22)
    ref = None
    for K in (1, 3, 9, 0):
        loss, g = tp.ringpass_adjoint(c0, lat, beam, None, 9, params, sigma=SIGMA, aperture=0.02,
                                      checkpoint_every=K)
        st = tp.adjoint_stats()
        if K:
            assert st["checkpoint_every"] == K and st["segments"] == math.ceil(9 / K)
        assert st["checkpoint_bytes"] == (st["segments"] - 1) * 128 * 48
        if ref is None:
            ref = (loss, g)
        else:
            assert loss == ref[0]
            assert np.abs(g - ref[1]).max() <= 1e-10 * np.abs(ref[1]).max()


def test_checkpoint_interval_autotuner_trials_then_settles():
    """checkpoint_every = 0: the first gradient calls of a configuration each
    time one candidate K (1, 2, 4, 8), later calls keep the fastest whose
    reconstruction error stayed small; tuned and fixed-K gradients agree within
    1e-10 of the largest component."""
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    params = W.magnet_indices(lat)
    c0 = W.gaussian(160, seed=23)
    _, gref = tp.ringpass_adjoint(c0, lat, beam, None, 12, params, sigma=SIGMA, aperture=0.02, checkpoint_every=1)
    assert tp.adjoint_stats()["k_tuning"] == 0
    ks, states = [], []
    for _ in range(6):
        _, g = tp.ringpass_adjoint(c0, lat, beam, None, 12, params, sigma=SIGMA, aperture=0.02, checkpoint_every=0)
        st = tp.adjoint_stats()
        ks.append(st["checkpoint_every"])
        states.append(st["k_tuning"])
        assert np.abs(g - gref).max() <= 1e-10 * np.abs(gref).max()
    assert ks[:4] == [1, 2, 4, 8] and states[:4] == [1, 1, 1, 1]
    assert states[4:] == [2, 2] and ks[4] == ks[5] and ks[4] in (1, 2, 4, 8)
    assert tp.adjoint_stats()["tuned_ms"] > 0


def test_adjoint_with_losses():
    """Dynamic-aperture grid particles: some are lost, and the gradient is taken
    over the oracle's survivor set."""
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    params = W.magnet_indices(lat)[:8]
    c0 = np.asfortranarray(np.concatenate([W.gaussian(64, seed=23), W.da_grid(12, 12, half=0.019)]))
    lost0 = np.zeros(len(c0), np.int64)
    lost0[3] = 1  # lost before the call: not tracked, not counted as alive
    loss, g, cout, lout = tp.ringpass_adjoint(c0, lat, beam, lost0, 6, params, sigma=SIGMA, lost_weight=LW,
                                              aperture=0.02, return_state=True)
    rloss, rg, rsurv = oracle_grad(lat, c0, beam, 6, params, 0.02, lost0=lost0)
    assert 0 < int((lout == 1).sum()) - 1 < len(c0) - 1
    assert int((lout == 0).sum()) == rsurv
    assert abs(loss - rloss) <= 1e-12 * abs(rloss)
    assert_grad_close(g, rg)


def test_adjoint_linearised_drift_fodo():
    lat, beam = W.fodo_ring(cells=2), W.fodo_beam()
    params = W.magnet_indices(lat)
    c0 = W.gaussian(128, seed=24)
    loss, g = tp.ringpass_adjoint(c0, lat, beam, None, 5, params, sigma=SIGMA, aperture=0.05, exact=False)
    rloss, rg, _ = oracle_grad(lat, c0, beam, 5, params, 0.05, exact=False)
    assert abs(loss - rloss) <= 1e-12 * abs(rloss)
    assert_grad_close(g, rg)


def mixed_lattice():
    """Every element kind with a reverse map: SBend edges (methods 1, 2, 3),
    thin multipole, octupole, exact bend with kicks and no fringe, straight
    exact bend, RF with length."""
    E = tp
    return tp.Lattice([
        E.Drift(0.4),
        E.SBend(0.9, 0.15, 0.03, 0.02, fint1=0.5, fint2=0.4, gap=0.02, fringe_bend_entrance=1, fringe_bend_exit=2,
                polynom_b=[0.0, 0.3, 0.0, 0.0], max_order=1),
        E.Quadrupole(0.4, 1.3),
        E.SBend(0.7, -0.08, 0.01, 0.0, fint1=0.3, gap=0.03, fringe_bend_entrance=3, fringe_bend_exit=3),
        E.Sextupole(0.2, 25.0),
        E.ThinMultipole(0.0, [0.0, 0.0, 0.0, 0.0], [0.0, 0.1, 4.0, 0.0], max_order=2),
        E.Octupole(0.2, 300.0),
        E.ExactSBend(1.0, 0.1, 0.02, 0.04, polynom_b=[0.0, 0.2, 0.0, 0.0], max_order=1, gk=0.02,
                     fringe_bend_entrance=1, fringe_bend_exit=1),
        E.Quadrupole(0.4, -1.1),
        E.ExactSBend(0.5, 0.0, 0.0, 0.0),
        E.RFCavity(0.2, 2e6, 500e6, 0.002, philag=0.3, energy=3.5e9),
        E.Drift(0.5),
    ])


def test_adjoint_every_reverse_map():
    lat, beam = mixed_lattice(), tp.Beam(3.5e9)
    params = [2, 4, 6, 8]
    c0 = W.gaussian(128, seed=25)
    loss, g = tp.ringpass_adjoint(c0, lat, beam, None, 4, params, checkpoint_every=1, sigma=SIGMA, aperture=0.05)
    rloss, rg, _ = oracle_grad(lat, c0, beam, 4, params, 0.05)
    assert abs(loss - rloss) <= 1e-12 * abs(rloss)
    assert_grad_close(g, rg)
    assert tp.adjoint_stats()["reconstruction_error"] < 1e-12


def test_adjoint_time_dependent_strengths():
    """A quadrupole k1 ramp and an RF voltage modulation evaluated per turn;
    the gradient of the ramped quadrupole is with respect to a shift of its k1
    at every turn."""
    base = W.dba_ring(cells=2)
    elems = list(base.elements)
    qi = next(i for i, e in enumerate(elems) if e.kind == "QUADRUPOLE")
    ri = len(elems) - 1
    elems[qi] = tp.timed(elems[qi], k1=lambda ctx, k0=elems[qi].k1: k0 * (1 + 0.01 * ctx.turn / 10))
    elems[ri] = tp.timed(elems[ri], volt=lambda ctx, v0=elems[ri].volt: v0 * (1 + 0.05 * math.sin(2 * math.pi * ctx.turn / 200)))
    lat, beam = tp.Lattice(elems), W.dba_beam()
    params = W.magnet_indices(base)
    c0 = W.gaussian(128, seed=26)
    loss, g = tp.ringpass_adjoint(c0, lat, beam, None, 7, params, sigma=SIGMA, aperture=0.02, turn=2)
    vals = np.array([[elems[qi].updates["k1"](tp.TimeContext(0.0, t)),
                      elems[ri].updates["volt"](tp.TimeContext(0.0, t))] for t in range(2, 9)])
    rloss, rg, _ = oracle_grad(base, c0, beam, 7, params, 0.02, sched=([qi, 1, ri, 5], 2, vals), turn0=2)
    assert abs(loss - rloss) <= 1e-12 * abs(rloss)
    assert_grad_close(g, rg)


def test_adjoint_against_central_differences():
    """d loss / d k from central differences of the GPU forward loss."""
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    params = W.magnet_indices(lat)
    c0 = W.gaussian(256, seed=27)
    _, g = tp.ringpass_adjoint(c0, lat, beam, None, 6, params, sigma=SIGMA, aperture=0.02)
    elems = list(lat.elements)
    for j in (0, 3, 6, 9):
        e = params[j]
        k = elems[e].k
        h = 1e-7 * abs(k)
        vals = []
        for sgn in (1, -1):
            var = list(elems)
            var[e] = type(elems[e])(elems[e].L, k + sgn * h, name=elems[e].name)
            l, _ = tp.ringpass_adjoint(c0, tp.Lattice(var), beam, None, 6, [], sigma=SIGMA, aperture=0.02)
            assert tp.last_stats()["survivors"] == 256
            vals.append(l)
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[j]) <= 1e-5 * max(abs(g[j]), 1e-3 * np.abs(g).max()), (j, fd, g[j])


def test_batched_adjoint_equals_lattice_by_lattice():
    variants = W.dba_variants(nvar=4, seed=5, n_base=200, cells_range=(2, 4))
    batch = tp.Batch([v for v, _ in variants])
    beam = W.dba_beam()
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([W.gaussian(n, seed=30 + i) for i, n in enumerate(counts)]))
    params = [W.magnet_indices(v) for v, _ in variants]
    loss, grads = batch.ringpass_adjoint(coords, poff, np.full(len(counts), tp.beti(beam)), None, 5, params,
                                         checkpoint_every=1, sigma=SIGMA, aperture=0.02)
    for i, (lat, n) in enumerate(variants):
        l1, g1 = tp.ringpass_adjoint(np.asfortranarray(coords[poff[i]:poff[i + 1]]), lat, beam, None, 5, params[i],
                                     checkpoint_every=1, sigma=SIGMA, aperture=0.02)
        assert loss[i] == l1
        assert np.array_equal(grads[i], g1)


def test_batched_time_dependent_adjoint():
    """The time-dependent batched adjoint workload at small size: per-variant
    loss and gradient equal the single-lattice adjoint, and the dual-number
    oracle for one variant."""
    variants = W.dba_variants(nvar=3, seed=8, n_base=120, cells_range=(2, 3))
    nt = 12
    lats = [W.time_dependent(v, nt) for v, _ in variants]
    batch = tp.Batch(lats)
    beam = W.dba_beam()
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([W.gaussian(n, seed=50 + i) for i, n in enumerate(counts)]))
    params = [W.magnet_indices(v) for v, _ in variants]
    loss, grads = batch.ringpass_adjoint(coords, poff, np.full(len(counts), tp.beti(beam)), None, nt, params,
                                         sigma=SIGMA, aperture=0.02, checkpoint_every=5)
    for i, lat in enumerate(lats):
        c = np.asfortranarray(coords[poff[i]:poff[i + 1]])
        l1, g1 = tp.ringpass_adjoint(c, lat, beam, None, nt, params[i], sigma=SIGMA, aperture=0.02,
                                     checkpoint_every=5)
        assert loss[i] == l1 and np.array_equal(grads[i], g1)
    # variant 0 against the oracle with the same per-turn values
    base, _ = variants[0]
    td = lats[0]
    fields, cols = [], []
    for j, e in enumerate(td.elements):
        if isinstance(e, tp.TimeVaryingElement):
            for name in e.updates:
                fields += [j, 1 if name == "k1" else 5]
                cols.append([float(e.updates[name](tp.TimeContext(0.0, t))) for t in range(nt)])
    vals = np.array(cols).T
    c0 = np.asfortranarray(coords[:counts[0]])
    rloss, rg, _ = oracle_grad(base, c0, beam, nt, params[0], 0.02, sched=(fields, 0, vals))
    assert abs(loss[0] - rloss) <= 1e-12 * abs(rloss)
    assert_grad_close(grads[0], rg)


def test_tangent_maps_match_oracle_and_are_symplectic():
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    orbits = np.concatenate([np.zeros((1, 6)), W.gaussian(7, seed=31)])
    M, err = tp.one_turn_jacobian(lat, beam, orbits)
    R = oracle_ref.jacobian(lat, orbits, tp.beti(beam))
    assert np.abs(M - R).max() <= 1e-9 * np.abs(R).max()
    assert (err < 1e-10).all()
    for i in range(len(orbits)):
        assert abs(err[i] - oracle_ref.symplectic_error(M[i])) < 1e-12
    # several turns
    M3, _ = tp.one_turn_jacobian(lat, beam, orbits[:3], nturns=3)
    R3 = oracle_ref.jacobian(lat, orbits[:3], tp.beti(beam), nturns=3)
    assert np.abs(M3 - R3).max() <= 1e-8 * np.abs(R3).max()


def test_tangent_map_of_the_full_ring():
    lat, beam = W.dba_ring(), W.dba_beam()
    M, err = tp.one_turn_jacobian(lat, beam, np.zeros((1, 6)))
    R = oracle_ref.jacobian(lat, np.zeros((1, 6)), tp.beti(beam))
    assert np.abs(M - R).max() <= 1e-9 * np.abs(R).max()
    assert err[0] < 1e-9
    # linearly stable in both transverse planes (the ring's design condition)
    assert abs(np.trace(M[0][:2, :2])) < 2 and abs(np.trace(M[0][2:4, 2:4])) < 2


def test_lost_orbit_gives_nan_tangent_map():
    lat, beam = W.dba_ring(cells=1), W.dba_beam()
    M, err = tp.one_turn_jacobian(lat, beam, np.array([[0.0] * 6, [1.5, 0, 0, 0, 0, 0]]))
    assert np.isfinite(M[0]).all() and np.isnan(M[1]).all() and np.isnan(err[1])


def test_adjoint_rejects_what_it_cannot_differentiate():
    lat, beam = W.dba_ring(cells=1), W.dba_beam()
    c0 = W.gaussian(32, seed=1)
    drift = next(i for i, e in enumerate(lat.elements) if e.kind == "DRIFT")
    with pytest.raises(ValueError):
        tp.ringpass_adjoint(c0, lat, beam, None, 2, [drift], sigma=SIGMA)
    with pytest.raises(ValueError):
        tp.ringpass_adjoint(c0, lat, beam, None, 2, [10 ** 6], sigma=SIGMA)
