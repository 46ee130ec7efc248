"""TPSA map tracking on the GPU (tp_tpsa_ringpass) against the CPU oracle
(oracle/tp_tpsa_oracle.hpp: the CTPS pass! methods of
ext/TrackPadPolySeriesExt.jl in the restated series algebra).

Both evaluate the same operations in the same order without FMA
contraction, so the coefficients must agree bit for bit; the tests assert
equality (np.array_equal) and report the largest difference otherwise.
"""
import numpy as np
import pytest

import oracle_ref as O
from conftest import tp
from test_tpsa_oracle import linear_kinds_lattice

pytestmark = pytest.mark.gpu
W = __import__("trackpad_b200.workloads", fromlist=["x"])

E0 = 3.5e9


def all_kinds_lattice():
    """Every kind with a CTPS pass! method, edges of all methods with fringe
    correction, both wakes, and a misalignment row."""
    acc = tp.AccelCavity(0.0, volt=2.5e6, freq=500e6, h=1200.0, phis=0.2, energy=E0)
    q = tp.Quadrupole(0.4, 1.2)
    q._misalign_init([-2e-5, 0, 1e-5, 0, 0, 0], [2e-5, 0, -1e-5, 0, 0, 0], None, None)
    return tp.Lattice(list(linear_kinds_lattice().elements) + [
        q,
        tp.SBend(0.9, 0.15, 0.03, 0.02, fint1=0.5, fint2=0.4, gap=0.05, fringe_bend_entrance=3, fringe_bend_exit=2,
                 polynom_b=[0.0, -0.3, 1.5, 0.0], max_order=2),
        tp.SBend(0.7, -0.08, 0.01, 0.0, fint1=0.3, gap=0.03, fringe_bend_entrance=2, fringe_bend_exit=3),
        tp.StrongGaussianBeam(1e-3, 0.511e6, 1, 10, 6e9, (3e-4, 4e-4), nzslice=3, zslice_npar=[0.2, 0.5, 0.3],
                              xoffsets=[1e-5, 0, -2e-5]),
        tp.LongitudinalRLCWake(freq=1.2e9, Rshunt=2e5, Q0=3.5, scale=2e-19),
        tp.LongitudinalWake(list(np.linspace(0, 3e-11, 40)), list(1e13 * np.cos(np.linspace(0, 6, 40))),
                            fliphalf=-1.0, scale=1e-19),
        tp.QuadrupoleSC(0.3, k1=0.5),
        tp.DriftSC(0.2),
        acc,
        tp.Drift(0.4),
    ])


def _refs(n, seed):
    return np.concatenate([np.zeros((1, 6)),
                           W.gaussian(n - 1, seed=seed, sigma=(1e-4, 1e-5, 1e-4, 1e-5, 1e-3, 1e-4))])


def _oracle_maps(lat, refs, order, nturns=1, sched=None, turn0=0):
    maps = np.ascontiguousarray(np.stack([O.tpsa_variables(r, order) for r in refs]))
    assert O.tpsa_ringpass(lat, maps, tp.beti(tp.Beam(E0)), order, nturns=nturns, sched=sched, turn0=turn0) == 0
    return maps


def _assert_same(dev, ref):
    if not np.array_equal(dev, ref, equal_nan=True):
        scale = np.abs(ref).max()
        err = np.abs(dev - ref).max()
        raise AssertionError(f"series differ: max |dev - ref| = {err:.3e} (max |ref| = {scale:.3e})")


# order 5 is the first whose products are dealt to threads by pair count
@pytest.mark.parametrize("order", [1, 2, 4, 5])
def test_every_kind_matches_oracle_bitwise(order):
    lat = all_kinds_lattice()
    refs = _refs(5, 3)
    dev = tp.tpsa.ringpass(lat, [tp.polyseries_variables(r, order) for r in refs], tp.Beam(E0), 1)
    _assert_same(np.stack([m.coef for m in dev]), _oracle_maps(lat, refs, order))


def test_several_turns_and_high_order():
    lat = linear_kinds_lattice()
    refs = _refs(3, 5)
    for order, nturns in ((3, 4), (6, 1)):
        arr = np.stack([tp.polyseries_variables(r, order).coef for r in refs])
        dev = tp.tpsa.ringpass(lat, arr, tp.Beam(E0), nturns, order=order)
        _assert_same(dev, _oracle_maps(lat, refs, order, nturns=nturns))


def test_order_seven_uses_the_global_pool():
    lat = tp.Lattice([tp.Drift(0.3), tp.Quadrupole(0.4, 1.2), tp.Sextupole(0.2, 25.0), tp.Drift(0.5)])
    refs = _refs(2, 7)
    dev = tp.tpsa.ringpass(lat, [tp.polyseries_variables(r, 7) for r in refs], tp.Beam(E0), 1)
    _assert_same(np.stack([m.coef for m in dev]), _oracle_maps(lat, refs, 7))


def test_many_maps_in_one_call_equal_one_by_one():
    lat = linear_kinds_lattice()
    refs = _refs(300, 9)
    all_ = tp.tpsa.one_turn_maps(lat, tp.Beam(E0), refs, order=2)
    for i in (0, 1, 150, 299):
        one = tp.polyseries_one_turn_map(lat, tp.Beam(E0), refs[i], order=2)
        assert np.array_equal(one.coef, all_[i].coef)


def test_time_dependent_strengths():
    base = linear_kinds_lattice()
    qi = next(i for i, e in enumerate(base.elements) if e.kind == "QUADRUPOLE")
    k1 = base.elements[qi].k1
    els = list(base.elements)
    els[qi] = tp.timed(els[qi], k1=lambda ctx: k1 * (1.0 + 0.01 * ctx.turn))
    lat = tp.Lattice(els)
    refs = _refs(2, 11)
    dev = tp.tpsa.ringpass(lat, [tp.polyseries_variables(r, 2) for r in refs], tp.Beam(E0), 3, turn=2)
    vals = np.array([[els[qi].updates["k1"](tp.TimeContext(0.0, t))] for t in (2, 3, 4)])
    sched = ([qi, 1], 2, vals)  # field 1: the main strength k
    _assert_same(np.stack([m.coef for m in dev]), _oracle_maps(base, refs, 2, nturns=3, sched=sched, turn0=2))


def test_first_order_part_is_the_tangent_map():
    lat = linear_kinds_lattice()
    r0 = np.array([1e-4, -2e-5, 5e-5, 1e-5, 1e-3, 2e-4])
    m = tp.polyseries_one_turn_map(lat, tp.Beam(E0), r0, order=3)
    M, _ = tp.one_turn_jacobian(lat, tp.Beam(E0), r0[None, :])
    assert np.abs(m.jacobian() - M[0]).max() <= 1e-12 * np.abs(M[0]).max()
    # evaluating the series at a small deviation reproduces particle tracking
    dx = np.array([1e-6, 2e-7, -1e-6, 1e-7, 1e-5, -2e-6])
    c = np.asfortranarray((r0 + dx)[None, :])
    tp.linepass_(c, lat, tp.Beam(E0), np.zeros(1, np.int64))
    assert np.abs(m(dx) - c[0]).max() < 1e-13


def test_kinds_without_a_series_method_are_rejected():
    lat = tp.Lattice([tp.Drift(0.2), tp.ExactSBend(1.0, 0.1)])
    with pytest.raises(tp._abi.TrackPadError) as ei:
        tp.polyseries_one_turn_map(lat, tp.Beam(E0), order=2)
    assert ei.value.status == tp._abi.TP_EUNSUPPORTED


def test_work_statistics():
    lat = all_kinds_lattice()
    refs = _refs(3, 13)
    tp.tpsa.ringpass(lat, [tp.polyseries_variables(r, 3) for r in refs], tp.Beam(E0), 1)
    st = tp.tpsa.last_stats()
    assert st["maps"] == 3 and st["order"] == 3 and st["coefficients"] == 84
    assert st["series_mul"] > 0 and st["flops"] > 0 and st["kernel_ms"] > 0
    assert 6 < st["slots_used"] <= st["slots"]


def test_core_kinds_fit_the_small_pool():
    """Tables of the integrator core use the 18-series pool: drifts, multipoles
    up to octupole, thin kicks of order 3, bends with all edge methods, RF."""
    lat = tp.Lattice([
        tp.Drift(0.3), tp.Quadrupole(0.4, 1.2), tp.Sextupole(0.2, 25.0), tp.Octupole(0.2, 300.0),
        tp.ThinMultipole(0.0, [0.0, 0.01, 0.0, 0.5], [0.0, 0.1, 4.0, 30.0], max_order=3),
        tp.SBend(0.9, 0.15, 0.03, 0.02, fint1=0.5, fint2=0.4, gap=0.05, fringe_bend_entrance=3, fringe_bend_exit=2,
                 polynom_b=[0.0, -0.3, 1.5, 10.0], max_order=3),
        tp.SBend(0.7, -0.08, 0.01, 0.0, fringe_bend_entrance=1, fringe_bend_exit=1),
        tp.RFCavity(0.2, 2e6, 500e6, 0.002, philag=0.3, energy=E0),
        tp.Drift(0.5),
    ])
    refs = _refs(3, 17)
    for order in (2, 4):
        dev = tp.tpsa.ringpass(lat, [tp.polyseries_variables(r, order) for r in refs], tp.Beam(E0), 2)
        st = tp.tpsa.last_stats()
        assert st["slots"] == 18 and st["slots_used"] <= 18
        _assert_same(np.stack([m.coef for m in dev]), _oracle_maps(lat, refs, order, nturns=2))


def test_later_calls_size_the_pool_by_the_slots_used():
    """The first call on a lattice program and order runs the full 18-series
    pool and records the slots it used; later calls size the pool to that
    (more maps resident per SM) and give the same bits."""
    lat = W.fodo_ring()
    beam = tp.Beam(E0)
    refs = _refs(40, 23)
    outs, seen = [], []
    for _ in range(2):
        dev = tp.tpsa.ringpass(lat, [tp.polyseries_variables(r, 5) for r in refs], beam, 1)
        st = tp.tpsa.last_stats()
        seen.append((st["slots"], st["slots_used"]))
        outs.append(np.stack([m.coef for m in dev]))
    assert seen[0][0] == 18 and 6 < seen[0][1] < 18
    assert seen[1][0] == max(7, seen[0][1])
    assert np.array_equal(outs[0], outs[1])
    _assert_same(outs[1][:8], _oracle_maps(lat, refs[:8], 5, nturns=1))
