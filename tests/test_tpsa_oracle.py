"""Pins of the TPSA oracle (oracle/tp_tpsa_oracle.hpp), which restates the
truncated power series algebra of PolySeries (not vendored with the
reference) and the CTPS pass! methods of ext/TrackPadPolySeriesExt.jl.

  * series identities of the restated algebra;
  * univariate Taylor coefficients against closed forms;
  * the constant part of a tracked map against the particle oracle (1e-13);
  * the first-order part against the dual-number Jacobian of the particle
    maps (1e-12), on lattices where the extension's formulas are the
    particle ones (edges without fringe-field correction, no wakes);
  * the second-order part against central differences of that Jacobian.
"""
import math

import numpy as np
import pytest

import oracle_ref as O
from conftest import tp

W = __import__("trackpad_b200.workloads", fromlist=["x"])


def _rand_series(order, a0, seed, scale=0.1):
    m = O.tpsa_set_order(order)
    a = np.random.default_rng(seed).standard_normal(m) * scale
    a[0] = a0
    return a


@pytest.mark.parametrize("order", [1, 3, 6])
def test_series_identities(order):
    a = _rand_series(order, 1.3, 1)
    one = np.zeros_like(a)
    one[0] = 1.0
    s = O.tpsa_op("sqrt", a)
    assert np.allclose(O.tpsa_op("mul", s, s), a, rtol=0, atol=1e-14)
    r = O.tpsa_op("rsqrt", a)
    assert np.allclose(O.tpsa_op("mul", O.tpsa_op("mul", r, r), a), one, rtol=0, atol=1e-14)
    assert np.allclose(O.tpsa_op("mul", O.tpsa_op("inv", a), a), one, rtol=0, atol=1e-14)
    assert np.allclose(O.tpsa_op("div", a, a), one, rtol=0, atol=1e-14)
    e = O.tpsa_op("mul", O.tpsa_op("exp", a), O.tpsa_op("exp", -a))
    assert np.allclose(e, one, rtol=0, atol=1e-13)
    sn, cs = O.tpsa_op("sin", a), O.tpsa_op("cos", a)
    assert np.allclose(O.tpsa_op("mul", sn, sn) + O.tpsa_op("mul", cs, cs), one, rtol=0, atol=1e-14)


def test_univariate_taylor_coefficients():
    order = 7
    mono = O.tpsa_monomials(order)
    a = np.zeros(len(mono))
    a[0], a[1] = 0.4, 1.0  # x0 + x
    xk = [int(np.where((mono[:, 0] == k) & (mono[:, 1:].sum(1) == 0))[0][0]) for k in range(order + 1)]
    sn = O.tpsa_op("sin", a)
    ex = O.tpsa_op("exp", a)
    sq = O.tpsa_op("sqrt", a)
    for k in range(order + 1):
        d = [math.sin, math.cos, lambda t: -math.sin(t), lambda t: -math.cos(t)][k % 4](0.4)
        assert abs(sn[xk[k]] - d / math.factorial(k)) < 1e-15
        assert abs(ex[xk[k]] - math.exp(0.4) / math.factorial(k)) < 1e-15 * math.exp(0.4)
        binom = math.prod(0.5 - j for j in range(k)) / math.factorial(k)
        assert abs(sq[xk[k]] - binom * 0.4 ** (0.5 - k)) < 1e-13 * abs(binom * 0.4 ** (0.5 - k)) + 1e-16
    # truncation: the product of two degree-4 monomials vanishes at order 7
    b = np.zeros(len(mono))
    b[int(np.where((mono[:, 0] == 4) & (mono[:, 1:].sum(1) == 0))[0][0])] = 1.0
    assert not O.tpsa_op("mul", b, b).any()


def linear_kinds_lattice():
    """Kinds whose CTPS pass! is the particle pass! in series arithmetic (edges
    of method 1 without fringe-field correction, where fy is a number)."""
    acc = tp.AccelCavity(0.0, volt=2.5e6, freq=500e6, h=1200.0, phis=0.2, energy=3.5e9)
    return tp.Lattice([
        tp.Drift(0.3),
        tp.Quadrupole(0.4, 1.2),
        tp.SBend(0.9, 0.15, 0.03, 0.02, fringe_bend_entrance=1, fringe_bend_exit=1, polynom_b=[0.0, 0.3, 0.0, 0.0],
                 max_order=1),
        tp.Sextupole(0.2, 25.0),
        tp.Octupole(0.2, 300.0),
        tp.ThinMultipole(0.0, [0.0, 0.0, 0.0, 0.0], [0.0, 0.1, 4.0, 0.0], max_order=2),
        tp.Solenoid(0.5, 0.8),
        tp.Corrector(0.4, 1.5e-4, -2.2e-4),
        tp.Quadrupole(0.4, -1.1),
        tp.Translation(0.0, dx=1e-4, dy=-2e-4, ds=3e-3),
        tp.YRotation(0.0, angle=0.002),
        tp.CrabCavity(0.3, volt=2e6, freq=500e6, phi=0.1, energy=3.5e9),
        acc,
        tp.LongitudinalRFMap(2e-4, acc),
        tp.LorentzBoost(0.003),
        tp.InvLorentzBoost(0.003),
        tp.StrongThinGaussianBeam(1e-6, 1e-3, 1.2e-3, xoffset=1e-4, yoffset=-2e-4),
        tp.RFCavity(0.2, 2e6, 500e6, 0.002, philag=0.3, energy=3.5e9),
        tp.Drift(0.5),
    ])


def _track_map(lat, x0, beti, order, nturns=1):
    maps = O.tpsa_variables(x0, order)[None].copy()
    assert O.tpsa_ringpass(lat, maps, beti, order, nturns=nturns) == 0
    return maps[0]


def test_constant_and_first_order_parts_match_the_particle_oracle():
    lat, beam = linear_kinds_lattice(), tp.Beam(3.5e9)
    beti = tp.beti(beam)
    x0 = np.array([1e-4, -2e-5, 5e-5, 1e-5, 1e-3, 2e-4])
    m = _track_map(lat, x0, beti, 3)
    c = np.asfortranarray(x0[None, :].copy())
    O.ringpass(lat, c, np.zeros(1, np.int64), beti, 1)
    assert np.allclose(m[:, 0], c[0], rtol=1e-13, atol=1e-18)
    J = O.jacobian(lat, x0[None, :], beti)[0]
    assert np.abs(m[:, 1:7] - J).max() <= 1e-12 * np.abs(J).max()


def test_second_order_part_against_differences_of_the_jacobian():
    lat, beam = linear_kinds_lattice(), tp.Beam(3.5e9)
    beti = tp.beti(beam)
    x0 = np.array([1e-4, -2e-5, 5e-5, 1e-5, 1e-3, 2e-4])
    order = 2
    mono = O.tpsa_monomials(order)
    m = _track_map(lat, x0, beti, order)
    h = np.array([1e-6, 1e-7, 1e-6, 1e-7, 1e-5, 1e-6])
    H = np.zeros((6, 6, 6))  # H[c, i, j] = d^2 f_c / dx_i dx_j
    for j in range(6):
        xp, xm = x0.copy(), x0.copy()
        xp[j] += h[j]
        xm[j] -= h[j]
        Jp = O.jacobian(lat, xp[None, :], beti)[0]
        Jm = O.jacobian(lat, xm[None, :], beti)[0]
        H[:, :, j] = (Jp - Jm) / (2 * h[j])
    for k in range(7, len(mono)):
        e = mono[k]
        idx = np.nonzero(e)[0]
        if len(idx) == 1:
            i = j = idx[0]
            want = H[:, i, i] / 2.0
        else:
            i, j = idx
            want = H[:, i, j]
        scale = np.abs(H).max()
        assert np.abs(m[:, k] - want).max() <= 1e-5 * scale, (k, e)


def test_edges_and_wakes_follow_the_extension():
    """Edge fy from the constant parts of delta, px; wakes at the constant part of z."""
    beam = tp.Beam(3.5e9)
    beti = tp.beti(beam)
    x0 = np.array([1e-4, 2e-5, 5e-5, 0.0, 1e-3, 2e-4])
    edge = tp.Lattice([tp.SBend(0.9, 0.15, 0.03, 0.02, fint1=0.5, fint2=0.4, gap=0.05, fringe_bend_entrance=3,
                                fringe_bend_exit=2)])
    m = _track_map(edge, x0, beti, 2)
    J = O.jacobian(edge, x0[None, :], beti)[0]
    # the particle Jacobian has d py / d delta from fy(delta); the series map does not
    assert abs(m[3, 6] - J[3, 5]) > 1e-9
    wake = tp.Lattice([tp.LongitudinalRLCWake(freq=1.2e9, Rshunt=2e5, Q0=3.5, scale=2e-19)])
    m = _track_map(wake, np.array([0, 0, 0, 0, -1e-3, 0.0]), beti, 2)
    assert m[5, 5] == 0.0 and m[5, 0] != 0.0  # no z dependence, a constant kick


def test_unsupported_kinds_are_reported():
    maps = O.tpsa_variables(np.zeros(6), 1)[None].copy()
    lat = tp.Lattice([tp.ExactSBend(1.0, 0.1)])
    assert O.tpsa_ringpass(lat, maps, 1.0, 1) == -2


def test_library_monomial_order_matches_the_oracle():
    """The device library orders coefficients as the oracle does (host-only calls)."""
    for order in (0, 1, 3, 6):
        assert tp.tpsa.coefficients(order) == math.comb(order + 6, 6)
        assert np.array_equal(tp.tpsa.monomials(order), O.tpsa_monomials(order))
    with pytest.raises(tp._abi.TrackPadError):
        tp.tpsa.coefficients(11)
