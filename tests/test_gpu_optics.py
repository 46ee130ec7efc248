"""Optics from device tangent maps against the oracle's dual-number maps.

Tolerances: maps 1e-9 of the largest entry; tunes 1e-11 (a function of the
map entries); chromaticity by the reference's finite difference in the
momentum offset (dpp = 1e-8), so its rounding error is ~1e-13 / 1e-8: 1e-4
relative; closed orbits: fixed point of the oracle's own one-turn map to 1e-10.
"""
import numpy as np
import pytest

import oracle_ref
from conftest import tp

pytestmark = pytest.mark.gpu
W = __import__("trackpad_b200.workloads", fromlist=["x"])


def _oracle_tunes(lat, beam, ref):
    M = oracle_ref.jacobian(lat, np.asarray(ref)[None, :], tp.beti(beam))[0]
    return tp.optics.tune_from_map(M), M


def test_one_turn_map_and_tunes():
    lat, beam = W.dba_ring(), W.dba_beam()
    M = tp.optics.one_turn_map(lat, beam)
    (qx, qy), R = _oracle_tunes(lat, beam, np.zeros(6))
    assert np.abs(M - R).max() <= 1e-9 * np.abs(R).max()
    gx, gy = tp.optics.gettune(lat, beam)
    assert abs(gx - qx) < 1e-11 and abs(gy - qy) < 1e-11
    # 20 cells of the DBA cell with tunes 0.309 / 0.396 per cell
    assert abs(gx - (20 * 0.309) % 1.0) < 0.02 and abs(gy - (20 * 0.396) % 1.0) < 0.02


def test_chromaticity_matches_oracle_maps():
    lat, beam = W.dba_ring(cells=4), W.dba_beam()
    xi = tp.optics.getchrom(lat, beam)
    (qx0, qy0), _ = _oracle_tunes(lat, beam, np.zeros(6))
    (qx1, qy1), _ = _oracle_tunes(lat, beam, np.array([0, 0, 0, 0, 0, 1e-8]))
    ref = ((qx1 - qx0) / 1e-8, (qy1 - qy0) / 1e-8)
    for a, b in zip(xi, ref):
        assert abs(a - b) <= 1e-4 * abs(b) + 1e-6


def test_closed_orbits_are_fixed_points_of_the_oracle_map():
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    bt = tp.beti(beam)
    x4 = tp.optics.find_closed_orbit_4d(lat, beam, dp=1e-3)
    r = np.asfortranarray(np.array([[x4[0], x4[1], x4[2], x4[3], 0.0, 1e-3]]))
    l = np.zeros(1, np.int64)
    oracle_ref.ringpass(lat, r, l, bt, 1)
    assert l[0] == 0 and np.abs(r[0, :4] - x4).max() < 1e-10
    assert abs(x4[0]) > 1e-6  # dispersion moves the off-momentum orbit
    x6 = tp.optics.find_closed_orbit_6d(lat, beam, x0=np.array([0, 0, 0, 0, 0, 1e-4]))
    r = np.asfortranarray(x6[None, :].copy())
    oracle_ref.ringpass(lat, r, np.zeros(1, np.int64), bt, 1)
    assert np.abs(r[0] - x6).max() < 1e-9


def test_batched_maps_at_many_momenta():
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    refs = np.zeros((9, 6))
    refs[:, 5] = np.linspace(-2e-3, 2e-3, 9)
    M, err = tp.optics.one_turn_maps(lat, beam, refs)
    R = oracle_ref.jacobian(lat, refs, tp.beti(beam))
    assert np.abs(M - R).max() <= 1e-9 * np.abs(R).max()
    assert (err < 1e-10).all()


def test_finite_difference_map_is_the_references_bit_for_bit():
    """method="fd" tracks the reference's 12 orbits on the device; the tracking
    is bit-identical to the oracle's, so the matrix is too."""
    lat, beam = W.dba_ring(cells=3), W.dba_beam()
    ref = np.array([2e-5, -1e-6, 1e-5, 0.0, 1e-4, 5e-4])
    M = tp.optics.one_turn_map(lat, beam, ref, method="fd")
    c = tp.optics.fd_orbits(ref)
    oracle_ref.ringpass(lat, c, np.zeros(12, np.int64), tp.beti(beam), 1, aperture=(1.0, 1.0))
    assert np.array_equal(M, tp.optics.fd_assemble(c))
    E = tp.optics.one_turn_map(lat, beam, ref)
    assert np.abs(M - E).max() < 1e-6 * np.abs(E).max()
