"""Reverse maps of the element kinds outside the integrator core and of
misalignment rows, on the GPU through the C ABI.

Checkers: the oracle's forward-mode dual numbers (oracle/tp_oracle.hpp with a
dual scalar) for the tangent maps and for the loss gradients, on the same
survivor set.  Tolerances as in test_gpu_adjoint.py: tangent maps 1e-9 of the
largest entry, gradients 1e-8 of the largest component, the loss 1e-12
relative; the rebuilt states (inverse maps, the crab cavity's fixed point,
the wiggler's shears and radiation root) must come back to the stored ones
within 1e-11.
"""
import math

import numpy as np
import pytest

import oracle_ref
from conftest import tp
from test_gpu_adjoint import LW, SIGMA, assert_grad_close, oracle_grad

pytestmark = pytest.mark.gpu
W = __import__("trackpad_b200.workloads", fromlist=["x"])

E0 = 3.5e9
BEAM_SIGMA = (1e-4, 1e-5, 1e-4, 1e-5, 3e-3, 1e-4)


def kinds_lattice(strong=True, rad=0):
    """Every kind with a reverse map in tp_reverse_kinds.cuh, between
    quadrupoles (the gradient parameters).  strong=False scales the frame
    changes down so that particles survive several turns."""
    acc = tp.AccelCavity(0.0, volt=2.5e6, freq=500e6, h=1200.0, phis=0.2, energy=E0)
    f = 1.0 if strong else 0.01
    return tp.Lattice([
        tp.Drift(0.3),
        tp.Quadrupole(0.4, 1.2),
        tp.Solenoid(0.5, 0.8),
        tp.Solenoid(0.2, 0.0),
        tp.Corrector(0.4, 1.5e-4, -2.2e-4),
        tp.Quadrupole(0.4, -1.1),
        tp.Translation(0.0, dx=1e-3 * f, dy=-2e-3 * f, ds=3e-3),
        tp.YRotation(0.0, angle=0.02 * f),
        tp.CrabCavity(0.3, volt=2e6, freq=500e6, phi=0.1, energy=E0),
        tp.CrabCavity(0.0, volt=1e6, freq=400e6, phi=-0.2, energy=E0),
        acc,
        tp.LongitudinalRFMap(2e-4, acc),
        tp.LorentzBoost(0.03 * f),
        tp.InvLorentzBoost(0.03 * f),
        tp.StrongThinGaussianBeam(1e-6, 1e-3, 1.2e-3, xoffset=1e-4, yoffset=-2e-4),
        tp.StrongGaussianBeam(1e-3, 0.511e6, 1, 10, 6e9, (3e-4, 4e-4), nzslice=4,
                              zslice_npar=[0.1, 0.4, 0.3, 0.2], xoffsets=[1e-5, 0, -2e-5, 3e-5]),
        tp.Quadrupole(0.4, 0.9),
        tp.LongitudinalRLCWake(freq=1.2e9, Rshunt=2e5, Q0=3.5, scale=2e-19),
        tp.LongitudinalWake(list(np.linspace(0, 3e-11, 40)), list(1e13 * np.cos(np.linspace(0, 6, 40))),
                            fliphalf=-1.0, scale=1e-19),
        tp.LongitudinalWake([0.0, 5e-12, 2e-12, 1e-11], [1e13, 2e12, 6e12, -1e12], fliphalf=-1.0, scale=2e-19),
        tp.LBend(0.9, 0.15, 0.03, 0.02, K=0.8, by_error=1e-4, fint1=0.5, fint2=0.4, full_gap=0.05),
        tp.LBend(0.9, 0.15, 0.03, 0.02, K=-0.9),
        tp.Quadrupole(0.4, -0.8),
        tp.Wiggler(0.2, lw=0.05, Bmax=0.9, Nsteps=3, By=(1, 1, 1, 1, 1, 0, 2, -1, 0, 3, 3, 1),
                   Bx=(1, 1, 1, 2, 2, 0), energy=E0, rad=rad),
        tp.Drift(0.5),
    ])


def _orbits(n, seed):
    return np.concatenate([np.zeros((1, 6)), W.gaussian(n - 1, seed=seed, sigma=BEAM_SIGMA)])


@pytest.mark.parametrize("rad", [0, 1])
def test_tangent_maps_of_every_kind_match_oracle(rad):
    lat, beam = kinds_lattice(rad=rad), tp.Beam(E0)
    orbits = _orbits(6, 41)
    M, err = tp.one_turn_jacobian(lat, beam, orbits)
    R = oracle_ref.jacobian(lat, orbits, tp.beti(beam))
    assert np.isfinite(M).all()
    assert np.abs(M - R).max() <= 1e-9 * np.abs(R).max()
    assert tp.adjoint_stats()["reconstruction_error"] < 1e-11
    # the reported ||M^T J M - J|| is that of the returned map (the boosts,
    # the crab cavity's phase at the pre-drift z and the radiation are not
    # symplectic, so there is no bound on the value itself)
    for i in range(len(orbits)):
        assert abs(err[i] - oracle_ref.symplectic_error(M[i])) <= 1e-12 * max(1.0, err[i])


@pytest.mark.parametrize("kind", ["solenoid", "corrector", "translation", "yrotation", "crab", "crab_thin", "accel",
                                  "lrf", "lorentz", "invlorentz", "stgb", "sgb", "rlc", "tabwake", "lbend",
                                  "wiggler", "wiggler_rad"])
def test_tangent_map_of_each_kind(kind):
    """One element between two drifts, so that a failing kind is named."""
    lat_all = kinds_lattice(rad=1 if kind == "wiggler_rad" else 0)
    pick = {"solenoid": 2, "corrector": 4, "translation": 6, "yrotation": 7, "crab": 8, "crab_thin": 9,
            "accel": 10, "lrf": 11, "lorentz": 12, "invlorentz": 13, "stgb": 14, "sgb": 15, "rlc": 17,
            "tabwake": 18, "lbend": 20, "wiggler": 23, "wiggler_rad": 23}[kind]
    els = [tp.Drift(0.2), lat_all.elements[pick], tp.Drift(0.3)]
    if kind == "lrf":
        els.insert(1, lat_all.elements[10])
    lat, beam = tp.Lattice(els), tp.Beam(E0)
    orbits = _orbits(4, 43)
    M, _ = tp.one_turn_jacobian(lat, beam, orbits)
    R = oracle_ref.jacobian(lat, orbits, tp.beti(beam))
    assert np.abs(M - R).max() <= 1e-10 * np.abs(R).max(), kind
    assert tp.adjoint_stats()["reconstruction_error"] < 1e-12


def test_adjoint_through_every_kind_matches_dual_oracle():
    lat, beam = kinds_lattice(strong=False), tp.Beam(E0)
    params = [i for i, e in enumerate(lat.elements) if e.kind == "QUADRUPOLE"]
    c0 = W.gaussian(192, seed=45, sigma=BEAM_SIGMA)
    loss, g = tp.ringpass_adjoint(c0, lat, beam, None, 4, params, checkpoint_every=1, sigma=SIGMA, lost_weight=LW, aperture=0.05)[:2]
    rloss, rg, rsurv = oracle_grad(lat, c0, beam, 4, params, 0.05)
    assert rsurv > 100
    assert abs(loss - rloss) <= 1e-12 * abs(rloss)
    assert_grad_close(g, rg)
    assert tp.adjoint_stats()["reconstruction_error"] < 1e-11


def _roll(theta):
    c, s = math.cos(theta), math.sin(theta)
    R = np.eye(6)
    R[0, 0] = R[1, 1] = R[2, 2] = R[3, 3] = c
    R[0, 2] = R[1, 3] = s
    R[2, 0] = R[3, 1] = -s
    return R


def misaligned_dba(cells=2, seed=7):
    """DBA cells with a random offset and roll on every magnet (the usual
    error-study rows: t1 = -offset, r1 = roll, r2 = roll^-1, t2 = +offset),
    and one general (non-orthogonal) entrance matrix."""
    lat = W.dba_ring(cells=cells)
    rng = np.random.default_rng(seed)
    els = list(lat.elements)
    first = True
    for e in els:
        if getattr(e, "_misalignable", False) and e.kind in ("QUADRUPOLE", "SEXTUPOLE", "SBEND"):
            dx, dy = rng.normal(0, 3e-5, 2)
            th = rng.normal(0, 2e-4)
            r1 = _roll(th)
            if first:  # a sheared, scaled row: needs the general inverse
                r1 = r1 @ (np.eye(6) + 1e-3 * rng.standard_normal((6, 6)))
                first = False
            e._misalign_init([-dx, 0, -dy, 0, 0, 0], [dx, 0, dy, 0, 0, 0], r1, np.linalg.inv(_roll(th)))
    return tp.Lattice(els)


def test_adjoint_with_misalignment_rows_matches_dual_oracle():
    lat, beam = misaligned_dba(), W.dba_beam()
    assert lat.pack()[3] > 0  # misalignment rows present
    params = W.magnet_indices(lat)
    c0 = W.gaussian(256, seed=47)
    loss, g = tp.ringpass_adjoint(c0, lat, beam, None, 6, params, checkpoint_every=1, sigma=SIGMA, lost_weight=LW, aperture=0.02)[:2]
    rloss, rg, _ = oracle_grad(lat, c0, beam, 6, params, 0.02)
    assert abs(loss - rloss) <= 1e-12 * abs(rloss)
    assert_grad_close(g, rg)
    assert tp.adjoint_stats()["reconstruction_error"] < 1e-11


def test_tangent_maps_with_misalignment_rows():
    lat, beam = misaligned_dba(cells=1), W.dba_beam()
    orbits = _orbits(5, 49)
    M, err = tp.one_turn_jacobian(lat, beam, orbits)
    R = oracle_ref.jacobian(lat, orbits, tp.beti(beam))
    assert np.abs(M - R).max() <= 1e-9 * np.abs(R).max()


def test_singular_misalignment_row_is_rejected():
    lat = W.dba_ring(cells=1)
    els = list(lat.elements)
    q = next(i for i, e in enumerate(els) if e.kind == "QUADRUPOLE")
    r1 = np.eye(6)
    r1[5, 5] = 0.0  # delta dropped: no inverse map
    els[q]._misalign_init(None, None, r1, None)
    with pytest.raises(tp._abi.TrackPadError) as ei:
        tp.one_turn_jacobian(tp.Lattice(els), W.dba_beam(), np.zeros((1, 6)))
    assert ei.value.status == tp._abi.TP_EUNSUPPORTED
