"""Properties that pin the oracle without the reference: analytic limits,
symplecticity, time reversibility, loss semantics and the known answers of the
reference tests that do not need JuTrack."""
import math

import numpy as np
import pytest

import oracle_ref
from conftest import tp

W = __import__("trackpad_b200.workloads", fromlist=["x"])


def beti_of(e):
    return tp.beti(tp.Beam(e))


def test_beam_matches_reference_formula():
    # Beam(energy): gamma = (E + m)/m (kinetic energy), beta = sqrt(1 - 1/gamma^2)
    b = tp.Beam(3.0e9)
    assert b.gamma == (3.0e9 + tp.M_ELECTRON) / tp.M_ELECTRON
    assert oracle_ref.lib().orc_beam_beti(3.0e9, tp.M_ELECTRON) == tp.beti(b)


def test_drift_is_linear_in_length():
    r0 = np.array([1e-3, 2e-4, -5e-4, 1e-4, 0.0, 1e-4])
    bt = beti_of(3e9)
    a = oracle_ref.submap(0, r0, 1.0, 0.0, bt)
    b = oracle_ref.submap(0, oracle_ref.submap(0, r0, 0.5, 0.0, bt), 0.5, 0.0, bt)
    assert np.allclose(a, b, rtol=0, atol=1e-18)
    # x advances by L * px / pz with pz = sqrt(1 + 2 delta beti + delta^2 - px^2 - py^2)
    pz = math.sqrt(1 + 2 * r0[5] * bt + r0[5] ** 2 - r0[1] ** 2 - r0[3] ** 2)
    assert a[0] == pytest.approx(r0[0] + r0[1] / pz, rel=1e-15)


def test_quadrupole_thin_lens_limit():
    # A short quadrupole focuses like a thin lens of strength k1*L at small amplitude.
    bt = beti_of(3e9)
    L, k1 = 1e-3, 2.0
    q = tp.Quadrupole(L, k1)
    M = oracle_ref.jacobian([q.pack()], np.zeros(6), bt)[0]
    assert M[1, 0] == pytest.approx(-k1 * L, rel=1e-5)
    assert M[3, 2] == pytest.approx(k1 * L, rel=1e-5)


def test_fodo_cell_matches_thick_lens_matrices():
    """On the design orbit the linear part of a FODO cell is the product of the
    thick-lens matrices (Yoshida-4 with 10 steps is accurate to ~1e-9 here)."""
    bt = beti_of(1e9)
    lat = W.fodo_ring(cells=1)
    M = oracle_ref.jacobian(lat, np.zeros(6), bt)[0]

    def quad(k, L):
        w = math.sqrt(abs(k))
        if k > 0:
            return np.array([[math.cos(w * L), math.sin(w * L) / w], [-w * math.sin(w * L), math.cos(w * L)]])
        return np.array([[math.cosh(w * L), math.sinh(w * L) / w], [w * math.sinh(w * L), math.cosh(w * L)]])

    D = np.array([[1.0, 2.0], [0.0, 1.0]])
    mx = D @ quad(-1.2, 0.5) @ D @ quad(1.2, 0.5)
    my = D @ quad(1.2, 0.5) @ D @ quad(-1.2, 0.5)
    assert np.allclose(M[0:2, 0:2], mx, atol=1e-8)
    assert np.allclose(M[2:4, 2:4], my, atol=1e-8)
    assert abs(np.trace(mx)) / 2 < 1  # stable, as required by the FODO ring workload


@pytest.mark.parametrize("name", ["fodo", "dba_cell", "dba_ring"])
def test_jacobians_are_symplectic(name):
    if name == "fodo":
        lat, bt = W.fodo_ring(), beti_of(1e9)
    elif name == "dba_cell":
        lat, bt = W.dba_ring(cells=1, rf=False), beti_of(3e9)
    else:
        lat, bt = W.dba_ring(), beti_of(3e9)
    orbits = np.array([[0, 0, 0, 0, 0, 0], [1e-4, 1e-5, -1e-4, 2e-5, 1e-3, 1e-4]], dtype=float)
    for M in oracle_ref.jacobian(lat, orbits, bt):
        assert oracle_ref.symplectic_error(M) < 1e-10


def test_dba_ring_is_stable_in_6d():
    lat, bt = W.dba_ring(), beti_of(3e9)
    M = oracle_ref.jacobian(lat, np.zeros(6), bt)[0]
    ev = np.linalg.eigvals(M)
    assert np.allclose(np.abs(ev), 1.0, atol=1e-9)
    tunes = np.sort(np.abs(np.angle(ev)) / (2 * np.pi))
    assert 0 < tunes[0] < 0.05  # synchrotron tune


@pytest.mark.parametrize("which,a0,a1", [(0, 2.25, 0.0), (1, 0.10471975511965977, 0.1), (3, 0.05, 0.0),
                                         (5, 0.05, 1.2)])
def test_submaps_are_time_reversible(which, a0, a1):
    """drift(-L), exact body(-L), yrot(-phi), kick(-K) invert their maps: the
    inverse maps of the adjoint's reverse sweep."""
    bt = beti_of(3e9)
    r0 = np.array([1e-3, 2e-4, -5e-4, 1e-4, 3e-4, 1e-4])
    if which == 1:
        r1 = oracle_ref.submap(1, r0, a0, a1, bt)
        back = oracle_ref.submap(1, r1, a0, -a1, bt)
    elif which == 5:
        r1 = oracle_ref.submap(5, r0, a0, a1, bt)
        back = oracle_ref.submap(5, r1, -a0, a1, bt)
    else:
        r1 = oracle_ref.submap(which, r0, a0, a1, bt)
        back = oracle_ref.submap(which, r1, -a0, a1, bt)
    assert np.allclose(back, r0, rtol=0, atol=1e-15)


def test_bend_edge_inverse_is_opposite_wedge():
    bt = beti_of(3e9)
    h = 2 * math.pi / 40 / 1.5
    r0 = np.array([1e-3, 2e-4, -5e-4, 1e-4, 3e-4, 1e-4])
    r1 = oracle_ref.submap(2, r0, h, -0.0785, bt)
    back = oracle_ref.submap(2, r1, h, 0.0785, bt)
    assert np.allclose(back, r0, rtol=0, atol=1e-14)


def test_loss_freezes_entrance_coordinates():
    """linepass!: a lost particle keeps the coordinates of the entrance of the
    element where it was lost (src/lattice.jl:281-284)."""
    bt = beti_of(1e9)
    elems = [tp.Drift(1.0).pack(), tp.Drift(1.0).pack()]
    c = np.asfortranarray([[0.0, 0.6, 0.0, 0.0, 0.0, 0.0], [0.0, 0.1, 0.0, 0.0, 0.0, 0.0]])
    lost = np.zeros(2, dtype=np.int64)
    lt = np.full(2, -1, np.int32)
    le = np.full(2, -1, np.int32)
    oracle_ref.ringpass(elems, c, lost, bt, 1, lost_turn=lt, lost_elem=le)
    assert lost.tolist() == [1, 0]
    assert le.tolist() == [1, -1] and lt.tolist() == [0, -1]
    assert c[0, 0] == pytest.approx(0.6 / math.sqrt(1 - 0.36), rel=1e-12)  # after drift 1, before drift 2


def test_flag_other_than_one_counts_as_alive():
    bt = beti_of(1e9)
    c = np.asfortranarray(np.zeros((3, 6)))
    c[:, 1] = 1e-3
    lost = np.array([0, 1, 2], dtype=np.int64)
    oracle_ref.ringpass([tp.Drift(1.0).pack()], c, lost, bt, 1)
    assert c[0, 0] > 0 and c[1, 0] == 0 and c[2, 0] > 0


def test_aperture_is_rectangular_and_strict():
    bt = beti_of(1e9)
    c = np.asfortranarray(np.zeros((3, 6)))
    c[:, 0] = [0.02, 0.0200001, -0.0199]
    lost = np.zeros(3, dtype=np.int64)
    oracle_ref.ringpass([tp.Marker().pack()], c, lost, bt, 1, aperture=(0.02, 0.01))
    assert lost.tolist() == [0, 1, 0]


def test_schedule_materializes_each_turn():
    """Known answer of test/verify_time_dependence.jl:65-73: ringpass over a
    timed lattice equals the per-turn materialised lattices applied in turn."""
    bt = beti_of(3e9)
    d = tp.Drift(1.0)
    q = tp.Quadrupole(0.4, 0.6, num_int_steps=8)
    elems = [d.pack(), q.pack(), d.pack()]
    k = [0.6 + 0.2 * math.sin(0.1 * t) + 0.01 * (4 + t) for t in range(3)]
    c = np.asfortranarray([[1e-3, 2e-4, 5e-4, -1e-4, 0.0, 0.0]])
    lost = np.zeros(1, np.int64)
    oracle_ref.ringpass(elems, c, lost, bt, 3, turn0=4, sched=([1, 1], 4, np.array(k).reshape(3, 1)))
    m = np.asfortranarray([[1e-3, 2e-4, 5e-4, -1e-4, 0.0, 0.0]])
    for t in range(3):
        qt = tp.Quadrupole(0.4, k[t], num_int_steps=8)
        oracle_ref.ringpass([d.pack(), qt.pack(), d.pack()], m, np.zeros(1, np.int64), bt, 1)
    assert np.array_equal(c, m)


def test_time_parameter_known_answer():
    """test/verify_time_dependence.jl:21-26: p = 2 + 0.5 sin(t) + 0.1 turn."""
    t, n = tp.Time(), tp.Turn()
    p = 2.0 + 0.5 * t.__class__(lambda c: math.sin(c.real_time)) + 0.1 * n
    assert p(0.0) == pytest.approx(2.0, abs=1e-15)
    assert p(tp.TimeContext(math.pi / 2, turn=3)) == pytest.approx(2.8, abs=1e-15)
