"""The host mirror of the reference interface: constructors, defaults, packing."""
import math

import numpy as np
import pytest

from conftest import tp

abi = tp._abi


def test_constructor_defaults_follow_reference():
    q = tp.Quadrupole(0.5, 1.2)
    assert (q.max_order, q.num_int_steps, q.k1) == (1, 10, 1.2)          # quad.jl:29
    s = tp.Sextupole(0.25, 30.0)
    assert (s.max_order, s.num_int_steps) == (2, 10)                      # multipole.jl:29
    o = tp.Octupole(0.2, 3.0)
    assert o.max_order == 3
    b = tp.SBend(1.0, 0.1)
    assert (b.max_order, b.fringe_bend_entrance, b.fringe_bend_exit) == (0, 1, 1)  # bend.jl:36-39
    eb = tp.ExactSBend(1.0, 0.1)
    assert eb.gk == 0.0 and eb.name == "ESBEND"
    rf = tp.RFCavity(0.0, 1e6, 5e8)
    assert rf.energy == 0.0 and rf.h == 1.0                               # rf.jl:17-18
    assert tp.CrabCavity(0.1, freq=5e8).k == pytest.approx(2 * math.pi * 5e8 / 2.99792458e8)


def test_rectangular_bends_split_angle():
    rb = tp.RBend(0.9, 0.15)
    assert rb.e1 == rb.e2 == 0.075
    er = tp.ERBend(0.9, 0.15)
    assert isinstance(er, tp.ExactSBend) and er.e1 == er.e2 == 0.075


def test_kickers():
    h = tp.HKicker(xkick=2.5e-4)
    v = tp.VKicker(ykick=-1.5e-4)
    assert (h.xkick, h.ykick, v.xkick, v.ykick) == (2.5e-4, 0.0, 0.0, -1.5e-4)


def test_pack_roundtrip():
    q = tp.Quadrupole(0.5, -0.8, kick_angle=[1e-4, -2e-4], polynom_a=[0, 0.05, 0, 0])
    e = q.pack()
    assert e.kind == abi.KIND["QUADRUPOLE"] and e.k == -0.8 and e.L == 0.5
    assert list(e.kick_angle) == [1e-4, -2e-4] and e.polynom_a[1] == 0.05
    assert e.misalign_index == -1


def test_misalignment_packs_into_side_table():
    d = tp.Drift(1.0, t1=[1e-3, 0, 0, 0, 0, 0])
    lat = tp.Lattice([tp.Drift(1.0), d])
    arr, n, marr, nm, aux = lat.pack()
    assert nm == 1 and arr[1].misalign_index == 0 and marr[0].t1[0] == 1e-3


def test_timed_rejects_unknown_fields():
    q = tp.Quadrupole(0.4, 0.6)
    with pytest.raises(ValueError):
        tp.timed(q, kk=1.0)
    qt = tp.timed(q, k1=lambda ctx: 0.6 + 0.01 * ctx.turn)
    assert tp.materialize(qt, tp.TimeContext(1.0, 5)).k1 == pytest.approx(0.65)
    assert tp.materialize(qt, 0.0).k1 == pytest.approx(0.6)


def test_spos_and_length():
    lat = tp.Lattice([tp.Drift(1.0), tp.Quadrupole(0.5, 1.0), tp.Marker()])
    assert tp.spos(lat) == [0.0, 1.0, 1.5, 1.5]
    assert lat.total_length() == 1.5


def test_tracking_rejects_bad_arrays():
    lat = tp.Lattice([tp.Drift(1.0)])
    beam = tp.Beam(1e9)
    with pytest.raises(TypeError):
        tp.ringpass_(np.zeros((4, 6), dtype=np.float32), lat, beam, np.zeros(4, np.int64), 1)
    with pytest.raises(ValueError):
        tp.ringpass_(np.zeros((4, 5)), lat, beam, np.zeros(4, np.int64), 1)
    with pytest.raises(TypeError):
        tp.ringpass_(np.zeros((4, 6)), lat, beam, np.zeros(4, np.int32), 1)


def test_tune_from_a_known_2x2_map():
    """twiss_from_2x2 (src/optics.jl:123-149) on R(mu) in Twiss form."""
    import math
    for mu, beta, alpha in ((0.3, 12.0, 0.4), (2.0, 3.5, -1.2), (4.5, 7.0, 0.0)):
        g = (1 + alpha * alpha) / beta
        M = np.array([[math.cos(mu) + alpha * math.sin(mu), beta * math.sin(mu)],
                      [-g * math.sin(mu), math.cos(mu) - alpha * math.sin(mu)]])
        b, a, m, q = tp.optics.twiss_from_2x2(M)
        assert abs(b - beta) < 1e-12 and abs(a - alpha) < 1e-12
        assert abs(q - (mu / (2 * math.pi)) % 1.0) < 1e-14
    with pytest.raises(ValueError):
        tp.optics.twiss_from_2x2(np.array([[2.0, 1.0], [1.0, 1.0]]))


def test_fd_map_assembly_against_the_oracle():
    """fd_orbits/fd_assemble (the reference's one_turn_map, src/optics.jl:110-121)
    with the oracle as the tracker agree with the oracle's dual-number map to
    the truncation error of h = 1e-8 central differences."""
    import oracle_ref
    W = __import__("trackpad_b200.workloads", fromlist=["x"])
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    ref = np.array([1e-5, 0.0, -2e-5, 0.0, 0.0, 1e-4])
    c = tp.optics.fd_orbits(ref)
    assert c.flags.f_contiguous and c.shape == (12, 6)
    assert np.array_equal(c[4], ref + 1e-8 * np.eye(6)[2]) and np.array_equal(c[5], ref - 1e-8 * np.eye(6)[2])
    oracle_ref.ringpass(lat, c, np.zeros(12, np.int64), tp.beti(beam), 1)
    M = tp.optics.fd_assemble(c)
    R = oracle_ref.jacobian(lat, ref[None, :], tp.beti(beam))[0]
    assert np.abs(M - R).max() < 1e-6 * np.abs(R).max()


def test_device_calls_run_on_the_callers_current_stream(monkeypatch):
    """With device arrays and no stream given, tp_opts.stream is PyTorch's
    current stream of the arrays' device; handle 0 (PyTorch's default stream)
    becomes NULL, the context stream, which is ordered with it.  Host arrays
    and an explicit stream are left as given."""
    import torch

    class _S:
        def __init__(self, h):
            self.cuda_stream = h

    seen = []
    handles = {None: 0, 3: 0xABC0}
    monkeypatch.setattr(torch.cuda, "current_stream", lambda d=None: seen.append(d) or _S(handles[d]))
    o = tp.tracking._opts(None, True, False, True, device_index=3)
    assert o.stream == 0xABC0 and seen == [3]
    o = tp.tracking._opts(None, True, False, True)
    assert not o.stream
    o = tp.tracking._opts(None, True, False, True, stream=0x55, device_index=3)
    assert o.stream == 0x55 and seen == [3, None]
    o = tp.tracking._opts(None, True, False, False)
    assert not o.stream and seen == [3, None]
