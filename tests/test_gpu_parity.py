"""GPU tracking against the oracle and the golden fixtures, through the C ABI.

Default build (no FMA contraction; transcendental functions from the shared
fdlibm-method implementation, exp/sinh/cosh included): coordinates, loss
flags, turn and element of loss are bit-identical to the oracle for every map.

FMA-contraction build (opt-in): 1e-9 relative (per coordinate, scaled by the
column's largest magnitude) after one turn on regular orbits -- the exact
bend's x update is a difference of O(1) terms, so a changed rounding shows up at
1e-11..1e-10 -- and identical losses except for particles within 1e-10 of an edge.
"""
import numpy as np
import pytest

import oracle_ref
from conftest import col_rel_err, golden_lattice, tp, unhex

pytestmark = pytest.mark.gpu
W = __import__("trackpad_b200.workloads", fromlist=["x"])

USES_EXP = set()  # exp now comes from the shared libm too: no exception left


def _run_case(c, contract):
    lat = golden_lattice(c)
    coords = np.asfortranarray(unhex(c["input"]))
    n = coords.shape[0]
    lost = np.zeros(n, np.int64)
    lt = np.full(n, -1, np.int32)
    le = np.full(n, -1, np.int32)
    beam = tp.Beam(c["energy"])
    tp.ringpass_(coords, lat, beam, lost, c["nturns"], aperture=tuple(c["aperture"]), lost_turn=lt, lost_elem=le,
                 contract=contract)
    return coords, lost, lt, le


@pytest.mark.parametrize("contract", [False, True])
def test_golden_cases(golden, contract):
    for c in golden["cases"]:
        coords, lost, lt, le = _run_case(c, contract)
        ref = unhex(c["output"])
        assert lost.tolist() == c["lost"], c["name"]
        assert lt.tolist() == c["lost_turn"], c["name"]
        assert le.tolist() == c["lost_elem"], c["name"]
        if not contract and c["name"] not in USES_EXP:
            assert np.array_equal(coords, ref), f"{c['name']}: default build not bit-identical"
        else:
            err = col_rel_err(coords, ref)
            tol = 1e-12 if not contract else 1e-9
            assert err < tol, f"{c['name']}: relative error {err}"


def _compare(lat, beam, coords0, nturns, aperture, rtol, contract=False, regular=None, rtol_other=None, **kw):
    """GPU vs oracle.  `regular` (bool mask) marks the regular orbits held to
    `rtol`; the other particles (large amplitudes near the dynamic-aperture
    boundary, where a one-ulp difference of a libm call grows by orders of
    magnitude per turn) are held to `rtol_other`."""
    c = coords0.copy(order="F")
    n = c.shape[0]
    lost = np.zeros(n, np.int64)
    lt = np.full(n, -1, np.int32)
    le = np.full(n, -1, np.int32)
    tp.ringpass_(c, lat, beam, lost, nturns, aperture=aperture, lost_turn=lt, lost_elem=le, contract=contract, **kw)
    r = coords0.copy(order="F")
    rl = np.zeros(n, np.int64)
    rlt = np.full(n, -1, np.int32)
    rle = np.full(n, -1, np.int32)
    edge = np.full(n, np.inf)
    oracle_ref.ringpass(lat, r, rl, tp.beti(beam), nturns, aperture=aperture, lost_turn=rlt, lost_elem=rle,
                        min_edge=edge, exact=kw.get("exact", True))
    if not contract:
        # Default build: the same bits as the oracle, lost particles included.
        assert np.array_equal(lost, rl) and np.array_equal(lt, rlt) and np.array_equal(le, rle)
        assert np.array_equal(c, r), f"not bit-identical: max relative difference {col_rel_err(c, r)}"
        return c, lost, st_of()
    # Loss bookkeeping must agree except for particles that came within 1e-10 of an edge.
    mism = (lost != rl) | (lt != rlt) | (le != rle)
    assert not (mism & (edge > 1e-10)).any(), f"{int(mism.sum())} loss mismatches away from the edges"
    ok = (lost == 0) & (rl == 0)
    if regular is None:
        regular = np.ones(n, bool)
    for mask, tol in ((ok & regular, rtol), (ok & ~regular, rtol_other)):
        if mask.any() and tol is not None:
            err = col_rel_err(c[mask], r[mask])
            assert err < tol, f"relative error {err} (tolerance {tol})"
    return c, lost, st_of()


def st_of():
    return tp.last_stats()


def test_fodo_ring_cpu_workload():
    """FODO ring on 1 GeV electrons: 10,000 Gaussian particles, 100 turns,
    aperture 0.05 m (the CPU-runnable workload), against the oracle."""
    lat, beam = W.fodo_ring(), W.fodo_beam()
    coords = W.gaussian(10000, seed=0)
    _, lost, st = _compare(lat, beam, coords, 100, 0.05, 1e-10)
    assert st["particles"] == 10000 and st["units"] == 10000 * 32 * 100
    assert st["element_passes"] == int((lost == 0).sum()) * 32 * 100 or lost.any()


@pytest.mark.parametrize("contract", [False, True])
def test_dba_one_turn(contract):
    """DBA ring, one turn.  Regular orbits (the Gaussian core): 1e-12 relative for
    the default build, 1e-10 with FMA contraction.  Dynamic-aperture grid
    particles: identical losses, coordinates within 1e-8."""
    lat, beam = W.dba_ring(), W.dba_beam()
    core, grid = W.gaussian(2048, seed=0), W.da_grid(32, 32)
    coords = np.asfortranarray(np.concatenate([core, grid]))
    regular = np.arange(len(coords)) < len(core)
    _compare(lat, beam, coords, 1, 0.02, 1e-9 if contract else 1e-12, contract=contract, regular=regular,
             rtol_other=1e-7)


def test_dba_ten_turns_with_losses():
    lat, beam = W.dba_ring(), W.dba_beam()
    core, grid = W.gaussian(512, seed=1), W.da_grid(24, 24)
    coords = np.asfortranarray(np.concatenate([core, grid]))
    regular = np.arange(len(coords)) < len(core)
    c, lost, st = _compare(lat, beam, coords, 10, 0.02, 1e-11, regular=regular, rtol_other=1e-6)
    assert 0 < lost.sum() < len(lost)
    assert st["survivors"] == int((lost == 0).sum())
    # maps evaluated: every turn of a survivor, and up to the element of loss of a lost particle
    c2 = coords.copy(order="F")
    l2 = np.zeros(len(c2), np.int64)
    lt = np.full(len(c2), -1, np.int32)
    le = np.full(len(c2), -1, np.int32)
    tp.ringpass_(c2, lat, beam, l2, 10, aperture=0.02, lost_turn=lt, lost_elem=le)
    expect = int((l2 == 0).sum()) * len(lat) * 10 + int((lt[l2 == 1].astype(np.int64) * len(lat) + le[l2 == 1] + 1).sum())
    assert tp.last_stats()["element_passes"] == expect


@pytest.mark.parametrize("schedule", [1, 2])
@pytest.mark.parametrize("block", [32, 64, 128])
def test_schedules_and_blocks_agree_bitwise(schedule, block):
    """Static and lane-refill scheduling at every block size give identical bits."""
    lat, beam = W.dba_ring(cells=4), W.dba_beam()
    coords0 = np.asfortranarray(np.concatenate([W.gaussian(3000, seed=2), W.da_grid(20, 20)]))
    ref = coords0.copy(order="F")
    rl = np.zeros(len(ref), np.int64)
    tp.ringpass_(ref, lat, beam, rl, 5, aperture=0.02, schedule=1, block_size=128)
    c = coords0.copy(order="F")
    l = np.zeros(len(c), np.int64)
    tp.ringpass_(c, lat, beam, l, 5, aperture=0.02, schedule=schedule, block_size=block)
    assert np.array_equal(l, rl) and np.array_equal(c, ref)


def test_ringpass_equals_repeated_linepass():
    """ringpass!(n) == n x linepass! (src/lattice.jl:305-317)."""
    lat, beam = W.dba_ring(cells=3), W.dba_beam()
    c0 = np.asfortranarray(np.concatenate([W.gaussian(500, seed=4), W.da_grid(10, 10)]))
    a = c0.copy(order="F")
    la = np.zeros(len(a), np.int64)
    tp.ringpass_(a, lat, beam, la, 4, aperture=0.02)
    b = c0.copy(order="F")
    lb = np.zeros(len(b), np.int64)
    for t in range(4):
        tp.linepass_(b, lat, beam, lb, turn=t, aperture=0.02)
    assert np.array_equal(la, lb) and np.array_equal(a, b)


def test_edge_cases():
    lat, beam = W.fodo_ring(), W.fodo_beam()
    # N = 0 and nturns = 0 are no-ops
    tp.ringpass_(np.zeros((0, 6), order="F"), lat, beam, np.zeros(0, np.int64), 10)
    c = W.gaussian(100, seed=5)
    c0 = c.copy()
    tp.ringpass_(c, lat, beam, np.zeros(100, np.int64), 0)
    assert np.array_equal(c, c0)
    # pre-lost particles are untouched; flags other than 1 count as alive
    flags = np.array([1, 2] * 50, np.int64)
    tp.ringpass_(c, lat, beam, flags, 3)
    assert np.array_equal(c[0::2], c0[0::2]) and not np.array_equal(c[1::2], c0[1::2])
    assert flags[1::2].tolist() == [2] * 50
    # every particle lost on the first element keeps its input coordinates
    big = np.asfortranarray(np.full((33, 6), 0.0))
    big[:, 0] = 2.0
    fl = np.zeros(33, np.int64)
    tp.ringpass_(big, lat, beam, fl, 5)
    assert fl.tolist() == [1] * 33 and (big[:, 0] == 2.0).all()
    # ragged sizes
    for n in (1, 31, 33, 257):
        cc = W.gaussian(n, seed=n)
        _compare(lat, beam, cc, 2, 0.05, 1e-12)


def test_row_major_input_is_updated_in_place():
    lat, beam = W.fodo_ring(cells=1), W.fodo_beam()
    c = np.ascontiguousarray(W.gaussian(64, seed=6))
    ref = np.asfortranarray(c)
    tp.ringpass_(c, lat, beam, np.zeros(64, np.int64), 2)
    oracle_ref.ringpass(lat, ref, np.zeros(64, np.int64), tp.beti(beam), 2)
    assert col_rel_err(c, ref) < 1e-12


def test_device_pointers_match_host_path():
    import torch
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    host = W.gaussian(4096, seed=7)
    dev = torch.from_numpy(np.ascontiguousarray(host.T)).cuda()  # (6, N) rows = columns of the N x 6 matrix
    lost_d = torch.zeros(4096, dtype=torch.int64, device="cuda")
    tp.ringpass_(dev.T, lat, beam, lost_d, 3, aperture=0.02)
    lost_h = np.zeros(4096, np.int64)
    tp.ringpass_(host, lat, beam, lost_h, 3, aperture=0.02)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy().T, host) and np.array_equal(lost_d.cpu().numpy(), lost_h)


@pytest.mark.parametrize("side_stream", [False, True])
def test_device_inputs_filled_on_the_torch_stream_are_ordered(side_stream):
    """Inputs written by PyTorch on its current stream (the default one, or a
    side stream set with torch.cuda.stream) behind a ~25 ms kernel, then
    tracked at once without a synchronize: the call must see the filled
    inputs, not the NaN coordinates and set loss flags they replace."""
    import torch
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    host = W.gaussian(4096, seed=8)
    init = torch.from_numpy(np.ascontiguousarray(host.T)).cuda()
    lost_h = np.zeros(4096, np.int64)
    tp.ringpass_(host, lat, beam, lost_h, 3, aperture=0.02)
    coords = torch.full_like(init, float("nan"))
    lost = torch.ones(4096, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    side = torch.cuda.Stream() if side_stream else torch.cuda.current_stream()
    with torch.cuda.stream(side):
        torch.cuda._sleep(50_000_000)  # a bounded spin of 5e7 clock cycles
        coords.copy_(init)
        lost.zero_()
        tp.ringpass_(coords.T, lat, beam, lost, 3, aperture=0.02)
    torch.cuda.synchronize()
    assert np.array_equal(coords.cpu().numpy().T, host) and np.array_equal(lost.cpu().numpy(), lost_h)


def test_linearised_drift_option():
    lat, beam = W.fodo_ring(cells=2), W.fodo_beam()
    c = W.gaussian(256, seed=8)
    _compare(lat, beam, c, 3, 0.05, 1e-12, exact=False)


def test_time_dependent_schedule():
    """timed quadrupole k1 and RF voltage, evaluated per turn (as materialize
    does per linepass! call), against the oracle with the same per-turn values."""
    import math
    base = W.dba_ring(cells=2)
    elems = list(base.elements)
    qi = next(i for i, e in enumerate(elems) if e.kind == "QUADRUPOLE")
    ri = len(elems) - 1
    elems[qi] = tp.timed(elems[qi], k1=lambda ctx, k0=elems[qi].k1: k0 * (1 + 0.01 * ctx.turn / 20))
    elems[ri] = tp.timed(elems[ri], volt=lambda ctx, v0=elems[ri].volt: v0 * (1 + 0.05 * math.sin(2 * math.pi * ctx.turn / 200)))
    lat = tp.Lattice(elems)
    beam = W.dba_beam()
    c0 = W.gaussian(300, seed=9)
    c = c0.copy(order="F")
    lost = np.zeros(300, np.int64)
    tp.ringpass_(c, lat, beam, lost, 6, turn=3, aperture=0.02)
    vals = np.array([[elems[qi].updates["k1"](tp.TimeContext(0.0, t)), elems[ri].updates["volt"](tp.TimeContext(0.0, t))]
                     for t in range(3, 9)])
    r = c0.copy(order="F")
    rl = np.zeros(300, np.int64)
    oracle_ref.ringpass(base, r, rl, tp.beti(beam), 6, turn0=3, aperture=0.02,
                        sched=([qi, 1, ri, 5], 3, vals))
    assert np.array_equal(lost, rl)
    assert col_rel_err(c, r) < 1e-12


def test_batched_equals_lattice_by_lattice():
    """One ragged batched launch == each variant tracked on its own, bit for bit."""
    variants = W.dba_variants(nvar=6, seed=3, n_base=300)
    batch = tp.Batch([v for v, _ in variants])
    beam = W.dba_beam()
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([W.gaussian(n, seed=10 + i) for i, n in enumerate(counts)]))
    ref = coords.copy(order="F")
    lost = np.zeros(len(coords), np.int64)
    for use_graph in (False, True, True):
        c = coords.copy(order="F")
        l = np.zeros(len(c), np.int64)
        batch.ringpass_(c, poff, np.full(len(counts), tp.beti(beam)), l, 4, aperture=0.02, use_graph=use_graph)
        st = tp.last_stats()
        assert st["units"] == sum(n * len(v) * 4 for v, n in variants)
        for i, (lat, n) in enumerate(variants):
            s = slice(poff[i], poff[i + 1])
            rc = np.asfortranarray(ref[s])
            rl = np.zeros(n, np.int64)
            tp.ringpass_(rc, lat, beam, rl, 4, aperture=0.02, schedule=1)
            assert np.array_equal(c[s], rc) and np.array_equal(l[s], rl)


@pytest.mark.parametrize("schedule", [1, 2])
def test_batched_schedules_with_losses_equal_lattice_by_lattice(schedule):
    """Static tiles and pooled refill (lanes of a variant refilled from that
    variant's particles after losses) give the same bits as each variant alone."""
    variants = W.dba_variants(nvar=5, seed=4, n_base=200, cells_range=(2, 5))
    batch = tp.Batch([v for v, _ in variants])
    beam = W.dba_beam()
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([np.concatenate([W.gaussian(n // 2, seed=60 + i),
                                                               W.da_grid(1, n - n // 2, half=0.019)])
                                               for i, n in enumerate(counts)]))
    c = coords.copy(order="F")
    l = np.zeros(len(c), np.int64)
    lt = np.full(len(c), -1, np.int32)
    le = np.full(len(c), -1, np.int32)
    batch.ringpass_(c, poff, np.full(len(counts), tp.beti(beam)), l, 12, aperture=0.02, lost_turn=lt, lost_elem=le,
                    schedule=schedule, use_graph=False)
    assert tp.last_stats()["schedule"] == schedule
    assert 0 < l.sum() < len(l)
    for i, (lat, n) in enumerate(variants):
        s = slice(poff[i], poff[i + 1])
        rc = np.asfortranarray(coords[s])
        rl = np.zeros(n, np.int64)
        rlt = np.full(n, -1, np.int32)
        rle = np.full(n, -1, np.int32)
        tp.ringpass_(rc, lat, beam, rl, 12, aperture=0.02, lost_turn=rlt, lost_elem=rle, schedule=1)
        assert np.array_equal(c[s], rc) and np.array_equal(l[s], rl)
        assert np.array_equal(lt[s], rlt) and np.array_equal(le[s], rle)


def test_autotuned_launch_settles_and_keeps_results():
    """schedule = min_blocks = 0: the first multi-turn calls try static and
    refill at 7 resident blocks per SM, then 8, 6 and 5 blocks with the faster
    schedule; later calls keep the fastest; every call gives the same bits."""
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    c0 = np.asfortranarray(np.concatenate([W.gaussian(300, seed=70), W.da_grid(16, 16)]))
    seen, outs = [], []
    for _ in range(8):
        c = c0.copy(order="F")
        l = np.zeros(len(c), np.int64)
        tp.ringpass_(c, lat, beam, l, 6, aperture=0.02)
        st = tp.last_stats()
        seen.append((st["schedule"], st["min_blocks"]))
        outs.append((c, l))
    assert seen[0] == (1, 7) and seen[1] == (2, 7)
    assert [m for _, m in seen[2:5]] == [8, 6, 5] and seen[2][0] == seen[3][0] == seen[4][0]
    assert seen[5] == seen[6] == seen[7] and seen[5] in seen[:5]
    for c, l in outs[1:]:
        assert np.array_equal(c, outs[0][0]) and np.array_equal(l, outs[0][1])


@pytest.mark.parametrize("minb", [5, 6, 7, 8])
def test_every_occupancy_instance_gives_the_same_bits(minb):
    """The kernel instances sized for 5, 6, 7 and 8 resident blocks per SM, single
    lattice and batched, bit-identical to the oracle / to each other."""
    lat, beam = W.dba_ring(cells=3), W.dba_beam()
    c0 = np.asfortranarray(np.concatenate([W.gaussian(500, seed=71), W.da_grid(12, 12)]))
    c = c0.copy(order="F")
    l = np.zeros(len(c), np.int64)
    tp.ringpass_(c, lat, beam, l, 5, aperture=0.02, schedule=2, min_blocks=minb)
    assert tp.last_stats()["min_blocks"] == minb
    r = c0.copy(order="F")
    rl = np.zeros(len(r), np.int64)
    oracle_ref.ringpass(lat, r, rl, tp.beti(beam), 5, aperture=(0.02, 0.02))
    assert np.array_equal(c, r) and np.array_equal(l, rl)
    variants = W.dba_variants(nvar=3, seed=12, n_base=200, cells_range=(2, 4))
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([W.gaussian(n, seed=80 + i) for i, n in enumerate(counts)]))
    batch = tp.Batch([v for v, _ in variants])
    outs = []
    for m in (7, minb):
        cb = coords.copy(order="F")
        lb = np.zeros(len(cb), np.int64)
        batch.ringpass_(cb, poff, np.full(3, tp.beti(beam)), lb, 5, aperture=0.02, schedule=2, min_blocks=m,
                        use_graph=True)
        assert tp.last_stats()["min_blocks"] == m
        outs.append((cb, lb))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_batched_time_dependent_equals_lattice_by_lattice():
    """Variants with a ramped quadrupole family and a modulated RF voltage in one
    batched launch == each variant on its own; a new turn range rebuilds the
    batch's per-turn tables (and its CUDA graph)."""
    variants = W.dba_variants(nvar=3, seed=7, n_base=150, cells_range=(2, 3))
    lats = [W.time_dependent(v, 40) for v, _ in variants]
    batch = tp.Batch(lats)
    beam = W.dba_beam()
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([W.gaussian(n, seed=40 + i) for i, n in enumerate(counts)]))
    for turn0, use_graph in ((2, True), (2, True), (9, True), (9, False)):
        c = coords.copy(order="F")
        l = np.zeros(len(c), np.int64)
        batch.ringpass_(c, poff, np.full(len(counts), tp.beti(beam)), l, 6, turn=turn0, aperture=0.02,
                        use_graph=use_graph)
        for i, lat in enumerate(lats):
            s = slice(poff[i], poff[i + 1])
            rc = np.asfortranarray(coords[s])
            rl = np.zeros(counts[i], np.int64)
            tp.ringpass_(rc, lat, beam, rl, 6, turn=turn0, aperture=0.02, schedule=1)
            assert np.array_equal(c[s], rc) and np.array_equal(l[s], rl)


def test_array_field_kinds_bitwise():
    """LBend (both signs of the gradient), StrongGaussianBeam slices, the
    resonator wake, sorted / unsorted tabulated wakes and wigglers (vertical
    harmonics, radiation), over a beam whose z spans the wake tables, against
    the oracle bit for bit."""
    lat = tp.Lattice([
        tp.LBend(0.9, 0.15, 0.03, 0.02, K=0.8, by_error=1e-4, fint1=0.5, fint2=0.4, full_gap=0.05),
        tp.Drift(0.5),
        tp.LBend(0.9, 0.15, 0.03, 0.02, K=-0.9),
        tp.StrongGaussianBeam(1e-3, 0.511e6, 1, 10, 6e9, (3e-4, 4e-4), nzslice=4,
                              zslice_npar=[0.1, 0.4, 0.3, 0.2], xoffsets=[1e-5, 0, -2e-5, 3e-5]),
        tp.LongitudinalRLCWake(freq=1.2e9, Rshunt=2e5, Q0=3.5, scale=2e-19),
        tp.LongitudinalWake(list(np.linspace(0, 3e-11, 40)), list(1e13 * np.cos(np.linspace(0, 6, 40))),
                            fliphalf=-1.0, scale=1e-19),
        tp.LongitudinalWake([0.0, 5e-12, 2e-12, 1e-11], [1e13, 2e12, 6e12, -1e12], fliphalf=-1.0, scale=2e-19),
        tp.Quadrupole(0.4, 1.1),
        tp.Wiggler(0.2, lw=0.05, Bmax=0.9, Nsteps=3, By=(1, 1, 1, 1, 1, 0, 2, -1, 0, 3, 3, 1),
                   Bx=(1, 1, 1, 2, 2, 0), energy=3.5e9),
        tp.Wiggler(0.2, lw=0.1, Bmax=1.4, Nsteps=2, energy=3.5e9, rad=1),
    ])
    beam = tp.Beam(3.5e9)
    c = W.gaussian(4096, seed=77, sigma=(1e-4, 1e-5, 1e-4, 1e-5, 3e-3, 1e-4))
    _compare(lat, beam, c, 3, 0.05, 1e-12)


def test_unsupported_schedule_outside_range():
    base = W.dba_ring(cells=1)
    elems = list(base.elements)
    elems[1] = tp.timed(elems[1], k1=lambda ctx: 1.0)
    lat = tp.Lattice(elems)
    lat.set_schedule(0.0, 0.0, 0, 2)
    c = W.gaussian(10, seed=1)
    import ctypes as C
    o = tp.tracking._opts(None, True, False, False)
    st = tp._abi.lib().tp_ringpass(tp.context(), lat.handle, c.ctypes.data_as(C.c_void_p), 10,
                                   np.zeros(10, np.int64).ctypes.data_as(C.c_void_p), None, None,
                                   C.c_double(1.0001), 5, C.c_double(0), C.c_double(0), 0, C.byref(o))
    assert st == tp._abi.TP_ERANGE


def test_table_in_shared_memory_or_l1_gives_the_same_bits():
    """tp_opts.table_in_smem only moves the element table (shared memory by a
    bulk copy, or the L1 cache): tracking and gradients are bit-identical."""
    lat, beam = W.dba_ring(cells=2), W.dba_beam()
    c0 = W.gaussian(4096, seed=5)
    params = W.magnet_indices(lat)
    out = []
    for flag in (False, True):
        tp.tracking.TABLE_IN_SMEM = flag
        try:
            c = np.asfortranarray(c0.copy())
            lost = np.zeros(len(c), np.int64)
            tp.ringpass_(c, lat, beam, lost, 5, aperture=0.02)
            loss, g = tp.ringpass_adjoint(c0, lat, beam, None, 3, params, checkpoint_every=1, sigma=1e-4, aperture=0.02)[:2]
            out.append((c, lost, loss, g))
        finally:
            tp.tracking.TABLE_IN_SMEM = False
    (c1, l1, s1, g1), (c2, l2, s2, g2) = out
    assert np.array_equal(c1, c2, equal_nan=True) and np.array_equal(l1, l2)
    assert s1 == s2 and np.array_equal(g1, g2)


def test_bounds_checked_kernels_give_the_same_bits():
    """tp_opts.bounds_check runs the kernels that check every element-table
    record (inside its table or turn block) and particle index before reading
    them: on valid inputs they give the default build's bits, single lattice
    (with a per-turn schedule) and batched, and report no violation."""
    base = W.dba_ring(cells=2)
    lat = W.time_dependent(base, 8)
    beam = W.dba_beam()
    c0 = np.asfortranarray(np.concatenate([W.gaussian(400, seed=90), W.da_grid(10, 10)]))
    outs = []
    for bc in (False, True):
        c = c0.copy(order="F")
        l = np.zeros(len(c), np.int64)
        lt = np.full(len(c), -1, np.int32)
        tp.ringpass_(c, lat, beam, l, 8, aperture=0.02, lost_turn=lt, bounds_check=bc)
        outs.append((c, l, lt))
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
    variants = W.dba_variants(nvar=4, seed=14, n_base=150, cells_range=(2, 4))
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([W.gaussian(n, seed=95 + i) for i, n in enumerate(counts)]))
    batch = tp.Batch([v for v, _ in variants])
    bo = []
    for bc in (False, True):
        cb = coords.copy(order="F")
        lb = np.zeros(len(cb), np.int64)
        batch.ringpass_(cb, poff, np.full(4, tp.beti(beam)), lb, 6, aperture=0.02, schedule=2, use_graph=True,
                        bounds_check=bc)
        bo.append((cb, lb))
    assert np.array_equal(bo[0][0], bo[1][0]) and np.array_equal(bo[0][1], bo[1][1])


def test_batched_refill_folds_are_tuned_and_keep_the_bits():
    """Pooled refill with fewer warps per variant (1/2 and 1/4 of the 32-particle
    tiles, each warp refilling from the variant's pool more often): the tuner
    times folds 1, 2, 4 on the first calls and keeps one; every call gives the
    same bits."""
    variants = W.dba_variants(nvar=5, seed=16, n_base=300, cells_range=(2, 5))
    counts = [n for _, n in variants]
    poff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = np.asfortranarray(np.concatenate([np.concatenate([W.gaussian(n - n // 4, seed=110 + i),
                                                               W.da_grid(1, n // 4, half=0.019)])
                                               for i, n in enumerate(counts)]))
    batch = tp.Batch([v for v, _ in variants])
    beam = W.dba_beam()
    seen, outs = [], []
    for _ in range(5):
        c = coords.copy(order="F")
        l = np.zeros(len(c), np.int64)
        lt = np.full(len(c), -1, np.int32)
        batch.ringpass_(c, poff, np.full(5, tp.beti(beam)), l, 10, aperture=0.02, lost_turn=lt, schedule=2,
                        min_blocks=7, use_graph=True)
        seen.append(tp.last_stats()["refill_fold"])
        outs.append((c, l, lt))
    assert seen[:3] == [1, 2, 4] and seen[3] == seen[4] and seen[3] in (1, 2, 4)
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert np.array_equal(a, b)
    assert 0 < outs[0][1].sum() < len(coords)
