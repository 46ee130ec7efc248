"""Synthetic workloads of the tracking benchmarks (seeded, no external data).

  fodo_ring()      FODO ring on 1 GeV electrons: QF(0.5 m, +1.2) D(2.0) QD(0.5 m, -1.2) D(2.0), 8 cells.
  dba_ring()       DBA storage ring on 3 GeV electrons: 20 cells of 25 m, 401 elements with the RF cavity.
  dba_variants()   ragged batch of DBA rings (4..20 cells, strengths perturbed by U[-2%, 2%]).
  time_dependent() a lattice whose Q1 quadrupole family ramps k1 linearly by +1% over a run and whose RF
                   voltage is modulated by 5% with a 200-turn period (the time-dependent adjoint workload).
  gaussian()       seeded 6D Gaussian beam in the reference's N x 6 column-major layout.
  da_grid()        dynamic-aperture grid of (x, y) amplitudes, other coordinates zero.

Random numbers come from numpy's counter-based Philox generator, so every
workload is a pure function of its seed.
"""
import math

import numpy as np

from .elements import C_LIGHT, Drift, ExactSBend, Quadrupole, RFCavity, Sextupole
from .tracking import Beam, Lattice, timed

SIGMA = (1e-4, 1e-5, 1e-4, 1e-5, 1e-3, 1e-4)  # x, px, y, py, z, delta

# DBA strengths: k1 of the three quadrupole families and k2 of the two
# sextupole families.  Drawn by oracle/search_dba.py (Philox seed 0, k1 from
# +-U[0.5, 2.5] m^-2, k2 from +-U[20, 60] m^-3) as the first draw whose linear
# cell map is stable with |trace/2| <= 0.9, whose cell tunes (0.309, 0.396) keep
# 0.04 away from the third- and fourth-order resonances the sextupoles of every
# cell drive, and on which a 256-particle Gaussian beam survives 300 turns.
DBA_FAMILIES = {
    "Q1": 1.3067877421264442,
    "Q2": -0.8455488336578774,
    "Q3": 1.0102025344289203,
    "S1": 38.679376805147385,
    "S2": -29.5033306060304,
}
DBA_CELL = ["D", "Q1", "D", "Q2", "D", "B", "S1", "Q3", "S2", "D", "D", "S2", "Q3", "S1", "B", "D", "Q2", "D", "Q1", "D"]
DBA_CELL_LENGTH = 25.0
DBA_ENERGY = 3.0e9        # kinetic energy [eV] of Beam(3e9)
DBA_RF_VOLT = 3.0e6
DBA_HARMONIC = 500.0


def fodo_ring(cells=8):
    """FODO ring (32 elements for 8 cells); Yoshida-4 with 10 steps per quadrupole."""
    elems = []
    for _ in range(cells):
        elems += [Quadrupole(0.5, 1.2, name="QF"), Drift(2.0, name="D"), Quadrupole(0.5, -1.2, name="QD"),
                  Drift(2.0, name="D")]
    return Lattice(elems, name="FODO")


def fodo_beam():
    """Beam(1.0e9): the reference default energy (src/lattice.jl:208)."""
    return Beam(1.0e9)


def dba_ring(cells=20, strengths=None, rf=True):
    """DBA ring: `cells` x 20 elements + one thin RF cavity (3 MV, harmonic 500).

    `strengths`, if given, maps the element index (within the ring) of every
    quadrupole and sextupole to its strength; the default uses DBA_FAMILIES.
    Element kinds: ExactSBend(1.5 m, 2pi/40, e1 = e2 = angle/2, fringe on, gk 0),
    Quadrupole(0.5 m), Sextupole(0.25 m), Drift(2.25 m).
    """
    ang = 2.0 * math.pi / 40.0
    elems = []
    for _c in range(cells):
        for tag in DBA_CELL:
            i = len(elems)
            if tag == "D":
                elems.append(Drift(2.25, name="D"))
            elif tag == "B":
                elems.append(ExactSBend(1.5, ang, ang / 2, ang / 2, name="B", gk=0.0))
            elif tag[0] == "Q":
                k = strengths[i] if strengths is not None else DBA_FAMILIES[tag]
                elems.append(Quadrupole(0.5, k, name=tag))
            else:
                k = strengths[i] if strengths is not None else DBA_FAMILIES[tag]
                elems.append(Sextupole(0.25, k, name=tag))
    if rf:
        circ = cells * DBA_CELL_LENGTH
        elems.append(RFCavity(0.0, DBA_RF_VOLT, DBA_HARMONIC * C_LIGHT / circ, 0.0, h=DBA_HARMONIC, philag=0.0,
                              energy=DBA_ENERGY, name="RF"))
    return Lattice(elems, name=f"DBA{cells}")


def dba_beam():
    return Beam(DBA_ENERGY)


def magnet_indices(lat, kinds=("QUADRUPOLE", "SEXTUPOLE")):
    """Indices of the quadrupoles and sextupoles of a lattice (gradient parameters)."""
    return [i for i, e in enumerate(lat.elements) if e.kind in kinds]


def dba_variants(nvar=256, seed=1, n_base=4096, perturb=0.02, cells_range=(4, 20)):
    """Ragged batch: cells ~ U{4..20}, every quadrupole/sextupole strength scaled by
    (1 + U[-perturb, perturb]), particle count round(n_base * U[0.25, 1])."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for _v in range(nvar):
        cells = int(rng.integers(cells_range[0], cells_range[1] + 1))
        base = dba_ring(cells)
        strengths = {}
        for i in magnet_indices(base):
            strengths[i] = base.elements[i].k * (1.0 + rng.uniform(-perturb, perturb))
        npart = int(round(n_base * rng.uniform(0.25, 1.0)))
        out.append((dba_ring(cells, strengths), npart))
    return out


def time_dependent(lat, nturns, family="Q1", ramp=0.01, rf_depth=0.05, rf_period=200.0):
    """`lat` with k1 of every quadrupole named `family` ramped linearly by
    `ramp` (relative) over `nturns` turns, and the RF voltage modulated by
    `rf_depth` with a period of `rf_period` turns: per-turn field functions
    (timed / Turn(), src/time_dependence.jl:46, 147-155)."""
    elems = list(lat.elements)
    for i, e in enumerate(elems):
        if e.kind == "QUADRUPOLE" and e.name == family:
            elems[i] = timed(e, k1=lambda ctx, k0=e.k1: k0 * (1.0 + ramp * ctx.turn / nturns))
        elif e.kind == "RFCAVITY":
            elems[i] = timed(e, volt=lambda ctx, v0=e.volt: v0 * (1.0 + rf_depth *
                                                                 math.sin(2.0 * math.pi * ctx.turn / rf_period)))
    return Lattice(elems, name=lat.name + "_TD")


def gaussian(n, seed=0, sigma=SIGMA):
    """N x 6 float64 Gaussian beam, column-major (Fortran order) like a Julia Matrix."""
    rng = np.random.Generator(np.random.Philox(seed))
    a = np.empty((n, 6), dtype=np.float64, order="F")
    for c in range(6):
        a[:, c] = rng.standard_normal(n) * sigma[c]
    return a


def da_grid(nx=512, ny=512, half=0.02):
    """Grid of (x, y) in [-half, half]^2 (linspace), other coordinates zero."""
    xs = np.linspace(-half, half, nx)
    ys = np.linspace(-half, half, ny)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    a = np.zeros((nx * ny, 6), dtype=np.float64, order="F")
    a[:, 0] = X.reshape(-1)
    a[:, 2] = Y.reshape(-1)
    return a


def dba_particles(n_gauss=1 << 20, grid=512, seed=0):
    """The DBA tracking input: n_gauss Gaussian particles followed by the DA grid."""
    parts = [gaussian(n_gauss, seed)]
    if grid:
        parts.append(da_grid(grid, grid))
    return np.asfortranarray(np.concatenate(parts, axis=0))
