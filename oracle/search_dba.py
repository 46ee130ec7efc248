"""Seeded search for the strengths of the DBA storage-ring workload.

TEST INFRASTRUCTURE: runs the CPU oracle.  Its output is the table of strengths
hard-coded in trackpad.jl_b200/workloads.py (DBA_FAMILIES); rerun it to
reproduce them:  python oracle/search_dba.py

Cell (25 m, 20 elements): D Q1 D Q2 D B S1 Q3 S2 D D S2 Q3 S1 B D Q2 D Q1 D with
ExactSBend B (L 1.5 m, angle 2pi/40, edge angles angle/2, fringe on, gk 0),
quadrupoles of 0.5 m, sextupoles of 0.25 m and drifts of 2.25 m.  Quadrupole
k1 are drawn from +-U[0.5, 2.5] m^-2 and sextupole k2 from +-U[20, 60] m^-3
with a counter-based generator (numpy Philox, seed 0).  A draw is accepted when
  * the linear one-turn map of the cell (forward-mode tangent of the oracle) is
    stable in both planes with margin, |trace/2| <= 0.9;
  * the cell tunes nu = mu/2pi keep 0.04 away from the resonances every cell's
    sextupoles drive coherently: 3 nu_x, nu_x + 2 nu_y, nu_x - 2 nu_y, 2 nu_y
    and 4 nu_x, 4 nu_y not within 0.04 of an integer;
  * 256 particles of the workload's Gaussian beam survive 300 turns of the
    full 20-cell ring with its RF cavity (aperture 0.02 m).
"""
import ctypes as C
import importlib.util
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _abi():
    spec = importlib.util.spec_from_file_location("_tp_abi", os.path.join(ROOT, "trackpad.jl_b200", "_abi.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _oracle():
    return C.CDLL(os.path.join(HERE, "_build", "libtp_oracle.so"))


def cell(k):
    q1, q2, q3, s1, s2 = k
    ang = 2 * math.pi / 40
    D = dict(kind="DRIFT", L=2.25)
    Q = lambda kk: dict(kind="QUADRUPOLE", L=0.5, k=kk, max_order=1, num_int_steps=10)
    S = lambda kk: dict(kind="SEXTUPOLE", L=0.25, k=kk, max_order=2, num_int_steps=10)
    B = dict(kind="EXACT_SBEND", L=1.5, angle=ang, e1=ang / 2, e2=ang / 2, num_int_steps=10,
             fringe_bend_entrance=1, fringe_bend_exit=1, gk=0.0)
    return [D, Q(q1), D, Q(q2), D, B, S(s1), Q(q3), S(s2), D, D, S(s2), Q(q3), S(s1), B, D, Q(q2), D, Q(q1), D]


def jacobian(elems, beti, nturns=1):
    abi, O = _abi(), _oracle()
    arr = abi.elem_array(elems)
    orbit = np.zeros(6)
    jac = np.zeros(36)
    O.orc_jacobian(arr, C.c_int64(len(elems)), None, C.c_int64(0), None, 0, 0, 0, None,
                   orbit.ctypes.data_as(C.c_void_p), C.c_int64(1), C.c_double(beti), nturns, 0, 1,
                   jac.ctypes.data_as(C.c_void_p))
    return jac.reshape(6, 6).T  # column-major -> M[i, j]


def cell_tunes(M):
    nus = []
    for i in (0, 2):
        c = (M[i, i] + M[i + 1, i + 1]) / 2
        mu = math.acos(max(-1.0, min(1.0, c)))
        if M[i, i + 1] < 0:
            mu = 2 * math.pi - mu
        nus.append(mu / (2 * math.pi))
    return nus


def near_integer(v, tol=0.04):
    return abs(v - round(v)) < tol


def survives(q, s, beti, nturns=300, npart=256):
    abi, O = _abi(), _oracle()
    elems = cell(list(q) + list(s)) * 20
    elems.append(dict(kind="RFCAVITY", L=0.0, volt=3e6, freq=500 * 2.99792458e8 / 500.0, h=500.0, lag=0.0,
                      philag=0.0, energy=3e9))
    arr = abi.elem_array(elems)
    rng = np.random.Generator(np.random.Philox(0))
    sig = (1e-4, 1e-5, 1e-4, 1e-5, 1e-3, 1e-4)
    c = np.empty((npart, 6), order="F")
    for k in range(6):
        c[:, k] = rng.standard_normal(npart) * sig[k]
    lost = np.zeros(npart, np.int64)
    O.orc_ringpass(arr, C.c_int64(len(elems)), None, C.c_int64(0), None, 0, 0, 0, None,
                   c.ctypes.data_as(C.c_void_p), C.c_int64(npart), lost.ctypes.data_as(C.c_void_p), None, None,
                   None, C.c_double(beti), nturns, 0, 1, C.c_double(0.02), C.c_double(0.02), 0)
    return int(lost.sum()) == 0


def main():
    gamma = (3.0e9 + 0.51099895069e6) / 0.51099895069e6
    beti = 1.0 / math.sqrt(1.0 - 1.0 / (gamma * gamma))
    rng = np.random.Generator(np.random.Philox(0))
    for trial in range(200000):
        q = rng.uniform(0.5, 2.5, 3) * rng.choice([-1.0, 1.0], 3)
        s = rng.uniform(20.0, 60.0, 2) * np.array([1.0, -1.0])
        M = jacobian(cell(list(q) + list(s)), beti)
        tx, ty = (M[0, 0] + M[1, 1]) / 2, (M[2, 2] + M[3, 3]) / 2
        if not (abs(tx) <= 0.9 and abs(ty) <= 0.9):
            continue
        nx, ny = cell_tunes(M)
        if any(near_integer(v) for v in (3 * nx, nx + 2 * ny, nx - 2 * ny, 2 * ny, 4 * nx, 4 * ny)):
            continue
        if not survives(q, s, beti):
            continue
        print(f"trial {trial}: k1 = {q.tolist()}, k2 = {s.tolist()}, cos(mu) = ({tx:.4f}, {ty:.4f}), "
              f"cell tunes = ({nx:.4f}, {ny:.4f})")
        return q, s
    sys.exit("no cell found")


if __name__ == "__main__":
    main()
