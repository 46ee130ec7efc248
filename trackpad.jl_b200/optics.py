"""Optics from device tangent maps: one-turn map, tunes, chromaticity, closed orbit.

The reference builds these from finite-difference maps, 12 single-particle
linepass calls per 6x6 map (one_turn_map, src/optics.jl:110-121; gettune
:278-283; getchrom :300-312; find_closed_orbit_6d/4d :335-389).  Here every
map is the exact tangent map of the tracked maps, computed on the GPU for any
number of reference orbits in one call (tp_one_turn_jacobian), so tunes at
many momenta, or every Newton step of a closed-orbit search, cost one launch
pair.  Names, arguments and error behaviour follow the reference.
"""
import math

import numpy as np

from . import tracking


def one_turn_map(lat, beam, reference=None, nturns=1, method="exact", h=1e-8):
    """6x6 one-turn map about `reference` (default zeros).

    method="exact": the exact tangent map of the tracked maps (device reverse
    sweep).  method="fd": the reference's own estimate (src/optics.jl:110-121),
    central differences (linepass(r + h e_i) - linepass(r - h e_i)) / 2h, with
    the 12 orbits tracked in one device call; since the tracking is
    bit-identical to the reference's maps, so is this matrix."""
    ref = np.zeros(6) if reference is None else np.asarray(reference, dtype=np.float64).reshape(6)
    if method == "fd":
        return _fd_map(lat, beam, ref, nturns, h)
    if method != "exact":
        raise ValueError("method must be 'exact' or 'fd'")
    M, _ = tracking.one_turn_jacobian(lat, beam, ref[None, :], nturns=nturns)
    if np.isnan(M[0]).any():
        raise ValueError("the reference orbit is lost within the turn")
    return M[0]


def fd_orbits(reference, h=1e-8):
    """The 12 orbits of the central-difference map: rows 2i, 2i+1 are
    reference + h e_i and reference - h e_i."""
    ref = np.asarray(reference, dtype=np.float64).reshape(6)
    out = np.empty((12, 6), dtype=np.float64, order="F")
    for i in range(6):
        e = np.zeros(6)
        e[i] = 1.0
        out[2 * i] = ref + h * e
        out[2 * i + 1] = ref - h * e
    return out


def fd_assemble(tracked, h=1e-8):
    """M[:, i] = (rp_i - rm_i) / (2h) from the tracked `fd_orbits`."""
    M = np.empty((6, 6))
    for i in range(6):
        M[:, i] = (tracked[2 * i] - tracked[2 * i + 1]) / (2.0 * h)
    return M


def _fd_map(lat, beam, ref, nturns, h):
    c = fd_orbits(ref, h)
    lost = np.zeros(12, np.int64)
    if nturns == 1:
        tracking.linepass_(c, lat, beam, lost)
    else:
        tracking.ringpass_(c, lat, beam, lost, nturns)
    if lost.any():
        raise ValueError("the reference orbit is lost within the turn")
    return fd_assemble(c, h)


def one_turn_maps(lat, beam, references, nturns=1):
    """Tangent maps about many reference orbits ((n, 6)) in one launch pair;
    returns (M of shape (n, 6, 6), symplecticity error per orbit)."""
    return tracking.one_turn_jacobian(lat, beam, np.atleast_2d(references), nturns=nturns)


def twiss_from_2x2(M):
    """(beta, alpha, mu, tune) of a 2x2 block (src/optics.jl:123-149):
    cos(mu) = trace/2, beta = M12/sin(mu), with mu -> 2pi - mu when beta <= 0."""
    tr = (M[0, 0] + M[1, 1]) / 2.0
    if abs(tr) >= 1.0:
        raise ValueError(f"unstable 2x2 map: |trace/2| = {abs(tr)} >= 1")
    mu = math.acos(min(1.0, max(-1.0, tr)))
    sinmu = math.sin(mu)
    if abs(sinmu) < math.sqrt(np.finfo(float).eps):
        raise ValueError(f"degenerate map: sin(mu) = {sinmu}")
    beta = M[0, 1] / sinmu
    alpha = (M[0, 0] - M[1, 1]) / (2.0 * sinmu)
    if beta <= 0.0:
        mu = 2.0 * math.pi - mu
        sinmu = math.sin(mu)
        beta = M[0, 1] / sinmu
        alpha = (M[0, 0] - M[1, 1]) / (2.0 * sinmu)
    return beta, alpha, mu, (mu / (2.0 * math.pi)) % 1.0


def tune_from_map(M):
    """(Qx, Qy) from the uncoupled 2x2 blocks of a 6x6 map."""
    return twiss_from_2x2(M[0:2, 0:2])[3], twiss_from_2x2(M[2:4, 2:4])[3]


def gettune(lat, beam, reference=None):
    """(Qx, Qy) of the one-turn map about `reference` (src/optics.jl:278-283)."""
    return tune_from_map(one_turn_map(lat, beam, reference))


def getchrom(lat, beam, dp=0.0, reference=None, dpp=1e-8):
    """Chromaticity (xi_x, xi_y): the change of the tunes with the momentum
    offset, (Q(dp + dpp) - Q(dp)) / dpp as in src/optics.jl:300-312; both maps
    come from one device call."""
    ref = np.zeros(6) if reference is None else np.asarray(reference, dtype=np.float64).reshape(6).copy()
    refs = np.array([ref, ref])
    refs[0, 5] = dp
    refs[1, 5] = dp + dpp
    M, _ = one_turn_maps(lat, beam, refs)
    (qx0, qy0), (qx1, qy1) = tune_from_map(M[0]), tune_from_map(M[1])
    return (qx1 - qx0) / dpp, (qy1 - qy0) / dpp


def _pass_once(lat, beam, r):
    c = np.array(r, dtype=np.float64, order="F", copy=True).reshape(1, 6)  # never the caller's array
    lost = np.zeros(1, np.int64)
    tracking.linepass_(c, lat, beam, lost)
    if lost[0]:
        raise ValueError("the orbit is lost within the turn")
    return c[0].copy()


def find_closed_orbit_6d(lat, beam, x0=None, tol=1e-10, maxiter=20, reg=1e-12):
    """6-D closed orbit by Newton iteration, x <- x + (I - J + reg I)^-1 (f(x) - x),
    with J the exact tangent map (src/optics.jl:335-357 uses finite differences)."""
    x = np.zeros(6) if x0 is None else np.asarray(x0, dtype=np.float64).reshape(6).copy()
    eye = np.eye(6)
    for _ in range(maxiter):
        fx = _pass_once(lat, beam, x)
        d = fx - x
        if np.linalg.norm(d) < tol:
            return x
        J = one_turn_map(lat, beam, x)
        x = x + np.linalg.solve(eye - J + reg * eye, d)
    return x


def find_closed_orbit_4d(lat, beam, dp=0.0, x0=None, tol=1e-10, maxiter=20, reg=1e-12):
    """4-D closed orbit (x, px, y, py) at fixed momentum offset `dp`
    (src/optics.jl:364-389), z = 0 at the start of each trial."""
    x = np.zeros(4) if x0 is None else np.asarray(x0, dtype=np.float64).reshape(4).copy()
    eye = np.eye(4)
    for _ in range(maxiter):
        r = np.array([x[0], x[1], x[2], x[3], 0.0, dp])
        fx = _pass_once(lat, beam, r)[:4]
        d = fx - x
        if np.linalg.norm(d) < tol:
            return x
        J = one_turn_map(lat, beam, r)[:4, :4]
        x = x + np.linalg.solve(eye - J + reg * eye, d)
    return x
