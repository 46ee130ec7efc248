"""Truncated power series (TPSA) maps on the device.

The reference's PolySeries extension (ext/TrackPadPolySeriesExt.jl) tracks a
vector of six CTPS values through the lattice: polyseries_variables builds
the identity map about a point, linepass / ringpass carry it through the
elements, and polyseries_one_turn_map is the Taylor map of one turn to a
chosen order.  Here the maps are tracked on the GPU (tp_tpsa_ringpass), many
at once: each map is six series of M = C(order + 6, 6) coefficients, in the
monomial order of `monomials(order)` (by degree, then exponent vectors in
descending lexicographic order).
"""
import ctypes as C

import numpy as np

from . import _abi
from . import tracking


def coefficients(order):
    """M, the number of coefficients of a series of this order."""
    m = C.c_int64()
    _abi.check(_abi.lib().tp_tpsa_coefficients(int(order), C.byref(m)), "tp_tpsa_coefficients")
    return int(m.value)


def monomials(order):
    """(M, 6) exponents of the monomials in coefficient order."""
    e = np.zeros((coefficients(order), 6), np.int32)
    _abi.check(_abi.lib().tp_tpsa_monomials(int(order), e.ctypes.data_as(C.c_void_p)), "tp_tpsa_monomials")
    return e


class TpsaMap:
    """Six truncated power series (x, px, y, py, z, delta) of the six
    phase-space variables: coef[c, k] multiplies monomial k of `monomials`."""

    def __init__(self, coef, order):
        self.order = int(order)
        self.coef = np.ascontiguousarray(coef, dtype=np.float64).reshape(6, coefficients(order))

    @property
    def monomials(self):
        return monomials(self.order)

    def constant(self):
        """The map of the expansion point (the tracked orbit)."""
        return self.coef[:, 0].copy()

    def jacobian(self):
        """The first-order part: the 6x6 tangent map."""
        return self.coef[:, 1:7].copy()

    def __call__(self, dx):
        """Evaluate the truncated series at a deviation dx (6,) or (n, 6)."""
        d = np.atleast_2d(np.asarray(dx, dtype=np.float64))
        mono = self.monomials
        terms = np.prod(d[:, None, :] ** mono[None, :, :], axis=2)  # (n, M)
        out = terms @ self.coef.T
        return out[0] if np.ndim(dx) == 1 else out


def polyseries_variables(x0=None, order=1):
    """The identity map about x0 (CTPS(x0[i], i) for each variable)."""
    m = coefficients(order)
    c = np.zeros((6, m))
    x = np.zeros(6) if x0 is None else np.asarray(x0, dtype=np.float64).reshape(6)
    for i in range(6):
        c[i, 0] = x[i]
        c[i, 1 + i] = 1.0
    return TpsaMap(c, order)


def ringpass(lat, maps, beam, nturns, *, order=None, turn=0, time=0.0, dt_turn=0.0):
    """nturns passes of series maps (a TpsaMap, a list of them, or an array
    (nmaps, 6, M) with `order`); returns new maps of the same form."""
    if not isinstance(lat, tracking.Lattice):
        lat = tracking.Lattice(lat)
    single = isinstance(maps, TpsaMap)
    if single or (isinstance(maps, (list, tuple)) and maps and isinstance(maps[0], TpsaMap)):
        lst = [maps] if single else list(maps)
        order = lst[0].order
        arr = np.ascontiguousarray(np.stack([m.coef for m in lst]))
    else:
        if order is None:
            raise ValueError("order is required for a coefficient array")
        arr = np.array(maps, dtype=np.float64, order="C", copy=True)
    m = coefficients(order)
    if arr.ndim != 3 or arr.shape[1:] != (6, m):
        raise ValueError(f"maps must have shape (nmaps, 6, {m})")
    lat.set_schedule(time, dt_turn, turn, max(int(nturns), 1))
    st = _abi.lib().tp_tpsa_ringpass(tracking.context(), lat.handle, arr.ctypes.data_as(C.c_void_p), arr.shape[0],
                                     int(order), C.c_double(tracking.beti(beam)), int(nturns), int(turn))
    _abi.check(st, "tp_tpsa_ringpass")
    if single:
        return TpsaMap(arr[0], order)
    if isinstance(maps, (list, tuple)):
        return [TpsaMap(a, order) for a in arr]
    return arr


def linepass(lat, maps, beam, *, order=None, turn=0, time=0.0):
    """One pass (linepass of CTPS coordinates, ext/TrackPadPolySeriesExt.jl:654-663)."""
    return ringpass(lat, maps, beam, 1, order=order, turn=turn, time=time)


def polyseries_one_turn_map(lat, beam, r0=None, order=1):
    """Taylor map of one turn about r0 to `order` (:701-705)."""
    return linepass(lat, polyseries_variables(r0, order), beam)


def one_turn_maps(lat, beam, references, order=1):
    """Taylor maps about many reference orbits ((n, 6)) in one device call."""
    refs = np.atleast_2d(np.asarray(references, dtype=np.float64))
    return ringpass(lat, [polyseries_variables(r, order) for r in refs], beam, 1)


def last_stats():
    """Work and device time of the last ringpass on this thread."""
    st = _abi.TpTpsaStats()
    _abi.check(_abi.lib().tp_tpsa_last_stats(C.byref(st)), "tp_tpsa_last_stats")
    return {f: getattr(st, f) for f, _ in st._fields_}
