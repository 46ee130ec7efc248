"""ctypes wrapper of the CPU oracle (oracle/_build/libtp_oracle.so) for the tests.

Test infrastructure: the checker the GPU results are compared with.
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_build", "libtp_oracle.so")
_lib = None

P = C.c_void_p


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            import subprocess
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
        _lib = C.CDLL(LIB)
        _lib.orc_beam_beti.restype = C.c_double
        _lib.orc_beam_beti.argtypes = [C.c_double, C.c_double]
        _lib.orc_ringpass.argtypes = [P, C.c_int64, P, C.c_int64, P, C.c_int32, C.c_int32, C.c_int32, P, P, C.c_int64,
                                      P, P, P, P, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                      C.c_int32]
        _lib.orc_count_flops.argtypes = [P, C.c_int64, P, C.c_int64, C.c_double, C.c_int32, P, P, P]
        _lib.orc_jacobian.argtypes = [P, C.c_int64, P, C.c_int64, P, C.c_int32, C.c_int32, C.c_int32, P, P,
                                      C.c_int64, C.c_double, C.c_int32, C.c_int32, C.c_int32, P]
        _lib.orc_loss_and_dk.argtypes = [P, C.c_int64, P, C.c_int64, P, C.c_int32, C.c_int32, C.c_int32, P, P,
                                         C.c_int64, P, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                         C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32, P, P, P]
        _lib.orc_pass_elements.argtypes = [P, C.c_int64, P, C.c_int64, P, C.c_int64, C.c_double, C.c_int32]
        _lib.orc_submap.argtypes = [C.c_int32, P, C.c_double, C.c_double, C.c_double]
        _lib.orc_max_threads.restype = C.c_int
        _lib.orc_set_aux.argtypes = [P, C.c_int64]
        _lib.orc_tpsa_set_order.argtypes = [C.c_int32]
        _lib.orc_tpsa_monomials.argtypes = [P]
        _lib.orc_tpsa_op.argtypes = [C.c_int32, P, P, P]
        _lib.orc_tpsa_ringpass.argtypes = [P, C.c_int64, P, C.c_int64, P, C.c_int32, C.c_int32, C.c_int32, P, P,
                                           C.c_int64, C.c_double, C.c_int32, C.c_int32]
        _lib.orc_tpsa_error.restype = C.c_char_p
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(P)


def _packed(lat):
    """(elems, n, mis, nmis) from a Lattice or a list of element dicts; the
    elements' array fields are handed to the oracle (orc_set_aux) for the call
    that follows."""
    if hasattr(lat, "pack"):
        arr, n, marr, nm, aux = lat.pack()
    else:
        import importlib
        abi = importlib.import_module("trackpad_b200._abi")
        arr, aux = abi.elem_array_aux(lat)
        n, marr, nm = len(lat), None, 0
    aux = np.ascontiguousarray(aux, dtype=np.float64)
    lib().orc_set_aux(aux.ctypes.data_as(P) if len(aux) else None, len(aux))  # the oracle copies it
    return arr, n, (marr if nm else None), nm


def _schedule(sched):
    if sched is None:
        return None, 0, 0, 0, None
    fields, turn0, values = sched
    f = np.ascontiguousarray(fields, dtype=np.int32).reshape(-1)
    v = np.ascontiguousarray(values, dtype=np.float64)
    return f, len(f) // 2, int(turn0), v.shape[0], v


def ringpass(lat, coords, lost, beti, nturns, turn0=0, aperture=(0.0, 0.0), lost_turn=None, lost_elem=None,
             min_edge=None, exact=True, nthreads=0, sched=None):
    """ringpass! of the oracle, in place on a Fortran-ordered (N, 6) array."""
    assert coords.flags.f_contiguous and coords.dtype == np.float64
    arr, n, mis, nm = _packed(lat)
    f, nf, st0, snt, sv = _schedule(sched)
    if np.isscalar(aperture):
        aperture = (aperture, aperture)
    rc = lib().orc_ringpass(arr, n, mis, nm, _ptr(f), nf, st0, snt, _ptr(sv), _ptr(coords), coords.shape[0],
                            _ptr(lost), _ptr(lost_turn), _ptr(lost_elem), _ptr(min_edge), beti, int(nturns),
                            int(turn0), 1 if exact else 0, float(aperture[0]), float(aperture[1]), int(nthreads))
    assert rc == 0


def count_flops(lat, beti, r0=(1e-4, 2e-4, 3e-4, -1e-4, 5e-5, 2e-4), exact=True):
    arr, n, mis, nm = _packed(lat)
    out = np.zeros(max(n, 1))
    tr = np.zeros(max(n, 1))
    r = np.array(r0, dtype=np.float64)
    lib().orc_count_flops(arr, n, mis, nm, beti, 1 if exact else 0, _ptr(r), _ptr(out), _ptr(tr))
    return out[:n], tr[:n]


def jacobian(lat, orbits, beti, nturns=1, turn0=0, exact=True, sched=None):
    """(n, 6, 6) tangent maps about each orbit (orbits: (n, 6))."""
    arr, n, mis, nm = _packed(lat)
    f, nf, st0, snt, sv = _schedule(sched)
    orb = np.asfortranarray(np.atleast_2d(orbits), dtype=np.float64)
    m = orb.shape[0]
    jac = np.zeros((m, 36))
    lib().orc_jacobian(arr, n, mis, nm, _ptr(f), nf, st0, snt, _ptr(sv), _ptr(orb), m, beti, int(nturns), int(turn0),
                       1 if exact else 0, _ptr(jac))
    return np.transpose(jac.reshape(m, 6, 6), (0, 2, 1))


def loss_and_dk(lat, coords0, lost0, beti, nturns, param_elem, sigma, lost_weight, aperture=(0.0, 0.0), turn0=0,
                exact=True, nthreads=0, sched=None):
    arr, n, mis, nm = _packed(lat)
    f, nf, st0, snt, sv = _schedule(sched)
    c0 = np.asfortranarray(coords0, dtype=np.float64)
    l0 = np.ascontiguousarray(lost0, dtype=np.int64)
    loss, dloss, surv = C.c_double(), C.c_double(), C.c_int64()
    lib().orc_loss_and_dk(arr, n, mis, nm, _ptr(f), nf, st0, snt, _ptr(sv), _ptr(c0), c0.shape[0], _ptr(l0), beti,
                          int(nturns), int(turn0), 1 if exact else 0, float(aperture[0]), float(aperture[1]),
                          float(sigma), float(lost_weight), int(param_elem), int(nthreads), C.byref(loss),
                          C.byref(dloss), C.byref(surv))
    return loss.value, dloss.value, surv.value


def pass_elements(elems, coords, beti, exact=True):
    arr, n, mis, nm = _packed(elems)
    lib().orc_pass_elements(arr, n, mis, nm, _ptr(coords), coords.shape[0], beti, 1 if exact else 0)


def submap(which, r, a0, a1, beti):
    v = np.array(r, dtype=np.float64)
    assert lib().orc_submap(int(which), _ptr(v), float(a0), float(a1), float(beti)) == 0
    return v


SYMPLECTIC_J = np.zeros((6, 6))
for _i, _s in enumerate((1.0, 1.0, -1.0)):
    SYMPLECTIC_J[2 * _i, 2 * _i + 1] = _s
    SYMPLECTIC_J[2 * _i + 1, 2 * _i] = -_s


def symplectic_error(M):
    """||M^T J M - J||_max with J = diag(J2, J2, -J2): in the reference's
    coordinates z is conjugate to delta with the sign of -c*dt."""
    return float(np.abs(M.T @ SYMPLECTIC_J @ M - SYMPLECTIC_J).max())


# ---------------------------------------------------------------------------
# TPSA (truncated power series) oracle
# ---------------------------------------------------------------------------
TPSA_OPS = {"mul": 0, "div": 1, "inv": 2, "sqrt": 3, "rsqrt": 4, "exp": 5, "sin": 6, "cos": 7}


def tpsa_set_order(order):
    """Set the series order; returns M, the number of coefficients."""
    m = lib().orc_tpsa_set_order(int(order))
    assert m > 0
    return m


def tpsa_monomials(order):
    m = tpsa_set_order(order)
    e = np.zeros((m, 6), np.int32)
    lib().orc_tpsa_monomials(_ptr(e))
    return e


def tpsa_op(op, a, b=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    out = np.zeros_like(a)
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.float64)
    assert lib().orc_tpsa_op(TPSA_OPS[op], _ptr(a), _ptr(bb), _ptr(out)) == 0
    return out


def tpsa_variables(x0, order):
    """(6, M) coefficients of the six variables about x0 (CTPS(x0[i], i))."""
    m = tpsa_set_order(order)
    r = np.zeros((6, m))
    for i in range(6):
        r[i, 0] = x0[i]
        r[i, 1 + i] = 1.0
    return r


def tpsa_ringpass(lat, maps, beti, order, nturns=1, turn0=0, sched=None):
    """Series maps (nmaps, 6, M) through nturns passes, in place; returns the status."""
    tpsa_set_order(order)
    arr, n, mis, nm = _packed(lat)
    f, nf, st0, snt, sv = _schedule(sched)
    assert maps.flags.c_contiguous and maps.dtype == np.float64
    st = lib().orc_tpsa_ringpass(arr, n, mis, nm, _ptr(f), nf, st0, snt, _ptr(sv), _ptr(maps),
                                 maps.shape[0], beti, int(nturns), int(turn0))
    if st == -3:
        raise RuntimeError(lib().orc_tpsa_error().decode())
    return st
