"""ctypes mirror of include/trackpad_b200.h and loader of the native library.

The library is built in-tree (``libtrackpad_b200.so`` next to this file).  There
is no CPU fallback: if the library is missing, every tracking call raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtrackpad_b200.so")

# enum tp_status
TP_OK = 0
TP_EINVAL = -1
TP_ENOMEM = -2
TP_EUNSUPPORTED = -3
TP_ECUDA = -4
TP_ETIMEOUT = -5
TP_EDEVICE = -6
TP_ENODEV = -7
TP_ERANGE = -8

# enum tp_kind
KINDS = [
    "MARKER", "DRIFT", "QUADRUPOLE", "SEXTUPOLE", "OCTUPOLE", "THIN_MULTIPOLE", "SBEND", "EXACT_SBEND",
    "RFCAVITY", "SOLENOID", "CORRECTOR", "TRANSLATION", "YROTATION", "CRAB_CAVITY", "ACCEL_CAVITY",
    "LONGITUDINAL_RF_MAP", "LORENTZ_BOOST", "INV_LORENTZ_BOOST", "SPACE_CHARGE", "DRIFT_SC", "QUADRUPOLE_SC",
    "SEXTUPOLE_SC", "OCTUPOLE_SC", "SBEND_SC", "STRONG_THIN_GAUSSIAN_BEAM", "LBEND", "WIGGLER",
    "STRONG_GAUSSIAN_BEAM", "LONGITUDINAL_RLC_WAKE", "LONGITUDINAL_WAKE",
]
KIND = {name: i for i, name in enumerate(KINDS)}

# enum tp_field
FIELDS = {
    "L": 0, "k": 1, "k1": 1, "k2": 1, "k3": 1, "angle": 2, "e1": 3, "e2": 4, "volt": 5, "freq": 6, "lag": 7,
    "philag": 8, "energy": 9, "num_int_steps": 10,
}
FIELD_POLYNOM_A0 = 11
FIELD_POLYNOM_B0 = 15

TP_LOSS_BEAM_SIZE = 0
FLOPS_PER_TRANSCENDENTAL = 20


class TpElem(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("max_order", C.c_int32), ("num_int_steps", C.c_int32),
        ("fringe_bend_entrance", C.c_int32), ("fringe_bend_exit", C.c_int32), ("misalign_index", C.c_int32),
        ("iparam", C.c_int32 * 2),
        ("L", C.c_double), ("k", C.c_double), ("angle", C.c_double), ("e1", C.c_double), ("e2", C.c_double),
        ("fint1", C.c_double), ("fint2", C.c_double), ("gap", C.c_double), ("gk", C.c_double),
        ("polynom_a", C.c_double * 4), ("polynom_b", C.c_double * 4), ("kick_angle", C.c_double * 2),
        ("volt", C.c_double), ("freq", C.c_double), ("h", C.c_double), ("lag", C.c_double),
        ("philag", C.c_double), ("energy", C.c_double), ("param", C.c_double * 8),
    ]


class TpMisalign(C.Structure):
    _fields_ = [("t1", C.c_double * 6), ("t2", C.c_double * 6), ("r1", C.c_double * 36), ("r2", C.c_double * 36)]


class TpOpts(C.Structure):
    _fields_ = [
        ("size", C.c_int32), ("exact_hamiltonian", C.c_int32), ("device_pointers", C.c_int32),
        ("fp_contract", C.c_int32), ("block_size", C.c_int32), ("min_blocks", C.c_int32), ("schedule", C.c_int32),
        ("table_in_smem", C.c_int32), ("aperture_x", C.c_double), ("aperture_y", C.c_double), ("stream", C.c_void_p),
        ("bounds_check", C.c_int32), ("reserved0", C.c_int32),
    ]


class TpStats(C.Structure):
    _fields_ = [
        ("particles", C.c_int64), ("survivors", C.c_int64), ("element_passes", C.c_int64), ("units", C.c_double),
        ("flops", C.c_double), ("kernel_ms", C.c_double), ("total_ms", C.c_double), ("h2d_bytes", C.c_int64),
        ("d2h_bytes", C.c_int64), ("block_size", C.c_int32), ("min_blocks", C.c_int32), ("grid", C.c_int32),
        ("launches", C.c_int32), ("schedule", C.c_int32), ("fp_contract", C.c_int32), ("refill_fold", C.c_int32),
        ("bounds_check", C.c_int32),
    ]


class TpLossSpec(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("sigma", C.c_double), ("lost_weight", C.c_double)]


class TpAdjointStats(C.Structure):
    _fields_ = [
        ("checkpoint_every", C.c_int32), ("segments", C.c_int32), ("checkpoint_bytes", C.c_int64),
        ("particles", C.c_int64), ("units", C.c_double), ("forward_ms", C.c_double), ("reverse_ms", C.c_double),
        ("reconstruction_error", C.c_double), ("launches", C.c_int32), ("k_tuning", C.c_int32),
        ("tuned_ms", C.c_double),
    ]


def elem_from_dict(d, aux=None):
    """Fill a TpElem from a dict with reference field names (kind given by name).
    An "aux" entry (list of floats: the element's array fields) is appended to
    `aux` and referenced by iparam[0] (offset) and iparam[1] (length)."""
    e = TpElem()
    e.kind = KIND[d["kind"]] if isinstance(d["kind"], str) else int(d["kind"])
    e.misalign_index = -1
    for key, val in d.items():
        if key == "kind":
            continue
        if key == "aux":
            if aux is None:
                raise ValueError("this element has array fields: pack it with elem_array_aux")
            e.iparam[0] = len(aux)
            e.iparam[1] = len(val)
            aux.extend(float(v) for v in val)
            continue
        if key in ("polynom_a", "polynom_b", "kick_angle", "param", "iparam"):
            arr = getattr(e, key)
            for i, v in enumerate(val):
                arr[i] = v
        else:
            setattr(e, key, val)
    return e


def elem_array(dicts):
    return elem_array_aux(dicts)[0]


def elem_array_aux(dicts):
    """(TpElem array, aux list) of a list of element dicts."""
    arr = (TpElem * max(len(dicts), 1))()
    aux = []
    for i, d in enumerate(dicts):
        arr[i] = d if isinstance(d, TpElem) else elem_from_dict(d, aux)
    return arr, aux


P = C.c_void_p
class TpTpsaStats(C.Structure):
    _fields_ = [("maps", C.c_int64), ("order", C.c_int32), ("coefficients", C.c_int32), ("pairs", C.c_int64),
                ("series_mul", C.c_double), ("series_lin", C.c_double), ("flops", C.c_double),
                ("kernel_ms", C.c_double), ("grid", C.c_int32), ("block", C.c_int32), ("shared_pool", C.c_int32),
                ("slots", C.c_int32), ("slots_used", C.c_int32), ("reserved", C.c_int32)]


_SIGS = {
    "tp_abi_version": (C.c_int, []),
    "tp_strerror": (C.c_char_p, [C.c_int]),
    "tp_last_error_string": (C.c_char_p, []),
    "tp_device_count": (C.c_int, []),
    "tp_ctx_create": (C.c_int, [C.c_int, C.POINTER(P)]),
    "tp_ctx_destroy": (C.c_int, [P]),
    "tp_last_stats": (C.c_int, [P, C.POINTER(TpStats)]),
    "tp_beam_beti": (C.c_int, [C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "tp_lattice_create": (C.c_int, [P, C.c_int64, P, C.c_int64, C.POINTER(P)]),
    "tp_lattice_create_ex": (C.c_int, [P, C.c_int64, P, C.c_int64, P, C.c_int64, C.POINTER(P)]),
    "tp_lattice_destroy": (C.c_int, [P]),
    "tp_lattice_length": (C.c_int, [P, C.POINTER(C.c_int64)]),
    "tp_lattice_flops": (C.c_int, [P, P]),
    "tp_lattice_set_schedule": (C.c_int, [P, P, C.c_int32, C.c_int32, C.c_int32, P]),
    "tp_linepass": (C.c_int, [P, P, P, C.c_int64, P, P, P, C.c_double, C.c_double, C.c_int32, P]),
    "tp_ringpass": (C.c_int, [P, P, P, C.c_int64, P, P, P, C.c_double, C.c_int32, C.c_double, C.c_double,
                              C.c_int32, P]),
    "tp_batch_create": (C.c_int, [P, P, C.c_int32, C.POINTER(P)]),
    "tp_batch_destroy": (C.c_int, [P]),
    "tp_ringpass_batched": (C.c_int, [P, P, P, P, P, P, P, P, C.c_int32, C.c_double, C.c_double, C.c_int32,
                                      C.c_int32, P]),
    "tp_ringpass_adjoint": (C.c_int, [P, P, P, C.c_int64, P, C.c_double, C.c_int32, C.c_double, C.c_double,
                                      C.c_int32, P, C.c_int32, P, C.c_int32, P, P, P, P, P]),
    "tp_ringpass_adjoint_batched": (C.c_int, [P, P, P, P, P, P, C.c_int32, C.c_double, C.c_double, C.c_int32,
                                              P, P, P, C.c_int32, P, P, P]),
    "tp_one_turn_jacobian": (C.c_int, [P, P, P, C.c_int64, C.c_double, C.c_int32, C.c_int32, P, P, P]),
    "tp_last_adjoint_stats": (C.c_int, [C.POINTER(TpAdjointStats)]),
    "tp_probe_fp64_peak": (C.c_int, [P, C.POINTER(C.c_double)]),
    "tp_ringpass_noalloc": (C.c_int, [P, P, C.c_int64, P, P, P, C.c_double, C.c_int32, C.c_int32, C.c_double,
                                      C.c_double, P]),
    "tp_tpsa_coefficients": (C.c_int, [C.c_int32, C.POINTER(C.c_int64)]),
    "tp_tpsa_monomials": (C.c_int, [C.c_int32, P]),
    "tp_tpsa_ringpass": (C.c_int, [P, P, P, C.c_int64, C.c_int32, C.c_double, C.c_int32, C.c_int32]),
    "tp_tpsa_last_stats": (C.c_int, [C.POINTER(TpTpsaStats)]),
}

_lib = None


def lib():
    """Load the native library once; raise loudly if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"native library {LIB_PATH} is missing; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` (there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class TrackPadError(RuntimeError):
    """Raised for a non-zero tp_status; `.status` holds the code."""

    def __init__(self, status, where):
        L = lib()
        msg = L.tp_strerror(status).decode()
        extra = L.tp_last_error_string().decode()
        super().__init__(f"{where}: {msg}" + (f" ({extra})" if extra else ""))
        self.status = status


def check(status, where):
    if status != TP_OK:
        if status == TP_EINVAL:
            raise ValueError(f"{where}: invalid argument ({lib().tp_last_error_string().decode()})")
        raise TrackPadError(status, where)
    return status
