"""Beam, Lattice, time-varying fields and the drop-in tracking calls.

Mirrors TrackPad.jl's multi-particle interface:
  linepass!(coords, lat, beam, lost_flags; time, turn)   -> linepass_(...)
  ringpass!(coords, lat, beam, lost_flags, nturns; ...)  -> ringpass_(...)
(src/lattice.jl:260-317).  `coords` is an N x 6 float64 array in the
reference's layout (column-major: each of x, px, y, py, z, delta is a
contiguous column) and is updated in place; `lost_flags` is int64 with 1 =
lost.  All computation runs on the GPU through libtrackpad_b200.so; there is no
CPU path.
"""
import ctypes as C
import math
import threading

import numpy as np

from . import _abi
from .elements import M_ELECTRON, AbstractElement

# ---------------------------------------------------------------------------
# Beam (src/lattice.jl:33-61)
# ---------------------------------------------------------------------------


class Beam:
    """Beam(energy; mass=M_ELECTRON, charge=-1.0).  `energy` is kinetic: gamma = (E + m)/m."""

    def __init__(self, energy, *, mass=M_ELECTRON, charge=-1.0):
        self.energy, self.mass, self.charge = float(energy), float(mass), float(charge)
        self.gamma = (self.energy + self.mass) / self.mass
        self.beta = math.sqrt(1.0 - 1.0 / (self.gamma * self.gamma))


def beti(beam):
    """1/beta (src/lattice.jl:61)."""
    return 1.0 / beam.beta


# ---------------------------------------------------------------------------
# Time dependence (src/time_dependence.jl)
# ---------------------------------------------------------------------------


class TimeContext:
    """Evaluation context of time-dependent parameters (time_dependence.jl:10-15)."""

    def __init__(self, real_time, turn=0):
        self.real_time, self.turn = float(real_time), int(turn)


class TimeDependentParam:
    """A parameter given as a function of a TimeContext (time_dependence.jl:32-38)."""

    def __init__(self, f):
        self.f = f if callable(f) else (lambda _ctx, _v=f: _v)

    def __call__(self, ctx):
        if not isinstance(ctx, TimeContext):
            ctx = TimeContext(ctx, 0)
        return self.f(ctx)

    def _op(self, other, fn):
        o = other if isinstance(other, TimeDependentParam) else TimeDependentParam(other)
        return TimeDependentParam(lambda ctx: fn(self(ctx), o(ctx)))

    def __add__(self, o): return self._op(o, lambda a, b: a + b)
    def __radd__(self, o): return self._op(o, lambda a, b: b + a)
    def __sub__(self, o): return self._op(o, lambda a, b: a - b)
    def __rsub__(self, o): return self._op(o, lambda a, b: b - a)
    def __mul__(self, o): return self._op(o, lambda a, b: a * b)
    def __rmul__(self, o): return self._op(o, lambda a, b: b * a)
    def __truediv__(self, o): return self._op(o, lambda a, b: a / b)
    def __rtruediv__(self, o): return self._op(o, lambda a, b: b / a)
    def __neg__(self): return TimeDependentParam(lambda ctx: -self(ctx))


def Time():
    """The physical-time parameter (time_dependence.jl:40)."""
    return TimeDependentParam(lambda ctx: ctx.real_time)


def Turn():
    """The turn-index parameter (time_dependence.jl:46)."""
    return TimeDependentParam(lambda ctx: ctx.turn)


_FIELD_ALIASES = {"k1": "k", "k2": "k", "k3": "k"}


class TimeVaryingElement(AbstractElement):
    """An element whose fields vary with (time, turn): timed(elem; field=f)."""

    def __init__(self, base, updates):
        self.base = base
        self.updates = updates

    def materialize(self, ctx):
        import copy
        e = copy.copy(self.base)
        for k, v in self.updates.items():
            setattr(e, k, type(getattr(self.base, k))(v(ctx)))
        return e

    def get_length(self):
        return self.base.get_length()


def timed(elem, **fields):
    """timed(elem; field=f) (time_dependence.jl:147-155): unknown fields raise."""
    ups = {}
    for k, v in fields.items():
        if not hasattr(elem, k):
            raise ValueError(f"{type(elem).__name__} has no field `{k}`")
        if _schedule_field(elem, k) is None:
            raise ValueError(f"field `{k}` of {type(elem).__name__} cannot vary on the device")
        ups[k] = v if isinstance(v, TimeDependentParam) else TimeDependentParam(v)
    return TimeVaryingElement(elem, ups)


def materialize(elem, t):
    """materialize(elem, t) (time_dependence.jl:163-175)."""
    ctx = t if isinstance(t, TimeContext) else TimeContext(t, 0)
    return elem.materialize(ctx) if isinstance(elem, TimeVaryingElement) else elem


def _schedule_field(elem, name):
    if name in ("k1", "k2", "k3"):
        return _abi.FIELDS["k"]
    if name in ("ks", "xkick", "ykick"):
        return None
    return _abi.FIELDS.get(name)


# ---------------------------------------------------------------------------
# Native handles
# ---------------------------------------------------------------------------
_ctx_lock = threading.Lock()
_contexts = {}


def context(device=None):
    """The library context of a CUDA device (created on first use)."""
    if device is None:
        device = 0
        try:
            import torch
            if torch.cuda.is_available():
                device = torch.cuda.current_device()
        except ImportError:  # pragma: no cover
            pass
    with _ctx_lock:
        if device not in _contexts:
            h = C.c_void_p()
            _abi.check(_abi.lib().tp_ctx_create(int(device), C.byref(h)), "tp_ctx_create")
            _contexts[device] = h
        return _contexts[device]


def last_stats(device=None):
    st = _abi.TpStats()
    _abi.check(_abi.lib().tp_last_stats(context(device), C.byref(st)), "tp_last_stats")
    return {f: getattr(st, f) for f, _ in st._fields_}


class Lattice:
    """Lattice(elements) (src/lattice.jl:87-99).  Owns the compiled native table."""

    def __init__(self, elements, *, name="LATTICE"):
        self.elements = list(elements)
        self.name = name
        self._handle = None
        self._sched_key = None

    @classmethod
    def from_records(cls, records, name="LATTICE", misalign=None):
        """A lattice from raw C-ABI records (dicts with tp_elem field names, or
        TpElem).  `misalign` lists the misalignment rows (dicts of t1, t2: 6
        values; r1, r2: 36 values, column-major) that the records'
        misalign_index select."""
        lat = cls([], name=name)
        lat._records = list(records)
        lat._mis_rows = list(misalign or [])
        return lat

    def __len__(self):
        return len(self._records) if getattr(self, "_records", None) is not None else len(self.elements)

    def __getitem__(self, i):
        return self.elements[i]

    def __iter__(self):
        return iter(self.elements)

    def total_length(self, time=0.0, turn=0):
        ctx = TimeContext(time, turn)
        return sum(float(materialize(e, ctx).get_length()) for e in self.elements)

    def has_time_dependence(self):
        return any(isinstance(e, TimeVaryingElement) for e in self.elements)

    def _static_elements(self):
        return [e.base if isinstance(e, TimeVaryingElement) else e for e in self.elements]

    def pack(self):
        """(tp_elem array, n, misalignment array, nmis, aux float64 array)."""
        if getattr(self, "_records", None) is not None:
            arr, aux = _abi.elem_array_aux(self._records)
            rows = getattr(self, "_mis_rows", [])
            marr = (_abi.TpMisalign * max(len(rows), 1))()
            for k, row in enumerate(rows):
                for f, n in (("t1", 6), ("t2", 6), ("r1", 36), ("r2", 36)):
                    vals = [float(v) for v in row[f]]
                    if len(vals) != n:
                        raise ValueError(f"misalignment row {k}: {f} needs {n} values")
                    getattr(marr[k], f)[:] = vals
            return arr, len(self._records), marr, len(rows), np.asarray(aux, dtype=np.float64)
        elems = self._static_elements()
        arr = (_abi.TpElem * max(len(elems), 1))()
        mis = []
        aux = []
        for i, e in enumerate(elems):
            arr[i] = e.pack(aux)
            if e.has_misalignment():
                arr[i].misalign_index = len(mis)
                mis.append(e.misalignment())
        marr = (_abi.TpMisalign * max(len(mis), 1))(*mis)
        return arr, len(elems), marr, len(mis), np.asarray(aux, dtype=np.float64)

    @property
    def handle(self):
        if self._handle is None:
            arr, n, marr, nm, aux = self.pack()
            h = C.c_void_p()
            _abi.check(_abi.lib().tp_lattice_create_ex(arr, n, marr if nm else None, nm,
                                                       aux.ctypes.data_as(C.c_void_p) if len(aux) else None,
                                                       len(aux), C.byref(h)), "tp_lattice_create_ex")
            self._handle = h
        return self._handle

    def set_schedule(self, time, dt_turn, turn0, nturns):
        """Evaluate every time-varying field at each turn (the materialize step of
        linepass!, src/lattice.jl:267) and hand the table to the library."""
        if not self.has_time_dependence():
            return
        key = (float(time), float(dt_turn), int(turn0), int(nturns))
        if key == self._sched_key:
            return
        fields = []
        for i, e in enumerate(self.elements):
            if isinstance(e, TimeVaryingElement):
                for name in e.updates:
                    fields.append((i, name, _schedule_field(e.base, name)))
        vals = np.empty((nturns, len(fields)), dtype=np.float64)
        for t in range(nturns):
            ctx = TimeContext(time + t * dt_turn, turn0 + t)
            for j, (i, name, _f) in enumerate(fields):
                vals[t, j] = float(self.elements[i].updates[name](ctx))
        f = np.array([[i, fid] for i, _n, fid in fields], dtype=np.int32).reshape(-1)
        _abi.check(_abi.lib().tp_lattice_set_schedule(self.handle, f.ctypes.data_as(C.c_void_p), len(fields),
                                                      int(turn0), int(nturns),
                                                      vals.ctypes.data_as(C.c_void_p)), "tp_lattice_set_schedule")
        self._sched_key = key

    def flops_per_element(self):
        out = np.zeros(max(len(self), 1), dtype=np.float64)  # noqa: E501
        _abi.check(_abi.lib().tp_lattice_flops(self.handle, out.ctypes.data_as(C.c_void_p)), "tp_lattice_flops")
        return out[:len(self)]

    def __del__(self):
        if self._handle is not None and _abi._lib is not None:
            try:
                _abi.lib().tp_lattice_destroy(self._handle)
            except Exception:  # pragma: no cover
                pass


def spos(lat, time=0.0, turn=0):
    """s-position of each element boundary (src/lattice.jl:331-338)."""
    ctx = TimeContext(time, turn)
    s = [0.0]
    for e in lat.elements:
        s.append(s[-1] + float(materialize(e, ctx).get_length()))
    return s


# ---------------------------------------------------------------------------
# Tracking calls
# ---------------------------------------------------------------------------
# Stage element tables into shared memory (tp_opts.table_in_smem); off by
# default, where the tables are read through the L1 cache.
TABLE_IN_SMEM = False


def _opts(aperture, exact, contract, device, block_size=0, schedule=0, stream=None, device_index=None,
          min_blocks=0, bounds_check=False):
    """tp_opts of a call.  With device arrays and no stream given, the call runs
    on PyTorch's current stream of that device, so the kernels follow the work
    that wrote the inputs there; PyTorch's default stream has handle 0, which
    selects the context stream, a blocking stream ordered with it."""
    if device and stream is None:
        import torch
        stream = torch.cuda.current_stream(device_index).cuda_stream or None
    o = _abi.TpOpts()
    o.table_in_smem = 1 if TABLE_IN_SMEM else 0
    o.size = C.sizeof(_abi.TpOpts)
    o.exact_hamiltonian = 1 if exact else 0
    o.device_pointers = 1 if device else 0
    o.fp_contract = 1 if contract else 0
    o.block_size = int(block_size)
    o.schedule = int(schedule)
    o.min_blocks = int(min_blocks)
    o.bounds_check = 1 if bounds_check else 0
    if aperture is not None:
        ax, ay = (aperture, aperture) if np.isscalar(aperture) else aperture
        o.aperture_x, o.aperture_y = float(ax), float(ay)
    o.stream = stream
    return o


class _Buffers:
    """Resolve coords/lost_flags into pointers; host arrays in the reference's
    column-major layout are used in place, others through a copy-back."""

    def __init__(self, coords, lost_flags, lost_turn, lost_elem):
        self.device = False
        self._copyback = []
        try:
            import torch
            is_t = isinstance(coords, torch.Tensor)
        except ImportError:  # pragma: no cover
            is_t = False
        if is_t:
            self._init_torch(coords, lost_flags, lost_turn, lost_elem)
        else:
            self._init_numpy(coords, lost_flags, lost_turn, lost_elem)

    def _init_numpy(self, coords, lost_flags, lost_turn, lost_elem):
        coords_a = coords
        if not isinstance(coords, np.ndarray) or coords.dtype != np.float64:
            raise TypeError("coords must be a float64 numpy array (N x 6)")
        if coords.ndim != 2 or coords.shape[1] != 6:
            raise ValueError("coords must have shape (N, 6)")
        if not coords.flags.f_contiguous:
            coords_a = np.asfortranarray(coords)
            self._copyback.append((coords, coords_a))
        if not isinstance(lost_flags, np.ndarray) or lost_flags.dtype != np.int64 or lost_flags.shape != (coords.shape[0],):
            raise TypeError("lost_flags must be an int64 numpy vector of length N")
        lf = lost_flags if lost_flags.flags.c_contiguous else np.ascontiguousarray(lost_flags)
        if lf is not lost_flags:
            self._copyback.append((lost_flags, lf))
        self.n = coords.shape[0]
        self.keep = [coords_a, lf]
        self.coords = coords_a.ctypes.data_as(C.c_void_p)
        self.lost = lf.ctypes.data_as(C.c_void_p)
        self.lost_turn = self._i32(lost_turn)
        self.lost_elem = self._i32(lost_elem)

    def _i32(self, a):
        if a is None:
            return None
        if not isinstance(a, np.ndarray) or a.dtype != np.int32 or a.shape != (self.n,) or not a.flags.c_contiguous:
            raise TypeError("lost_turn / lost_elem must be contiguous int32 vectors of length N")
        self.keep.append(a)
        return a.ctypes.data_as(C.c_void_p)

    def _init_torch(self, coords, lost_flags, lost_turn, lost_elem):
        import torch
        if not coords.is_cuda:
            raise TypeError("torch tensors must be on a CUDA device (use numpy arrays for host memory)")
        if coords.dtype != torch.float64:
            raise TypeError("coords must be float64")
        if coords.dim() != 2 or coords.shape[1] != 6 or coords.stride() != (1, coords.shape[0]):
            raise ValueError("device coords must be an (N, 6) column-major view, e.g. torch.empty(6, N).T")
        if lost_flags.dtype != torch.int64 or lost_flags.shape != (coords.shape[0],) or not lost_flags.is_contiguous():
            raise TypeError("lost_flags must be a contiguous int64 CUDA vector of length N")
        self.device = True
        self.n = coords.shape[0]
        self.keep = [coords, lost_flags]
        self.coords = C.c_void_p(coords.data_ptr())
        self.lost = C.c_void_p(lost_flags.data_ptr())
        self.lost_turn = None if lost_turn is None else C.c_void_p(lost_turn.data_ptr())
        self.lost_elem = None if lost_elem is None else C.c_void_p(lost_elem.data_ptr())
        self.device_index = coords.device.index

    def finish(self):
        for orig, tmp in self._copyback:
            orig[...] = tmp


def ringpass_(coords, lat, beam, lost_flags, nturns, *, time=0.0, dt_turn=0.0, turn=0, aperture=None,
              lost_turn=None, lost_elem=None, exact=True, contract=False, block_size=0, schedule=0, stream=None,
              min_blocks=0, bounds_check=False):
    """ringpass!(coords, lat, beam, lost_flags, nturns; time, dt_turn, turn) on the GPU.

    Extra keywords: `aperture` (half width, or (ax, ay)) adds the rectangular
    aperture check beside check_lost; `lost_turn`/`lost_elem` (int32, length N)
    receive the turn and 0-based element of each loss; `exact=False` selects the
    linearised drift (USE_EXACT_HAMILTONIAN = false); `contract=True` runs the
    kernel built with FMA contraction (faster; its rounding differs from the
    reference's operation order); `schedule` (1 static, 2 lane refill) and
    `min_blocks` (kernel instance sized for 8, 7, 6 or 5 resident blocks per SM)
    fix what the autotuner otherwise picks (0); `bounds_check=True` runs the
    kernels that check every element-table record and particle index before
    reading it (a violation raises with TP_EDEVICE).
    """
    if not isinstance(lat, Lattice):
        lat = Lattice(lat)
    nturns = int(nturns)
    if nturns < 0:
        raise ValueError("nturns must be >= 0")
    b = _Buffers(coords, lost_flags, lost_turn, lost_elem)
    lat.set_schedule(time, dt_turn, turn, max(nturns, 1))
    dev = b.device_index if b.device else None
    o = _opts(aperture, exact, contract, b.device, block_size, schedule, stream, device_index=dev,
              min_blocks=min_blocks, bounds_check=bounds_check)
    st = _abi.lib().tp_ringpass(context(dev), lat.handle, b.coords, b.n, b.lost, b.lost_turn, b.lost_elem,
                                C.c_double(beti(beam)), nturns, C.c_double(time), C.c_double(dt_turn), int(turn),
                                C.byref(o))
    _abi.check(st, "tp_ringpass")
    b.finish()
    return None


def linepass_(coords, lat, beam, lost_flags, *, time=0.0, turn=0, **kw):
    """linepass!(coords, lat, beam, lost_flags; time, turn) on the GPU."""
    if not isinstance(lat, Lattice):
        lat = Lattice(lat)
    b = _Buffers(coords, lost_flags, kw.pop("lost_turn", None), kw.pop("lost_elem", None))
    lat.set_schedule(time, 0.0, turn, 1)
    dev = b.device_index if b.device else None
    o = _opts(kw.get("aperture"), kw.get("exact", True), kw.get("contract", False), b.device, kw.get("block_size", 0),
              kw.get("schedule", 0), kw.get("stream"), device_index=dev)
    st = _abi.lib().tp_linepass(context(dev), lat.handle, b.coords, b.n, b.lost, b.lost_turn, b.lost_elem,
                                C.c_double(beti(beam)), C.c_double(time), int(turn), C.byref(o))
    _abi.check(st, "tp_linepass")
    b.finish()
    return None


class Batch:
    """Many lattice variants tracked in one launch (tp_batch)."""

    def __init__(self, lattices, device=None):
        self.lattices = [l if isinstance(l, Lattice) else Lattice(l) for l in lattices]
        self.device = device
        hs = (C.c_void_p * len(self.lattices))(*[l.handle for l in self.lattices])
        h = C.c_void_p()
        _abi.check(_abi.lib().tp_batch_create(context(device), hs, len(self.lattices), C.byref(h)), "tp_batch_create")
        self._handle = h

    def ringpass_(self, coords, poff, betis, lost_flags, nturns, *, time=0.0, dt_turn=0.0, turn=0, aperture=None,
                  lost_turn=None, lost_elem=None, exact=True, contract=False, use_graph=True, block_size=0,
                  schedule=0, stream=None, min_blocks=0, bounds_check=False):
        """ringpass! of every variant in one launch; variant v owns particles
        poff[v]..poff[v+1].  Time-dependent variants are evaluated per turn."""
        b = _Buffers(coords, lost_flags, lost_turn, lost_elem)
        for lat in self.lattices:
            lat.set_schedule(time, dt_turn, turn, max(int(nturns), 1))
        poff = np.ascontiguousarray(poff, dtype=np.int64)
        betis = np.ascontiguousarray(betis, dtype=np.float64)
        if poff.shape != (len(self.lattices) + 1,) or betis.shape != (len(self.lattices),):
            raise ValueError("poff must have nvar+1 entries and betis nvar entries")
        if poff[-1] != b.n:
            raise ValueError("poff[-1] must equal the number of particles")
        o = _opts(aperture, exact, contract, b.device, block_size, schedule, stream,
                  device_index=b.device_index if b.device else None, min_blocks=min_blocks,
                  bounds_check=bounds_check)
        st = _abi.lib().tp_ringpass_batched(context(self.device), self._handle, b.coords,
                                            poff.ctypes.data_as(C.c_void_p), b.lost, b.lost_turn, b.lost_elem,
                                            betis.ctypes.data_as(C.c_void_p), int(nturns), C.c_double(0.0),
                                            C.c_double(0.0), int(turn), 1 if use_graph else 0, C.byref(o))
        _abi.check(st, "tp_ringpass_batched")
        b.finish()

    def ringpass_adjoint(self, coords0, poff, betis, lost0, nturns, params, *, sigma, lost_weight=1e3, time=0.0,
                         dt_turn=0.0, turn=0, aperture=None, exact=True, checkpoint_every=0, stream=None):
        """Per-variant loss and gradient in one launch (see ringpass_adjoint).

        params[v] lists the parameter elements of variant v.  Returns
        (loss[nvar], [grad_v for each variant]).
        """
        cp, lp, n, dev, keep = _adj_inputs(coords0, lost0)
        poff = np.ascontiguousarray(poff, dtype=np.int64)
        betis = np.ascontiguousarray(betis, dtype=np.float64)
        nv = len(self.lattices)
        if poff.shape != (nv + 1,) or betis.shape != (nv,) or poff[-1] != n:
            raise ValueError("poff must have nvar+1 entries ending at N and betis nvar entries")
        if len(params) != nv:
            raise ValueError("params needs one list per variant")
        for lat in self.lattices:
            lat.set_schedule(time, dt_turn, turn, max(int(nturns), 1))
        flat = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.int32).reshape(-1) for p in params])
                                    if nv else np.zeros(0, np.int32), dtype=np.int32)
        pof = np.zeros(nv + 1, dtype=np.int32)
        pof[1:] = np.cumsum([len(p) for p in params])
        loss = np.zeros(nv)
        grad = np.zeros(max(len(flat), 1))
        o = _opts(aperture, exact, False, dev is not None, stream=stream, device_index=dev)
        ls = _loss_spec(sigma, lost_weight)
        st = _abi.lib().tp_ringpass_adjoint_batched(
            context(self.device), self._handle, cp, poff.ctypes.data_as(C.c_void_p), lp,
            betis.ctypes.data_as(C.c_void_p), int(nturns), C.c_double(0.0), C.c_double(0.0), int(turn),
            flat.ctypes.data_as(C.c_void_p), pof.ctypes.data_as(C.c_void_p), C.byref(ls), int(checkpoint_every),
            loss.ctypes.data_as(C.c_void_p), grad.ctypes.data_as(C.c_void_p), C.byref(o))
        _abi.check(st, "tp_ringpass_adjoint_batched")
        return loss, [grad[pof[v]:pof[v + 1]].copy() for v in range(nv)]

    def __del__(self):
        if getattr(self, "_handle", None) is not None and _abi._lib is not None:
            try:
                _abi.lib().tp_batch_destroy(self._handle)
            except Exception:  # pragma: no cover
                pass


# ---------------------------------------------------------------------------
# Derivatives: adjoint gradient of a beam loss, one-turn Jacobian
# ---------------------------------------------------------------------------
def _adj_inputs(coords0, lost0):
    """(coords pointer, lost pointer, n, device index or None, keep-alive list)."""
    try:
        import torch
        is_t = isinstance(coords0, torch.Tensor)
    except ImportError:  # pragma: no cover
        is_t = False
    if is_t:
        if not coords0.is_cuda or coords0.dtype != torch.float64 or coords0.dim() != 2 or coords0.shape[1] != 6 \
                or coords0.stride() != (1, coords0.shape[0]):
            raise ValueError("device coords0 must be an (N, 6) float64 column-major CUDA view")
        n = coords0.shape[0]
        if lost0 is not None and (lost0.dtype != torch.int64 or lost0.shape != (n,) or not lost0.is_contiguous()):
            raise TypeError("lost0 must be a contiguous int64 CUDA vector of length N")
        return (C.c_void_p(coords0.data_ptr()), None if lost0 is None else C.c_void_p(lost0.data_ptr()), n,
                coords0.device.index, [coords0, lost0])
    c = np.asfortranarray(coords0, dtype=np.float64)
    if c.ndim != 2 or c.shape[1] != 6:
        raise ValueError("coords0 must have shape (N, 6)")
    n = c.shape[0]
    keep = [c]
    lp = None
    if lost0 is not None:
        l = np.ascontiguousarray(lost0, dtype=np.int64)
        if l.shape != (n,):
            raise ValueError("lost0 must have length N")
        keep.append(l)
        lp = l.ctypes.data_as(C.c_void_p)
    return c.ctypes.data_as(C.c_void_p), lp, n, None, keep


def _loss_spec(sigma, lost_weight):
    ls = _abi.TpLossSpec()
    ls.kind = 0
    ls.sigma = float(sigma)
    ls.lost_weight = float(lost_weight)
    return ls


def ringpass_adjoint(coords0, lat, beam, lost0, nturns, params, *, sigma, lost_weight=1e3, time=0.0, dt_turn=0.0,
                     turn=0, aperture=None, exact=True, checkpoint_every=0, return_state=False, stream=None):
    """Loss of a tracked beam and its gradient with respect to element strengths.

    loss = mean over the particles that survive `nturns` of (x^2 + y^2)/sigma^2
           + lost_weight * (lost / alive at start)
    `params` lists element indices (0-based) of Quadrupoles, Sextupoles or
    Octupoles; grad[j] = d loss / d k of params[j] (k1, k2 or k3), with the
    survivor set held fixed.  A time-dependent strength is shifted by the same
    amount at every turn.  coords0/lost0 are read only (numpy host arrays or
    CUDA tensors).  Returns (loss, grad), plus (coords, lost_flags) after the
    forward pass when `return_state` is set.
    """
    if not isinstance(lat, Lattice):
        lat = Lattice(lat)
    cp, lp, n, dev, keep = _adj_inputs(coords0, lost0)
    lat.set_schedule(time, dt_turn, turn, max(int(nturns), 1))
    prm = np.ascontiguousarray(params, dtype=np.int32).reshape(-1)
    grad = np.zeros(max(len(prm), 1))
    loss = C.c_double()
    out_c = out_l = None
    ocp = olp = None
    if return_state:
        if dev is None:
            out_c = np.zeros((n, 6), order="F")
            out_l = np.zeros(n, dtype=np.int64)
            ocp, olp = out_c.ctypes.data_as(C.c_void_p), out_l.ctypes.data_as(C.c_void_p)
        else:
            import torch
            out_c = torch.empty((6, n), dtype=torch.float64, device=f"cuda:{dev}").T
            out_l = torch.empty(n, dtype=torch.int64, device=f"cuda:{dev}")
            ocp, olp = C.c_void_p(out_c.data_ptr()), C.c_void_p(out_l.data_ptr())
    o = _opts(aperture, exact, False, dev is not None, stream=stream, device_index=dev)
    ls = _loss_spec(sigma, lost_weight)
    st = _abi.lib().tp_ringpass_adjoint(context(dev), lat.handle, cp, n, lp, C.c_double(beti(beam)), int(nturns),
                                        C.c_double(time), C.c_double(dt_turn), int(turn),
                                        prm.ctypes.data_as(C.c_void_p), len(prm), C.byref(ls), int(checkpoint_every),
                                        C.byref(loss), grad.ctypes.data_as(C.c_void_p), ocp, olp, C.byref(o))
    _abi.check(st, "tp_ringpass_adjoint")
    if return_state:
        return loss.value, grad[:len(prm)], out_c, out_l
    return loss.value, grad[:len(prm)]


def one_turn_jacobian(lat, beam, orbits, *, nturns=1, turn=0, time=0.0, dt_turn=0.0, exact=True):
    """Tangent maps of `nturns` passes about each orbit and their symplecticity.

    The exact counterpart of one_turn_map (src/optics.jl:110-121, finite
    differences there).  orbits: (n, 6).  Returns (M, err) with M of shape
    (n, 6, 6) and err[i] = ||M^T J M - J||_max, J = diag(J2, J2, -J2).  An
    orbit lost on the way gives NaN.
    """
    if not isinstance(lat, Lattice):
        lat = Lattice(lat)
    orb = np.asfortranarray(np.atleast_2d(orbits), dtype=np.float64)
    n = orb.shape[0]
    lat.set_schedule(time, dt_turn, turn, max(int(nturns), 1))
    jac = np.zeros((n, 36))
    err = np.zeros(n)
    o = _opts(None, exact, False, False)
    st = _abi.lib().tp_one_turn_jacobian(context(), lat.handle, orb.ctypes.data_as(C.c_void_p), n,
                                         C.c_double(beti(beam)), int(nturns), int(turn),
                                         jac.ctypes.data_as(C.c_void_p), err.ctypes.data_as(C.c_void_p), C.byref(o))
    _abi.check(st, "tp_one_turn_jacobian")
    return np.transpose(jac.reshape(n, 6, 6), (0, 2, 1)), err


def adjoint_stats():
    """Statistics of the last adjoint or Jacobian call on this thread."""
    st = _abi.TpAdjointStats()
    _abi.check(_abi.lib().tp_last_adjoint_stats(C.byref(st)), "tp_last_adjoint_stats")
    return {f: getattr(st, f) for f, _ in st._fields_}


def probe_fp64_peak(device=None):
    """Measured FP64 FMA throughput of the device in TFLOP/s."""
    v = C.c_double()
    _abi.check(_abi.lib().tp_probe_fp64_peak(context(device), C.byref(v)), "tp_probe_fp64_peak")
    return v.value
