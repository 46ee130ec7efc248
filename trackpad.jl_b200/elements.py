"""Element types with TrackPad.jl's field names and constructor defaults.

Each class mirrors one reference struct (src/elements/*.jl) and packs itself
into the C-ABI record `tp_elem` (include/trackpad_b200.h).  Constructors take
the same positional and keyword arguments as the Julia constructors.
"""
import math

from . import _abi

C_LIGHT = 2.99792458e8          # src/elements/rf.jl:28
M_ELECTRON = 0.51099895069e6    # src/lattice.jl:42
M_PROTON = 938.27208816e6       # src/lattice.jl:43
TWO_PI = 2.0 * math.pi


def _vec(v, n, name):
    if v is None:
        return [0.0] * n
    v = [float(x) for x in v]
    if len(v) != n:
        raise ValueError(f"{name} must have {n} entries")
    return v


def _mat(m, name):
    """6x6 matrix (nested rows or flat column-major 36) -> column-major list."""
    if m is None:
        return [0.0] * 36
    try:
        import numpy as np
        a = np.asarray(m, dtype=float)
        if a.shape == (6, 6):
            return [float(x) for x in a.flatten(order="F")]
        if a.shape == (36,):
            return [float(x) for x in a]
    except ImportError:  # pragma: no cover
        pass
    raise ValueError(f"{name} must be a 6x6 matrix")


class AbstractElement:
    """Base of every element (src/elements/core.jl:1)."""

    kind = None
    _misalignable = False

    def _misalign_init(self, t1, t2, r1, r2):
        self.t1 = _vec(t1, 6, "t1")
        self.t2 = _vec(t2, 6, "t2")
        self.r1 = _mat(r1, "r1")
        self.r2 = _mat(r2, "r2")

    def has_misalignment(self):
        return self._misalignable and any(v != 0.0 for v in self.t1 + self.t2 + self.r1 + self.r2)

    def _fields(self):
        """Dict of tp_elem fields (reference names)."""
        raise NotImplementedError

    def pack(self, aux=None):
        """The tp_elem record; array fields are appended to `aux`."""
        d = self._fields()
        d["kind"] = self.kind
        return _abi.elem_from_dict(d, aux)

    def misalignment(self):
        m = _abi.TpMisalign()
        for i in range(6):
            m.t1[i] = self.t1[i]
            m.t2[i] = self.t2[i]
        for i in range(36):
            m.r1[i] = self.r1[i]
            m.r2[i] = self.r2[i]
        return m

    def get_length(self):
        return getattr(self, "L", 0.0)

    def __repr__(self):
        return f"{type(self).__name__}({getattr(self, 'name', '')})"


class Marker(AbstractElement):
    kind = "MARKER"

    def __init__(self, *, name="MARKER"):
        self.name = name

    def _fields(self):
        return {}


class Drift(AbstractElement):
    """src/elements/drift.jl:21-34"""
    kind = "DRIFT"
    _misalignable = True

    def __init__(self, L, *, name="DRIFT", t1=None, t2=None, r1=None, r2=None, r_apertures=None, e_apertures=None):
        self.name, self.L = name, float(L)
        self._misalign_init(t1, t2, r1, r2)
        self.r_apertures = _vec(r_apertures, 6, "r_apertures")
        self.e_apertures = _vec(e_apertures, 6, "e_apertures")

    def _fields(self):
        return {"L": self.L}


class _Multipole(AbstractElement):
    _misalignable = True
    _strength = None
    _default_order = 1

    def __init__(self, L, k, *, name=None, polynom_a=None, polynom_b=None, max_order=None, num_int_steps=10, rad=0,
                 fringe_entrance=0, fringe_exit=0, t1=None, t2=None, r1=None, r2=None, r_apertures=None,
                 e_apertures=None, kick_angle=None):
        self.name = name or self.kind
        self.L = float(L)
        setattr(self, self._strength, float(k))
        self.polynom_a = _vec(polynom_a, 4, "polynom_a")
        self.polynom_b = _vec(polynom_b, 4, "polynom_b")
        self.max_order = self._default_order if max_order is None else int(max_order)
        self.num_int_steps = int(num_int_steps)
        self.rad, self.fringe_entrance, self.fringe_exit = int(rad), int(fringe_entrance), int(fringe_exit)
        self._misalign_init(t1, t2, r1, r2)
        self.r_apertures = _vec(r_apertures, 6, "r_apertures")
        self.e_apertures = _vec(e_apertures, 6, "e_apertures")
        self.kick_angle = _vec(kick_angle, 2, "kick_angle")

    @property
    def k(self):
        return getattr(self, self._strength)

    def _fields(self):
        return {"L": self.L, "k": self.k, "polynom_a": self.polynom_a, "polynom_b": self.polynom_b,
                "max_order": self.max_order, "num_int_steps": self.num_int_steps, "kick_angle": self.kick_angle}


class Quadrupole(_Multipole):
    """src/elements/quad.jl:26-47 (max_order 1, num_int_steps 10)."""
    kind, _strength, _default_order = "QUADRUPOLE", "k1", 1


class Sextupole(_Multipole):
    """src/elements/multipole.jl:26-47 (max_order 2)."""
    kind, _strength, _default_order = "SEXTUPOLE", "k2", 2


class Octupole(_Multipole):
    """src/elements/multipole.jl:72-93 (max_order 3)."""
    kind, _strength, _default_order = "OCTUPOLE", "k3", 3


class ThinMultipole(AbstractElement):
    """src/elements/multipole.jl:118-139"""
    kind = "THIN_MULTIPOLE"
    _misalignable = True

    def __init__(self, L, polynom_a, polynom_b, *, name="MULTIPOLE", max_order=1, num_int_steps=1, rad=0,
                 fringe_entrance=0, fringe_exit=0, t1=None, t2=None, r1=None, r2=None, r_apertures=None,
                 e_apertures=None, kick_angle=None):
        self.name, self.L = name, float(L)
        self.polynom_a = _vec(polynom_a, 4, "polynom_a")
        self.polynom_b = _vec(polynom_b, 4, "polynom_b")
        self.max_order, self.num_int_steps = int(max_order), int(num_int_steps)
        self._misalign_init(t1, t2, r1, r2)
        self.kick_angle = _vec(kick_angle, 2, "kick_angle")

    def _fields(self):
        return {"L": self.L, "polynom_a": self.polynom_a, "polynom_b": self.polynom_b, "max_order": self.max_order,
                "num_int_steps": self.num_int_steps}


class SBend(AbstractElement):
    """src/elements/bend.jl:33-64 (max_order 0, num_int_steps 10, Brown edges on)."""
    kind = "SBEND"
    _misalignable = True

    def __init__(self, L, angle, e1=0.0, e2=0.0, *, name="SBEND", polynom_a=None, polynom_b=None, max_order=0,
                 num_int_steps=10, rad=0, fint1=0.0, fint2=0.0, gap=0.0, fringe_bend_entrance=1, fringe_bend_exit=1,
                 fringe_quad_entrance=0, fringe_quad_exit=0, fringe_int_m0=None, fringe_int_p0=None, t1=None,
                 t2=None, r1=None, r2=None, r_apertures=None, e_apertures=None, kick_angle=None):
        self.name = name
        self.L, self.angle, self.e1, self.e2 = float(L), float(angle), float(e1), float(e2)
        self.polynom_a = _vec(polynom_a, 4, "polynom_a")
        self.polynom_b = _vec(polynom_b, 4, "polynom_b")
        self.max_order, self.num_int_steps, self.rad = int(max_order), int(num_int_steps), int(rad)
        self.fint1, self.fint2, self.gap = float(fint1), float(fint2), float(gap)
        self.fringe_bend_entrance, self.fringe_bend_exit = int(fringe_bend_entrance), int(fringe_bend_exit)
        self.fringe_quad_entrance, self.fringe_quad_exit = int(fringe_quad_entrance), int(fringe_quad_exit)
        self._misalign_init(t1, t2, r1, r2)
        self.kick_angle = _vec(kick_angle, 2, "kick_angle")

    def _fields(self):
        return {"L": self.L, "angle": self.angle, "e1": self.e1, "e2": self.e2, "polynom_a": self.polynom_a,
                "polynom_b": self.polynom_b, "max_order": self.max_order, "num_int_steps": self.num_int_steps,
                "fint1": self.fint1, "fint2": self.fint2, "gap": self.gap,
                "fringe_bend_entrance": self.fringe_bend_entrance, "fringe_bend_exit": self.fringe_bend_exit,
                "kick_angle": self.kick_angle}


def RBend(L, angle, **kw):
    """src/elements/bend.jl:81: e1 = e2 = angle/2."""
    return SBend(L, angle, angle / 2, angle / 2, **kw)


class ExactSBend(SBend):
    """src/elements/bend.jl:118-149 (adds gk)."""
    kind = "EXACT_SBEND"

    def __init__(self, L, angle, e1=0.0, e2=0.0, *, name="ESBEND", gk=0.0, **kw):
        super().__init__(L, angle, e1, e2, name=name, **kw)
        self.gk = float(gk)

    def _fields(self):
        d = super()._fields()
        d["gk"] = self.gk
        return d


def ERBend(L, angle, **kw):
    """src/elements/SCelements.jl:339: e1 = e2 = angle/2."""
    return ExactSBend(L, angle, angle / 2, angle / 2, **kw)


class RFCavity(AbstractElement):
    """src/elements/rf.jl:16-21 (energy defaults to 0: no kick)."""
    kind = "RFCAVITY"

    def __init__(self, L, volt, freq, lag=0.0, *, name="RFCA", h=1.0, philag=0.0, energy=0.0):
        self.name = name
        self.L, self.volt, self.freq, self.lag = float(L), float(volt), float(freq), float(lag)
        self.h, self.philag, self.energy = float(h), float(philag), float(energy)

    def _fields(self):
        return {"L": self.L, "volt": self.volt, "freq": self.freq, "h": self.h, "lag": self.lag,
                "philag": self.philag, "energy": self.energy}


class Solenoid(AbstractElement):
    kind = "SOLENOID"
    _misalignable = True

    def __init__(self, L, ks, *, name="SOLENOID", t1=None, t2=None, r1=None, r2=None):
        self.name, self.L, self.ks = name, float(L), float(ks)
        self._misalign_init(t1, t2, r1, r2)

    def _fields(self):
        return {"L": self.L, "param": [self.ks] + [0.0] * 7}


class Corrector(AbstractElement):
    kind = "CORRECTOR"
    _misalignable = True

    def __init__(self, L, hk, vk, *, name="CORRECTOR", t1=None, t2=None, r1=None, r2=None):
        self.name, self.L, self.xkick, self.ykick = name, float(L), float(hk), float(vk)
        self._misalign_init(t1, t2, r1, r2)

    def _fields(self):
        return {"L": self.L, "param": [self.xkick, self.ykick] + [0.0] * 6}


def HKicker(*, name="HKICKER", L=0.0, xkick=0.0):
    """src/elements/corrector.jl:34-36"""
    return Corrector(L, xkick, 0.0, name=name)


def VKicker(*, name="VKICKER", L=0.0, ykick=0.0):
    """src/elements/corrector.jl:43-45"""
    return Corrector(L, 0.0, ykick, name=name)


class Translation(AbstractElement):
    kind = "TRANSLATION"

    def __init__(self, L, *, name="TRANSLATION", dx=0.0, dy=0.0, ds=0.0):
        self.name, self.L, self.dx, self.dy, self.ds = name, float(L), float(dx), float(dy), float(ds)

    def _fields(self):
        return {"L": self.L, "param": [self.dx, self.dy, self.ds] + [0.0] * 5}


class YRotation(AbstractElement):
    kind = "YROTATION"

    def __init__(self, L, *, name="YROTATION", angle=0.0):
        self.name, self.L, self.angle = name, float(L), float(angle)

    def _fields(self):
        return {"L": self.L, "angle": self.angle}


class CrabCavity(AbstractElement):
    """src/elements/rf.jl:46-54: k = 2pi*freq/c."""
    kind = "CRAB_CAVITY"

    def __init__(self, L, *, name="CRABCAVITY", volt=0.0, freq=0.0, phi=0.0, errors=None, energy=1.0e9):
        self.name, self.L, self.volt, self.freq = name, float(L), float(volt), float(freq)
        self.k = TWO_PI * self.freq / C_LIGHT
        self.phi, self.errors, self.energy = float(phi), _vec(errors, 2, "errors"), float(energy)

    def _fields(self):
        return {"L": self.L, "volt": self.volt, "freq": self.freq, "energy": self.energy,
                "param": [self.k, self.phi, self.errors[0], self.errors[1]] + [0.0] * 4}


class AccelCavity(AbstractElement):
    """src/elements/rf.jl:80-88: k = 2pi*freq/c."""
    kind = "ACCEL_CAVITY"

    def __init__(self, L, *, name="ACCELCAVITY", volt=0.0, freq=0.0, h=1.0, phis=0.0, energy=1.0e9):
        self.name, self.L, self.volt, self.freq = name, float(L), float(volt), float(freq)
        self.k = TWO_PI * self.freq / C_LIGHT
        self.h, self.phis, self.energy = float(h), float(phis), float(energy)

    def _fields(self):
        return {"L": self.L, "volt": self.volt, "freq": self.freq, "h": self.h, "energy": self.energy,
                "param": [self.k, self.phis] + [0.0] * 6}


class LongitudinalRFMap(AbstractElement):
    """src/elements/rf.jl:97-100; k and h of the linked element via _rf_k/_rf_h (tracking.jl:1565-1573)."""
    kind = "LONGITUDINAL_RF_MAP"

    def __init__(self, alphac, rf):
        self.alphac, self.rf = float(alphac), rf

    def _fields(self):
        rf = self.rf
        if isinstance(rf, RFCavity):
            k, h = TWO_PI * rf.freq / C_LIGHT, rf.h
        elif isinstance(rf, AccelCavity):
            k, h = rf.k, rf.h
        elif isinstance(rf, CrabCavity):
            k, h = rf.k, 1.0
        else:
            k, h = 0.0, 1.0
        return {"param": [self.alphac, k, h] + [0.0] * 5}

    def get_length(self):
        return 0.0


class LorentzBoost(AbstractElement):
    """src/elements/beambeam.jl:14-19"""
    kind = "LORENTZ_BOOST"

    def __init__(self, angle, *, name="LORENTZBOOST", mode=0):
        self.name, self.angle, self.mode = name, float(angle), int(mode)
        self.cosang, self.tanang = math.cos(self.angle), math.tan(self.angle)

    def _fields(self):
        return {"param": [self.angle, self.cosang, 0.0, self.tanang] + [0.0] * 4, "iparam": [self.mode, 0]}

    def get_length(self):
        return 0.0


class InvLorentzBoost(AbstractElement):
    """src/elements/beambeam.jl:38-43"""
    kind = "INV_LORENTZ_BOOST"

    def __init__(self, angle, *, name="INVLORENTZBOOST", mode=0):
        self.name, self.angle, self.mode = name, float(angle), int(mode)
        self.sinang, self.cosang = math.sin(self.angle), math.cos(self.angle)

    def _fields(self):
        return {"param": [self.angle, self.cosang, self.sinang, 0.0] + [0.0] * 4, "iparam": [self.mode, 0]}

    def get_length(self):
        return 0.0


class SpaceCharge(AbstractElement):
    kind = "SPACE_CHARGE"

    def __init__(self, L, *, name="SPACECHARGE", effective_len=0.0, Nl=10, Nm=10, a=1.0, b=1.0):
        self.name, self.L = name, float(L)
        self.effective_len, self.Nl, self.Nm, self.a, self.b = float(effective_len), int(Nl), int(Nm), float(a), float(b)

    def _fields(self):
        return {"L": self.L}


class DriftSC(Drift):
    kind = "DRIFT_SC"

    def __init__(self, L, *, name="DRIFT_SC", a=1.0, b=1.0, Nl=10, Nm=10, Nsteps=1, **kw):
        super().__init__(L, name=name, **kw)
        self.a, self.b, self.Nl, self.Nm, self.Nsteps = float(a), float(b), int(Nl), int(Nm), int(Nsteps)


class _MultipoleSC(AbstractElement):
    _misalignable = True
    _default_order = 1

    def __init__(self, L, *, name=None, k0=0.0, k1=0.0, k2=0.0, k3=0.0, polynom_a=None, max_order=None,
                 num_int_steps=10, rad=0, fringe_entrance=0, fringe_exit=0, t1=None, t2=None, r1=None, r2=None,
                 r_apertures=None, e_apertures=None, kick_angle=None, a=1.0, b=1.0, Nl=10, Nm=10, Nsteps=1):
        self.name = name or self.kind
        self.L, self.k0, self.k1, self.k2, self.k3 = float(L), float(k0), float(k1), float(k2), float(k3)
        self.polynom_a = _vec(polynom_a, 4, "polynom_a")
        self.max_order = self._default_order if max_order is None else int(max_order)
        self.num_int_steps = int(num_int_steps)
        self._misalign_init(t1, t2, r1, r2)
        self.kick_angle = _vec(kick_angle, 2, "kick_angle")
        self.a, self.b, self.Nl, self.Nm, self.Nsteps = float(a), float(b), int(Nl), int(Nm), int(Nsteps)

    def _fields(self):
        return {"L": self.L, "polynom_a": self.polynom_a, "max_order": self.max_order,
                "num_int_steps": self.num_int_steps, "kick_angle": self.kick_angle,
                "param": [self.k0, self.k1, self.k2, self.k3] + [0.0] * 4}


class QuadrupoleSC(_MultipoleSC):
    kind, _default_order = "QUADRUPOLE_SC", 1


class SextupoleSC(_MultipoleSC):
    kind, _default_order = "SEXTUPOLE_SC", 2


class OctupoleSC(_MultipoleSC):
    kind, _default_order = "OCTUPOLE_SC", 3


class SBendSC(SBend):
    kind = "SBEND_SC"

    def __init__(self, L, angle, e1=0.0, e2=0.0, *, name="SBEND_SC", a=1.0, b=1.0, Nl=10, Nm=10, Nsteps=1, **kw):
        super().__init__(L, angle, e1, e2, name=name, **kw)
        self.a, self.b, self.Nl, self.Nm, self.Nsteps = float(a), float(b), int(Nl), int(Nm), int(Nsteps)


def RBendSC(L, angle, **kw):
    """src/elements/SCelements.jl:332"""
    return SBendSC(L, angle, angle / 2, angle / 2, **kw)


class StrongThinGaussianBeam(AbstractElement):
    kind = "STRONG_THIN_GAUSSIAN_BEAM"

    def __init__(self, amplitude, rmssizex, rmssizey, *, name="STRONGTHINGAUSSIANBEAM", zloc=0.0, xoffset=0.0,
                 yoffset=0.0):
        self.name = name
        self.amplitude, self.rmssizex, self.rmssizey = float(amplitude), float(rmssizex), float(rmssizey)
        self.zloc, self.xoffset, self.yoffset = float(zloc), float(xoffset), float(yoffset)

    def _fields(self):
        return {"param": [self.amplitude, self.rmssizex, self.rmssizey, self.xoffset, self.yoffset, 0.0, 0.0, 0.0]}

    def get_length(self):
        return 0.0


class LBend(AbstractElement):
    """src/elements/SCelements.jl:346-383 (linear combined-function bend, method-1 edges)."""
    kind = "LBEND"
    _misalignable = True

    def __init__(self, L, angle, e1=0.0, e2=0.0, *, name="LBEND", K=0.0, by_error=0.0, fint1=0.0, fint2=0.0,
                 full_gap=0.0, t1=None, t2=None, r1=None, r2=None, r_apertures=None, e_apertures=None):
        self.name = name
        self.L, self.angle, self.e1, self.e2 = float(L), float(angle), float(e1), float(e2)
        self.K, self.by_error = float(K), float(by_error)
        self.fint1, self.fint2, self.full_gap = float(fint1), float(fint2), float(full_gap)
        self._misalign_init(t1, t2, r1, r2)

    def _fields(self):
        return {"L": self.L, "angle": self.angle, "e1": self.e1, "e2": self.e2, "fint1": self.fint1,
                "fint2": self.fint2, "gap": self.full_gap, "param": [self.K, self.by_error] + [0.0] * 6}


class StrongGaussianBeam(AbstractElement):
    """src/elements/beambeam.jl:83-121: Gaussian kicks of nzslice slices."""
    kind = "STRONG_GAUSSIAN_BEAM"

    def __init__(self, charge, mass, atomnum, num_particle, total_energy, beamsize, *, name="STRONGGAUSSIANBEAM",
                 nzslice=1, zslice_center=None, zslice_npar=None, xoffsets=None, yoffsets=None):
        self.name = name
        self.charge, self.mass, self.atomnum = float(charge), float(mass), float(atomnum)
        self.num_particle = int(num_particle)
        self.total_energy = float(total_energy)
        self.beamsize = [float(beamsize[0]), float(beamsize[1])]
        self.nzslice = int(nzslice)
        n = self.nzslice
        self.zslice_center = ([-1.0 + 2.0 * i / (n - 1) for i in range(n)] if n > 1 else [-1.0] * n) \
            if zslice_center is None else [float(v) for v in zslice_center]
        self.zslice_npar = [1.0 / max(n, 1)] * n if zslice_npar is None else [float(v) for v in zslice_npar]
        self.xoffsets = [0.0] * n if xoffsets is None else [float(v) for v in xoffsets]
        self.yoffsets = [0.0] * n if yoffsets is None else [float(v) for v in yoffsets]

    def _fields(self):
        n = max(self.nzslice, 0)
        # the pass reads slice i's weight and offsets, or 1/nzslice and 0 past the arrays' ends
        w = [self.zslice_npar[i] if i < len(self.zslice_npar) else 1.0 / n for i in range(n)]
        xo = [self.xoffsets[i] if i < len(self.xoffsets) else 0.0 for i in range(n)]
        yo = [self.yoffsets[i] if i < len(self.yoffsets) else 0.0 for i in range(n)]
        return {"param": [self.charge, self.total_energy, self.beamsize[0], self.beamsize[1]] + [0.0] * 4,
                "aux": w + xo + yo}

    def get_length(self):
        return 0.0


class LongitudinalRLCWake(AbstractElement):
    """src/elements/wake.jl:6-18: resonator wake, a function of each particle's z."""
    kind = "LONGITUDINAL_RLC_WAKE"

    def __init__(self, *, name="LONGITUDINALRLCWAKE", freq=1.0e9, Rshunt=1.0e6, Q0=1.0, scale=0.0):
        self.name = name
        self.freq, self.Rshunt, self.Q0, self.scale = float(freq), float(Rshunt), float(Q0), float(scale)

    def _fields(self):
        return {"param": [self.freq, self.Rshunt, self.Q0, self.scale] + [0.0] * 4}

    def get_length(self):
        return 0.0


class LongitudinalWake(AbstractElement):
    """src/elements/wake.jl:44-58: tabulated wake, interpolated at each particle's z."""
    kind = "LONGITUDINAL_WAKE"

    def __init__(self, times, wakefields, *, name="LONGITUDINALWAKE", fliphalf=-1.0, scale=0.0):
        if len(times) != len(wakefields):
            raise ValueError("times and wakefields must have the same length")
        if len(times) < 2:
            raise ValueError("LongitudinalWake requires at least two samples")
        self.name = name
        self.times = [float(v) for v in times]
        self.wakefields = [float(v) for v in wakefields]
        self.fliphalf, self.scale = float(fliphalf), float(scale)

    def _fields(self):
        return {"param": [self.fliphalf, self.scale] + [0.0] * 6, "aux": self.times + self.wakefields}

    def get_length(self):
        return 0.0


class Wiggler(AbstractElement):
    """src/elements/wiggler.jl:6-44: harmonics By / Bx of six integers each
    (_, amplitude, kx/kw, ky/kw, kz/kw, phase)."""
    kind = "WIGGLER"
    _misalignable = True

    def __init__(self, L, *, name="WIGGLER", lw=0.0, Bmax=0.0, Nsteps=10, By=(1, 1, 0, 1, 1, 0), Bx=(),
                 energy=1.0e9, rad=0, t1=None, t2=None, r1=None, r2=None):
        self.name = name
        self.L, self.lw, self.Bmax, self.Nsteps = float(L), float(lw), float(Bmax), int(Nsteps)
        self.By = [int(v) for v in By]
        self.Bx = [int(v) for v in Bx]
        self.NHharm, self.NVharm = len(self.By) // 6, len(self.Bx) // 6
        self.energy, self.rad = float(energy), int(rad)
        self._misalign_init(t1, t2, r1, r2)

    def _fields(self):
        by = [float(v) for v in self.By[:6 * self.NHharm]]
        bx = [float(v) for v in self.Bx[:6 * self.NVharm]]
        return {"L": self.L, "num_int_steps": self.Nsteps, "param": [self.lw, self.Bmax, self.energy] + [0.0] * 5,
                "aux": [float(self.NHharm), float(self.NVharm), float(self.rad)] + by + bx}


ELEMENT_TYPES = [Marker, Drift, Quadrupole, Sextupole, Octupole, ThinMultipole, SBend, ExactSBend, RFCavity,
                 Solenoid, Corrector, Translation, YRotation, CrabCavity, AccelCavity, LongitudinalRFMap,
                 LorentzBoost, InvLorentzBoost, SpaceCharge, DriftSC, QuadrupoleSC, SextupoleSC, OctupoleSC,
                 SBendSC, StrongThinGaussianBeam, LBend, StrongGaussianBeam, LongitudinalRLCWake, LongitudinalWake,
                 Wiggler]
