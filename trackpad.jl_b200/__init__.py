"""trackpad_b200 -- B200 multi-particle tracking engine for TrackPad.jl.

The package directory is `trackpad.jl_b200/`; load it under the module name
`trackpad_b200` (see `load()` in the repository's entry scripts).  The public
names mirror TrackPad.jl (`linepass!` -> `linepass_`, `ringpass!` -> `ringpass_`).
"""
from . import _abi, checkpoint, optics, sharding, tpsa
from .elements import (AbstractElement, AccelCavity, Corrector, CrabCavity, Drift, DriftSC, ERBend, ExactSBend,
                       HKicker, InvLorentzBoost, LongitudinalRFMap, LorentzBoost, M_ELECTRON, M_PROTON, Marker,
                       Octupole, OctupoleSC, Quadrupole, QuadrupoleSC, RBend, RBendSC, RFCavity, SBend, SBendSC,
                       Sextupole, SextupoleSC, Solenoid, SpaceCharge, StrongThinGaussianBeam, ThinMultipole,
                       Translation, VKicker, YRotation, LBend, StrongGaussianBeam, LongitudinalRLCWake,
                       LongitudinalWake, Wiggler)
from .tracking import (Batch, Beam, Lattice, Time, TimeContext, TimeDependentParam, TimeVaryingElement, Turn,
                       adjoint_stats, beti, context, last_stats, linepass_, materialize, one_turn_jacobian,
                       probe_fp64_peak, ringpass_, ringpass_adjoint, spos, timed)
from .tpsa import polyseries_one_turn_map, polyseries_variables

__all__ = [n for n in dir() if not n.startswith("_")]
