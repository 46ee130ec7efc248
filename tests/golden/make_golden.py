"""Generate the golden fixtures in this folder.

An independent pure-Python transcription of TrackPad.jl's per-particle maps
(src/tracking.jl) and of linepass!/ringpass! (src/lattice.jl:260-317), written
separately from the C++ oracle so that the two transcriptions check each other.
Python floats are IEEE binary64 with no fused multiply-add; sin, cos, tan, asin
and atan come from fdlibm_py (the published fdlibm method, the one the kernels
and the oracle implement), so the oracle must reproduce these numbers bit for bit.

The cases are the reference's own parity tests, run on its own 10-particle
fixture (test/verify_elements.jl:10-21, energy 3.5e9 eV):
  * every element case of test/verify_elements.jl:48-118 this engine supports,
  * the FODO line of test/verify_fodo.jl:30-39,
  * the DBA line of test/verify_dba.jl:31-44,
  * the single bends of test/verify_bend.jl:25-28 and
    test/verify_exact_bend.jl:24-28,
plus multi-turn and loss cases on the same fixture.

Usage:  python tests/golden/make_golden.py   (writes golden_*.json here)
"""
import json
import math
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import fdlibm_py as fm  # noqa: E402

NAN = float("nan")
COORD_LIMIT = 1.0  # tracking.jl:25
ANGLE_LIMIT = 1.0  # tracking.jl:26
DRIFT1 = 0.6756035959798286638  # tracking.jl:29-32
DRIFT2 = -0.1756035959798286639
KICK1 = 1.351207191959657328
KICK2 = -1.702414383919314656
C_LIGHT = 2.99792458e8  # elements/rf.jl:28
M_ELECTRON = 0.51099895069e6  # lattice.jl:42
TWO_PI = 2.0 * math.pi
EPS = 2.220446049250313e-16

PARTICLES = [  # test/verify_elements.jl:10-21 (rows = particles)
    [1.0e-4, 2.0e-4, 3.0e-4, -1.0e-4, 5.0e-5, 2.0e-4],
    [-2.2e-4, 1.7e-4, -1.1e-4, 2.3e-4, -7.0e-5, 1.0e-4],
    [3.5e-4, -2.1e-4, 8.0e-5, -1.8e-4, 1.4e-4, -2.6e-4],
    [-4.0e-4, 2.9e-4, 1.6e-4, 9.0e-5, -1.2e-4, 3.1e-4],
    [5.2e-4, -3.3e-4, -2.4e-4, 1.1e-4, 2.6e-4, -3.7e-4],
    [-6.1e-4, 4.4e-4, 2.7e-4, -2.5e-4, -3.0e-4, 4.5e-4],
    [7.0e-4, -5.2e-4, -3.1e-4, 3.4e-4, 3.3e-4, -5.0e-4],
    [-8.0e-4, 6.0e-4, 3.9e-4, -4.2e-4, -3.8e-4, 5.8e-4],
    [9.1e-4, -6.7e-4, -4.6e-4, 5.1e-4, 4.4e-4, -6.3e-4],
    [-9.8e-4, 7.3e-4, 5.3e-4, -5.9e-4, -4.9e-4, 7.1e-4],
]


def beti_of(energy, mass=M_ELECTRON):
    """Beam(energy): gamma=(E+m)/m, beta=sqrt(1-1/gamma^2); beti=1/beta (lattice.jl:50-61)."""
    gamma = (energy + mass) / mass
    beta = math.sqrt(1.0 - 1.0 / (gamma * gamma))
    return 1.0 / beta


def nan6():
    return (NAN,) * 6


# --------------------------------------------------------------------------
# Element constructors with the reference defaults (src/elements/*.jl)
# --------------------------------------------------------------------------
def elem(kind, **kw):
    e = dict(kind=kind, max_order=0, num_int_steps=0, fringe_bend_entrance=0, fringe_bend_exit=0,
             misalign_index=-1, iparam=[0, 0], L=0.0, k=0.0, angle=0.0, e1=0.0, e2=0.0, fint1=0.0,
             fint2=0.0, gap=0.0, gk=0.0, polynom_a=[0.0] * 4, polynom_b=[0.0] * 4, kick_angle=[0.0, 0.0],
             volt=0.0, freq=0.0, h=0.0, lag=0.0, philag=0.0, energy=0.0, param=[0.0] * 8)
    e.update(kw)
    return e


def Marker():
    return elem("MARKER")


def Drift(L):
    return elem("DRIFT", L=float(L))


def Quadrupole(L, k1, num_int_steps=10, max_order=1):  # elements/quad.jl:26-47
    return elem("QUADRUPOLE", L=float(L), k=float(k1), num_int_steps=num_int_steps, max_order=max_order)


def Sextupole(L, k2, num_int_steps=10, max_order=2):  # elements/multipole.jl:26-47
    return elem("SEXTUPOLE", L=float(L), k=float(k2), num_int_steps=num_int_steps, max_order=max_order)


def Octupole(L, k3, num_int_steps=10, max_order=3):  # elements/multipole.jl:72-93
    return elem("OCTUPOLE", L=float(L), k=float(k3), num_int_steps=num_int_steps, max_order=max_order)


def ThinMultipole(L, pa, pb, max_order=1):  # elements/multipole.jl:118-139
    return elem("THIN_MULTIPOLE", L=float(L), polynom_a=[float(v) for v in pa],
                polynom_b=[float(v) for v in pb], max_order=max_order, num_int_steps=1)


def SBend(L, angle, e1=0.0, e2=0.0, num_int_steps=10, fbe=1, fbx=1, fint1=0.0, fint2=0.0, gap=0.0):
    return elem("SBEND", L=float(L), angle=float(angle), e1=float(e1), e2=float(e2), num_int_steps=num_int_steps,
                fringe_bend_entrance=fbe, fringe_bend_exit=fbx, fint1=fint1, fint2=fint2, gap=gap)


def RBend(L, angle, **kw):  # elements/bend.jl:81
    return SBend(L, angle, angle / 2, angle / 2, **kw)


def ExactSBend(L, angle, e1=0.0, e2=0.0, num_int_steps=10, gk=0.0, fbe=1, fbx=1):
    return elem("EXACT_SBEND", L=float(L), angle=float(angle), e1=float(e1), e2=float(e2),
                num_int_steps=num_int_steps, gk=float(gk), fringe_bend_entrance=fbe, fringe_bend_exit=fbx)


def ERBend(L, angle, **kw):  # elements/SCelements.jl:339
    return ExactSBend(L, angle, angle / 2, angle / 2, **kw)


def RFCavity(L, volt, freq, lag=0.0, h=1.0, philag=0.0, energy=0.0):  # elements/rf.jl:16-21
    return elem("RFCAVITY", L=float(L), volt=float(volt), freq=float(freq), lag=float(lag), h=float(h),
                philag=float(philag), energy=float(energy))


def Solenoid(L, ks):
    return elem("SOLENOID", L=float(L), param=[float(ks)] + [0.0] * 7)


def Corrector(L, hk, vk):
    return elem("CORRECTOR", L=float(L), param=[float(hk), float(vk)] + [0.0] * 6)


def Translation(L, dx=0.0, dy=0.0, ds=0.0):
    return elem("TRANSLATION", L=float(L), param=[dx, dy, ds] + [0.0] * 5)


def YRotation(L, angle=0.0):
    return elem("YROTATION", L=float(L), angle=float(angle))


def CrabCavity(L, volt=0.0, freq=0.0, phi=0.0, energy=1.0e9):  # elements/rf.jl:46-53
    k = TWO_PI * freq / C_LIGHT
    return elem("CRAB_CAVITY", L=float(L), volt=volt, freq=freq, energy=energy,
                param=[k, phi, 0.0, 0.0] + [0.0] * 4)


def AccelCavity(L, volt=0.0, freq=0.0, h=1.0, phis=0.0, energy=1.0e9):  # elements/rf.jl:80-87
    k = TWO_PI * freq / C_LIGHT
    return elem("ACCEL_CAVITY", L=float(L), volt=volt, freq=freq, h=h, energy=energy,
                param=[k, phis] + [0.0] * 6)


def LongitudinalRFMap(alphac, rf):  # _rf_k/_rf_h: tracking.jl:1565-1573
    if rf["kind"] == "RFCAVITY":
        k, h = TWO_PI * rf["freq"] / C_LIGHT, rf["h"]
    elif rf["kind"] == "ACCEL_CAVITY":
        k, h = rf["param"][0], rf["h"]
    elif rf["kind"] == "CRAB_CAVITY":
        k, h = rf["param"][0], 1.0
    else:
        k, h = 0.0, 1.0
    return elem("LONGITUDINAL_RF_MAP", param=[alphac, k, h] + [0.0] * 5)


def LorentzBoost(angle, mode=0):  # elements/beambeam.jl:14-19
    return elem("LORENTZ_BOOST", param=[angle, fm.cos(angle), 0.0, fm.tan(angle)] + [0.0] * 4, iparam=[mode, 0])


def InvLorentzBoost(angle, mode=0):  # elements/beambeam.jl:38-43
    return elem("INV_LORENTZ_BOOST", param=[angle, fm.cos(angle), fm.sin(angle), 0.0] + [0.0] * 4,
                iparam=[mode, 0])


def DriftSC(L):
    return elem("DRIFT_SC", L=float(L))


def QuadrupoleSC(L, k0=0.0, k1=0.0, k2=0.0, k3=0.0, max_order=1, num_int_steps=10):
    return elem("QUADRUPOLE_SC", L=float(L), param=[k0, k1, k2, k3] + [0.0] * 4, max_order=max_order,
                num_int_steps=num_int_steps)


def SextupoleSC(L, k0=0.0, k1=0.0, k2=0.0, k3=0.0, max_order=2, num_int_steps=10):
    return elem("SEXTUPOLE_SC", L=float(L), param=[k0, k1, k2, k3] + [0.0] * 4, max_order=max_order,
                num_int_steps=num_int_steps)


def OctupoleSC(L, k0=0.0, k1=0.0, k2=0.0, k3=0.0, max_order=3, num_int_steps=10):
    return elem("OCTUPOLE_SC", L=float(L), param=[k0, k1, k2, k3] + [0.0] * 4, max_order=max_order,
                num_int_steps=num_int_steps)


def SBendSC(L, angle, e1=0.0, e2=0.0, num_int_steps=10):
    return elem("SBEND_SC", L=float(L), angle=float(angle), e1=float(e1), e2=float(e2),
                num_int_steps=num_int_steps, fringe_bend_entrance=1, fringe_bend_exit=1)


def SpaceCharge(L):
    return elem("SPACE_CHARGE", L=float(L))


def StrongThinGaussianBeam(amplitude, rmssizex, rmssizey, xoffset=0.0, yoffset=0.0):
    return elem("STRONG_THIN_GAUSSIAN_BEAM", param=[amplitude, rmssizex, rmssizey, xoffset, yoffset, 0.0, 0.0, 0.0])


# --------------------------------------------------------------------------
# Maps (src/tracking.jl), written over 6-tuples
# --------------------------------------------------------------------------
def LBend(L, angle, e1=0.0, e2=0.0, K=0.0, by_error=0.0, fint1=0.0, fint2=0.0, full_gap=0.0):  # SCelements.jl:366-377
    return elem("LBEND", L=L, angle=angle, e1=e1, e2=e2, fint1=fint1, fint2=fint2, gap=full_gap,
                param=[K, by_error] + [0.0] * 6)


def StrongGaussianBeam(charge, total_energy, beamsize, npar, xoff, yoff):  # beambeam.jl:101-114
    return elem("STRONG_GAUSSIAN_BEAM", param=[charge, total_energy, beamsize[0], beamsize[1]] + [0.0] * 4,
                aux=list(npar) + list(xoff) + list(yoff))


def LongitudinalRLCWake(freq=1.0e9, Rshunt=1.0e6, Q0=1.0, scale=0.0):  # wake.jl:14-18
    return elem("LONGITUDINAL_RLC_WAKE", param=[freq, Rshunt, Q0, scale] + [0.0] * 4)


def LongitudinalWake(times, wakefields, fliphalf=-1.0, scale=0.0):  # wake.jl:52-58
    return elem("LONGITUDINAL_WAKE", param=[fliphalf, scale] + [0.0] * 6, aux=list(times) + list(wakefields))


def lbend_body(r, L, grd, b_angle, by_error):  # tracking.jl:1076-1150
    if L == 0.0:
        return r
    p_norm = 1.0 / (1.0 + r[5])
    Kx = b_angle / L
    G1 = (Kx * Kx + grd) * p_norm
    G2 = -grd * p_norm
    tol = 1.4901161193847656e-08
    MHD, M12, M21, MVD, M34, M43 = 1.0, L, 0.0, 1.0, L, 0.0
    arg1 = sqrtG1 = 0.0
    if abs(G1) >= tol:
        if G1 > 0.0:
            sqrtG1 = math.sqrt(G1)
            arg1 = L * sqrtG1
            MHD, M12, M21 = fm.cos(arg1), fm.sin(arg1) / sqrtG1, -fm.sin(arg1) * sqrtG1
        else:
            sqrtG1 = math.sqrt(-G1)
            arg1 = L * sqrtG1
            MHD, M12, M21 = fm.cosh(arg1), fm.sinh(arg1) / sqrtG1, fm.sinh(arg1) * sqrtG1
    if abs(G2) >= tol:
        if G2 > 0.0:
            sq = math.sqrt(G2)
            a2 = L * sq
            MVD, M34, M43 = fm.cos(a2), fm.sin(a2) / sq, -fm.sin(a2) * sq
        else:
            sq = math.sqrt(-G2)
            a2 = L * sq
            MVD, M34, M43 = fm.cosh(a2), fm.sinh(a2) / sq, fm.sinh(a2) * sq
    x, xpr, y, ypr = r[0], r[1] * p_norm, r[2], r[3] * p_norm
    dterm = r[5] * p_norm - by_error
    x_new = MHD * x + M12 * xpr
    px_new = (M21 * x + MHD * xpr) / p_norm
    if abs(G1) < tol:
        x_new += dterm * L * L * Kx / 2
        px_new += dterm * L * Kx / p_norm
    elif G1 > 0.0:
        x_new += dterm * (1.0 - fm.cos(arg1)) * Kx / G1
        px_new += dterm * fm.sin(arg1) * Kx / (sqrtG1 * p_norm)
    else:
        x_new += dterm * (1.0 - fm.cosh(arg1)) * Kx / G1
        px_new += dterm * fm.sinh(arg1) * Kx / (sqrtG1 * p_norm)
    y_new = MVD * y + M34 * ypr
    py_new = (M43 * y + MVD * ypr) / p_norm
    z_new = r[4] + xpr * xpr * (L + MHD * M12) / 4
    if abs(G1) >= tol:
        z_new += (L - MHD * M12) * (x * x * G1 + dterm * dterm * Kx * Kx / G1 - 2 * x * Kx * dterm) / 4
        z_new += M12 * M21 * (x * xpr - xpr * dterm * Kx / G1) / 2
        z_new += Kx * x * M12 + xpr * (1.0 - MHD) * Kx / G1 + dterm * (L - M12) * Kx * Kx / G1
    z_new += ((L - MVD * M34) * y * y * G2 + ypr * ypr * (L + MVD * M34)) / 4
    z_new += M34 * M43 * y * ypr / 2
    return (x_new, px_new, y_new, py_new, z_new, r[5])


def interpolate(x, xs, ys):  # _linear_interpolate, wake.jl:68-84
    if x <= xs[0]:
        return ys[0] + (ys[1] - ys[0]) / (xs[1] - xs[0]) * (x - xs[0])
    if x >= xs[-1]:
        n = len(xs)
        return ys[n - 1] + (ys[n - 1] - ys[n - 2]) / (xs[n - 1] - xs[n - 2]) * (x - xs[n - 1])
    for i in range(1, len(xs)):
        if x < xs[i]:
            return ys[i - 1] + (ys[i] - ys[i - 1]) / (xs[i] - xs[i - 1]) * (x - xs[i - 1])
    return ys[-1]


def Wiggler(L, lw=0.0, Bmax=0.0, Nsteps=10, By=(1, 1, 0, 1, 1, 0), Bx=(), energy=1.0e9, rad=0):  # wiggler.jl:23-44
    return elem("WIGGLER", L=L, num_int_steps=Nsteps, param=[lw, Bmax, energy] + [0.0] * 5,
                aux=[float(len(By) // 6), float(len(Bx) // 6), float(rad)] + [float(v) for v in By]
                + [float(v) for v in Bx])


def sinc_taylor(x):  # tracking.jl:1226-1229
    x2 = x * x
    return 1.0 - x2 / 6 * (1.0 - x2 / 20 * (1.0 - x2 / 42 * (1.0 - x2 / 72)))


def wig_harmonics(e):
    a = e["aux"]
    nh, nv = int(a[0]), int(a[1])
    by = [a[3 + 6 * i: 9 + 6 * i] for i in range(nh)]
    bx = [a[3 + 6 * nh + 6 * i: 9 + 6 * nh + 6 * i] for i in range(nv)]
    return by, bx


def wig_ax_axpy(e, x, y, Zw, Aw, Po):  # tracking.jl:1231-1280
    by, bx = wig_harmonics(e)
    kw = TWO_PI / e["param"][0]
    ax = axpy = 0.0
    for h in by:
        HCw = h[1] * Aw / Po
        kx, ky, kz, tz = h[2] * kw, h[3] * kw, h[4] * kw, h[5]
        cx, chy, sz = fm.cos(kx * x), fm.cosh(ky * y), fm.sin(kz * Zw + tz)
        ax += HCw * (kw / kz) * cx * chy * sz
        shy = fm.sinh(ky * y)
        sxkx = fm.sin(kx * x) / kx if abs(kx / kw) > 1e-6 else x * sinc_taylor(kx * x)
        axpy += HCw * (kw / kz) * ky * sxkx * shy * sz
    for h in bx:
        VCw = h[1] * Aw / Po
        kx, ky, kz, tz = h[2] * kw, h[3] * kw, h[4] * kw, h[5]
        shx, sy, sz = fm.sinh(kx * x), fm.sin(ky * y), fm.sin(kz * Zw + tz)
        ax += VCw * (kw / kz) * (ky / kx) * shx * sy * sz
        chx, cy = fm.cosh(kx * x), fm.cos(ky * y)
        axpy += VCw * (kw / kz) * ((ky / kx) * (ky / kx)) * chx * cy * sz
    return ax, axpy


def wig_ay_aypx(e, x, y, Zw, Aw, Po):  # tracking.jl:1282-1331
    by, bx = wig_harmonics(e)
    kw = TWO_PI / e["param"][0]
    ay = aypx = 0.0
    for h in by:
        HCw = h[1] * Aw / Po
        kx, ky, kz, tz = h[2] * kw, h[3] * kw, h[4] * kw, h[5]
        sx, shy, sz = fm.sin(kx * x), fm.sinh(ky * y), fm.sin(kz * Zw + tz)
        ay += HCw * (kw / kz) * (kx / ky) * sx * shy * sz
        cx, chy = fm.cos(kx * x), fm.cosh(ky * y)
        aypx += HCw * (kw / kz) * ((kx / ky) * (kx / ky)) * cx * chy * sz
    for h in bx:
        VCw = h[1] * Aw / Po
        kx, ky, kz, tz = h[2] * kw, h[3] * kw, h[4] * kw, h[5]
        chx, cy, sz = fm.cosh(kx * x), fm.cos(ky * y), fm.sin(kz * Zw + tz)
        ay += VCw * (kw / kz) * chx * cy * sz
        shx = fm.sinh(kx * x)
        syky = fm.sin(ky * y) / ky if abs(ky / kw) > 1e-6 else y * sinc_taylor(ky * y)
        aypx += VCw * (kw / kz) * kx * shx * syky * sz
    return ay, aypx


def wig_map_2nd(e, r, dl, Zw, Aw, Po):  # tracking.jl:1333-1378
    delta = r[5]
    inv1pd = 1.0 / (1.0 + delta)
    dld = dl * inv1pd
    dl2 = dl / 2
    dl2d = dl2 * inv1pd
    Zw += dl2
    x, px, y, py, z = r[0], r[1], r[2], r[3], r[4]
    ay, aypx = wig_ay_aypx(e, x, y, Zw, Aw, Po)
    px -= aypx
    py -= ay
    y += dl2d * py
    z += (dl2d / 2) * (py * py) * inv1pd
    ay, aypx = wig_ay_aypx(e, x, y, Zw, Aw, Po)
    px += aypx
    py += ay
    ax, axpy = wig_ax_axpy(e, x, y, Zw, Aw, Po)
    px -= ax
    py -= axpy
    x += dld * px
    z += (dld / 2) * (px * px) * inv1pd
    ax, axpy = wig_ax_axpy(e, x, y, Zw, Aw, Po)
    px += ax
    py += axpy
    ay, aypx = wig_ay_aypx(e, x, y, Zw, Aw, Po)
    px -= aypx
    py -= ay
    y += dl2d * py
    z += (dl2d / 2) * (py * py) * inv1pd
    ay, aypx = wig_ay_aypx(e, x, y, Zw, Aw, Po)
    px += aypx
    py += ay
    Zw += dl2
    return (x, px, y, py, z, delta), Zw


def wig_B(e, x, y, Zw):  # tracking.jl:1400-1449 (Bz unused)
    by, bx = wig_harmonics(e)
    kw = TWO_PI / e["param"][0]
    PB0 = e["param"][1]
    Bxv = Byv = 0.0
    for h in by:
        HCw = h[1]
        kx, ky, kz, tz = h[2] * kw, h[3] * kw, h[4] * kw, h[5]
        sx, cx, chy, shy = fm.sin(kx * x), fm.cos(kx * x), fm.cosh(ky * y), fm.sinh(ky * y)
        cz = fm.cos(kz * Zw + tz)
        Bxv += PB0 * HCw * (kx / ky) * sx * shy * cz
        Byv -= PB0 * HCw * cx * chy * cz
    for h in bx:
        VCw = h[1]
        kx, ky, kz, tz = h[2] * kw, h[3] * kw, h[4] * kw, h[5]
        shx, chx, sy, cy = fm.sinh(kx * x), fm.cosh(kx * x), fm.sin(ky * y), fm.cos(ky * y)
        cz = fm.cos(kz * Zw + tz)
        Bxv += PB0 * VCw * chx * cy * cz
        Byv -= PB0 * VCw * (ky / kx) * shx * sy * cz
    return Bxv, Byv


def wig_rad_block(e, r, Zw, Aw, Po, srCoef, SL):  # tracking.jl:1451-1463, 1477-1483
    ax, _ = wig_ax_axpy(e, r[0], r[2], Zw, Aw, Po)
    ay, _ = wig_ay_aypx(e, r[0], r[2], Zw, Aw, Po)
    r = (r[0], r[1] - ax, r[2], r[3] - ay, r[4], r[5])
    Bxv, Byv = wig_B(e, r[0], r[2], Zw)
    B2 = Bxv * Bxv + Byv * Byv
    if B2 != 0.0:
        H = Po * M_ELECTRON / C_LIGHT
        irho2 = B2 / (H * H)
        dFactor = (1.0 + r[5]) * (1.0 + r[5])
        dDelta = -srCoef * dFactor * irho2 * SL
        sc = 1.0 + dDelta
        r = (r[0], r[1] * sc, r[2], r[3] * sc, r[4], r[5] + dDelta)
    return (r[0], r[1] + ax, r[2], r[3] + ay, r[4], r[5])


def wiggler(e, r):  # tracking.jl:1380-1398, 1465-1503, 1509-1525
    lw, Bmax, energy = e["param"][:3]
    rad = int(e["aux"][2])
    PN = e["num_int_steps"]
    Nw = round(e["L"] / lw)  # Python round: half to even, as Julia's round(Int, x)
    Nstep = PN * max(1, Nw)
    dl = lw / PN
    dl1, dl0 = dl * 1.3512071919596573, dl * -1.7024143839193146
    Aw = 1e-9 * C_LIGHT / (M_ELECTRON * 1e-9) / TWO_PI * lw * Bmax
    Zw = 0.0
    if rad == 1:
        gamma = energy / M_ELECTRON
        Po = math.sqrt(gamma * gamma - 1.0)
        srCoef = (2.0 / 3.0) * 2.8179403205e-15 * (gamma * gamma * gamma)
        r = wig_rad_block(e, r, Zw, Aw, Po, srCoef, dl)
        for _ in range(Nstep):
            for d in (dl1, dl0, dl1):
                r, Zw = wig_map_2nd(e, r, d, Zw, Aw, Po)
            r = wig_rad_block(e, r, Zw, Aw, Po, srCoef, dl)
        return r
    Po = math.sqrt((energy / M_ELECTRON) * (energy / M_ELECTRON) - 1.0)
    for _ in range(Nstep):
        for d in (dl1, dl0, dl1):
            r, Zw = wig_map_2nd(e, r, d, Zw, Aw, Po)
    return r


def lost_check(r):  # tracking.jl:49-52
    return (math.isnan(r[0]) or abs(r[0]) > COORD_LIMIT or abs(r[2]) > COORD_LIMIT
            or abs(r[1]) > ANGLE_LIMIT or abs(r[3]) > ANGLE_LIMIT)


def drift(r, L, beti):  # tracking.jl:87-99 (exact Hamiltonian branch)
    x, px, y, py, z, d = r
    pz2 = 1.0 + 2.0 * d * beti + d * d - px * px - py * py
    if pz2 <= 0.0:
        return nan6()
    nl = L / math.sqrt(pz2)
    return (x + nl * px, px, y + nl * py, py, z + nl * (beti + d) - L * beti, d)


def horner(pa, pb, order, x, y):  # shared Horner loop of tracking.jl:243-305
    re, im = pb[order], pa[order]
    for i in range(order - 1, -1, -1):
        re, im = re * x - im * y + pb[i], im * x + re * y + pa[i]
    return re, im


def thin_kick(r, pa, pb, K, order):  # strthinkick, tracking.jl:284-305
    re, im = horner(pa, pb, order, r[0], r[2])
    return (r[0], r[1] - K * re, r[2], r[3] + K * im, r[4], r[5])


def bend_kick(r, pa, pb, K, irho, order, beti):  # bndthinkick, tracking.jl:243-270
    re, im = horner(pa, pb, order, r[0], r[2])
    return (r[0], r[1] - K * (re - (r[5] - r[0] * irho) * irho), r[2], r[3] + K * im,
            r[4] + K * irho * r[0] * beti, r[5])


def yoshida(r, L, steps, drift_fn, kick_fn):  # tracking.jl:317-375
    sl = L / float(steps)
    l1, l2, k1, k2 = sl * DRIFT1, sl * DRIFT2, sl * KICK1, sl * KICK2
    for _ in range(steps):
        r = drift_fn(r, l1)
        r = kick_fn(r, k1)
        r = drift_fn(r, l2)
        r = kick_fn(r, k2)
        r = drift_fn(r, l2)
        r = kick_fn(r, k1)
        r = drift_fn(r, l1)
    return r


def folded(e, pa, pb):  # kick_angle folding, tracking.jl:396-411
    pa, pb = list(pa), list(pb)
    if e["L"] > 0.0:
        pb[0] = pb[0] - fm.sin(e["kick_angle"][0]) / e["L"]
        pa[0] = pa[0] + fm.sin(e["kick_angle"][1]) / e["L"]
    return pa, pb


def edge(r, irho, ang, fint, gap, method, at_exit):  # tracking.jl:160-221
    if fint == 0.0 or gap == 0.0 or method == 0:
        fc = 0.0
    else:
        se, ce = fm.sin(ang), fm.cos(ang)
        fc = irho * gap * fint * (1.0 + se * se) / ce
    fx = irho * fm.tan(ang)
    opd = 1.0 + r[5]
    if method == 2:
        fy = irho * fm.tan(ang - fc / opd) / opd
    elif method == 3:
        fy = irho * fm.tan(ang - fc - r[1] / opd) if at_exit else irho * fm.tan(ang - fc + r[1] / opd)
    else:
        fy = irho * fm.tan(ang - fc / opd)
    return (r[0], r[1] + r[0] * fx, r[2], r[3] - r[2] * fy, r[4], r[5])


def pxyz(dp1, px, py):  # tracking.jl:717-720
    v = dp1 * dp1 - px * px - py * py
    return math.sqrt(v) if v > 0.0 else 0.0


def jclamp(v):  # Julia clamp(v, -1, 1); NaN passes through
    return 1.0 if v > 1.0 else (-1.0 if v < -1.0 else v)


def yrot(r, phi, beti):  # tracking.jl:727-745
    if phi == 0.0:
        return r
    x, px, y, py, z, d = r
    dp1 = beti + d
    c, s = fm.cos(phi), fm.sin(phi)
    pz = pxyz(dp1, px, py)
    p = c * pz - s * px
    return (x * pz / p, s * pz + c * px, y + x * py * s / p, py, z + dp1 * x * s / p, d)


def fringe(r, irho, gk, beti):  # bend_fringe, tracking.jl:752-815
    x, px, y, py, z, d = r
    b0 = irho
    dp1 = beti + d
    pz = pxyz(dp1, px, py)
    xp, yp = px / pz, py / pz
    t1 = 1.0 + xp * xp * (2.0 + yp * yp)
    t2 = xp / (1.0 + yp * yp)
    phi = -b0 * fm.tan(b0 * gk * t1 * pz - fm.atan(t2))
    px2, py2, pz2 = px * px, py * py, pz * pz
    pz4 = pz2 * pz2
    s2 = py2 + pz2
    arg = (b0 * gk * (pz4 + px2 * (py2 + 2.0 * pz2))) / (pz2 * pz) - fm.atan(px * pz / (py2 + pz2))
    sec = 1.0 / fm.cos(arg)
    psec = sec * sec
    py4 = py2 * py2
    py6 = py4 * py2
    pz5 = pz4 * pz
    pz6 = pz4 * pz2
    s2sq = s2 * s2
    den = pz5 * (py4 + px2 * pz2 + 2.0 * py2 * pz2 + pz4)
    dpx = -(b0 * (px2 * pz4 * (py2 - pz2) - pz6 * (py2 + pz2)
                  + b0 * gk * px * (pz2 * s2sq * (2.0 * py2 + 3.0 * pz2)
                                    + px2 * px2 * (3.0 * py2 * pz2 + 2.0 * pz4)
                                    + px2 * (3.0 * py6 + 8.0 * py4 * pz2 + 9.0 * py2 * pz4 + 5.0 * pz6)))) * psec
    dpx = dpx / den
    dpy = -(b0 * py * (px * pz4 * (py2 + pz2)
                       + b0 * gk * (-(pz4 * s2sq) + px2 * px2 * (3.0 * py2 * pz2 + 4.0 * pz4)
                                    + px2 * (3.0 * py6 + 10.0 * py4 * pz2 + 11.0 * py2 * pz4 + 3.0 * pz6)))) * psec
    dpy = dpy / den
    dd = (b0 * dp1 * (px * pz4 * (py2 - pz2)
                      + b0 * gk * (-(pz4 * s2sq) + px2 * px2 * (3.0 * py2 * pz2 + 2.0 * pz4)
                                   + px2 * (3.0 * py6 + 8.0 * py4 * pz2 + 7.0 * py2 * pz4 + pz6)))) * psec
    dd = dd / den
    yf = (2.0 * y) / (1.0 + math.sqrt(1.0 - 2.0 * dpy * y))
    return (x + 0.5 * dpx * (yf * yf), px, yf, py - phi * yf, z - 0.5 * dd * (yf * yf), d)


def wedge(r, h, theta, beti):  # bend_edge, tracking.jl:822-851
    if abs(h) < 1e-6:
        return r
    x, px, y, py, z, d = r
    dp1 = beti + d
    c, s = fm.cos(theta), fm.sin(theta)
    pz = pxyz(dp1, px, py)
    d2 = pxyz(dp1, 0.0, py)
    pxn = px * c + (pz - h * x) * s
    das = fm.asin(jclamp(px / d2)) - fm.asin(jclamp(pxn / d2))
    num = x * (px * fm.sin(2.0 * theta) + s * s * (2.0 * pz - h * x))
    den = pxyz(dp1, pxn, py) + pz * c - px * s
    return (x * c + num / den, pxn, y + py * (theta / h + das / h), py, z + dp1 / h * (theta + das), d)


def body(r, h, L, beti):  # exact_bend_body, tracking.jl:858-894
    x, px, y, py, z, d = r
    dp1 = beti + d
    pz = pxyz(dp1, px, py)
    if abs(h) < 1e-6:
        nl = L / pz
        return (x + px * nl, px, y + py * nl, py, z + nl * dp1 - L * beti, d)
    pzmx = pz - (1.0 + x * h)
    cs, sn = fm.cos(h * L), fm.sin(h * L)
    pxn = px * cs + pzmx * sn
    d2 = pxyz(dp1, 0.0, py)
    das = L + (fm.asin(jclamp(px / d2)) - fm.asin(jclamp(pxn / d2))) / h
    xn = (pxyz(dp1, pxn, py) - pzmx * cs + px * sn - 1.0) / h
    return (xn, pxn, y + py * das, py, z + dp1 * das - L * beti, d)


# Kinds whose pass! starts with apply_misalignment(r, elem.t1) (and `elem.r1 * r`
# when r1 is not all zero) and ends with `elem.r2 * r` and apply_misalignment(r,
# elem.t2): tracking.jl:115-132, 386-427, 438-459, 470-491, 529-570, 579-607,
# 616-633, 657-706, 901-973, 981-1060, 1152-1170, 1509-1525.
MISALIGNED_KINDS = {"DRIFT", "QUADRUPOLE", "SEXTUPOLE", "OCTUPOLE", "SOLENOID", "CORRECTOR", "THIN_MULTIPOLE",
                    "SBEND", "EXACT_SBEND", "DRIFT_SC", "QUADRUPOLE_SC", "SEXTUPOLE_SC", "OCTUPOLE_SC", "SBEND_SC",
                    "LBEND", "WIGGLER"}


def add_t(r, t):  # apply_misalignment(r, t) = r + t, tracking.jl:64-66
    return tuple(r[i] + t[i] for i in range(6))


def mat_vec(R, r):
    """SMatrix{6,6} * SVector{6}: R stored column-major (R[i + 6 j] is row i,
    column j); each row summed over the columns left to right."""
    out = []
    for i in range(6):
        acc = R[i] * r[0]
        for j in range(1, 6):
            acc = acc + R[i + 6 * j] * r[j]
        out.append(acc)
    return tuple(out)


def apply_pass(e, r, beti, mis=None):
    """pass!(elem, r, beti): misalignment (when the element has a row) around the map."""
    row = mis[e["misalign_index"]] if (mis and e.get("misalign_index", -1) >= 0) else None
    if row is None or e["kind"] not in MISALIGNED_KINDS:
        return apply_map(e, r, beti)
    r = add_t(r, row["t1"])
    if any(v != 0.0 for v in row["r1"]):
        r = mat_vec(row["r1"], r)
    if e["kind"] in ("SBEND_SC", "LBEND") and e["L"] == 0.0:
        return nan6()
    r = apply_map(e, r, beti)
    if any(v != 0.0 for v in row["r2"]):
        r = mat_vec(row["r2"], r)
    return add_t(r, row["t2"])


def apply_map(e, r, beti):
    """The map of pass!(elem, r, beti) between the misalignments, for every supported element kind."""
    kind = e["kind"]
    if kind in ("MARKER", "SPACE_CHARGE"):
        return r
    if kind in ("DRIFT", "DRIFT_SC"):
        return drift(r, e["L"], beti)
    if kind in ("QUADRUPOLE", "SEXTUPOLE", "OCTUPOLE", "QUADRUPOLE_SC", "SEXTUPOLE_SC", "OCTUPOLE_SC"):
        pb = list(e["polynom_b"])
        pa = list(e["polynom_a"])
        order = e["max_order"]
        if kind == "QUADRUPOLE":
            pb[1] = e["k"]
            pa, pb = folded(e, pa, pb)
        elif kind == "SEXTUPOLE":
            pb[2] = e["k"] / 2.0
        elif kind == "OCTUPOLE":
            pb[3] = e["k"] / 6.0
        else:  # SC family: (k0, k1, k2/2, k3/6), tracking.jl:993-1039
            p = e["param"]
            pb = [p[0], p[1], p[2] / 2.0, p[3] / 6.0]
            if kind == "QUADRUPOLE_SC":
                pa, pb = folded(e, pa, pb)
            order = min(max(order, 0), 3)
        return yoshida(r, e["L"], e["num_int_steps"], lambda q, l: drift(q, l, beti),
                       lambda q, kk: thin_kick(q, pa, pb, kk, order))
    if kind == "THIN_MULTIPOLE":
        return thin_kick(r, e["polynom_a"], e["polynom_b"], 1.0, e["max_order"])
    if kind in ("SBEND", "SBEND_SC"):
        if kind == "SBEND_SC" and e["L"] == 0.0:
            return nan6()
        order = e["max_order"] if kind == "SBEND" else min(max(e["max_order"], 0), 3)
        irho = e["angle"] / e["L"]
        pa, pb = folded(e, e["polynom_a"], e["polynom_b"])
        if e["fringe_bend_entrance"] != 0:
            r = edge(r, irho, e["e1"], e["fint1"], e["gap"], e["fringe_bend_entrance"], False)
        r = yoshida(r, e["L"], e["num_int_steps"], lambda q, l: drift(q, l, beti),
                    lambda q, kk: bend_kick(q, pa, pb, kk, irho, order, beti))
        if e["fringe_bend_exit"] != 0:
            r = edge(r, irho, e["e2"], e["fint2"], e["gap"], e["fringe_bend_exit"], True)
        return r
    if kind == "EXACT_SBEND":
        irho = e["angle"] / e["L"]
        r = yrot(r, e["e1"], beti)
        if e["fringe_bend_entrance"] != 0:
            r = fringe(r, irho, e["gk"], beti)
        r = wedge(r, irho, -e["e1"], beti)
        if e["num_int_steps"] == 0:
            r = body(r, irho, e["L"], beti)
        else:
            pa, pb = folded(e, e["polynom_a"], e["polynom_b"])
            r = yoshida(r, e["L"], e["num_int_steps"], lambda q, l: body(q, irho, l, beti),
                        lambda q, kk: thin_kick(q, pa, pb, kk, e["max_order"]))
        r = wedge(r, irho, -e["e2"], beti)
        if e["fringe_bend_exit"] != 0:
            r = fringe(r, -irho, e["gk"], beti)
        return yrot(r, e["e2"], beti)
    if kind == "RFCAVITY":  # tracking.jl:502-518
        beta = 1.0 / beti
        if e["L"] > 0.0:
            r = drift(r, e["L"] / 2.0, beti)
        if e["energy"] > 0.0:
            nv = e["volt"] / e["energy"]
            ph = TWO_PI * e["freq"] * ((r[4] - e["lag"]) / C_LIGHT) - e["philag"]
            r = r[:5] + (r[5] - nv * fm.sin(ph) / (beta * beta),)
        if e["L"] > 0.0:
            r = drift(r, e["L"] / 2.0, beti)
        return r
    if kind == "SOLENOID":  # tracking.jl:529-570
        ks, L = e["param"][0], e["L"]
        if ks == 0.0:
            return drift(r, L, beti)
        x, px, y, py, z, d = r
        pn = 1.0 / (1.0 + d)
        xpr, ypr = px * pn, py * pn
        H = ks * pn / 2.0
        S, C = fm.sin(L * H), fm.cos(L * H)
        xn = x * C * C + xpr * C * S / H + y * C * S + ypr * S * S / H
        pxn = (-x * H * C * S + xpr * C * C - y * H * S * S + ypr * C * S) / pn
        yn = -x * C * S - xpr * S * S / H + y * C * C + ypr * C * S / H
        pyn = (x * H * S * S - xpr * C * S - y * C * S * H + ypr * C * C) / pn
        zn = z + L * (H * H * (x * x + y * y) + 2.0 * H * (xpr * y - ypr * x) + xpr * xpr + ypr * ypr) / 2.0
        return (xn, pxn, yn, pyn, zn, d)
    if kind == "CORRECTOR":  # tracking.jl:579-607
        xk, yk = e["param"][0], e["param"][1]
        x, px, y, py, z, d = r
        pn = 1.0 / (1.0 + d)
        nl = e["L"] * pn
        zn = z + nl * pn * (xk * xk / 3.0 + yk * yk / 3.0 + px * px + py * py + px * xk + py * yk) / 2.0
        return (x + nl * (px + xk / 2.0), px + xk, y + nl * (py + yk / 2.0), py + yk, zn, d)
    if kind == "TRANSLATION":  # tracking.jl:1182-1192
        x, px, y, py, z, d = r
        dx, dy, ds = e["param"][0], e["param"][1], e["param"][2]
        pz2 = 1.0 + 2.0 * d * beti + d * d - px * px - py * py
        if pz2 <= 0.0:
            return nan6()
        pz = math.sqrt(pz2)
        return (x - (dx + ds * px / pz), px, y - (dy + ds * py / pz), py, z + ds * (beti + d) / pz, d)
    if kind == "YROTATION":  # tracking.jl:1194-1218
        ang = -e["angle"]
        if ang == 0.0:
            return r
        x, px, y, py, z, d = r
        ca, sa, ta = fm.cos(ang), fm.sin(ang), fm.tan(ang)
        pz2 = 1.0 + 2.0 * d * beti + d * d - px * px - py * py
        if pz2 <= 0.0:
            return nan6()
        pz = math.sqrt(pz2)
        ptt = 1.0 - ta * px / pz
        if abs(ptt) < math.sqrt(EPS):
            return nan6()
        return (x / (ca * ptt), ca * px + sa * pz, y + ta * x * py / (pz * ptt), py,
                z + ta * x * (beti + d) / (pz * ptt), d)
    if kind == "CRAB_CAVITY":  # tracking.jl:1531-1547
        k, phi0, er1, er2 = e["param"][0], e["param"][1], e["param"][2], e["param"][3]
        volt = e["volt"] * (1.0 + er1)
        phi = phi0 + er2
        E = max(abs(e["energy"]), EPS)
        ang = k * r[4] + phi
        if e["L"] > 0.0:
            r = drift(r, e["L"] / 2.0, beti)
        pxn = r[1] + (volt / E) * fm.sin(ang * beti)
        dn = r[5] - (k * volt / E * beti) * r[0] * fm.cos(ang * beti)
        r = (r[0], pxn, r[2], r[3], r[4], dn)
        if e["L"] > 0.0:
            r = drift(r, e["L"] / 2.0, beti)
        return r
    if kind == "ACCEL_CAVITY":  # tracking.jl:1549-1559
        beta = 1.0 / beti
        b2 = beta * beta
        if b2 <= EPS:
            return r
        E = max(abs(e["energy"]), EPS)
        k, phis = e["param"][0], e["param"][1]
        sv = fm.sin(k * r[4] + phis) - fm.sin(phis)
        return r[:5] + (r[5] + (e["volt"] / (b2 * E)) * sv,)
    if kind == "LONGITUDINAL_RF_MAP":  # tracking.jl:1575-1585
        alphac, k, h = e["param"][0], e["param"][1], e["param"][2]
        if abs(k) <= EPS:
            return r
        beta = 1.0 / beti
        eta = alphac - (1.0 - beta * beta)
        return r[:4] + (r[4] - (TWO_PI * h * eta / k) * r[5], r[5])
    if kind == "LORENTZ_BOOST":  # tracking.jl:1587-1595
        if e["iparam"][0] != 0:
            return r
        ic = 1.0 / e["param"][1]
        ta = e["param"][3]
        return (r[0] + ta * r[4], r[1] * ic, r[2], r[3] * ic, r[4] * ic, r[5] - ta * r[1])
    if kind == "INV_LORENTZ_BOOST":  # tracking.jl:1597-1604
        if e["iparam"][0] != 0:
            return r
        c, s = e["param"][1], e["param"][2]
        return (r[0] - s * r[4], r[1] * c, r[2], r[3] * c, r[4] * c, r[5] + s * r[1])
    if kind == "STRONG_THIN_GAUSSIAN_BEAM":  # tracking.jl:1610-1619
        amp, sx, sy, xo, yo = e["param"][:5]
        sx2, sy2 = max(sx * sx, EPS), max(sy * sy, EPS)
        dx, dy = r[0] - xo, r[2] - yo
        g = amp * fm.exp(-0.5 * (dx * dx / sx2 + dy * dy / sy2))
        return (r[0], r[1] - g * dx / sx2, r[2], r[3] - g * dy / sy2, r[4], r[5])
    if kind == "LBEND":  # tracking.jl:1152-1170
        if e["L"] == 0.0:
            return nan6()
        irho = e["angle"] / e["L"]
        r = edge(r, irho, e["e1"], e["fint1"], e["gap"], 1, False)
        r = lbend_body(r, e["L"], e["param"][0], e["angle"], e["param"][1])
        return edge(r, irho, e["e2"], e["fint2"], e["gap"], 1, True)
    if kind == "STRONG_GAUSSIAN_BEAM":  # tracking.jl:1621-1641
        a = e["aux"]
        nz = len(a) // 3
        if nz <= 0:
            return r
        sx2, sy2 = max(e["param"][2] ** 2, EPS), max(e["param"][3] ** 2, EPS)
        factor = e["param"][0] / max(abs(e["param"][1]), EPS)
        px, py = r[1], r[3]
        for i in range(nz):
            dx, dy = r[0] - a[nz + i], r[2] - a[2 * nz + i]
            g = a[i] * fm.exp(-0.5 * (dx * dx / sx2 + dy * dy / sy2))
            px -= factor * g * dx / sx2
            py -= factor * g * dy / sy2
        return (r[0], px, r[2], py, r[4], r[5])
    if kind == "LONGITUDINAL_RLC_WAKE":  # tracking.jl:1647-1654, wake.jl:27-37
        freq, rsh, q0, scale = e["param"][:4]
        if scale == 0.0:
            return r
        t = min(r[4] / C_LIGHT, 0.0)
        q0p = math.sqrt(q0 * q0 - 0.25)
        w0 = TWO_PI * freq
        w0p = w0 / q0 * q0p
        wf = 0.0 if t > 0.0 else rsh * w0 / q0 * (fm.cos(w0p * t) + fm.sin(w0p * t) / (2 * q0p)) * \
            fm.exp(w0 * t / (2 * q0))
        return (r[0], r[1], r[2], r[3], r[4], r[5] - scale * wf)
    if kind == "WIGGLER":
        return wiggler(e, r)
    if kind == "LONGITUDINAL_WAKE":  # tracking.jl:1656-1663, wake.jl:86-91
        flip, scale = e["param"][:2]
        if scale == 0.0:
            return r
        n = len(e["aux"]) // 2
        xs, ys = e["aux"][:n], e["aux"][n:]
        t = r[4] / C_LIGHT
        wf = 0.0 if t > xs[0] * flip else interpolate(t * flip, xs, ys)
        return (r[0], r[1], r[2], r[3], r[4], r[5] - scale * wf)
    raise ValueError(kind)


def ringpass(elems, parts, beti, nturns=1, aperture=(0.0, 0.0), misalign=None):
    """ringpass!/linepass! (lattice.jl:260-317) on a list of particles;
    `misalign` lists the misalignment rows the elements' misalign_index select."""
    coords = [tuple(p) for p in parts]
    lost = [0] * len(coords)
    lost_turn = [-1] * len(coords)
    lost_elem = [-1] * len(coords)
    ax, ay = aperture
    for t in range(nturns):
        for ie, e in enumerate(elems):
            for i in range(len(coords)):
                if lost[i] == 1:
                    continue
                rn = apply_pass(e, coords[i], beti, misalign)
                out = lost_check(rn) or (ax > 0.0 and abs(rn[0]) > ax) or (ay > 0.0 and abs(rn[2]) > ay)
                if out:
                    lost[i], lost_turn[i], lost_elem[i] = 1, t, ie
                    continue
                coords[i] = rn
    return coords, lost, lost_turn, lost_elem


def hexify(rows):
    return [[float(v).hex() for v in row] for row in rows]


def case(name, elems, parts, energy, nturns=1, aperture=(0.0, 0.0), misalign=None):
    beti = beti_of(energy)
    out, lost, lt, le = ringpass(elems, parts, beti, nturns, aperture, misalign)
    d = dict(name=name, energy=energy, beti=beti.hex(), nturns=nturns, aperture=list(aperture),
             elements=elems, input=hexify(parts), output=hexify(out), lost=lost, lost_turn=lt, lost_elem=le)
    if misalign:
        d["misalign"] = [{k: [float(v).hex() for v in row[k]] for k in ("t1", "t2", "r1", "r2")}
                         for row in misalign]
    return d


def rot_xy(phi):
    """Roll about the beam axis by phi: (x, y) and (px, py) rotated alike (column-major 6x6)."""
    c, sn = math.cos(phi), math.sin(phi)
    m = [0.0] * 36
    for i in range(6):
        m[i + 6 * i] = 1.0
    for a, b in ((0, 2), (1, 3)):
        m[a + 6 * a], m[a + 6 * b] = c, sn
        m[b + 6 * a], m[b + 6 * b] = -sn, c
    return m


def general_matrix(seed):
    """A non-orthogonal matrix near the identity (column-major), deterministic."""
    m = [0.0] * 36
    v = seed
    for j in range(6):
        for i in range(6):
            v = (v * 1103515245 + 12345) % (1 << 31)
            m[i + 6 * j] = (1.0 if i == j else 0.0) + ((v / (1 << 31)) - 0.5) * 0.02
    return m


def misalignment_cases(energy):
    """Elements with offsets t1/t2 and rotations r1/r2 (the reference's Drift,
    Quadrupole, Sextupole, SBend, ExactSBend, ... misalignment fields)."""
    zero = [0.0] * 36
    offs = [(1.5e-4, -2.0e-5, -7.0e-5, 1.2e-5, 3.0e-5, 0.0), (-1.5e-4, 2.0e-5, 7.0e-5, -1.2e-5, -3.0e-5, 0.0)]
    rows = [
        dict(t1=list(offs[0]), t2=list(offs[1]), r1=rot_xy(2e-3), r2=rot_xy(-2e-3)),   # offset and roll
        dict(t1=list(offs[0]), t2=list(offs[1]), r1=zero, r2=zero),                     # offset only
        dict(t1=[0.0] * 6, t2=[0.0] * 6, r1=general_matrix(7), r2=general_matrix(11)),  # general matrices
        dict(t1=[2e-5, 0.0, -1e-5, 0.0, 0.0, 1e-6], t2=[0.0] * 6, r1=zero, r2=rot_xy(1e-3)),
    ]

    def mis(e, k):
        e = dict(e)
        e["misalign_index"] = k
        return e

    a = math.pi / 9
    dba = [Drift(2.0), mis(SBend(1.0, a, a / 2, a / 2), 1), Drift(0.5), mis(Quadrupole(0.4, 1.5), 0), Drift(0.5),
           mis(Quadrupole(0.4, -1.2), 2), Drift(0.5), mis(Quadrupole(0.4, 1.5), 3), Drift(0.5),
           mis(SBend(1.0, a, a / 2, a / 2), 0), Drift(2.0)]
    return [
        ("MisalignedQuadrupole", [mis(Quadrupole(0.4, 1.3), 0)], rows, 1),
        ("MisalignedSextupoleGeneral", [mis(Sextupole(0.4, 2.0), 2)], rows, 1),
        ("MisalignedDriftRotation", [mis(Drift(0.7), 2)], rows, 1),
        ("MisalignedSBend", [mis(SBend(0.9, 0.15, 0.03, 0.02), 1)], rows, 1),
        ("MisalignedExactSBend", [mis(ExactSBend(0.9, 0.15, 0.03, 0.02), 0)], rows, 1),
        ("MisalignedExactSBendGeneral", [mis(ExactSBend(1.5, 2.0 * math.pi / 40.0, math.pi / 40.0,
                                                        math.pi / 40.0), 2)], rows, 1),
        ("MisalignedOtherKinds", [mis(ThinMultipole(1.0, [0.0, 0.01, 0.0, 0.0], [1e-4, 0.2, 3.0, 0.0], max_order=2), 0),
                                  mis(Solenoid(0.5, 0.3), 1), mis(Corrector(0.3, 1e-4, -2e-4), 3),
                                  mis(QuadrupoleSC(0.4, k1=1.1), 2), mis(SBendSC(0.9, 0.15, 0.03, 0.02), 0),
                                  mis(DriftSC(0.6), 3), mis(Octupole(0.3, 40.0), 1),
                                  mis(LBend(0.9, 0.15, 0.03, 0.02, K=0.8), 2),
                                  mis(Wiggler(0.25, lw=0.05, Bmax=0.8, Nsteps=3, energy=3.5e9), 3)], rows, 1),
        ("MisalignedDBA_line_3passes", dba, rows, 3),
    ]


def element_cases(energy):
    """test/verify_elements.jl:52-118 (cases this engine supports)."""
    acc = AccelCavity(0.0, volt=2.5e6, freq=500.0e6, h=1200.0, phis=0.2, energy=energy)
    return [
        ("Marker", [Marker()]),
        ("Drift", [Drift(0.7)]),
        ("Quadrupole", [Quadrupole(0.4, 1.3, num_int_steps=10)]),
        ("Sextupole", [Sextupole(0.4, 2.0, num_int_steps=10)]),
        ("Octupole", [Octupole(0.4, -3.0, num_int_steps=10)]),
        ("ThinMultipole", [ThinMultipole(0.0, [0.0] * 4, [0.0, 0.2, -0.1, 0.05], max_order=3)]),
        ("SBend", [SBend(0.9, 0.15, 0.03, 0.02, num_int_steps=10)]),
        ("RBend", [RBend(0.9, 0.15, num_int_steps=10)]),
        ("ExactSBend", [ExactSBend(0.9, 0.15, 0.03, 0.02, num_int_steps=10)]),
        ("ERBend", [ERBend(0.9, 0.15, num_int_steps=10)]),
        ("RFCavity", [RFCavity(0.3, 2.0e6, 500.0e6, 0.002, h=1200.0, philag=0.3, energy=energy)]),
        ("CrabCavity", [CrabCavity(0.3, volt=2.0e6, freq=500.0e6, phi=0.1, energy=energy)]),
        ("AccelCavity", [acc]),
        ("LongitudinalRFMap", [LongitudinalRFMap(2.0e-4, acc)]),
        ("Solenoid", [Solenoid(0.5, 0.8)]),
        ("Corrector", [Corrector(0.4, 1.5e-4, -2.2e-4)]),
        ("HKicker", [Corrector(0.0, 2.5e-4, 0.0)]),
        ("VKicker", [Corrector(0.0, 0.0, -1.5e-4)]),
        ("Translation", [Translation(0.0, dx=1e-3, dy=-2e-3, ds=3e-3)]),
        ("YRotation", [YRotation(0.0, angle=0.02)]),
        ("LorentzBoost", [LorentzBoost(0.03)]),
        ("InvLorentzBoost", [InvLorentzBoost(0.03)]),
        ("DriftSC", [DriftSC(0.5)]),
        ("QuadrupoleSC", [QuadrupoleSC(0.4, k1=0.0)]),
        ("SextupoleSC", [SextupoleSC(0.3, k2=2.4)]),
        ("OctupoleSC", [OctupoleSC(0.2, k3=3.6)]),
        ("SBendSC", [SBendSC(1.0, 0.0, 0.0, 0.0)]),
        ("RBendSC", [SBendSC(1.2, 0.0, 0.0, 0.0)]),
        ("SpaceCharge", [SpaceCharge(0.9)]),
        ("StrongThinGaussianBeam", [StrongThinGaussianBeam(1.0e-6, 1.0e-3, 1.2e-3, 1.0e-4, -2.0e-4)]),
    ]


def extra_cases(energy):
    """Cases beyond the reference suite: other edge methods, kick angles, skew terms."""
    q = Quadrupole(0.5, -0.8)
    q["kick_angle"] = [1.0e-4, -2.0e-4]
    q["polynom_a"] = [0.0, 0.05, 0.0, 0.0]
    sb2 = SBend(0.9, 0.15, 0.03, 0.02, fbe=2, fbx=3, fint1=0.5, fint2=0.4, gap=0.05)
    sb2["polynom_b"] = [0.0, -0.3, 1.5, 0.0]
    sb2["max_order"] = 2
    eb = ExactSBend(1.5, 2.0 * math.pi / 40.0, math.pi / 40.0, math.pi / 40.0, gk=0.0)
    eb_gk = ExactSBend(0.9, 0.15, 0.03, 0.02, gk=0.6)
    eb_kick = ExactSBend(0.9, 0.15, 0.03, 0.02)
    eb_kick["kick_angle"] = [1.0e-4, 5.0e-5]
    eb0 = ExactSBend(0.9, 0.15, 0.03, 0.02, num_int_steps=0)
    return [
        ("QuadKickSkew", [q]),
        ("SBendMethods23", [sb2]),
        ("ExactSBendDBA", [eb]),
        ("ExactSBendGK", [eb_gk]),
        ("ExactSBendKick", [eb_kick]),
        ("ExactSBendNoSteps", [eb0]),
        ("RFNoEnergy", [RFCavity(0.2, 1.0e6, 500.0e6)]),
        ("LBendFocusing", [LBend(0.9, 0.15, 0.03, 0.02, K=0.8, by_error=1e-4, fint1=0.5, fint2=0.4,
                                 full_gap=0.05)]),
        ("LBendDefocusing", [LBend(0.9, 0.15, 0.03, 0.02, K=-0.9)]),
        ("LBendNoGradient", [LBend(1.2, 1e-5, 0.0, 0.0)]),
        ("StrongGaussianBeam", [StrongGaussianBeam(1.0e-3, 6.0e9, (3e-4, 4e-4), [0.2, 0.5, 0.3],
                                                   [1e-5, 0.0, -2e-5], [0.0, 3e-5, -1e-5])]),
        ("LongitudinalRLCWake", [LongitudinalRLCWake(1.2e9, 2.0e5, 3.5, 2e-19)]),
        ("LongitudinalWake", [LongitudinalWake([0.0, 2e-12, 5e-12, 1e-11, 3e-11],
                                               [1e13, 6e12, 2e12, -1e12, 0.0], fliphalf=-3.0, scale=1e-19)]),
        ("Wiggler", [Wiggler(1.0, lw=0.1, Bmax=1.2, Nsteps=5, energy=3.5e9)]),
        ("WigglerHV", [Wiggler(0.25, lw=0.05, Bmax=0.8, Nsteps=4, By=(1, 1, 1, 1, 1, 0, 2, -1, 0, 3, 3, 1),
                               Bx=(1, 1, 1, 2, 2, 0), energy=3.5e9)]),
        ("WigglerRad", [Wiggler(0.3, lw=0.1, Bmax=1.5, Nsteps=3, energy=3.5e9, rad=1)]),
        ("LongitudinalWakeUnsorted", [LongitudinalWake([0.0, 5e-12, 2e-12, 1e-11], [1e13, 2e12, 6e12, -1e12],
                                                       fliphalf=-4.0, scale=2e-19)]),
    ]


def fodo_line():  # test/verify_fodo.jl:30-39
    return [Drift(1.0), Quadrupole(1.0, -0.9, num_int_steps=10), Drift(1.0), SBend(0.6, math.pi / 15.0),
            Drift(1.0), Quadrupole(1.0, 0.3, num_int_steps=10), Drift(1.0)]


def dba_line():  # test/verify_dba.jl:31-44
    a = math.pi / 9
    dl, ds = Drift(2.0), Drift(0.5)
    b = SBend(1.0, a, a / 2, a / 2)
    qf, qd = Quadrupole(0.4, 1.5), Quadrupole(0.4, -1.2)
    return [dl, b, ds, qf, ds, qd, ds, qf, ds, b, dl]


def fodo_ring():
    """The FODO cell of the CPU workload: QF(0.5, +1.2) D(2.0) QD(0.5, -1.2) D(2.0), 8 cells."""
    cell = [Quadrupole(0.5, 1.2), Drift(2.0), Quadrupole(0.5, -1.2), Drift(2.0)]
    return cell * 8


def main():
    energy = 3.5e9
    parts = PARTICLES
    cases = []
    for name, elems in element_cases(energy) + extra_cases(energy):
        cases.append(case(name, elems, parts, energy))
    for name, elems, rows, nturns in misalignment_cases(energy):
        cases.append(case(name, elems, parts, energy, nturns=nturns, misalign=rows))
    cases.append(case("FODO_line", fodo_line(), parts, energy))
    cases.append(case("DBA_line", dba_line(), parts, energy))
    cases.append(case("Bend_pi4", [SBend(1.0, math.pi / 4, math.pi / 8, math.pi / 8)], parts, energy))
    cases.append(case("ExactBend_pi9", [ExactSBend(1.0, math.pi / 9, math.pi / 18, math.pi / 18)], parts, energy))
    cases.append(case("FODO_ring_10turns", fodo_ring(), parts, 1.0e9, nturns=10, aperture=(0.05, 0.05)))
    # Loss semantics: amplitudes scaled up so that some particles cross the
    # aperture or the angle limit at different turns and elements.
    big = [[v * s for v in p] for p, s in zip(parts, [1, 2, 4, 6, 8, 10, 12, 14, 1500, 8000])]
    cases.append(case("FODO_ring_losses", fodo_ring(), big, 1.0e9, nturns=6, aperture=(0.01, 0.0075)))
    # Sextupoles make the large amplitudes unstable over several turns.
    cell = [Quadrupole(0.5, 1.2), Sextupole(0.2, 100.0), Drift(2.0), Quadrupole(0.5, -1.2),
            Sextupole(0.2, -100.0), Drift(2.0)]
    big = [[v * s for v in p] for p, s in zip(parts, range(1, 11))]
    cases.append(case("FODO_sext_losses", cell * 8, big, 1.0e9, nturns=20, aperture=(0.02, 0.015)))
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden_cases.json"), "w") as f:
        json.dump(dict(generator="tests/golden/make_golden.py", mass=M_ELECTRON, cases=cases), f, indent=1)
    print("wrote", len(cases), "cases")


if __name__ == "__main__":
    main()
