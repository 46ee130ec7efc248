"""asin, sin, cos, tan, atan by the published fdlibm method, in pure Python.

The golden-fixture generator evaluates the reference maps with these functions,
the same method (and operation order) the CUDA kernels and the CPU oracle use,
so that the fixtures, the oracle and the GPU agree bit for bit.  Python floats
are IEEE binary64 and Python never fuses a multiply-add.

The coefficient tables and branch structure follow fdlibm, whose routines carry
this notice:

    Copyright (C) 1993 by Sun Microsystems, Inc. All rights reserved.

    Developed at SunPro, a Sun Microsystems, Inc. business.
    Permission to use, copy, modify, and distribute this
    software is freely granted, provided that this notice
    is preserved.
"""
import math
import struct

PIO2_HI = 1.57079632679489655800e+00
PIO2_LO = 6.12323399573676603587e-17
PIO4_HI = 7.85398163397448278999e-01
PS = [1.66666666666666657415e-01, -3.25565818622400915405e-01, 2.01212532134862925881e-01,
      -4.00555345006794114027e-02, 7.91534994289814532176e-04, 3.47933107596021167570e-05]
QS = [-2.40339491173441421878e+00, 2.02094576023350569471e+00, -6.88283971605453293030e-01,
      7.70381505559019352791e-02]
S = [-1.66666666666666324348e-01, 8.33333333332248946124e-03, -1.98412698298579493134e-04,
     2.75573137070700676789e-06, -2.50507602534068634195e-08, 1.58969099521155010221e-10]
Cc = [4.16666666666666019037e-02, -1.38888888888741095749e-03, 2.48015872894767294178e-05,
      -2.75573143513906633035e-07, 2.08757232129817482790e-09, -1.13596475577881948265e-11]
T = [3.33333333333334091986e-01, 1.33333333333201242699e-01, 5.39682539762260521377e-02,
     2.18694882948595424599e-02, 8.86323982359930005737e-03, 3.59207910759131235356e-03,
     1.45620945432529025516e-03, 5.88041240820264096874e-04, 2.46463134818469906812e-04,
     7.81794442939557092300e-05, 7.14072491382608190305e-05, -1.85586374855275456654e-05,
     2.59073051863633712884e-05]
PIO4 = 7.85398163397448278999e-01
PIO4LO = 3.06161699786838301793e-17
INVPIO2 = 6.36619772367581382433e-01
PIO2_1, PIO2_1T = 1.57079632673412561417e+00, 6.07710050650619224932e-11
PIO2_2, PIO2_2T = 6.07710050630396597660e-11, 2.02226624879595063154e-21
PIO2_3, PIO2_3T = 2.02226624871116645580e-21, 8.47842766036889956997e-32
ATANHI = [4.63647609000806093515e-01, 7.85398163397448278999e-01, 9.82793723247329054082e-01,
          1.57079632679489655800e+00]
ATANLO = [2.26987774529616870924e-17, 3.06161699786838301793e-17, 1.39033110312309984516e-17,
          6.12323399573676603587e-17]
AT = [3.33333333333329318027e-01, -1.99999999998764832476e-01, 1.42857142725034663711e-01,
      -1.11111104054623557880e-01, 9.09088713343650656196e-02, -7.69187620504482999495e-02,
      6.66107313738753120669e-02, -5.83357013379057348645e-02, 4.97687799461593236017e-02,
      -3.65315727442169155270e-02, 1.62858201153657823623e-02]


def _bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def _from(u):
    return struct.unpack("<d", struct.pack("<Q", u))[0]


def _hix(x):
    return (_bits(x) >> 32) & 0x7fffffff


def _clear_low(x):
    return _from(_bits(x) & 0xffffffff00000000)


def _neg(x):
    return _from(_bits(x) ^ 0x8000000000000000)


def _signbit(x):
    return _bits(x) >> 63


def _expo(x):
    return (_bits(x) >> 52) & 0x7ff


def _asin_p(t):
    return t * (PS[0] + t * (PS[1] + t * (PS[2] + t * (PS[3] + t * (PS[4] + t * PS[5])))))


def _asin_q(t):
    return 1.0 + t * (QS[0] + t * (QS[1] + t * (QS[2] + t * QS[3])))


def asin(x):
    ix = _hix(x)
    ax = abs(x)
    if ix >= 0x3ff00000:
        if ax == 1.0:
            return x * PIO2_HI + x * PIO2_LO
        return math.nan
    if ix < 0x3fe00000:
        if ix < 0x3e500000:
            return x
        t = x * x
        w = _asin_p(t) / _asin_q(t)
        return x + x * w
    w = 1.0 - ax
    t = w * 0.5
    p, q = _asin_p(t), _asin_q(t)
    s = math.sqrt(t)
    if ix >= 0x3fef3333:
        w = p / q
        r = PIO2_HI - (2.0 * (s + s * w) - PIO2_LO)
    else:
        f = _clear_low(s)
        c = (t - f * f) / (s + f)
        rr = p / q
        pp = 2.0 * s * rr - (PIO2_LO - 2.0 * c)
        qq = PIO4_HI - 2.0 * f
        r = PIO4_HI - (pp - qq)
    return _neg(r) if _signbit(x) else r


def _k_sin(x, y, has_tail):
    z = x * x
    v = z * x
    r = S[1] + z * (S[2] + z * (S[3] + z * (S[4] + z * S[5])))
    if not has_tail:
        return x + v * (S[0] + z * r)
    return x - ((z * (0.5 * y - v * r) - y) - v * S[0])


def _k_cos(x, y):
    z = x * x
    r = z * (Cc[0] + z * (Cc[1] + z * (Cc[2] + z * (Cc[3] + z * (Cc[4] + z * Cc[5])))))
    hz = 0.5 * z
    w = 1.0 - hz
    return w + (((1.0 - w) - hz) + (z * r - x * y))


def _k_tan(x, y, iy):
    hx = _bits(x) >> 32
    ix = hx & 0x7fffffff
    big = ix >= 0x3fe59428
    if ix < 0x3e300000:
        if iy == 1:
            return x
        w = x + y
        z = _clear_low(w)
        v = y - (z - x)
        a = -1.0 / w
        t = _clear_low(a)
        s = 1.0 + t * z
        return t + a * (s + t * v)
    neg_in = bool(hx >> 31)
    if big:
        if neg_in:
            x, y = _neg(x), _neg(y)
        z = PIO4 - x
        w = PIO4LO - y
        x = z + w
        y = 0.0
    z = x * x
    w = z * z
    r = T[1] + w * (T[3] + w * (T[5] + w * (T[7] + w * (T[9] + w * T[11]))))
    v = z * (T[2] + w * (T[4] + w * (T[6] + w * (T[8] + w * (T[10] + w * T[12])))))
    s = z * x
    r = y + z * (s * (r + v) + y)
    r = r + T[0] * s
    w = x + r
    if big:
        vv = float(iy)
        res = vv - 2.0 * (x - (w * w / (w + vv) - r))
        return _neg(res) if neg_in else res
    if iy == 1:
        return w
    zz = _clear_low(w)
    vv = r - (zz - x)
    a = -1.0 / w
    t = _clear_low(a)
    ss = 1.0 + t * zz
    return t + a * (ss + t * vv)


def _rem_pio2(x):
    t = abs(x)
    n = int(t * INVPIO2 + 0.5)
    fn = float(n)
    r = t - fn * PIO2_1
    w = fn * PIO2_1T
    j = _expo(t)
    a = r - w
    if j - _expo(a) > 16:
        tt = r
        w = fn * PIO2_2
        r = tt - w
        w = fn * PIO2_2T - ((tt - r) - w)
        a = r - w
        if j - _expo(a) > 49:
            tt = r
            w = fn * PIO2_3
            r = tt - w
            w = fn * PIO2_3T - ((tt - r) - w)
            a = r - w
    b = (r - a) - w
    if _signbit(x):
        return (-n) & 3, _neg(a), _neg(b)
    return n & 3, a, b


HI_PIO4 = 0x3fe921fb
HI_MEDIUM = 0x413921fb


def sin(x):
    ix = _hix(x)
    if ix <= HI_PIO4:
        if ix < 0x3e500000:
            return x
        return _k_sin(x, 0.0, False)
    if ix >= 0x7ff00000:
        return x - x
    if ix >= HI_MEDIUM:
        return math.sin(x)
    n, y0, y1 = _rem_pio2(x)
    return [lambda: _k_sin(y0, y1, True), lambda: _k_cos(y0, y1), lambda: _neg(_k_sin(y0, y1, True)),
            lambda: _neg(_k_cos(y0, y1))][n]()


def cos(x):
    ix = _hix(x)
    if ix <= HI_PIO4:
        if ix < 0x3e46a09e:
            return 1.0
        return _k_cos(x, 0.0)
    if ix >= 0x7ff00000:
        return x - x
    if ix >= HI_MEDIUM:
        return math.cos(x)
    n, y0, y1 = _rem_pio2(x)
    return [lambda: _k_cos(y0, y1), lambda: _neg(_k_sin(y0, y1, True)), lambda: _neg(_k_cos(y0, y1)),
            lambda: _k_sin(y0, y1, True)][n]()


def tan(x):
    ix = _hix(x)
    if ix <= HI_PIO4:
        return _k_tan(x, 0.0, 1)
    if ix >= 0x7ff00000:
        return x - x
    if ix >= HI_MEDIUM:
        return math.tan(x)
    n, y0, y1 = _rem_pio2(x)
    return _k_tan(y0, y1, -1 if (n & 1) else 1)


def atan(x):
    ix = _hix(x)
    negx = _signbit(x)
    if ix >= 0x44100000:
        if x != x:
            return x + x
        r = ATANHI[3] + ATANLO[3]
        return _neg(r) if negx else r
    if ix < 0x3fdc0000:
        if ix < 0x3e400000:
            return x
        idx = -1
    else:
        x = abs(x)
        if ix < 0x3ff30000:
            if ix < 0x3fe60000:
                idx = 0
                x = (2.0 * x - 1.0) / (2.0 + x)
            else:
                idx = 1
                x = (x - 1.0) / (x + 1.0)
        else:
            if ix < 0x40038000:
                idx = 2
                x = (x - 1.5) / (1.0 + 1.5 * x)
            else:
                idx = 3
                x = -1.0 / x
    z = x * x
    w = z * z
    s1 = z * (AT[0] + w * (AT[2] + w * (AT[4] + w * (AT[6] + w * (AT[8] + w * AT[10])))))
    s2 = w * (AT[1] + w * (AT[3] + w * (AT[5] + w * (AT[7] + w * AT[9]))))
    if idx < 0:
        return x - x * (s1 + s2)
    r = ATANHI[idx] - ((x * (s1 + s2) - ATANLO[idx]) - x)
    return _neg(r) if negx else r


# exp, expm1, sinh, cosh (fdlibm method; same reduction, polynomials and
# branch points as tp_libm.h)
LN2_HI, LN2_LO, INV_LN2 = 6.93147180369123816490e-01, 1.90821492927058770002e-10, 1.44269504088896338700e+00
EXP_P = [1.66666666666666019037e-01, -2.77777777770155933842e-03, 6.61375632143793436117e-05,
         -1.65339022054652515390e-06, 4.13813679705723846039e-08]
EXP_OVER, EXP_UNDER = 7.09782712893383973096e+02, -7.45133219101941108420e+02
EM1_Q = [-3.33333333333331316428e-02, 1.58730158725481460165e-03, -7.93650757867487942473e-05,
         4.00821782732936239552e-06, -2.01099218183624371326e-07]
TWO_M1000 = 9.33263618503218878990e-302


def _add_expo(y, k):
    return _from((_bits(y) + (k << 52)) & 0xffffffffffffffff)


def _trunc(v):
    return int(v)  # C conversion: toward zero


def exp(x):
    hx = _hix(x)
    neg = _signbit(x) == 1
    if hx >= 0x40862E42:
        if hx >= 0x7ff00000:
            if _bits(x) & 0x000fffffffffffff:
                return x + x
            return 0.0 if neg else x
        if x > EXP_OVER:
            return math.inf
        if x < EXP_UNDER:
            return 0.0
    hi = lo = 0.0
    k = 0
    if hx > 0x3fd62e42:
        if hx < 0x3FF0A2B2:
            hi = x + LN2_HI if neg else x - LN2_HI
            lo = -LN2_LO if neg else LN2_LO
            k = -1 if neg else 1
        else:
            k = _trunc(INV_LN2 * x + (-0.5 if neg else 0.5))
            t = float(k)
            hi = x - t * LN2_HI
            lo = t * LN2_LO
        r = hi - lo
    elif hx < 0x3e300000:
        return 1.0 + x
    else:
        r = x
    t = r * r
    c = r - t * (EXP_P[0] + t * (EXP_P[1] + t * (EXP_P[2] + t * (EXP_P[3] + t * EXP_P[4]))))
    if k == 0:
        return 1.0 - ((r * c) / (c - 2.0) - r)
    y = 1.0 - ((lo - (r * c) / (2.0 - c)) - hi)
    if k >= -1021:
        return _add_expo(y, k)
    return _add_expo(y, k + 1000) * TWO_M1000


def expm1(x):
    hx = _hix(x)
    neg = _signbit(x) == 1
    if hx >= 0x4043687A:
        if hx >= 0x40862E42:
            if hx >= 0x7ff00000:
                if _bits(x) & 0x000fffffffffffff:
                    return x + x
                return -1.0 if neg else x
            if x > EXP_OVER:
                return math.inf
        if neg:
            return -1.0
    c = 0.0
    k = 0
    if hx > 0x3fd62e42:
        if hx < 0x3FF0A2B2:
            if not neg:
                hi, lo, k = x - LN2_HI, LN2_LO, 1
            else:
                hi, lo, k = x + LN2_HI, -LN2_LO, -1
        else:
            k = _trunc(INV_LN2 * x + (-0.5 if neg else 0.5))
            t = float(k)
            hi = x - t * LN2_HI
            lo = t * LN2_LO
        x = hi - lo
        c = (hi - x) - lo
    elif hx < 0x3c900000:
        return x
    hfx = 0.5 * x
    hxs = x * hfx
    r1 = 1.0 + hxs * (EM1_Q[0] + hxs * (EM1_Q[1] + hxs * (EM1_Q[2] + hxs * (EM1_Q[3] + hxs * EM1_Q[4]))))
    t = 3.0 - r1 * hfx
    e = hxs * ((r1 - t) / (6.0 - x * t))
    if k == 0:
        return x - (x * e - hxs)
    e = x * (e - c) - c
    e = e - hxs
    if k == -1:
        return 0.5 * (x - e) - 0.5
    if k == 1:
        if x < -0.25:
            return -2.0 * (e - (x + 0.5))
        return 1.0 + 2.0 * (x - e)
    if k <= -2 or k > 56:
        y = 1.0 - (e - x)
        return _add_expo(y, k) - 1.0
    if k < 20:
        t1 = _from((0x3ff00000 - (0x200000 >> k)) << 32)
        return _add_expo(t1 - (e - x), k)
    t2 = _from(((0x3ff - k) << 20) << 32)
    y = x - (e + t2)
    y = y + 1.0
    return _add_expo(y, k)


def sinh(x):
    ix = _hix(x)
    if ix >= 0x7ff00000:
        return x + x
    h = -0.5 if _signbit(x) else 0.5
    ax = abs(x)
    if ix < 0x40360000:
        if ix < 0x3e300000:
            return x
        t = expm1(ax)
        if ix < 0x3ff00000:
            return h * (2.0 * t - (t * t) / (t + 1.0))
        return h * (t + t / (t + 1.0))
    if ix < 0x40862E42:
        return h * exp(ax)
    w = exp(0.5 * ax)
    return (h * w) * w


def cosh(x):
    ix = _hix(x)
    if ix >= 0x7ff00000:
        return x * x
    ax = abs(x)
    if ix < 0x3fd62e43:
        t = expm1(ax)
        w = 1.0 + t
        if ix < 0x3c800000:
            return w
        return 1.0 + (t * t) / (w + w)
    if ix < 0x40360000:
        t = exp(ax)
        return 0.5 * t + 0.5 / t
    if ix < 0x40862E42:
        return 0.5 * exp(ax)
    w = exp(0.5 * ax)
    return (0.5 * w) * w
