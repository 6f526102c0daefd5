"""The double-double pow/exp/log shared by the oracle and the engine
(pangu_b200/csrc/pgmath.h): correctly rounded against 60-digit decimal
arithmetic, and close to the C library's (which misrounds some results)."""
import ctypes as C
from decimal import Decimal, getcontext

import numpy as np

import pyoracle as po

getcontext().prec = 60
L = po.lib()
_D = C.POINTER(C.c_double)


def _pow(x, y):
    out = np.empty_like(x)
    L.or_pgm_pow(len(x), x.ctypes.data_as(_D), y.ctypes.data_as(_D), out.ctypes.data_as(_D))
    return out


def _exp(x):
    out = np.empty_like(x)
    L.or_pgm_exp(len(x), x.ctypes.data_as(_D), out.ctypes.data_as(_D))
    return out


def _log(x):
    out = np.empty_like(x)
    L.or_pgm_log(len(x), x.ctypes.data_as(_D), out.ctypes.data_as(_D))
    return out


def _is_correctly_rounded(v, exact):
    """|v - exact| <= half an ulp of v."""
    v = float(v)
    ulp = np.spacing(abs(v))
    return abs(Decimal(v) - exact) <= Decimal(ulp) / 2


def test_pow_correctly_rounded():
    rng = np.random.default_rng(7)
    x = 10 ** rng.uniform(-10, 6, 3000)
    y = rng.choice([5 / 3, -5 / 3, 4 / 3, -4 / 3, 2 / 3, -1.5, -2.5, 0.7, -1.4, 3.3], 3000)
    out = _pow(x, y)
    for xi, yi, oi in zip(x, y, out):
        exact = (Decimal(float(xi)).ln() * Decimal(float(yi))).exp()
        assert _is_correctly_rounded(oi, exact), (xi.hex(), yi.hex(), oi.hex())


def _pow_slow(x, y):
    out = np.empty_like(x)
    L.or_pgm_pow_slow(len(x), x.ctypes.data_as(_D), y.ctypes.data_as(_D),
                      out.ctypes.data_as(_D))
    return out


def test_fast_path_agrees_with_slow_path():
    """The table-driven fast path returns a result only when its error bound
    guarantees the rounding; it must then agree with the 2^-95 slow path
    everywhere: physics exponents over the floor-to-torus range of values,
    arbitrary exponents, and arguments near 1 and near table boundaries."""
    rng = np.random.default_rng(11)
    n = 400000
    cases = [
        (10 ** rng.uniform(-12, 6, n),
         rng.choice([5 / 3, -5 / 3, 4 / 3, -4 / 3, 1 / 3, 2 / 3, -1.5, -2.5, 0.7, -1.4, 3.3], n)),
        (10 ** rng.uniform(-300, 300, n), rng.uniform(-1.0, 1.0, n)),
        (10 ** rng.uniform(-6, 6, n), rng.uniform(-40.0, 40.0, n)),
        (1.0 + rng.uniform(-1e-3, 1e-3, n), rng.uniform(-1e4, 1e4, n)),
        (np.ldexp(rng.uniform(0.70, 1.42, n), rng.integers(-60, 60, n)),
         rng.uniform(-8.0, 8.0, n)),
    ]
    for x, y in cases:
        fast, slow = _pow(x, y), _pow_slow(x, y)
        bad = fast != slow
        assert not bad.any(), (x[bad][:3], y[bad][:3], fast[bad][:3], slow[bad][:3])


def _pow_fast(x, y):
    out = np.empty_like(x)
    ok = np.empty(len(x), dtype=np.int32)
    L.or_pgm_pow_fast(len(x), x.ctypes.data_as(_D), y.ctypes.data_as(_D),
                      out.ctypes.data_as(_D), ok.ctypes.data_as(C.POINTER(C.c_int)))
    return out, ok.astype(bool)


def test_fast_path_next_to_one():
    """The log intervals next to the one centred on 1 carry the largest
    relative error of the fast path's log (|ln m| down to 2^-10 with the
    product's low part up to 2^-53); large exponents magnify it in t."""
    rng = np.random.default_rng(12)
    n = 300000
    side = rng.choice([-1.0, 1.0], n)
    x = 1.0 + side * rng.uniform(1 / 1024, 3 / 1024, n)
    y = rng.uniform(-2.5e5, 2.5e5, n)
    fast, ok = _pow_fast(x, y)
    slow = _pow_slow(x, y)
    assert np.array_equal(fast[ok], slow[ok])
    for xi, yi, oi in list(zip(x[ok], y[ok], fast[ok]))[:300]:
        exact = (Decimal(float(xi)).ln() * Decimal(float(yi))).exp()
        assert _is_correctly_rounded(oi, exact), (xi.hex(), yi.hex(), oi.hex())


def test_fast_path_decides_almost_always():
    """With the physics exponents over the floor-to-torus range of values the
    fast path decides nearly every rounding (a warp waits for any lane that
    falls to the slow path)."""
    rng = np.random.default_rng(13)
    n = 400000
    x = 10 ** rng.uniform(-12, 6, n)
    y = rng.choice([-13 / 9, -4 / 3, -5 / 3, 13 / 9 - 4 / 3, 1 / 3, 0.7, -1.4, 3.3], n)
    fast, ok = _pow_fast(x, y)
    assert ok.mean() > 0.99999, ok.mean()
    assert np.array_equal(fast[ok], _pow(x[ok], y[ok]))


def test_log_table_binades():
    """The fast path sums L_j + r with an ordered (fast) two-sum: in every
    interval with L_j != 0, |L_j| lies in a higher binade than any |r|."""
    import math
    import os
    import re
    here = os.path.dirname(os.path.abspath(__file__))
    txt = open(os.path.join(here, "..", "pangu_b200", "csrc", "pgmath_tables.h")).read()
    m0 = float.fromhex(re.search(r"#define PGM_LOG_M0 (\S+)", txt).group(1))
    body = txt.split("PGM_LOG_TABLE_INIT {")[1].split("}")[0]
    vals = [0.0 if v == "0.0" else float.fromhex(v)
            for v in re.findall(r"(-?0x[0-9a-fp.+-]+|0\.0)", body)]
    for j in range(len(vals) // 3):
        inv, lh = vals[3 * j], vals[3 * j + 1]
        lo, hi = max(m0 + j / 512, 2 ** -0.5), min(m0 + (j + 1) / 512, 2 ** 0.5)
        rmax = max(abs(lo * inv - 1.0), abs(hi * inv - 1.0))
        assert rmax < 2 ** -9.49
        if lh == 0.0:
            assert inv == 1.0
            continue
        assert math.frexp(abs(lh))[1] > math.frexp(rmax)[1], j


def test_fast_path_error_bounds():
    """The bounds the fast path's rounding test relies on, against 60-digit
    decimals: the log within 2^-80.5 + 2^-84 |ln x| (arguments next to 1,
    at the edges of the table's intervals and of [1/sqrt2, sqrt2), and over
    the whole range), the exp within a relative 2^-76.9 (over |t| < 700,
    with the largest reduced arguments, and with a low part)."""
    rng = np.random.default_rng(14)
    n = 1500
    xs = np.concatenate([
        1.0 + rng.choice([-1.0, 1.0], n) * rng.uniform(1 / 1024, 3 / 1024, n),
        1.0 + rng.uniform(-1 / 1024, 1 / 1024, n),
        (361.5 + rng.integers(0, 363, n) + rng.choice([1e-7, -1e-7, 0.5], n)) / 512,
        10 ** rng.uniform(-300, 300, n),
        np.ldexp(rng.choice([2 ** -0.5, 2 ** 0.5], n) * (1 + rng.uniform(-1e-3, 1e-3, n)),
                 rng.integers(-5, 5, n)),
    ])
    hi, lo = np.empty_like(xs), np.empty_like(xs)
    L.or_pgm_log_fast(len(xs), xs.ctypes.data_as(_D), hi.ctypes.data_as(_D),
                      lo.ctypes.data_as(_D))
    two = Decimal(2)
    for x, h, l in zip(xs, hi, lo):
        exact = Decimal(float(x)).ln()
        err = abs(Decimal(float(h)) + Decimal(float(l)) - exact)
        assert err <= two ** Decimal("-80.5") + two ** -84 * abs(exact), float(x).hex()
    k = rng.integers(-120000, 120000, n)
    th = np.concatenate([rng.uniform(-699, 699, n),
                         (k + 0.5) * np.log(2) / 128 * (1 + rng.uniform(-1e-12, 1e-12, n)),
                         rng.uniform(-0.01, 0.01, n)])
    tl = th * np.concatenate([rng.uniform(-2 ** -43, 2 ** -43, n), np.zeros(n),
                              rng.uniform(-2 ** -52, 2 ** -52, n)])
    hi, lo = np.empty_like(th), np.empty_like(th)
    sc = np.empty(len(th), dtype=np.int32)
    L.or_pgm_exp_fast(len(th), th.ctypes.data_as(_D), tl.ctypes.data_as(_D),
                      hi.ctypes.data_as(_D), lo.ctypes.data_as(_D),
                      sc.ctypes.data_as(C.POINTER(C.c_int)))
    for a, b, h, l, s in zip(th, tl, hi, lo, sc):
        exact = (Decimal(float(a)) + Decimal(float(b))).exp()
        v = (Decimal(float(h)) + Decimal(float(l))) * two ** int(s)
        assert abs(v - exact) / exact <= two ** Decimal("-76.9"), (float(a).hex(), float(b).hex())


def test_exp_log_correctly_rounded():
    rng = np.random.default_rng(8)
    e = rng.uniform(-700, 700, 2000)
    for xi, oi in zip(e, _exp(e)):
        assert _is_correctly_rounded(oi, Decimal(float(xi)).exp())
    l = 10 ** rng.uniform(-300, 300, 2000)
    for xi, oi in zip(l, _log(l)):
        assert _is_correctly_rounded(oi, Decimal(float(xi)).ln())


def test_agrees_with_c_library_within_one_ulp():
    rng = np.random.default_rng(9)
    x = 10 ** rng.uniform(-12, 6, 200000)
    y = rng.uniform(-5, 5, 200000)
    ref = np.power(x, y)
    out = _pow(x, y)
    assert np.all(np.abs(out - ref) <= np.spacing(np.abs(ref)))
    assert np.mean(out == ref) > 0.9


def test_special_values():
    inf, nan = np.inf, np.nan
    xs = np.array([0.0, -0.0, 0.0, 1.0, 2.0, -2.0, -2.0, inf, inf, 0.5, 2.0, nan, 1.0, -8.0])
    ys = np.array([2.0, 3.0, -1.0, nan, 0.0, 3.0, 0.5, 2.0, -2.0, inf, -inf, 0.0, inf, 1 / 3])
    ref = np.power(xs, ys)
    out = _pow(xs, ys)
    np.testing.assert_array_equal(np.isnan(out), np.isnan(ref))
    ok = ~np.isnan(ref)
    np.testing.assert_array_equal(out[ok], ref[ok])
