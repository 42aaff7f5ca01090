"""The number format of the device-side result text (clast_format_tsv), run
on the host: every double the GPU writes must read exactly as the C
library's printf("%g") writes it (std::ostream's default, 6 significant
digits, round half to even); values whose rounding the device cannot decide
(only non-finite ones here) are left to the host, which uses printf itself."""
import ctypes as C

import numpy as np
import pytest

from clast_b200 import _native as N


@pytest.fixture(scope="module")
def fmt():
    lib = C.CDLL(N.LIB_PATH)
    f = lib.clast_format_g6_host
    f.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    libc = C.CDLL("libc.so.6")
    buf = C.create_string_buffer(64)

    def run(vals):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        out = np.zeros(32 * len(v), dtype=np.uint8)
        lens = np.zeros(len(v), dtype=np.int32)
        assert f(v.ctypes.data, len(v), out.ctypes.data, lens.ctypes.data) == 0
        bad, undecided = [], 0
        for i, x in enumerate(v):
            if lens[i] < 0:
                undecided += 1
                continue
            libc.snprintf(buf, 64, b"%g", C.c_double(x))
            got = bytes(out[32 * i:32 * i + lens[i]])
            if got != buf.value:
                bad.append((float(x), got, buf.value))
        return bad, undecided

    return run


def test_evalues(fmt):
    rng = np.random.default_rng(1)
    score = rng.integers(0, 600, 40000)
    ev = 0.71 * 1e8 * rng.integers(20, 10000, 40000) * np.exp(-1.37 * score)
    bad, und = fmt(ev)
    assert not bad and und == 0, bad[:5]


def test_match_percentages(fmt):
    rng = np.random.default_rng(2)
    m = rng.integers(-3000, 10000, 40000)
    q = rng.integers(1, 10000, 40000)
    bad, und = fmt((m * 100).astype(np.float64) / q)
    assert not bad and und == 0, bad[:5]


def test_exact_ties_and_edges(fmt):
    vals = [7900 / 128, 12.34375, 0.5, 2.5, 1234565.0, 12345650.0, 99999.95, 999999.5, 9999995.0, 1e-5, 1e-4,
            0.0001234565, 100000.0, 1e6, -0.0, 0.0, 123456789.0, 1e-300, 5e-324, 2.2250738585072014e-308,
            1.7976931348623157e308, -42.0]
    bad, und = fmt(vals)
    assert not bad and und == 0, bad
    bad, und = fmt([np.inf, -np.inf, np.nan])
    assert und == 3


def test_random_bit_patterns(fmt):
    rng = np.random.default_rng(3)
    x = rng.integers(0, 2 ** 63 - 1, 60000, dtype=np.int64).view(np.float64)
    x = x[np.isfinite(x)]
    bad, und = fmt(np.concatenate([x, -x[:1000]]))
    assert not bad and und == 0, bad[:5]


def test_near_decimal_midpoints(fmt):
    # nearest doubles to 7-digit decimals ending in 5: the hardest roundings;
    # a few may be left to the host, none may differ
    rng = np.random.default_rng(4)
    mant = rng.integers(1000000, 9999999, 20000) // 10 * 10 + 5
    ex = rng.integers(-40, 40, 20000)
    vals = np.array([float("%de%d" % (a, b)) for a, b in zip(mant, ex)])
    bad, und = fmt(vals)
    assert not bad, bad[:5]
    assert und < len(vals) // 20
