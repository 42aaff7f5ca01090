"""The %g formatter of the result text, run as a kernel on the GPU (the path
clast_format_tsv takes), against the C library's printf: every value the
device writes must read exactly as printf("%g") writes it."""
import ctypes as C

import numpy as np
import pytest

from clast_b200 import _native as N

pytestmark = pytest.mark.gpu


def test_device_digits_equal_printf(engine):
    lib = C.CDLL(N.LIB_PATH)
    f = lib.clast_format_g6_device
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    libc = C.CDLL("libc.so.6")
    rng = np.random.default_rng(11)
    score = rng.integers(0, 800, 30000)
    ev = 0.71 * 1e8 * rng.integers(20, 10000, 30000) * np.exp(-1.37 * score)
    pct = (rng.integers(-3000, 10000, 20000) * 100).astype(np.float64) / rng.integers(1, 10000, 20000)
    bits = rng.integers(0, 2 ** 63 - 1, 20000, dtype=np.int64).view(np.float64)
    edges = [7900 / 128, 12.34375, 0.5, 2.5, 1234565.0, 999999.5, 1e-5, 1e-4, 100000.0, 1e6, -0.0, 0.0, 5e-324,
             1.7976931348623157e308, 98.6667, 1.08231e-62, 0.00216598]
    v = np.ascontiguousarray(np.concatenate([ev, pct, bits[np.isfinite(bits)], edges]), dtype=np.float64)
    out = np.zeros(32 * len(v), dtype=np.uint8)
    lens = np.zeros(len(v), dtype=np.int32)
    assert f(engine.ctx, v.ctypes.data, len(v), out.ctypes.data, lens.ctypes.data) == 0
    buf = C.create_string_buffer(64)
    bad = []
    for i, x in enumerate(v):
        if lens[i] < 0:
            continue
        libc.snprintf(buf, 64, b"%g", C.c_double(x))
        got = bytes(out[32 * i:32 * i + lens[i]])
        if got != buf.value:
            bad.append((float(x), got, buf.value))
    assert (lens >= 0).mean() > 0.999
    assert not bad, bad[:5]
