"""clast_write_file (the result text's writer, used by the command line and
TsvText.write) on the host: every size and thread count gives the bytes
back exactly, an existing longer file is truncated, files that cannot be
mapped take positional writes, and an unwritable path is an error."""
import ctypes as C
import os

import numpy as np
import pytest

from clast_b200 import _native as N


@pytest.fixture(scope="module")
def lib():
    return N.load()


def write(lib, path, data, threads):
    buf = C.create_string_buffer(data, len(data)) if data else None
    return lib.clast_write_file(os.fsencode(path), C.cast(buf, C.c_void_p) if buf else None, len(data), threads)


@pytest.mark.parametrize("n", [0, 1, 4095, 4097, (4 << 20) + 3, (9 << 20) + 4097, 33 << 20])
@pytest.mark.parametrize("threads", [1, 3, 8])
def test_bytes_back_exactly(lib, tmp_path, n, threads):
    data = np.random.Generator(np.random.PCG64(n + threads)).integers(0, 256, size=n, dtype=np.uint8).tobytes()
    p = tmp_path / "out.tsv"
    assert write(lib, p, data, threads) == 0
    assert p.read_bytes() == data


def test_longer_file_is_truncated(lib, tmp_path):
    p = tmp_path / "out.tsv"
    p.write_bytes(b"x" * 100_000)
    assert write(lib, p, b"abc\n", 4) == 0
    assert p.read_bytes() == b"abc\n"


def test_unmappable_target_and_bad_path(lib, tmp_path):
    assert write(lib, "/dev/null", b"y" * (5 << 20), 4) == 0  # a device: positional writes
    assert write(lib, tmp_path / "no" / "such" / "dir.tsv", b"z", 2) != 0
    assert lib.clast_write_file(None, None, 0, 1) != 0
