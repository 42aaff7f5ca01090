"""Pins the oracle to the reference itself: the reference's own sources built
for the CPU (oracle/build_ref.py) and the oracle must write byte-identical
TSV files.  Skipped where the reference build is absent."""
import os

import pytest

import oracle as O
from _fasta import write_pair, write_quirky

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference CPU build absent (oracle/build_ref.py)")


def both(tmp, args):
    ro, oo = os.path.join(tmp, "ref.tsv"), os.path.join(tmp, "oracle.tsv")
    rc, log = O.run_ref(args + ["-o", ro])
    assert rc == 0, log[-2000:]
    rc, err = O.run_cli(args + ["-o", oo])
    assert rc == 0, err
    return open(ro, "rb").read(), open(oo, "rb").read()


@pytest.mark.parametrize("extra", [
    [],
    ["-local", "1"],
    ["-numOut", "2"],
    ["-cutOff", "-1", "-gap", "3"],
    ["-gap", "16"],
    ["-tRAM", "0.02", "-qRAM", "0.006"],
    ["-tVRAM", "0.012", "-qVRAM", "0.0015"],
    ["-lMer", "12", "-stride", "3", "-repeat", "4", "-width", "40"],
    ["-lMer", "21", "-stride", "1", "-repeat", "-1"],
])
def test_oracle_equals_reference(tmp_path, extra):
    tp, qp, _, _ = write_pair(str(tmp_path), 200 + len(extra), n_reads=120)
    a, b = both(str(tmp_path), ["-t", tp, "-q", qp] + extra)
    assert a.count(b"\n") > 30
    assert a == b


def test_oracle_equals_reference_quirky(tmp_path):
    tp, qps = write_quirky(str(tmp_path), 9)
    a, b = both(str(tmp_path), ["-t", tp, "-q"] + qps + ["-qRAM", "0.01"])
    assert a.count(b"\n") > 20
    assert a == b


def test_oracle_equals_reference_uneven(tmp_path):
    tp, qp, _, _ = write_pair(str(tmp_path), 300, n_reads=60, read_len=600, sub=0.05, indel=0.02)
    a, b = both(str(tmp_path), ["-t", tp, "-q", qp])
    assert a == b
