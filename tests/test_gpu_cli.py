"""The drop-in command line on the GPU against the oracle's: same FASTA in,
byte-identical TSV out.  Covers RAM loads, VRAM windows, local mode, numOut,
cutOff -1 and the FASTA loader's special cases."""
import os

import pytest

import oracle as O
from clast_b200 import api
from _fasta import write_adversarial, write_pair, write_quirky

pytestmark = pytest.mark.gpu


def run_both(tmp_path, args):
    og, oo = os.path.join(tmp_path, "gpu.tsv"), os.path.join(tmp_path, "oracle.tsv")
    rc, err = api.run_clast(args + ["-o", og])
    assert rc == 0, err
    rc, err = O.run_cli(args + ["-o", oo])
    assert rc == 0, err
    a, b = open(og, "rb").read(), open(oo, "rb").read()
    return a, b


@pytest.mark.parametrize("extra", [
    [],
    ["-local", "1"],
    ["-numOut", "1"],
    ["-cutOff", "-1", "-gap", "4"],
    ["-tRAM", "0.02", "-qRAM", "0.006"],            # several RAM loads on both sides
    ["-tVRAM", "0.012", "-qVRAM", "0.0015"],        # several VRAM windows per load
    ["-lMer", "12", "-stride", "3", "-repeat", "4", "-width", "40"],
])
def test_cli_matches_oracle(tmp_path, extra):
    tp, qp, _, _ = write_pair(str(tmp_path), 100 + len(extra))
    a, b = run_both(str(tmp_path), ["-t", tp, "-q", qp] + extra)
    assert b.count(b"\n") > 50
    assert a == b


def test_cli_quirky_fasta(tmp_path):
    tp, qps = write_quirky(str(tmp_path), 7)
    a, b = run_both(str(tmp_path), ["-t", tp, "-q"] + qps + ["-qRAM", "0.01"])
    assert b.count(b"\n") > 20
    assert a == b


@pytest.mark.parametrize("budgets", [[], ["-tRAM", "0.02", "-qRAM", "0.012"]])
def test_cli_adversarial_fasta(tmp_path, budgets):
    tp, qps = write_adversarial(str(tmp_path), 11)
    a, b = run_both(str(tmp_path), ["-t", tp, "-q"] + qps + budgets)
    assert b.count(b"\n") > 20
    assert a == b
