"""Golden fixtures: TSV files the reference itself wrote (its sources built
for the CPU, tests/golden/make_golden.py) for small seeded inputs.  The
oracle must reproduce them on the CPU, and the CUDA path on the GPU."""
import os

import pytest

import oracle as O
from clast_b200 import api

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(d for d in os.listdir(HERE) if os.path.isdir(os.path.join(HERE, d)))


def args_of(name, out):
    d = os.path.join(HERE, name)
    flags = open(os.path.join(d, "flags.txt")).read().split()
    return ["-t", os.path.join(d, "target.fa"), "-q", os.path.join(d, "query.fa"), "-o", out] + flags


def golden(name):
    return open(os.path.join(HERE, name, "reference.tsv"), "rb").read()


def test_cases_present():
    assert len(CASES) >= 5


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_tsv(name, tmp_path):
    out = str(tmp_path / "o.tsv")
    rc, err = O.run_cli(args_of(name, out))
    assert rc == 0, err
    assert open(out, "rb").read() == golden(name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_reproduces_reference_tsv(name, tmp_path):
    out = str(tmp_path / "g.tsv")
    rc, err = api.run_clast(args_of(name, out))
    assert rc == 0, err
    assert open(out, "rb").read() == golden(name)
