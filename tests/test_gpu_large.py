"""Parity at the window sizes of the large-genome configuration: two
chromosomes of 125 Mbp from the 3 Gbp shape (45 % repeats in families at
80-99 % identity, 1 % N blocks) in ONE target window of 250 Mbp
(-tRAM 260 -tVRAM 260, as that configuration needs), 6,000 reads of 150 bp.
At this size the index holds 50 M samples: its hash table is past 100 M
records, the filter is at its size cap with under 3 bits per key, and
entry offsets and record homes use their full ranges.  The drop-in command
line on the GPU and the oracle's command line must write the same bytes."""
import os

import numpy as np
import pytest

import oracle as O
from clast_b200 import api, synth

pytestmark = pytest.mark.gpu


def test_250_mbp_window_matches_oracle(tmp_path):
    rng = np.random.Generator(np.random.PCG64(0x1A76E))
    lens = np.array([125_000_000, 125_000_000], dtype=np.int64)
    t = synth.make_target(rng, int(lens.sum()), lengths=lens, n_frac=0.01, n_run_mean=1000.0, repeat_frac=0.45,
                          n_families=84, fam_ident=(0.80, 0.99))
    t.labels = ["chr1", "chr2"]
    q = synth.make_reads_fixed(rng, t, 6000)
    tp, qp = str(tmp_path / "t.fa"), str(tmp_path / "q.fa")
    t.to_fasta(tp)
    q.to_fasta(qp)
    flags = ["-tRAM", "260", "-tVRAM", "260"]
    og, oo = str(tmp_path / "g.tsv"), str(tmp_path / "o.tsv")
    rc, err = api.run_clast(["-t", tp, "-q", qp, "-o", og] + flags)
    assert rc == 0, err
    rc, err = O.run_cli(["-t", tp, "-q", qp, "-o", oo] + flags)
    assert rc == 0, err
    a, b = open(og, "rb").read(), open(oo, "rb").read()
    assert b.count(b"\n") > 5000
    assert a == b
