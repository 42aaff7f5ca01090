#!/usr/bin/env python3
"""Regenerates the golden fixtures in this directory.

Each case is a seeded synthetic target/query FASTA pair (clast_b200.synth)
plus the TSV that the reference itself writes for it: the reference's own
sources built for the CPU by oracle/build_ref.py (oracle/_ref/clast_ref).
Needs that build, i.e. the reference sources; the committed fixtures are used
wherever they are absent.

Usage: python tests/golden/make_golden.py
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402
from _fasta import write_pair, write_quirky  # noqa: E402

CASES = {
    # name: (input builder, extra flags)
    "default": (lambda d: write_pair(d, 901, target_bp=24_000, n_contigs=3, n_reads=60)[:2], []),
    "local": (lambda d: write_pair(d, 902, target_bp=24_000, n_contigs=3, n_reads=60)[:2], ["-local", "1"]),
    "small_l_wide_gap": (lambda d: write_pair(d, 903, target_bp=20_000, n_contigs=2, n_reads=50)[:2],
                         ["-lMer", "9", "-stride", "2", "-gap", "14", "-repeat", "6", "-numOut", "3"]),
    "loads_windows": (lambda d: write_pair(d, 904, target_bp=30_000, n_contigs=6, n_reads=80)[:2],
                      ["-tRAM", "0.012", "-qRAM", "0.008", "-tVRAM", "0.007", "-qVRAM", "0.002", "-cutOff", "-1"]),
    "quirky": (lambda d: (lambda t, qs: (t, qs[0]))(*write_quirky(d, 905)), ["-gap", "5"]),
}


def main():
    if not O.ref_available():
        sys.exit("the reference CPU build is missing: run python oracle/build_ref.py first")
    for name, (make, flags) in CASES.items():
        d = os.path.join(HERE, name)
        os.makedirs(d, exist_ok=True)
        tp, qp = make(d)
        os.replace(tp, os.path.join(d, "target.fa"))
        os.replace(qp, os.path.join(d, "query.fa"))
        for f in os.listdir(d):
            if f.endswith(".fa") and f not in ("target.fa", "query.fa"):
                os.remove(os.path.join(d, f))
        with open(os.path.join(d, "flags.txt"), "w") as fh:
            fh.write(" ".join(flags) + "\n")
        out = os.path.join(d, "reference.tsv")
        rc, log = O.run_ref(["-t", os.path.join(d, "target.fa"), "-q", os.path.join(d, "query.fa"), "-o", out]
                            + flags)
        if rc != 0:
            sys.exit("reference failed on %s: %s" % (name, log[-1000:]))
        print("%-18s %6d lines" % (name, sum(1 for _ in open(out))))


if __name__ == "__main__":
    main()
