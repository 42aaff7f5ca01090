"""Bit-exact parity on the benchmark configurations themselves, not only on
small cases: the drop-in command line on the GPU, and the whole-job API
(targets + map + format_tsv), against the oracle's command line (OpenMP on
the host cores), byte-identical TSV.

* small: the 1 Mbp single-record target with 0.1 % N runs and its 1,000
  reads of 150 bp (5 % decoys), in full, default settings.
* medium target: the 100 Mbp / 200-contig target with its repeat families, in
  full, and the first 250,000 of its reads -- two query RAM loads (32 Mbase
  per load) against both 64 Mbase target windows, at default settings.  At
  this size the index paths that only large windows reach run: the filter
  at its size cap, the seed partitions sized from the query and rerun
  when one overflows (the first map of a fresh context), and the deferred
  table-overflow check.
"""
import os
import time

import numpy as np
import pytest

import oracle as O
from clast_b200 import api, synth

pytestmark = pytest.mark.gpu

T_RAM, Q_RAM, T_VRAM, Q_VRAM = 64_000_000, 64_000_000, 64_000_000, 2_000_000  # defaults (common.hpp:12-15)


def write(tmp, t, q):
    tp, qp = os.path.join(tmp, "t.fa"), os.path.join(tmp, "q.fa")
    t.to_fasta(tp)
    q.to_fasta(qp)
    return tp, qp


def cli_pair(tmp, tp, qp, extra=()):
    og, oo = os.path.join(tmp, "gpu.tsv"), os.path.join(tmp, "oracle.tsv")
    rc, err = api.run_clast(["-t", tp, "-q", qp, "-o", og] + list(extra))
    assert rc == 0, err
    t0 = time.perf_counter()
    rc, err = O.run_cli(["-t", tp, "-q", qp, "-o", oo] + list(extra))
    assert rc == 0, err
    print("oracle: %.1f s" % (time.perf_counter() - t0))
    return open(og, "rb").read(), open(oo, "rb").read()


def api_text(engine, t, q):
    """targets + map + format_tsv on the same records (the bench's path)."""
    s = api.Setting(total_db=float(t.offsets[-1]))  # every non-'>' line of the FASTA is bases
    keep_t, t_loads = api.ram_loads(np.diff(t.offsets), T_RAM)
    keep_q, q_loads = api.ram_loads(np.diff(q.offsets), Q_RAM // 2)
    assert keep_t.all() and keep_q.all()
    T = engine.targets(s, t.bases, t.offsets, t_loads, T_VRAM)
    res = engine.map(s, T, q.bases, q.offsets, q_loads, Q_VRAM)
    text = engine.format_tsv(T, res, q.labels, t.labels)
    del res
    T.close()
    return text, q_loads


def test_small_config_in_full(tmp_path, engine):
    t, q = synth.workload("small")
    assert len(t) == 1 and t.offsets[-1] == 1_000_000 and len(q) == 1000
    assert (t.bases == ord("N")).any()
    tp, qp = write(str(tmp_path), t, q)
    a, b = cli_pair(str(tmp_path), tp, qp)
    assert b.count(b"\n") > 500
    assert a == b
    text, _ = api_text(engine, t, q)
    assert text == b


def test_small_config_local_mode(tmp_path):
    t, q = synth.workload("small")
    tp, qp = write(str(tmp_path), t, q)
    a, b = cli_pair(str(tmp_path), tp, qp, ["-local", "1"])
    assert b.count(b"\n") > 500
    assert a == b


def test_medium_target_two_query_loads(tmp_path, engine):
    t, q = synth.workload("medium", n_reads=250_000)
    assert len(t) == 200 and t.offsets[-1] == 100_000_000
    _, q_loads = api.ram_loads(np.diff(q.offsets), Q_RAM // 2)
    assert len(q_loads) == 2
    _, t_loads = api.ram_loads(np.diff(t.offsets), T_RAM)
    assert len(t_loads) == 2
    tp, qp = write(str(tmp_path), t, q)
    a, b = cli_pair(str(tmp_path), tp, qp)
    assert b.count(b"\n") > 300_000
    assert a == b
    text, _ = api_text(engine, t, q)
    assert text == b


def test_uneven_reads_in_full(tmp_path, engine):
    """Reads of 50 bp to 10 kbp (log-uniform, 1-12 % errors with indels: the
    batched uneven-read shape) against a 5 Mbp target through the drop-in
    command line and the whole-job API: hits taken longest first and the
    longest extended one per warp; the TSV is byte-identical to the
    oracle's."""
    rng = np.random.Generator(np.random.PCG64(31))
    t = synth.make_target(rng, 5_000_000, n_contigs=20, median=250_000)
    q = synth.make_reads(rng, t, 4000, log_uniform=(50, 10_000), err_range=(0.01, 0.12), decoy_frac=0.02)
    tp, qp = write(str(tmp_path), t, q)
    a, b = cli_pair(str(tmp_path), tp, qp)
    assert b.count(b"\n") > 3000
    assert a == b
    text, _ = api_text(engine, t, q)
    assert text == b
