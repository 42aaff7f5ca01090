"""The banded DP with one warp per hit (the band's anti-diagonal wavefront,
k_banded_dp_warp) against the one-thread-per-hit kernel and the oracle.

CLAST_DP_WARP=all sends every hit through the warp kernel, =off through the
thread kernels; unset, the split is chosen per batch (the longest hits one
per warp).  All three must give the oracle's hits exactly, for both passes
(hits whose seed sits at a read's start or end have an empty pass), both
modes (local: the first best cell in row-major order; global: the first best
column of the last row), narrow and wide bands, targets whose ends fall
inside the band ('X' beyond them), the bad-area letter and '-1' letters in
both sequences, and reads of 16 bp to 5 kbp."""
import os

import numpy as np
import pytest

import oracle as O
from clast_b200 import api, synth
from _cases import compare

pytestmark = pytest.mark.gpu


def uneven_case(seed, setting, n_reads=120, len_range=(40, 5000), letters=b"XRYENKZ"):
    rng = np.random.Generator(np.random.PCG64(seed))
    t = synth.make_target(rng, 60_000, n_contigs=4, median=12_000)
    q = synth.make_reads_var(rng, t, n_reads, len_range=len_range, decoy_frac=0.05)
    tseqs = [bytearray(t.seq(i).tobytes()) for i in range(len(t))]
    qseqs = [bytearray(q.seq(i).tobytes()) for i in range(len(q))]
    # reads at both ends of every contig (the band runs past the target's
    # ends) and very short ones (a pass of a few rows)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    for s in tseqs:
        for piece in (bytes(s[:700]), bytes(s[-900:]), bytes(s[5:5 + setting.lmer + 3]), bytes(s[-40:])):
            qseqs.append(bytearray(piece))
            qseqs.append(bytearray(piece.translate(comp)[::-1]))
    for s in tseqs + qseqs:
        for p in rng.integers(0, len(s), size=max(1, len(s) // 700)):
            s[p] = letters[int(rng.integers(0, len(letters)))]
    setting.total_db = float(sum(len(x) for x in tseqs))
    tl = api.SeqList(setting.lmer).add_targets([bytes(x) for x in tseqs])
    ql = api.SeqList(setting.lmer).add_queries([bytes(x) for x in qseqs])
    return setting, tl, ql


def hits(engine, s, tl, ql, mode):
    old = os.environ.get("CLAST_DP_WARP")
    if mode is None:
        os.environ.pop("CLAST_DP_WARP", None)
    else:
        os.environ["CLAST_DP_WARP"] = mode
    try:
        ix = engine.hash_table(s, tl, 0, len(tl.lengths))
        got = engine.hit_list(s, ix, ql, 0, len(ql.lengths) // 2)
        ix.close()
        return got
    finally:
        if old is None:
            os.environ.pop("CLAST_DP_WARP", None)
        else:
            os.environ["CLAST_DP_WARP"] = old


@pytest.mark.parametrize("gap", [2, 8, 16])
@pytest.mark.parametrize("local", [0, 1])
def test_warp_per_hit_equals_oracle(engine, gap, local):
    s, tl, ql = uneven_case(100 + gap + local, api.Setting(gap=gap, local=local))
    tbases, tgw, tln = tl.window(0, len(tl.lengths))
    qbases, qgw, qln = ql.window(0, len(ql.lengths))
    want = O.window_search(s, tbases, tgw, tln, 0, qbases, qgw, qln, 0)
    assert len(want["t_id"]) > 50
    for mode in ("all", "off", None):
        compare(hits(engine, s, tl, ql, mode), want)


@pytest.mark.parametrize("lmer,stride", [(8, 2), (20, 5)])
def test_warp_per_hit_other_lmers(engine, lmer, stride):
    s, tl, ql = uneven_case(300 + lmer, api.Setting(lmer=lmer, stride=stride, gap=12))
    tbases, tgw, tln = tl.window(0, len(tl.lengths))
    qbases, qgw, qln = ql.window(0, len(ql.lengths))
    want = O.window_search(s, tbases, tgw, tln, 0, qbases, qgw, qln, 0)
    compare(hits(engine, s, tl, ql, "all"), want)


def test_equal_lengths_and_one_read(engine):
    """Reads of one length (the all-or-none split on the host) and a single
    long read (one warp per hit by default)."""
    rng = np.random.Generator(np.random.PCG64(7))
    t = synth.make_target(rng, 80_000, n_contigs=2, median=40_000)
    for n, lo in ((300, 600), (1, 4000)):
        q = synth.make_reads_var(rng, t, n, len_range=(lo, lo + 1))
        s = api.Setting()
        s.total_db = float(t.offsets[-1])
        tl = api.SeqList(s.lmer).add_targets([t.seq(i).tobytes() for i in range(len(t))])
        ql = api.SeqList(s.lmer).add_queries([q.seq(i).tobytes() for i in range(len(q))])
        tbases, tgw, tln = tl.window(0, len(tl.lengths))
        qbases, qgw, qln = ql.window(0, len(ql.lengths))
        want = O.window_search(s, tbases, tgw, tln, 0, qbases, qgw, qln, 0)
        assert len(want["t_id"]) > 0
        for mode in ("all", None):
            compare(hits(engine, s, tl, ql, mode), want)


def test_whole_job_split_matches_thread_kernel(engine):
    """clast_map over uneven reads (length buckets, the split on the device,
    the autotuner's candidates): the same hits with and without the warp
    kernel."""
    rng = np.random.Generator(np.random.PCG64(9))
    t = synth.make_target(rng, 3_000_000, n_contigs=6, median=500_000)
    q = synth.make_reads_var(rng, t, 6000, len_range=(50, 8000), decoy_frac=0.05)
    s = api.Setting(total_db=float(t.offsets[-1]))
    _, t_loads = api.ram_loads(np.diff(t.offsets), 64_000_000)
    _, q_loads = api.ram_loads(np.diff(q.offsets), 32_000_000)
    T = engine.targets(s, t.bases, t.offsets, t_loads, 64_000_000)
    out, warp = {}, {}
    for mode in ("off", None, "all"):
        if mode is None:
            os.environ.pop("CLAST_DP_WARP", None)
        else:
            os.environ["CLAST_DP_WARP"] = mode
        try:
            r = engine.map(s, T, q.bases, q.offsets, q_loads, 2_000_000)
        finally:
            os.environ.pop("CLAST_DP_WARP", None)
        out[mode] = {f: np.array(r[f]) for f in api.MAP_FIELDS}
        del r
        st = engine.stats()
        warp[mode] = (st["dp_warp_hits"], st["hits"])
    T.close()
    assert len(out["off"]["score"]) > 1000
    # hits extended one per warp: none, some (the longest), every one
    assert warp["off"][0] == 0 and warp["all"][0] == warp["all"][1] > 0
    assert 0 <= warp[None][0] <= warp[None][1]
    for mode in (None, "all"):
        for f in api.MAP_FIELDS:
            assert np.array_equal(out[mode][f], out["off"][f]), (mode, f)


@pytest.mark.parametrize("lmer,gap,local", [(15, 8, 0), (15, 8, 1), (8, 4, 0), (11, 16, 0)])
def test_hits_entering_the_dp_equal_oracle(engine, lmer, gap, local):
    """The number of hits the seed filters pass to the DP equals the oracle's
    count after its isolate and duplicate filters: reads at both ends of every
    contig make the boundary filters drop seeds (stored as sentinels that
    sort last and are never filtered), and strands of every seed-count tier
    (one thread, one warp, shared memory) occur."""
    s, tl, ql = uneven_case(500 + lmer + gap + local, api.Setting(lmer=lmer, stride=2, gap=gap, local=local))
    tbases, tgw, tln = tl.window(0, len(tl.lengths))
    qbases, qgw, qln = ql.window(0, len(ql.lengths))
    want = O.window_search(s, tbases, tgw, tln, 0, qbases, qgw, qln, 0, stage=O.STAGE_FILTERED)
    before = engine.stats()["hits"]
    ix = engine.hash_table(s, tl, 0, len(tl.lengths))
    engine.hit_list(s, ix, ql, 0, len(ql.lengths) // 2)
    ix.close()
    got = engine.stats()["hits"] - before
    assert len(want["t_id"]) > 100
    assert got == len(want["t_id"])
