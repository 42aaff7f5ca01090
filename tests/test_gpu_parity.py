"""CUDA path against the oracle, one (target window, query window) pair at a
time, through the C ABI (clast_index_build + clast_search)."""
import numpy as np
import pytest

import oracle as O
from clast_b200 import api
from _cases import make_case, compare

pytestmark = pytest.mark.gpu


def run_pair(engine, s, tl, ql, tb=0, te=None, qb=0, qe=None):
    te = len(tl.lengths) if te is None else te
    qe = len(ql.lengths) // 2 if qe is None else qe
    ix = engine.hash_table(s, tl, tb, te)
    got = engine.hit_list(s, ix, ql, qb, qe)
    tbases, tgw, tln = tl.window(tb, te)
    qbases, qgw, qln = ql.window(2 * qb, 2 * qe)
    want = O.window_search(s, tbases, tgw, tln, tb, qbases, qgw, qln, 2 * qb)
    ix.close()
    return got, want


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_default_settings(engine, seed):
    s, tl, ql = make_case(seed)
    got, want = run_pair(engine, s, tl, ql)
    assert len(want["t_id"]) > 10
    compare(got, want)


@pytest.mark.parametrize("gap", [2, 5, 8, 12, 16])
@pytest.mark.parametrize("local", [0, 1])
def test_gap_and_mode(engine, gap, local):
    s, tl, ql = make_case(10 + gap, setting=api.Setting(gap=gap, local=local))
    got, want = run_pair(engine, s, tl, ql)
    assert len(want["t_id"]) > 0
    compare(got, want)


@pytest.mark.parametrize("lmer,stride", [(8, 3), (11, 1), (16, 4), (17, 2), (20, 7), (31, 5)])
def test_lmer_stride(engine, lmer, stride):
    s, tl, ql = make_case(20 + lmer, setting=api.Setting(lmer=lmer, stride=stride))
    got, want = run_pair(engine, s, tl, ql)
    compare(got, want)


@pytest.mark.parametrize("cut", [-1, 0, 3, 20])
def test_repeat_cut(engine, cut):
    s, tl, ql = make_case(30, setting=api.Setting(cut_repeat=cut, lmer=10, stride=2))
    got, want = run_pair(engine, s, tl, ql)
    compare(got, want)


def test_letters_and_bad_area(engine):
    # IUPAC, '-1' letters and 'X' in both target and reads
    s, tl, ql = make_case(40, letters=b"XRYENKZ")
    got, want = run_pair(engine, s, tl, ql)
    compare(got, want)


def test_windows_offsets(engine):
    # windows that do not start at id 0 (t_begin, q_begin shift every id)
    s, tl, ql = make_case(50, n_contigs=6, n_reads=60)
    got, want = run_pair(engine, s, tl, ql, tb=2, te=5, qb=10, qe=41)
    compare(got, want)


def test_small_lmer_out_of_window_reads(engine):
    # lMer 8 with gap 12: the DP reads bases before a window's first sequence
    # and past its last one (defined as 'N' in both implementations)
    s, tl, ql = make_case(60, setting=api.Setting(lmer=8, gap=12, stride=2), n_contigs=2)
    got, want = run_pair(engine, s, tl, ql)
    compare(got, want)


def test_no_cutoff_and_short_reads(engine):
    s, tl, ql = make_case(70, setting=api.Setting(cutoff=-1), read_len=40)
    got, want = run_pair(engine, s, tl, ql)
    compare(got, want)


def test_empty_query_hits(engine):
    # decoys only: no seeds at all
    s, tl, ql = make_case(80, decoy_frac=1.0)
    got, want = run_pair(engine, s, tl, ql)
    compare(got, want)


@pytest.mark.parametrize("local", [0, 1])
def test_uneven_read_lengths(engine, local):
    # log-uniform read lengths 50 bp - 4 kbp with per-read error rates 1-12 %
    # (the batched uneven-reads shape, scaled down for the oracle)
    s, tl, ql = make_case(61 + local, target_bp=300_000, n_contigs=4, n_reads=50,
                          setting=api.Setting(local=local), log_uniform=(50, 4000), err_range=(0.01, 0.12),
                          decoy_frac=0.0)
    assert max(ql.lengths) > 1000 and min(ql.lengths) < 200
    got, want = run_pair(engine, s, tl, ql)
    assert len(want["t_id"]) > 20
    compare(got, want)
