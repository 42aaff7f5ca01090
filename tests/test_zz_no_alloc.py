"""clast_search_noalloc (the library's fixed device scratch, caller-owned
host arrays) against clast_search, both through the C ABI, on the same
windows.  The file sorts last so that it also runs after every other GPU test
has used the device; it passes alone as well."""
import numpy as np
import pytest

from clast_b200 import api
from _cases import make_case

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 64 << 20  # CLAST_NOALLOC_SCRATCH_BYTES


def same(got, want):
    assert len(got["t_id"]) == len(want["t_id"]), (len(got["t_id"]), len(want["t_id"]))
    for f in api.HIT_FIELDS:
        if f == "evalue":
            np.testing.assert_allclose(got[f], want[f], rtol=1e-12, atol=0)
        else:
            np.testing.assert_array_equal(got[f], want[f], err_msg=f)


@pytest.fixture(scope="module")
def eng():
    e = api.Engine(0)
    yield e
    e.close()


def test_two_calls_in_a_row_match_clast_search(eng):
    s, tl, ql = make_case(7, target_bp=200_000, n_contigs=5, n_reads=600)
    ix = eng.hash_table(s, tl, 0, len(tl.lengths))
    nq = len(ql.lengths) // 2
    want = eng.hit_list(s, ix, ql, 0, nq)
    assert len(want["t_id"]) > 200
    first = eng.hit_list_noalloc(s, ix, ql, 0, nq, capacity=len(want["t_id"]) + 16)
    second = eng.hit_list_noalloc(s, ix, ql, 0, nq, capacity=len(want["t_id"]))
    same(first, want)
    same(second, want)
    # a smaller window next: nothing of the larger one may leak through the reused scratch
    want2 = eng.hit_list(s, ix, ql, 100, 130)
    got2 = eng.hit_list_noalloc(s, ix, ql, 100, 130, capacity=4096)
    same(got2, want2)
    ix.close()


@pytest.mark.parametrize("gap,local", [(3, 1), (12, 0)])
def test_other_settings(eng, gap, local):
    s, tl, ql = make_case(70 + gap, setting=api.Setting(gap=gap, local=local), letters=b"XRYN")
    ix = eng.hash_table(s, tl, 0, len(tl.lengths))
    nq = len(ql.lengths) // 2
    want = eng.hit_list(s, ix, ql, 0, nq)
    for _ in range(2):
        same(eng.hit_list_noalloc(s, ix, ql, 0, nq, capacity=len(want["t_id"]) + 1), want)
    ix.close()


def test_uneven_read_lengths(eng):
    # reads of 50 bp - 3 kbp: the DP takes the hits longest first here too
    s, tl, ql = make_case(71, target_bp=200_000, n_contigs=4, n_reads=60, log_uniform=(50, 3000),
                          err_range=(0.01, 0.12), decoy_frac=0.0)
    ix = eng.hash_table(s, tl, 0, len(tl.lengths))
    nq = len(ql.lengths) // 2
    want = eng.hit_list(s, ix, ql, 0, nq)
    assert len(want["t_id"]) > 20
    for _ in range(2):
        same(eng.hit_list_noalloc(s, ix, ql, 0, nq, capacity=len(want["t_id"])), want)
    ix.close()


def test_overlapping_calls_are_rejected_not_raced(eng):
    # two contexts on one device in two threads: the shared scratch admits one
    # call at a time; every call either returns clast_search's hits or is
    # rejected as overlapping, and a later call succeeds
    import threading
    s, tl, ql = make_case(8, target_bp=150_000, n_contigs=4, n_reads=400)
    ix = eng.hash_table(s, tl, 0, len(tl.lengths))
    nq = len(ql.lengths) // 2
    want = eng.hit_list(s, ix, ql, 0, nq)
    other = api.Engine(0)
    ix2 = other.hash_table(s, tl, 0, len(tl.lengths))
    outcomes, barrier = [], threading.Barrier(2)

    def worker(e, x):
        barrier.wait()
        for _ in range(6):
            try:
                got = e.hit_list_noalloc(s, x, ql, 0, nq, capacity=len(want["t_id"]))
                same(got, want)
                outcomes.append("ok")
            except api.ClastError as err:
                assert err.code == -1 and "scratch" in str(err), str(err)
                outcomes.append("busy")

    ts = [threading.Thread(target=worker, args=(eng, ix)), threading.Thread(target=worker, args=(other, ix2))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert len(outcomes) == 12 and "ok" in outcomes
    same(eng.hit_list_noalloc(s, ix, ql, 0, nq, capacity=len(want["t_id"])), want)
    ix2.close()
    other.close()
    ix.close()


def test_capacity_too_small_reports_count(eng):
    s, tl, ql = make_case(8)
    ix = eng.hash_table(s, tl, 0, len(tl.lengths))
    nq = len(ql.lengths) // 2
    want = eng.hit_list(s, ix, ql, 0, nq)
    n = len(want["t_id"])
    assert n > 2
    with pytest.raises(api.ClastError) as e:
        eng.hit_list_noalloc(s, ix, ql, 0, nq, capacity=n - 1)
    assert e.value.code == -1 and e.value.needed == n
    assert "capacity" in str(e.value)
    # the scratch is free again after the failed call
    same(eng.hit_list_noalloc(s, ix, ql, 0, nq, capacity=n), want)
    ix.close()


def test_empty_window(eng):
    s, tl, ql = make_case(9)
    ix = eng.hash_table(s, tl, 0, len(tl.lengths))
    got = eng.hit_list_noalloc(s, ix, ql, 3, 3, capacity=0)
    assert all(len(got[f]) == 0 for f in api.HIT_FIELDS)
    ix.close()


def test_window_beyond_scratch_is_rejected(eng):
    s, tl, _ql = make_case(9)
    ix = eng.hash_table(s, tl, 0, len(tl.lengths))
    n = SCRATCH_BYTES  # one byte of bases per byte of scratch already exceeds it with the 2-bit words
    half = n // 2
    bases = b"A" * n
    with pytest.raises(api.ClastError) as e:
        eng.hit_list_window_noalloc(s, ix, bases, [0, half], [half - 14, half - 14], 0, capacity=16)
    assert e.value.code == -1 and "use clast_search" in str(e.value)
    ix.close()
