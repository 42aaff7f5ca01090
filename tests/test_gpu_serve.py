"""The served form (clast_server_*) on the device: each request's hits are
the same alone and batched with others, and equal the oracle's result for
that request's reads; requests are batched as they arrive; a queued request
can be cancelled; admission keeps the estimated device bytes in flight within
the budget and rejects a request that can never fit."""
import time

import numpy as np
import pytest

from clast_b200 import api, synth
from _oracle_map import oracle_map

pytestmark = pytest.mark.gpu

Q_VRAM, Q_RAM = 60_000, 200_000


@pytest.fixture(scope="module")
def served_case():
    rng = np.random.Generator(np.random.PCG64(2024))
    t = synth.make_target(rng, 400_000, n_contigs=5, median=60_000, repeat_frac=0.05, n_families=4)
    pool = synth.make_reads_var(rng, t, 1500, len_range=(100, 3000), decoy_frac=0.05)
    reqs = synth.served_requests(rng, 14, pool, count_range=(1, 300))
    s = api.Setting(total_db=float(t.offsets[-1]))
    return s, t, pool, reqs


def sub(pool, a, b):
    return pool.bases[pool.offsets[a]:pool.offsets[b]], pool.offsets[a:b + 1] - pool.offsets[a]


def assert_same(got, want, rtol=0.0):
    np.testing.assert_array_equal(got["load_offsets"], want["load_offsets"])
    for f in api.MAP_FIELDS:
        if f == "evalue" and rtol:
            np.testing.assert_allclose(got[f], want[f], rtol=rtol, atol=0)
        else:
            np.testing.assert_array_equal(got[f], want[f], err_msg=f)


def test_alone_equals_mix_equals_oracle(engine, served_case):
    s, t, pool, reqs = served_case
    T = engine.targets(s, t.bases, t.offsets, [len(t)], 150_000)
    srv = api.Server(engine, T, s, lanes=2, q_vram=Q_VRAM, q_ram=Q_RAM, max_batch_bases=2_000_000)
    alone = []
    for (a, b) in reqs:  # one request at a time: a batch of one
        rid = srv.submit(*sub(pool, a, b))
        alone.append(srv.poll(rid, -1))
        srv.release(rid)
    ids = [srv.submit(*sub(pool, a, b)) for (a, b) in reqs]  # all at once: batched
    mix = [srv.poll(rid, -1) for rid in ids]
    st = srv.stats()
    for rid in ids:
        srv.release(rid)
    srv.close()
    T.close()
    assert st["max_batch_requests"] > 1, st
    tseqs = [t.seq(i).tobytes() for i in range(len(t))]
    total = 0
    for (a, b), x, y in zip(reqs, alone, mix):
        assert_same(x, y)
        qseqs = [pool.seq(i).tobytes() for i in range(a, b)]
        _, loads = api.ram_loads([len(q) for q in qseqs], Q_RAM)
        want = oracle_map(s, tseqs, [len(t)], 150_000, qseqs, loads, Q_VRAM)
        assert_same(x, want, rtol=1e-12)
        total += len(x["read"])
    assert total > 200


def test_cancel_queued_request(engine, served_case):
    s, t, pool, reqs = served_case
    T = engine.targets(s, t.bases, t.offsets, [len(t)], 150_000)
    big = synth.make_reads_fixed(np.random.Generator(np.random.PCG64(5)), t, 60_000)
    srv = api.Server(engine, T, s, lanes=1, q_vram=2_000_000, max_batch_bases=1)  # one request per batch
    r1 = srv.submit(big.bases, big.offsets)
    r2 = srv.submit(*sub(pool, 0, 50))
    srv.cancel(r2)  # the single lane is busy with r1
    with pytest.raises(api.ClastError) as e:
        srv.poll(r2, -1)
    assert e.value.code == api.ERR_CANCELLED
    assert srv.poll(r1, -1) is not None
    with pytest.raises(api.ClastError):
        srv.cancel(r1)  # finished: nothing to cancel
    srv.release(r1)
    srv.release(r2)
    with pytest.raises(api.ClastError):
        srv.poll(r1, 0)  # released
    srv.close()
    T.close()


def test_admission_by_device_budget(engine, served_case):
    s, t, pool, reqs = served_case
    T = engine.targets(s, t.bases, t.offsets, [len(t)], 150_000)
    # room for about one small request's estimate in flight at a time
    srv = api.Server(engine, T, s, lanes=3, q_vram=Q_VRAM, q_ram=Q_RAM, hbm_budget=24 << 20)
    big = synth.make_reads_fixed(np.random.Generator(np.random.PCG64(6)), t, 40_000)
    with pytest.raises(api.ClastError) as e:
        srv.submit(big.bases, big.offsets)  # 6 Mbp: its estimate alone exceeds the budget
    assert e.value.code == -3
    ids = [srv.submit(*sub(pool, a, min(b, a + 40))) for (a, b) in reqs]
    for rid in ids:
        assert srv.poll(rid, -1) is not None
        srv.release(rid)
    st = srv.stats()
    assert 0 < st["hbm_in_flight_max"] <= st["hbm_budget"] == 24 << 20
    srv.close()
    T.close()


def test_poll_without_wait_and_times(engine, served_case):
    s, t, pool, reqs = served_case
    T = engine.targets(s, t.bases, t.offsets, [len(t)], 150_000)
    srv = api.Server(engine, T, s, lanes=2, q_vram=Q_VRAM, q_ram=Q_RAM)
    t0 = time.monotonic_ns()
    rid = srv.submit(*sub(pool, 0, 200))
    res = srv.poll(rid, 0)
    while res is None:
        res = srv.poll(rid, 5)
    a, b, c = srv.times(rid)
    assert t0 <= a <= b <= c <= time.monotonic_ns()
    srv.release(rid)
    with pytest.raises(api.ClastError):
        srv.release(rid)
    srv.close()
    T.close()
