"""Host-side helpers that the bench and the served form rely on, on CPU:
the vectorised window layout equals CHostSeqList's, read sets can be made
for any range of one fixed sequence (the multi-GPU shards), and the request
read counts and lengths follow the served shape."""
import numpy as np

from clast_b200 import api, synth


def test_joint_layout_equals_seqlist():
    rng = np.random.Generator(np.random.PCG64(3))
    t = synth.make_target(rng, 20_000, n_contigs=4, median=4000)
    q = synth.make_reads(rng, t, 30, log_uniform=(5, 400))
    for l in (8, 15, 31):
        ql = api.SeqList(l).add_queries([q.seq(i).tobytes() for i in range(len(q))])
        for (a, b) in [(0, 30), (3, 17), (29, 30)]:
            B, G, L = ql.window(2 * a, 2 * b)
            b2, g2, l2 = api.joint_layout(q.bases, q.offsets, l, a, b, True)
            assert b2.tobytes() == B and (g2 == G).all() and (l2 == L).all(), (l, a, b)
        tl = api.SeqList(l).add_targets([t.seq(i).tobytes() for i in range(len(t))])
        B, G, L = tl.window(1, 4)
        b2, g2, l2 = api.joint_layout(t.bases, t.offsets, l, 1, 4, False)
        assert b2.tobytes() == B and (g2 == G).all() and (l2 == L).all()


def test_reads_for_any_range_are_slices_of_one_sequence():
    t, q = synth.workload("medium", scale=0.02, n_reads=140_000)
    _, q2 = synth.workload("medium", scale=0.02, n_reads=50_000, first=65_000)
    assert np.array_equal(q.bases[q.offsets[65_000]:q.offsets[115_000]], q2.bases)
    assert q2.labels[0] == "r65000" and len(q2) == 50_000


def test_served_request_shape():
    rng = np.random.Generator(np.random.PCG64(8))
    t = synth.make_target(rng, 2_000_000, n_contigs=4, median=500_000)
    pool = synth.make_reads_var(rng, t, 5000, len_range=(100, 5000))
    L = np.diff(pool.offsets)
    assert L.min() >= 100 and L.max() <= 5000
    reqs = synth.served_requests(rng, 500, pool)
    counts = np.array([b - a for a, b in reqs])
    assert counts.min() >= 1 and counts.max() <= 5000
    assert all(0 <= a < b <= len(pool) for a, b in reqs)
    # log-uniform counts: about as many requests below 100 reads as above
    assert 0.3 < np.mean(counts < 100) < 0.7
