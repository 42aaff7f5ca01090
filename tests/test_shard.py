"""Multi-GPU host logic on CPU: query-window sharding with a replicated index
and the rank-ordered merge, with world_size 2 over gloo.  The per-rank mapper
is the oracle's whole-job composition, so the test needs no device."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from clast_b200 import api, shard, synth


def brute_windows(lengths, load_sizes, l, q_vram):
    starts, r0 = [], 0
    for n in load_sizes:
        g = [0]
        for L in lengths[r0:r0 + n]:
            g.append(g[-1] + 2 * (L + l - 1))
        qb = 0
        while qb < n:
            qe = qb + 1
            while qe < n and g[qe + 1] - g[qb] < q_vram:
                qe += 1
            starts.append(r0 + qb)
            qb = qe
        r0 += n
    return starts


def test_query_windows_match_scheduler_rule():
    rng = np.random.default_rng(3)
    lengths = rng.integers(20, 400, size=500).tolist()
    for q_vram in (100, 1000, 5000, 10**6):
        for loads in ([500], [200, 300], [1] * 10 + [490]):
            assert shard.query_windows(lengths, loads, 15, q_vram) == brute_windows(lengths, loads, 15, q_vram)


def test_shards_cover_reads_on_window_boundaries():
    rng = np.random.default_rng(4)
    lengths = rng.integers(50, 300, size=1000)
    loads = [400, 600]
    starts = set(shard.query_windows(lengths, loads, 15, 3000))
    for world in (1, 2, 3, 8):
        sh = shard.shard_reads(lengths, loads, 15, 3000, world)
        assert sh[0][0] == 0 and sh[-1][1] == len(lengths)
        for (a, b, sizes, ids), nxt in zip(sh, sh[1:] + [None]):
            assert a in starts or a == len(lengths)
            assert sum(sizes) == b - a
            if nxt:
                assert nxt[0] == b


def _case():
    rng = np.random.Generator(np.random.PCG64(11))
    t = synth.make_target(rng, 30_000, n_contigs=4, median=6000)
    q = synth.make_reads(rng, t, 60)
    s = api.Setting(total_db=float(t.offsets[-1]))
    tseqs = [t.seq(i).tobytes() for i in range(len(t))]
    return s, t, q, tseqs


def _worker(rank, world, port, out_path):
    import torch.distributed as dist
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle"), os.path.join(root, "tests")]
    from _oracle_map import oracle_map
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    s, t, q, tseqs = _case()
    q_loads = [25, 35]

    def map_fn(b, o, ls):
        qseqs = [b[o[i]:o[i + 1]].tobytes() for i in range(len(o) - 1)]
        return oracle_map(s, tseqs, [len(tseqs)], 10**9, qseqs, ls, 2000)

    res = shard.map_sharded(map_fn, q.bases, q.offsets, q_loads, s.lmer, 2000, rank, world)
    if rank == 0:
        np.savez(out_path, **res)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_sharding_equals_single(tmp_path):
    import sys
    from _oracle_map import oracle_map
    s, t, q, tseqs = _case()
    qseqs = [q.seq(i).tobytes() for i in range(len(q))]
    want = oracle_map(s, tseqs, [len(tseqs)], 10**9, qseqs, [25, 35], 2000)
    assert len(want["read"]) > 20
    sock = socket.socket()
    sock.bind(("127.0.0.1", 0))
    port = sock.getsockname()[1]
    sock.close()
    out = str(tmp_path / "merged.npz")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    for f in list(api.MAP_FIELDS) + ["load_offsets"]:
        np.testing.assert_array_equal(got[f], want[f], err_msg=f)
