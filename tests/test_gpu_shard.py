"""Query sharding on the device path: the reads split by shard.shard_reads,
each shard mapped by Engine.map (clast_map), the shards merged by
shard.merge_shards, give the oracle's whole-job result.  The shards run one
after another on one GPU; on several GPUs each would be one rank's work."""
import numpy as np
import pytest

from clast_b200 import api, shard, synth
from _oracle_map import oracle_map

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_map_merges_to_oracle(engine, world):
    rng = np.random.Generator(np.random.PCG64(404))
    t = synth.make_target(rng, 200_000, n_contigs=5, median=30_000)
    q = synth.make_reads(rng, t, 900, log_uniform=(60, 600))
    s = api.Setting(total_db=float(t.offsets[-1]))
    q_loads, q_vram, t_vram = [300, 600], 20_000, 90_000
    T = engine.targets(s, t.bases, t.offsets, [len(t)], t_vram)
    lengths = np.diff(q.offsets)
    shards = shard.shard_reads(lengths, q_loads, s.lmer, q_vram, world)
    results = []
    for (a, b, sizes, _ids) in shards:
        sub_off = q.offsets[a:b + 1] - q.offsets[a]
        res = engine.map(s, T, q.bases[q.offsets[a]:q.offsets[b]], sub_off, sizes, q_vram)
        results.append({f: np.array(res[f]) for f in list(api.MAP_FIELDS) + ["load_offsets"]})
        del res
    merged = shard.merge_shards(results, shards, len(q_loads))
    T.close()
    want = oracle_map(s, [t.seq(i).tobytes() for i in range(len(t))], [len(t)], t_vram,
                      [q.seq(i).tobytes() for i in range(len(q))], q_loads, q_vram)
    assert len(want["read"]) > 200
    np.testing.assert_array_equal(merged["load_offsets"], want["load_offsets"])
    for f in api.MAP_FIELDS:
        if f == "evalue":
            np.testing.assert_allclose(merged[f], want[f], rtol=1e-12, atol=0)
        else:
            np.testing.assert_array_equal(merged[f], want[f], err_msg=f)


@pytest.mark.parametrize("group", ["2", "4"])
def test_several_windows_per_seeding_pass(engine, group, monkeypatch):
    # CLAST_SEED_WINDOWS > 1: the seeds of several target windows in one pass
    # over the query (k_seed_multi); the hits must equal the oracle's
    rng = np.random.Generator(np.random.PCG64(405))
    t = synth.make_target(rng, 300_000, n_contigs=7, median=40_000, repeat_frac=0.05, n_families=5)
    q = synth.make_reads(rng, t, 700, log_uniform=(60, 800))
    s = api.Setting(total_db=float(t.offsets[-1]))
    q_loads, q_vram, t_vram = [700], 30_000, 45_000  # five or more target windows
    monkeypatch.setenv("CLAST_SEED_WINDOWS", group)
    T = engine.targets(s, t.bases, t.offsets, [len(t)], t_vram)
    res = engine.map(s, T, q.bases, q.offsets, q_loads, q_vram)
    got = {f: np.array(res[f]) for f in list(api.MAP_FIELDS) + ["load_offsets"]}
    del res
    T.close()
    want = oracle_map(s, [t.seq(i).tobytes() for i in range(len(t))], [len(t)], t_vram,
                      [q.seq(i).tobytes() for i in range(len(q))], q_loads, q_vram)
    assert len(want["read"]) > 200
    for f in api.MAP_FIELDS:
        if f == "evalue":
            np.testing.assert_allclose(got[f], want[f], rtol=1e-12, atol=0)
        else:
            np.testing.assert_array_equal(got[f], want[f], err_msg=f)
