"""Index persistence: clast_targets_save / clast_targets_load round trip
through the C ABI gives the oracle's whole-job result (and the freshly built
indexes' one), a saved file passes the host-side checks, and a mismatched or
foreign file is rejected."""
import numpy as np
import pytest

from clast_b200 import api, synth
from _oracle_map import oracle_map

pytestmark = pytest.mark.gpu


def workload():
    rng = np.random.Generator(np.random.PCG64(91))
    t = synth.make_target(rng, 400_000, n_contigs=6, median=60_000)
    q = synth.make_reads(rng, t, 3000)
    s = api.Setting(total_db=float(t.offsets[-1]))
    return s, t, q


def run_map(engine, s, T, q):
    return engine.map(s, T, q.bases, q.offsets, [len(q)], 2_000_000)


def test_saved_index_maps_identically(engine, tmp_path):
    s, t, q = workload()
    T = engine.targets(s, t.bases, t.offsets, [len(t)], 150_000)  # several windows
    want = run_map(engine, s, T, q)
    assert len(want["read"]) > 100
    path = str(tmp_path / "targets.clastix")
    engine.save_targets(T, path)
    T.close()
    ok, why = api.verify_targets_file(s, path)
    assert ok, why
    T2 = engine.load_targets(s, path)
    ref = oracle_map(s, [t.seq(i).tobytes() for i in range(len(t))], [len(t)], 150_000,
                     [q.seq(i).tobytes() for i in range(len(q))], [len(q)], 2_000_000)
    for _ in range(2):
        got = run_map(engine, s, T2, q)
        assert set(got) == set(want)
        for f in want:
            np.testing.assert_array_equal(got[f], want[f], err_msg=f)
            if f == "evalue":
                np.testing.assert_allclose(got[f], ref[f], rtol=1e-12, atol=0)
            else:
                np.testing.assert_array_equal(got[f], ref[f], err_msg=f)
    T2.close()


def test_load_rejects_other_settings_and_foreign_files(engine, tmp_path):
    s, t, q = workload()
    T = engine.targets(s, t.bases, t.offsets, [len(t)], 150_000)
    path = str(tmp_path / "targets.clastix")
    engine.save_targets(T, path)
    T.close()
    with pytest.raises(api.ClastError) as e:
        engine.load_targets(api.Setting(lmer=14, total_db=s.total_db), path)
    assert e.value.code == -1
    bogus = tmp_path / "bogus.bin"
    bogus.write_bytes(b"not an index file at all")
    with pytest.raises(api.ClastError) as e:
        engine.load_targets(s, str(bogus))
    assert e.value.code == -1
    truncated = tmp_path / "truncated.clastix"
    truncated.write_bytes(open(path, "rb").read()[:1000])
    with pytest.raises(api.ClastError) as e:
        engine.load_targets(s, str(truncated))
    assert e.value.code == -1
