"""Seeded windows shared by the parity tests."""
import numpy as np

from clast_b200 import api, synth


def make_case(seed, target_bp=30_000, n_contigs=3, n_reads=40, read_len=150, setting=None, letters=None,
              **read_kw):
    """(setting, target SeqList, query SeqList): synthetic contigs and reads;
    ``letters`` sprinkles extra letters (e.g. b"XRYE") into both."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = synth.make_target(rng, target_bp, n_contigs=n_contigs, median=target_bp / max(1, n_contigs) * 0.8)
    q = synth.make_reads(rng, t, n_reads, length=read_len, **read_kw)
    tseqs = [bytearray(t.seq(i).tobytes()) for i in range(len(t))]
    qseqs = [bytearray(q.seq(i).tobytes()) for i in range(len(q))]
    if letters:
        for s in tseqs + qseqs:
            k = max(1, len(s) // 500)
            for p in rng.integers(0, len(s), size=k):
                s[p] = letters[int(rng.integers(0, len(letters)))]
    s = setting or api.Setting()
    s.total_db = float(sum(len(x) for x in tseqs))
    tl = api.SeqList(s.lmer).add_targets([bytes(x) for x in tseqs])
    ql = api.SeqList(s.lmer).add_queries([bytes(x) for x in qseqs])
    return s, tl, ql


def compare(got, want, rtol=1e-12):
    """Field-by-field equality; E-values within rtol (relative)."""
    import oracle as O
    assert len(got["t_id"]) == len(want["t_id"]), (len(got["t_id"]), len(want["t_id"]))
    for f in O.FIELDS:
        if f == "evalue":
            np.testing.assert_allclose(got[f], want[f], rtol=rtol, atol=0)
        else:
            bad = np.flatnonzero(got[f] != want[f])
            assert bad.size == 0, "field %s differs at %s: got %s want %s" % (
                f, bad[:5], got[f][bad[:5]], want[f][bad[:5]])
