"""Index files are checked on the host before anything is uploaded
(clast_targets_verify runs the checks of clast_targets_load without a
device): a file of another layout, other settings, or with any offset the
kernels would follow pointing outside its array is rejected.

The files here are written by a small writer of the documented layout
(clast_b200/csrc/clast_indexfile.cu), then edited one field at a time."""
import struct

import numpy as np
import pytest

from clast_b200 import api

KPAD = 64
NO_PAYLOAD = (1 << 64) - 1
MULTI = 1 << 63


def window(l=15, stride=5, n_seqs=2, seq_len=200):
    """A consistent one-load window: sequences, entries, a table whose
    records use single and multi payloads, a zero filter."""
    lengths = np.full(n_seqs, seq_len, dtype=np.int32)
    gateway = (np.arange(n_seqs) * (seq_len + l - 1)).astype(np.int32)
    n = int(n_seqs * (seq_len + l - 1))
    ns = n // stride
    nbuckets = max(1, ns)
    n_records = 2 * nbuckets + (1 << 16)
    entries = np.zeros((ns, 2), dtype=np.int32)
    entries[:, 0] = np.arange(ns) % n_seqs
    entries[:, 1] = np.arange(ns) % seq_len
    table = np.full((n_records, 2), NO_PAYLOAD, dtype=np.uint64)
    table[0] = (7, (1 << 32) | 5)               # single entry: sequence 1, index 5
    table[2] = (9, MULTI | (3 << 32) | 4)       # entries 3..6
    fshift = 52
    return dict(l=l, stride=stride, load=0, first=0, t_begin=0, nseqs=n_seqs, n=n, nbuckets=nbuckets,
                fshift=fshift, n_records=n_records, n_keys=ns, bases=b"N" * (n + 2 * KPAD), gateway=gateway,
                lengths=lengths, entries=entries, table=table, filter=np.zeros(1 << (64 - fshift), np.uint32))


def write(path, w, magic=b"CLASTIX2", layout=2, n_loads=1, trailing=b""):
    with open(path, "wb") as f:
        f.write(magic)
        f.write(struct.pack("<iiiiiq", layout, w["l"], w["stride"], 20, n_loads, 1))
        f.write(struct.pack("<iiiiqIiqqqq", w["load"], w["first"], w["t_begin"], w["nseqs"], w["n"], w["nbuckets"],
                            w["fshift"], w["n_records"], len(w["filter"]), len(w["entries"]), w["n_keys"]))
        f.write(w["bases"])
        f.write(np.ascontiguousarray(w["gateway"], np.int32).tobytes())
        f.write(np.ascontiguousarray(w["lengths"], np.int32).tobytes())
        f.write(np.ascontiguousarray(w["entries"], np.int32).tobytes())
        f.write(np.ascontiguousarray(w["table"], np.uint64).tobytes())
        f.write(np.ascontiguousarray(w["filter"], np.uint32).tobytes())
        f.write(trailing)


def verify(path, **kw):
    return api.verify_targets_file(api.Setting(**kw), str(path))


def test_consistent_file_passes(tmp_path):
    p = tmp_path / "ok.clastix"
    write(p, window())
    ok, why = verify(p)
    assert ok, why


def test_unused_entry_tail_is_not_checked(tmp_path):
    # the entry array is sized by the samples; entries past the kept ones
    # hold whatever the build left there and no record refers to them
    w = window()
    w["entries"][-5:] = (-7, 10 ** 6)
    p = tmp_path / "tail.clastix"
    write(p, w)
    ok, why = verify(p)
    assert ok, why


@pytest.mark.parametrize("edit,expect", [
    (dict(magic=b"CLASTIX1"), "older index layout"),
    (dict(magic=b"NOTANIDX"), "not a clast index file"),
    (dict(layout=3), "index layout 3"),
    (dict(trailing=b"\0"), "past its last window"),
])
def test_header_edits_rejected(tmp_path, edit, expect):
    p = tmp_path / "bad.clastix"
    write(p, window(), **edit)
    ok, why = verify(p)
    assert not ok and expect in why, why


def test_other_settings_rejected(tmp_path):
    p = tmp_path / "s.clastix"
    write(p, window())
    ok, why = verify(p, lmer=14)
    assert not ok and "other lMer" in why


def edited(field_fn):
    w = window()
    field_fn(w)
    return w


@pytest.mark.parametrize("name,fn,expect", [
    ("records", lambda w: w.update(n_records=w["n_records"] - 1, table=w["table"][:-1]), "record count"),
    ("buckets", lambda w: w.update(nbuckets=w["nbuckets"] + 1), "bucket count"),
    ("last_free", lambda w: w["table"].__setitem__(-1, (1, 0)), "last table record"),
    ("multi_past", lambda w: w["table"].__setitem__(2, (9, MULTI | (int(w["n_keys"]) - 2 << 32) | 4)),
     "points past the entries"),
    ("single_past", lambda w: w["table"].__setitem__(0, (7, (1 << 32) | 200)), "names no target base"),
    ("single_seq", lambda w: w["table"].__setitem__(0, (7, (5 << 32) | 1)), "names no target base"),
    ("gateway", lambda w: w["gateway"].__setitem__(1, w["n"] - 10), "outside the window"),
    ("length", lambda w: w["lengths"].__setitem__(0, 10_000), "outside the window"),
    ("entry", lambda w: w["entries"].__setitem__(3, (0, 999)), "entry 3"),  # inside record 2's range 3..6
    ("load", lambda w: w.update(load=1), "target load"),
    ("filter", lambda w: w.update(fshift=40), "filter size"),
])
def test_window_edits_rejected(tmp_path, name, fn, expect):
    p = tmp_path / ("%s.clastix" % name)
    write(p, edited(fn))
    ok, why = verify(p)
    assert not ok and expect in why, (name, why)


def test_truncated_file_rejected(tmp_path):
    p = tmp_path / "t.clastix"
    write(p, window())
    data = p.read_bytes()
    for cut in (10, 60, len(data) // 2, len(data) - 1):
        p.write_bytes(data[:cut])
        ok, why = verify(p)
        assert not ok and ("truncated" in why or "not a clast index" in why), (cut, why)
