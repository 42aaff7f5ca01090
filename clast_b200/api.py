"""Host-side mirror of the reference's in-process interface for the search path.

The reference (masayano/CLAST) drives its device work through four classes,
constructed by its scheduler for every (target window, query window) pair
(CHostSchedular.cu:141,169,187,196):

=====================================  ==========================================
reference                              here
=====================================  ==========================================
CHostSetting (CHostSetting.cuh:29-49)  :class:`Setting`
CHostSeqList_target / _query           :class:`SeqList` (``add_targets`` / ``add_queries``)
CDeviceHashTable(s, t, tb, te)         :meth:`Engine.hash_table`
CDeviceHitList(s, h, q, tb, 2*qb)      :meth:`Engine.hit_list` (+ ``getResult``)
CHostMapper/CHostSchedular/Holder      :meth:`Engine.targets` + :meth:`Engine.map`
``clast`` command line                 :func:`run_clast`
=====================================  ==========================================

All device work goes through libclast_b200.so (include/clast_gpu.h); a call
that fails raises :class:`ClastError` with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
import dataclasses
import time

import numpy as np

from . import _native as N

HIT_FIELDS = ("t_id", "t_idx", "q_id", "q_idx", "t_len", "q_len", "match", "score", "evalue")
MAP_FIELDS = ("read", "strand", "t_load", "t_seq", "t_idx", "q_idx", "t_len", "q_len", "match", "score", "evalue")


class ClastError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("clast error %d: %s" % (code, msg))
        self.code = code


@dataclasses.dataclass
class Setting:
    """The search settings of CHostSetting; defaults of common.hpp:12-43."""
    lmer: int = 15
    stride: int = 5
    cut_repeat: int = 20
    width: int = 100
    gap: int = 8
    local: int = 0
    cutoff: float = 10.0
    total_db: float = 0.0
    K: float = 0.71
    lambda_: float = 1.37

    def c(self) -> N.clast_params:
        return N.clast_params(self.lmer, self.stride, self.cut_repeat, self.width, self.gap, self.local,
                              float(self.cutoff), float(self.total_db), float(self.K), float(self.lambda_))


def ram_loads(lengths, budget: int):
    """RAM loads of CFASTALoader (CFASTALoader.cpp:43-87) for records of the
    given lengths: a record joins the current load while sum + length <
    budget, a record longer than the budget is skipped.  Returns (kept mask,
    records per load).  A record exactly as long as the budget would make the
    reference loop forever; that raises ValueError."""
    lengths = np.asarray(lengths, dtype=np.int64)
    keep = lengths <= budget
    loads, cur, tot = [], 0, 0
    for L in lengths[keep].tolist():
        if tot + L < budget:
            tot += L
            cur += 1
            continue
        if cur == 0:
            raise ValueError("a record is exactly as long as the RAM budget; the reference never terminates")
        loads.append(cur)
        cur, tot = 1, L
        if L == budget:
            raise ValueError("a record is exactly as long as the RAM budget; the reference never terminates")
    if cur:
        loads.append(cur)
    return keep, loads


def _comp(seq: bytes) -> bytes:
    """utilReverseSeq.cpp:3-19: reverse complement, non-ACGT -> N."""
    table = bytes.maketrans(b"ACGT", b"TGCA")
    out = seq[::-1].translate(table)
    return bytes(c if c in b"ACGT" else ord("N") for c in out) if any(c not in b"ACGT" for c in out) else out


_COMP_TABLE = np.full(256, ord("N"), dtype=np.uint8)
for _a, _b in zip(b"ACGT", b"TGCA"):
    _COMP_TABLE[_a] = _b


def joint_layout(bases, offsets, lmer: int, first: int, end: int, both_strands: bool):
    """The base array CHostSeqList::getBaseArray builds for records
    [first, end) of a one-strand set (utilAddSequence.cu:6-47): every
    sequence followed by its first l-1 bases ('N' past its end); with
    ``both_strands`` every record gives its '+' strand then its reverse
    complement (non-ACGT -> N, utilReverseSeq.cpp:3-19), as
    CHostSeqList_query::add does.  Returns (uint8 bases, int64 window-relative
    gateway, int32 lengths), vectorised."""
    offsets = np.asarray(offsets, dtype=np.int64)
    lens = np.diff(offsets[first:end + 1])
    k = 2 if both_strands else 1
    L = np.repeat(lens, k)
    src0 = np.repeat(offsets[first:end], k)
    rev = np.tile(np.array([False, True]), len(lens)) if both_strands else np.zeros(len(L), bool)
    per = L + lmer - 1
    gw = np.zeros(len(per), dtype=np.int64)
    if len(per) > 1:
        np.cumsum(per[:-1], out=gw[1:])
    total = int(per.sum()) if len(per) else 0
    sid = np.repeat(np.arange(len(per)), per)
    pos = np.arange(total, dtype=np.int64) - gw[sid]
    Ls = L[sid]
    kk = np.where(pos < Ls, pos, pos - Ls)           # index within the sequence (joint: its first bases)
    ok = kk < Ls
    r = rev[sid]
    src = src0[sid] + np.where(r, Ls - 1 - kk, kk)
    src = np.where(ok, src, 0)
    b = np.asarray(bases)[src] if total else np.zeros(0, np.uint8)
    b = np.where(r, _COMP_TABLE[b], b)
    out = np.where(ok, b, np.uint8(ord("N"))).astype(np.uint8)
    return out, gw, L.astype(np.int32)


class SeqList:
    """CHostSeqList: concatenated sequences, each followed by its first l-1
    bases (the joint, utilAddSequence.cu:6-47), with gateway prefix sums."""

    def __init__(self, lmer: int):
        self.l = lmer
        self.labels: list = []
        self.start_idx: list = []
        self._parts: list = []
        self.lengths: list = []
        self.gateway: list = []

    def _add(self, label, seq: bytes, start_idx=0):
        j = seq[: self.l - 1]
        j = j + b"N" * (self.l - 1 - len(j))
        self._parts.append(seq + j)
        self.labels.append(label)
        self.start_idx.append(start_idx)
        self.lengths.append(len(seq))
        if not self.gateway:
            self.gateway.append(0)
        self.gateway.append(self.gateway[-1] + len(seq) + self.l - 1)

    def add_targets(self, seqs, labels=None, start_idx=None):
        """CHostSeqList_target::add (CHostSeqList_target.cu:8-33)."""
        for i, s in enumerate(seqs):
            self._add(labels[i] if labels else "t%d" % len(self.labels), bytes(s),
                      start_idx[i] if start_idx else 0)
        return self

    def add_queries(self, seqs, labels=None):
        """CHostSeqList_query::add: '+' strand then the reverse complement
        (CHostSeqList_query.cu:11-54)."""
        for i, s in enumerate(seqs):
            lab = labels[i] if labels else "q%d" % (len(self.labels) // 2)
            self._add(lab, bytes(s))
            self._add(lab, _comp(bytes(s)))
        return self

    @property
    def bases(self) -> bytes:
        return b"".join(self._parts)

    def window(self, b: int, e: int):
        """getBaseArray/getGateway/getLengthArray(b, e) (CHostSeqList.cu:15-70):
        the base array of sequences b..e-1, window-relative starts, lengths."""
        g = self.gateway
        bases = self.bases[g[b]:g[e]]
        gw = np.asarray([g[i] - g[b] for i in range(b, e)], dtype=np.int32)
        ln = np.asarray(self.lengths[b:e], dtype=np.int32)
        return bases, gw, ln


def _ptr(b):
    """Pointer argument for bytes or a contiguous numpy array (no copy)."""
    if isinstance(b, np.ndarray):
        assert b.flags.c_contiguous
        return b.ctypes.data
    return b


def _hits_to_numpy(h: N.clast_hits) -> dict:
    n = int(h.n)
    out = {}
    for f in HIT_FIELDS:
        ptr = getattr(h, f)
        dt = np.float64 if f == "evalue" else np.int32
        out[f] = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)
    return out


class _MapResultOwner:
    """Keeps one clast_map result (pinned buffers of the context) alive while
    any of its numpy views exists; releases it afterwards."""

    def __init__(self, engine, r):
        self.engine = engine
        self.r = r

    def __del__(self):
        if self.r is not None and getattr(self.engine, "ctx", None):
            N.load().clast_map_result_free(C.byref(self.r))
        self.r = None


class TsvText:
    """A result text held in the library's pinned buffer (clast_format_tsv)."""

    def __init__(self, engine, t, n_loads):
        self._lib = engine._lib
        self.t = t
        n = int(t.n_bytes)
        self.n_bytes = n
        self.view = memoryview((C.c_char * max(n, 1)).from_address(t.text))[:n]
        self.load_offsets = np.ctypeslib.as_array(t.load_offsets, shape=(n_loads + 1,)).copy()

    def write(self, path, threads: int = 8):
        """The text as a new file at path (clast_write_file)."""
        rc = self._lib.clast_write_file(os.fsencode(path), self.t.text if self.n_bytes else None, self.n_bytes,
                                        threads)
        if rc != 0:
            raise OSError("cannot write %s" % path)

    def release(self):
        if self.t is not None:
            self.view = None
            self._lib.clast_tsv_free(C.byref(self.t))
            self.t = None

    __del__ = release


class MapResult(dict):
    """Fields of a clast_map result (numpy views of the library's pinned
    arrays); ``owner`` keeps the library result alive."""
    owner = None


def flat_labels(labels):
    """(chars, offsets) of a list of str / bytes labels (clast_labels)."""
    enc = [x.encode() if isinstance(x, str) else bytes(x) for x in labels]
    offsets = np.zeros(len(enc) + 1, dtype=np.int64)
    if enc:
        np.cumsum([len(x) for x in enc], out=offsets[1:])
    return b"".join(enc), offsets


def _map_result_arrays(engine, r, n_loads) -> dict:
    """Zero-copy numpy views of a clast_map result."""
    owner = _MapResultOwner(engine, r)
    n = int(r.n)
    out = MapResult()
    out.owner = owner
    out.n_loads = n_loads
    for f in MAP_FIELDS:
        ct = C.c_double if f == "evalue" else C.c_int32
        buf = (ct * max(n, 1)).from_address(C.cast(getattr(r, f), C.c_void_p).value)
        buf._owner = owner
        out[f] = np.frombuffer(buf, dtype=np.float64 if f == "evalue" else np.int32, count=n)
    lo = (C.c_int64 * (n_loads + 1)).from_address(C.cast(r.load_offsets, C.c_void_p).value)
    lo._owner = owner
    out["load_offsets"] = np.frombuffer(lo, dtype=np.int64, count=n_loads + 1)
    return out


class HashTable:
    """Resident index of one target window (CDeviceHashTable)."""

    def __init__(self, engine: "Engine", handle: int, t_begin: int):
        self.engine = engine
        self.handle = handle
        self.t_begin = t_begin

    def close(self):
        if self.handle:
            N.load().clast_index_free(self.handle)
            self.handle = None

    __del__ = close


class Targets:
    """Every target window of every RAM load, resident in HBM."""

    def __init__(self, handle, engine=None):
        self.handle = handle
        self.engine = engine  # the context must outlive its indexes

    def close(self):
        if self.handle:
            N.load().clast_targets_free(self.handle)
            self.handle = None

    __del__ = close


class Engine:
    """One device context (clast_ctx_create)."""

    def __init__(self, device: int = 0):
        lib = N.load()
        h = C.c_void_p()
        rc = lib.clast_ctx_create(device, C.byref(h))
        if rc != 0:
            raise ClastError(rc, "cannot create a context on device %d" % device)
        self._lib = lib
        self.ctx = h

    def close(self):
        if getattr(self, "ctx", None):
            self._lib.clast_ctx_destroy(self.ctx)
            self.ctx = None

    __del__ = close

    def _check(self, rc):
        if rc != 0:
            raise ClastError(rc, self._lib.clast_last_error(self.ctx).decode(errors="replace"))

    # -- the reference seam ------------------------------------------------
    def hash_table_window(self, s: Setting, bases, gateway, lengths, t_begin: int) -> HashTable:
        """``bases``: bytes or a contiguous uint8 numpy array (no copy)."""
        gw = np.ascontiguousarray(gateway, dtype=np.int32)
        ln = np.ascontiguousarray(lengths, dtype=np.int32)
        out = C.c_void_p()
        p = s.c()
        self._check(self._lib.clast_index_build(self.ctx, C.byref(p), _ptr(bases), len(bases), gw.ctypes.data,
                                                ln.ctypes.data, len(gw), t_begin, C.byref(out)))
        return HashTable(self, out.value, t_begin)

    def hash_table(self, s: Setting, targets: SeqList, t_begin: int, t_end: int) -> HashTable:
        """CDeviceHashTable(setting, targetList, t_begin, t_end)."""
        bases, gw, ln = targets.window(t_begin, t_end)
        return self.hash_table_window(s, bases, gw, ln, t_begin)

    def hit_list_window(self, s: Setting, ix: HashTable, q_bases: bytes, q_gateway, q_lengths,
                        q_begin: int) -> dict:
        gw = np.ascontiguousarray(q_gateway, dtype=np.int32)
        ln = np.ascontiguousarray(q_lengths, dtype=np.int32)
        h = N.clast_hits()
        p = s.c()
        self._check(self._lib.clast_search(self.ctx, ix.handle, C.byref(p), _ptr(q_bases), len(q_bases),
                                           gw.ctypes.data, ln.ctypes.data, len(gw), q_begin, C.byref(h)))
        try:
            return _hits_to_numpy(h)
        finally:
            self._lib.clast_hits_free(C.byref(h))

    def hit_list_window_noalloc(self, s: Setting, ix: HashTable, q_bases: bytes, q_gateway, q_lengths,
                                q_begin: int, capacity: int) -> dict:
        """clast_search_noalloc: hit_list_window on the library's fixed
        scratch, writing into host arrays of ``capacity`` hits owned here.
        Raises ClastError (with ``needed`` set when the capacity was short)."""
        gw = np.ascontiguousarray(q_gateway, dtype=np.int32)
        ln = np.ascontiguousarray(q_lengths, dtype=np.int32)
        cap = int(capacity)
        bufs = {f: np.empty(max(cap, 1), np.float64 if f == "evalue" else np.int32) for f in HIT_FIELDS}
        h = N.clast_hits()
        for f in HIT_FIELDS:
            ct = C.c_double if f == "evalue" else C.c_int32
            setattr(h, f, bufs[f].ctypes.data_as(C.POINTER(ct)))
        p = s.c()
        rc = self._lib.clast_search_noalloc(self.ctx, ix.handle, C.byref(p), q_bases, len(q_bases), gw.ctypes.data,
                                            ln.ctypes.data, len(gw), q_begin, cap, C.byref(h))
        if rc != 0:
            err = ClastError(rc, self._lib.clast_last_error(self.ctx).decode(errors="replace"))
            err.needed = int(h.n)
            raise err
        n = int(h.n)
        return {f: bufs[f][:n] for f in HIT_FIELDS}

    def hit_list_noalloc(self, s: Setting, ix: HashTable, queries: SeqList, q_begin: int, q_end: int,
                         capacity: int) -> dict:
        """hit_list through clast_search_noalloc."""
        bases, gw, ln = queries.window(2 * q_begin, 2 * q_end)
        return self.hit_list_window_noalloc(s, ix, bases, gw, ln, 2 * q_begin, capacity)

    def hit_list(self, s: Setting, ix: HashTable, queries: SeqList, q_begin: int, q_end: int) -> dict:
        """CDeviceSeqList_query(s, q, q_begin, q_end) + CDeviceHitList(s, h, q,
        t_begin, 2*q_begin) + getResult: the window's hits as numpy arrays
        (t_id, t_idx, q_id, q_idx, t_len, q_len, match, score, evalue)."""
        bases, gw, ln = queries.window(2 * q_begin, 2 * q_end)
        return self.hit_list_window(s, ix, bases, gw, ln, 2 * q_begin)

    # -- whole job ----------------------------------------------------------
    @staticmethod
    def _seqs(bases, offsets):
        """clast_seqs over a numpy array (host) or an object with a
        ``data_ptr()`` method on the context's GPU (e.g. a torch CUDA tensor)."""
        o = np.ascontiguousarray(offsets, dtype=np.int64)
        if hasattr(bases, "data_ptr"):
            dev = 1 if getattr(bases, "is_cuda", False) else 0
            ptr, keep = bases.data_ptr(), bases
        else:
            keep = np.ascontiguousarray(bases, dtype=np.uint8)
            dev, ptr = 0, keep.ctypes.data
        return N.clast_seqs(len(o) - 1, ptr, o.ctypes.data_as(C.POINTER(C.c_int64)), dev), (o, keep)

    def targets(self, s: Setting, bases, offsets: np.ndarray, load_sizes, t_vram: int) -> Targets:
        """Index of every target window (``bases``: numpy uint8, pinned or
        CUDA torch tensor)."""
        ls = np.ascontiguousarray(load_sizes, dtype=np.int64)
        seqs, _keep = self._seqs(bases, offsets)
        out = C.c_void_p()
        p = s.c()
        self._check(self._lib.clast_targets_create(self.ctx, C.byref(p), int(t_vram), C.byref(seqs), len(ls),
                                                   ls.ctypes.data, C.byref(out)))
        return Targets(out.value, self)

    def save_targets(self, targets: Targets, path: str) -> None:
        """clast_targets_save: every resident window index to one file."""
        self._check(self._lib.clast_targets_save(self.ctx, targets.handle, os.fsencode(path)))

    def load_targets(self, s: Setting, path: str) -> Targets:
        """clast_targets_load: indexes written by save_targets, for settings
        with the same lmer / stride / cut_repeat."""
        out = C.c_void_p()
        p = s.c()
        self._check(self._lib.clast_targets_load(self.ctx, C.byref(p), os.fsencode(path), C.byref(out)))
        return Targets(out.value, self)

    def map(self, s: Setting, targets: Targets, bases, offsets: np.ndarray, load_sizes, q_vram: int) -> dict:
        """Every read against every target window; hits per query load in
        the order CHostResultHolder::fixResult leaves them."""
        t0 = time.perf_counter()
        ls = np.ascontiguousarray(load_sizes, dtype=np.int64)
        seqs, _keep = self._seqs(bases, offsets)
        r = N.clast_map_result()
        p = s.c()
        t1 = time.perf_counter()
        self._check(self._lib.clast_map(self.ctx, targets.handle, C.byref(p), int(q_vram), C.byref(seqs), len(ls),
                                        ls.ctypes.data, C.byref(r)))
        t2 = time.perf_counter()
        out = _map_result_arrays(self, r, len(ls))
        self.last_map_py_ms = ((t1 - t0) * 1e3, (t2 - t1) * 1e3, (time.perf_counter() - t2) * 1e3)
        return out

    def format_tsv_text(self, targets: Targets, result: dict, read_labels, target_labels, start_idx=None,
                        num_out: int = -1) -> "TsvText":
        """clast_format_tsv, keeping the library's text buffer: a TsvText whose
        ``view`` is the text (valid until ``release()``), so that it can be
        written while the next map runs."""
        rl = read_labels if isinstance(read_labels, tuple) else flat_labels(read_labels)
        tl = target_labels if isinstance(target_labels, tuple) else flat_labels(target_labels)
        roff = np.ascontiguousarray(rl[1], dtype=np.int64)
        toff = np.ascontiguousarray(tl[1], dtype=np.int64)
        rlab = N.clast_labels(len(roff) - 1, C.cast(C.c_char_p(rl[0]), C.c_void_p),
                              roff.ctypes.data_as(C.POINTER(C.c_int64)))
        tlab = N.clast_labels(len(toff) - 1, C.cast(C.c_char_p(tl[0]), C.c_void_p),
                              toff.ctypes.data_as(C.POINTER(C.c_int64)))
        si = None if start_idx is None else np.ascontiguousarray(start_idx, dtype=np.int32)
        t = N.clast_tsv()
        self._check(self._lib.clast_format_tsv(self.ctx, targets.handle, C.byref(result.owner.r), result.n_loads,
                                               C.byref(rlab), C.byref(tlab), None if si is None else si.ctypes.data,
                                               int(num_out), C.byref(t)))
        return TsvText(self, t, result.n_loads)

    def format_tsv(self, targets: Targets, result: dict, read_labels, target_labels, start_idx=None,
                   num_out: int = -1, out=None):
        """clast_format_tsv: the reference's 10-column text of a map result
        (every query load in order).  ``read_labels`` / ``target_labels``:
        every read / target record given to map() / targets(), or their
        flat_labels() (chars, offsets).  Returns the text as bytes, or, with
        ``out`` (a binary file), writes it there straight from the library's
        buffer and returns its length.  The byte offset of every load's text
        is left in ``last_tsv_load_offsets``."""
        rl = read_labels if isinstance(read_labels, tuple) else flat_labels(read_labels)
        tl = target_labels if isinstance(target_labels, tuple) else flat_labels(target_labels)
        roff = np.ascontiguousarray(rl[1], dtype=np.int64)
        toff = np.ascontiguousarray(tl[1], dtype=np.int64)
        rlab = N.clast_labels(len(roff) - 1, C.cast(C.c_char_p(rl[0]), C.c_void_p),
                              roff.ctypes.data_as(C.POINTER(C.c_int64)))
        tlab = N.clast_labels(len(toff) - 1, C.cast(C.c_char_p(tl[0]), C.c_void_p),
                              toff.ctypes.data_as(C.POINTER(C.c_int64)))
        si = None if start_idx is None else np.ascontiguousarray(start_idx, dtype=np.int32)
        t = N.clast_tsv()
        self._check(self._lib.clast_format_tsv(self.ctx, targets.handle, C.byref(result.owner.r), result.n_loads,
                                               C.byref(rlab), C.byref(tlab), None if si is None else si.ctypes.data,
                                               int(num_out), C.byref(t)))
        try:
            n = int(t.n_bytes)
            self.last_tsv_load_offsets = np.ctypeslib.as_array(t.load_offsets, shape=(result.n_loads + 1,)).copy()
            if out is None:
                return C.string_at(t.text, n) if n else b""
            if isinstance(out, (str, bytes, os.PathLike)):
                if self._lib.clast_write_file(os.fsencode(out), t.text if n else None, n, 8) != 0:
                    raise OSError("cannot write %s" % os.fsdecode(out))
            elif n:
                out.write(memoryview((C.c_char * n).from_address(t.text)))
            return n
        finally:
            self._lib.clast_tsv_free(C.byref(t))

    def stats(self) -> dict:
        """clast_get_stats: CUDA-event timings and counts of the last
        targets()/map() calls."""
        st = N.clast_stats()
        self._check(self._lib.clast_get_stats(self.ctx, C.byref(st)))
        return {f: getattr(st, f) for f, _ in N.clast_stats._fields_}

    def trim(self) -> None:
        """clast_ctx_trim: hand back the device memory kept for reuse."""
        self._check(self._lib.clast_ctx_trim(self.ctx))

    def int32_peak(self) -> float:
        """Measured INT32 tera-ops/s of this GPU (clast_int32_peak)."""
        v = C.c_double()
        self._check(self._lib.clast_int32_peak(self.ctx, C.byref(v)))
        return v.value

    def last_map_stats(self):
        ms = C.c_double()
        k = C.c_int64()
        self._check(self._lib.clast_last_map_stats(self.ctx, C.byref(ms), C.byref(k)))
        return ms.value, k.value


PENDING = 1
ERR_CANCELLED = -5


class Server:
    """The served form (clast_server_*): resident targets, requests batched
    as they arrive, ``lanes`` batches on the GPU at once.  Results are dicts
    of MAP_FIELDS (read = record index within the request) plus
    ``load_offsets``, copied out of the library."""

    def __init__(self, engine: "Engine", targets: Targets, s: Setting, lanes: int = 4, q_vram: int = 2_000_000,
                 q_ram: int = 32_000_000, max_batch_bases: int = 8_000_000, hbm_budget: int = 0,
                 hbm_reserve: int = 0):
        self._lib = N.load()
        self.engine, self.targets = engine, targets
        self.q_ram = q_ram
        self._nloads = {}
        cfg = N.clast_server_config(lanes, q_vram, q_ram, 0, max_batch_bases, hbm_budget, hbm_reserve)
        p = s.c()
        h = C.c_void_p()
        engine._check(self._lib.clast_server_create(engine.ctx, targets.handle, C.byref(p), C.byref(cfg),
                                                    C.byref(h)))
        self.handle = h

    def _check(self, rc):
        if rc != 0:
            raise ClastError(rc, self._lib.clast_server_last_error(self.handle).decode(errors="replace"))

    def submit(self, bases, offsets) -> int:
        o = np.ascontiguousarray(offsets, dtype=np.int64)
        b = np.ascontiguousarray(bases, dtype=np.uint8)
        seqs = N.clast_seqs(len(o) - 1, b.ctypes.data, o.ctypes.data_as(C.POINTER(C.c_int64)), 0)
        rid = C.c_int64()
        self._check(self._lib.clast_server_submit(self.handle, C.byref(seqs), C.byref(rid)))
        # the request's RAM loads (the same rule the server applies)
        self._nloads[rid.value] = len(ram_loads(np.diff(o), self.q_ram)[1])
        return rid.value

    def poll(self, rid: int, timeout_ms: int = -1):
        """The request's hits when done, None while it is pending; raises
        ClastError when it failed or was cancelled."""
        r = N.clast_map_result()
        rc = self._lib.clast_server_poll(self.handle, int(rid), int(timeout_ms), C.byref(r))
        if rc == PENDING:
            return None
        self._check(rc)
        n = int(r.n)
        out = {}
        for f in MAP_FIELDS:
            dt = np.float64 if f == "evalue" else np.int32
            out[f] = np.ctypeslib.as_array(getattr(r, f), shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)
        nl = self._nloads.get(int(rid), 0)
        out["load_offsets"] = np.ctypeslib.as_array(r.load_offsets, shape=(nl + 1,)).copy()
        return out

    def cancel(self, rid: int) -> None:
        self._check(self._lib.clast_server_cancel(self.handle, int(rid)))

    def release(self, rid: int) -> None:
        self._check(self._lib.clast_server_release(self.handle, int(rid)))
        self._nloads.pop(int(rid), None)

    def times(self, rid: int):
        """(queued, started, finished) steady-clock ns (time.monotonic_ns)."""
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        self._check(self._lib.clast_server_times(self.handle, int(rid), C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def stats(self) -> dict:
        st = N.clast_server_stats()
        self._check(self._lib.clast_server_get_stats(self.handle, C.byref(st)))
        return {f: getattr(st, f) for f, _ in N.clast_server_stats._fields_}

    def close(self):
        if getattr(self, "handle", None):
            self._lib.clast_server_destroy(self.handle)
            self.handle = None

    __del__ = close


def verify_targets_file(s: Setting, path: str):
    """clast_targets_verify: (ok, reason) for an index file, on the host."""
    err = C.create_string_buffer(512)
    p = s.c()
    rc = N.load().clast_targets_verify(C.byref(p), os.fsencode(path), err, len(err))
    return rc == 0, err.value.decode(errors="replace")


def run_clast(argv) -> tuple:
    """The reference's command line (``clast -t T.fa -q Q.fa -o out.tsv ...``)
    on the GPU.  Returns (exit code, error message)."""
    lib = N.load()
    args = ["clast"] + [str(a) for a in argv]
    arr = (C.c_char_p * len(args))(*[a.encode() for a in args])
    err = C.create_string_buffer(1024)
    rc = lib.clast_cli_main(len(args), arr, err, len(err))
    return rc, err.value.decode(errors="replace")
