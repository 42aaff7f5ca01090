"""Seeded synthetic DNA workloads with the shapes of the benchmark configurations.

There is no public dataset behind these workloads; every target and read set
is generated from a fixed seed, so the same call gives the same bytes on any
machine.  Shapes:

* ``small``  -- one 1 Mbp target record of uniform ACGT with 0.1 % of bases in
  N runs (geometric length, mean 10); 1,000 reads of 150 bp sampled uniformly
  from it with 2 % substitutions and 0.5 % indel events (geometric length,
  mean 2), half reverse-complemented, 5 % uniform random decoys.
* ``medium`` -- 100 Mbp in 200 contigs with log-normal lengths (median 300 kbp),
  10 % of bases in 500 repeat families of 300 bp - 6 kbp copied at 85-99 %
  identity; 1,000,000 reads of 150 bp from the same error model.
* ``uneven`` -- the medium target; 200,000 reads with log-uniform lengths in
  50 bp - 10 kbp, per-read error rate uniform in 1-12 % (70 % substitutions,
  30 % indels).
* ``large``  -- a 3 Gbp genome of 24 chromosomes of 50-250 Mbp, 45 % of bases
  in 1,000 repeat families of 300 bp - 6 kbp at 80-99 % identity, 1 % of bases
  in N blocks (geometric length, mean 1 kbp); 5,000,000 reads of 150 bp
  (medium's error model).  Chromosomes are labelled ``chr<i>``.

Reads carry labels ``r<i>``; targets ``ctg<i>``.  Sizes scale with the
arguments so tests can use small versions of each shape.
"""
from __future__ import annotations

import dataclasses
import numpy as np

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)
_COMP = np.zeros(256, dtype=np.uint8)
_COMP[:] = ord("N")
for a, b in (("A", "T"), ("C", "G"), ("G", "C"), ("T", "A")):
    _COMP[ord(a)] = ord(b)


def revcomp(seq: np.ndarray) -> np.ndarray:
    """Reverse complement of an uint8 ASCII array (non-ACGT -> N)."""
    return _COMP[seq[::-1]]


@dataclasses.dataclass
class SeqSet:
    """Concatenated sequences: ``bases[offsets[i]:offsets[i+1]]`` is record i."""
    labels: list
    bases: np.ndarray      # uint8 ASCII, no separators
    offsets: np.ndarray    # int64, len(labels)+1

    def __len__(self):
        return len(self.labels)

    def seq(self, i: int) -> np.ndarray:
        return self.bases[self.offsets[i]:self.offsets[i + 1]]

    @property
    def lengths(self) -> np.ndarray:
        return np.diff(self.offsets)

    def to_fasta(self, path: str, width: int = 60) -> None:
        """Writes FASTA with ``width``-column sequence lines."""
        with open(path, "wb") as f:
            for i, lab in enumerate(self.labels):
                s = self.seq(i).tobytes()
                f.write(b">" + lab.encode() + b"\n")
                for k in range(0, len(s), width):
                    f.write(s[k:k + width] + b"\n")


def _rand_bases(rng, n):
    return ACGT[rng.integers(0, 4, size=n, dtype=np.uint8)]


def make_target(rng, total_bp: int, n_contigs: int = 1, median: float | None = None,
                n_frac: float = 0.001, n_run_mean: float = 10.0, repeat_frac: float = 0.0,
                n_families: int = 0, fam_len=(300, 6000), fam_ident=(0.85, 0.99), lengths=None) -> SeqSet:
    """Random contigs (log-normal lengths when ``n_contigs > 1``, or the given
    ``lengths``) with N runs and optional repeat families."""
    if lengths is not None:
        lens = np.asarray(lengths, dtype=np.int64)
    elif n_contigs == 1:
        lens = np.array([total_bp], dtype=np.int64)
    else:
        mean = total_bp / n_contigs
        med = median if median else mean * 0.6
        sigma = float(np.sqrt(max(2.0 * np.log(mean / med), 1e-6)))
        raw = rng.lognormal(np.log(med), sigma, size=n_contigs)
        lens = np.maximum((raw / raw.sum() * total_bp).astype(np.int64), 1000)
        lens[int(np.argmax(lens))] += total_bp - lens.sum()
    bases = _rand_bases(rng, int(lens.sum()))
    offsets = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    total = len(bases)
    # repeat families: consensus copies at per-copy identity, substitutions only
    if repeat_frac > 0 and n_families > 0:
        budget = int(repeat_frac * total)
        per_fam = budget // n_families
        for _ in range(n_families):
            flen = int(np.exp(rng.uniform(np.log(fam_len[0]), np.log(fam_len[1]))))
            cons = _rand_bases(rng, flen)
            ncopy = max(2, per_fam // flen)
            for _ in range(ncopy):
                ident = rng.uniform(*fam_ident)
                copy = cons.copy()
                mut = rng.random(flen) > ident
                copy[mut] = _rand_bases(rng, int(mut.sum()))
                c = int(rng.integers(0, len(lens)))
                if lens[c] <= flen:
                    continue
                at = offsets[c] + int(rng.integers(0, lens[c] - flen))
                bases[at:at + flen] = copy
    # N runs
    if n_frac > 0:
        n_runs = int(n_frac * total / n_run_mean)
        starts = rng.integers(0, total, size=n_runs)
        runs = rng.geometric(1.0 / n_run_mean, size=n_runs)
        for s, r in zip(starts, runs):
            bases[s:s + r] = ord("N")
    labels = ["ctg%d" % i for i in range(len(lens))]
    return SeqSet(labels, bases, offsets)


def chromosome_lengths(rng, n: int, total_bp: int, lo: int, hi: int):
    """n lengths in [lo, hi] summing to total_bp (uniform draws, rescaled)."""
    x = rng.uniform(lo, hi, size=n)
    x = x / x.sum() * total_bp
    x = np.clip(x, lo, hi).astype(np.int64)
    x[int(np.argmin(x))] += total_bp - int(x.sum())
    return x


def _mutate(rng, src: np.ndarray, out_len: int, sub: float, indel: float, indel_mean: float) -> np.ndarray:
    """Applies substitutions and indel events to ``src`` and returns the first
    ``out_len`` bases of the mutated sequence (``src`` is long enough)."""
    n = len(src)
    ev = np.flatnonzero(rng.random(n) < indel)
    if len(ev) == 0:
        seq = src.copy()
    else:
        parts, prev = [], 0
        for e in ev:
            if e < prev:
                continue
            ln = int(rng.geometric(1.0 / indel_mean))
            parts.append(src[prev:e])
            if rng.random() < 0.5:   # insertion before e
                parts.append(_rand_bases(rng, ln))
                prev = e
            else:                    # deletion of e .. e+ln-1
                prev = e + ln
        parts.append(src[prev:])
        seq = np.concatenate(parts)
    seq = seq[:out_len].copy()
    m = rng.random(len(seq)) < sub
    if m.any():
        # a substitution always changes the base
        cur = seq[m]
        shift = rng.integers(1, 4, size=int(m.sum()))
        idx = np.searchsorted(ACGT, cur)
        valid = (idx < 4) & (ACGT[np.minimum(idx, 3)] == cur)
        new = ACGT[(np.where(valid, idx, 0) + shift) % 4]
        seq[m] = new
    return seq


def make_reads(rng, target: SeqSet, n_reads: int, length=150, sub=0.02, indel=0.005,
               indel_mean=2.0, rev_frac=0.5, decoy_frac=0.05, log_uniform=None,
               err_range=None) -> SeqSet:
    """Reads sampled uniformly from the target (by base), with errors,
    reverse-complemented with probability ``rev_frac`` and replaced by random
    decoys with probability ``decoy_frac``.  ``log_uniform=(lo, hi)`` draws
    read lengths log-uniformly; ``err_range=(lo, hi)`` draws a per-read error
    rate split 70/30 between substitutions and indels."""
    tl = target.lengths
    cum = np.concatenate([[0], np.cumsum(tl)])
    seqs = []
    for i in range(n_reads):
        L = length if log_uniform is None else int(np.exp(rng.uniform(np.log(log_uniform[0]),
                                                                     np.log(log_uniform[1]))))
        s_rate, i_rate = sub, indel
        if err_range is not None:
            e = rng.uniform(*err_range)
            s_rate, i_rate = 0.7 * e, 0.3 * e / indel_mean
        if rng.random() < decoy_frac:
            seqs.append(_rand_bases(rng, L))
            continue
        need = L + 8 * int(np.ceil(L * i_rate * indel_mean)) + 16
        for _ in range(100):
            g = int(rng.integers(0, cum[-1]))
            c = int(np.searchsorted(cum, g, side="right") - 1)
            if tl[c] >= need:
                break
        else:
            c = int(np.argmax(tl))
        start = int(rng.integers(0, tl[c] - need + 1))
        src = target.bases[target.offsets[c] + start: target.offsets[c] + start + need]
        r = _mutate(rng, src, L, s_rate, i_rate, indel_mean)
        if rng.random() < rev_frac:
            r = revcomp(r)
        seqs.append(r)
    lens = np.array([len(s) for s in seqs], dtype=np.int64)
    offsets = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    bases = np.concatenate(seqs) if seqs else np.zeros(0, dtype=np.uint8)
    return SeqSet(["r%d" % i for i in range(n_reads)], bases, offsets)


def _mutated_batch(rng, target: SeqSet, B: int, length: int, M: int, sub, indel, indel_mean: float, ok, w):
    """B reads of `length` bases: sources of M bases at uniform target
    positions with substitutions and indel events (rates scalar or per read),
    vectorised.  Returns a (B, length) uint8 array."""
    tl = target.lengths
    sub = np.broadcast_to(np.asarray(sub, dtype=np.float64), (B,))[:, None]
    indel = np.broadcast_to(np.asarray(indel, dtype=np.float64), (B,))[:, None]
    c = ok[rng.choice(len(ok), size=B, p=w)]
    start = target.offsets[c] + (rng.random(B) * (tl[c] - M + 1)).astype(np.int64)
    src = target.bases[start[:, None] + np.arange(M)[None, :]]
    ev = rng.random((B, M)) < indel
    ins = ev & (rng.random((B, M)) < 0.5)
    dele = ev & ~ins
    ln = rng.geometric(1.0 / indel_mean, size=(B, M))
    diff = np.zeros((B, M + 1), dtype=np.int32)
    rb, rc = np.nonzero(dele)
    np.add.at(diff, (rb, rc), 1)
    np.add.at(diff, (rb, np.minimum(rc + ln[rb, rc], M)), -1)
    covered = np.cumsum(diff[:, :M], axis=1) > 0
    n_ins = np.where(ins & ~covered, ln, 0)
    emit = n_ins + (~covered).astype(np.int64)
    cs = np.cumsum(emit, axis=1)
    total = cs[:, -1]
    if (total < length).any():  # pathological deletions: fall back to the source
        short = total < length
        emit[short] = 1
        n_ins[short] = 0
        cs = np.cumsum(emit, axis=1)
    big = int(cs[:, -1].max()) + 1
    flat = (cs + (np.arange(B) * big)[:, None]).ravel()
    o = (np.arange(length)[None, :] + (np.arange(B) * big)[:, None]).ravel()
    j = np.searchsorted(flat, o, side="right").reshape(B, length) - np.arange(B)[:, None] * M
    j = np.minimum(j, M - 1)
    before = np.take_along_axis(cs, j, axis=1) - np.take_along_axis(emit, j, axis=1)
    rank = np.arange(length)[None, :] - before   # rank within position j's emission
    is_ins = rank < np.take_along_axis(n_ins, j, axis=1)
    r = np.take_along_axis(src, j, axis=1)
    r = np.where(is_ins, ACGT[rng.integers(0, 4, size=(B, length))], r)
    m = rng.random((B, length)) < sub
    idx = np.searchsorted(ACGT, r)
    valid = (idx < 4) & (ACGT[np.minimum(idx, 3)] == r)
    newb = ACGT[(np.where(valid, idx, 0) + rng.integers(1, 4, size=(B, length))) % 4]
    return np.where(m & valid, newb, r)


def make_reads_fixed(rng, target: SeqSet, n_reads: int, length=150, sub=0.02, indel=0.005, indel_mean=2.0,
                     rev_frac=0.5, decoy_frac=0.05, batch=65536, first: int = 0) -> SeqSet:
    """Vectorised fixed-length version of :func:`make_reads` (same error model:
    substitutions, indel events of geometric length, reverse strand, decoys).
    Reads come in batches of ``batch``, batch k drawn from its own stream
    (``rng``'s bit generator jumped k + 1 times), so reads [first, first +
    n_reads) of the sequence can be made without the ones before them."""
    base_bg = rng.bit_generator
    tl = target.lengths
    cum = np.concatenate([[0], np.cumsum(tl)])
    pad = 16 + 8 * int(np.ceil(length * indel * indel_mean))
    M = length + pad
    ok = np.flatnonzero(tl >= M)
    if ok.size == 0:
        raise ValueError("target contigs shorter than a read")
    w = tl[ok].astype(np.float64)
    w /= w.sum()
    out = np.empty((n_reads, length), dtype=np.uint8)
    k0 = first // batch
    for k in range(k0, (first + n_reads + batch - 1) // batch):
        rng = np.random.Generator(base_bg.jumped(k + 1))
        B = batch  # every batch draws `batch` reads: any range is a slice of the same sequence
        r = _mutated_batch(rng, target, B, length, M, sub, indel, indel_mean, ok, w)
        rev = rng.random(B) < rev_frac
        r[rev] = _COMP[r[rev, ::-1]]
        dec = rng.random(B) < decoy_frac
        r[dec] = ACGT[rng.integers(0, 4, size=(int(dec.sum()), length))]
        lo, hi = max(first, k * batch), min(first + n_reads, (k + 1) * batch)
        out[lo - first:hi - first] = r[lo - k * batch:hi - k * batch]
    offsets = np.arange(n_reads + 1, dtype=np.int64) * length
    return SeqSet(["r%d" % i for i in range(first, first + n_reads)], out.ravel(), offsets)


def make_reads_var(rng, target: SeqSet, n_reads: int, len_range=(100, 5000), sub=0.02, rev_frac=0.5,
                   decoy_frac=0.0) -> SeqSet:
    """Vectorised reads of log-uniform length in ``len_range`` sampled
    uniformly (by base) from the target, with substitutions at rate ``sub``
    (no indels), reverse-complemented with probability ``rev_frac``, random
    decoys with probability ``decoy_frac``."""
    lo, hi = len_range
    L = np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_reads)).astype(np.int64)
    tl = target.lengths
    ok = np.flatnonzero(tl > hi + 1)
    if ok.size == 0:
        raise ValueError("target contigs shorter than the longest read")
    w = tl[ok].astype(np.float64)
    w /= w.sum()
    c = ok[rng.choice(len(ok), size=n_reads, p=w)]
    start = target.offsets[c] + (rng.random(n_reads) * (tl[c] - L)).astype(np.int64)
    offsets = np.concatenate([[0], np.cumsum(L)]).astype(np.int64)
    total = int(offsets[-1])
    rid = np.repeat(np.arange(n_reads), L)
    k = np.arange(total, dtype=np.int64) - offsets[rid]
    rev = rng.random(n_reads) < rev_frac
    pos = np.where(rev[rid], start[rid] + L[rid] - 1 - k, start[rid] + k)
    b = target.bases[pos]
    b = np.where(rev[rid], _COMP[b], b)
    m = rng.random(total) < sub
    idx = np.searchsorted(ACGT, b)
    valid = (idx < 4) & (ACGT[np.minimum(idx, 3)] == b)
    newb = ACGT[(np.where(valid, idx, 0) + rng.integers(1, 4, size=total)) % 4]
    b = np.where(m & valid, newb, b).astype(np.uint8)
    dec = rng.random(n_reads) < decoy_frac
    if dec.any():
        dmask = dec[rid]
        b[dmask] = ACGT[rng.integers(0, 4, size=int(dmask.sum()))]
    return SeqSet(["r%d" % i for i in range(n_reads)], b, offsets)


def served_requests(rng, n_requests: int, pool: SeqSet, count_range=(1, 10_000)):
    """Read ranges of ``n_requests`` requests with log-uniform read counts in
    ``count_range``, taken one after another from ``pool`` (wrapping
    around): a list of (first read, end read)."""
    lo, hi = count_range
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size=n_requests)).astype(np.int64)
    counts = np.clip(counts, lo, min(hi, len(pool)))
    out, at = [], 0
    for c in counts:
        if at + c > len(pool):
            at = 0
        out.append((at, at + int(c)))
        at += int(c)
    return out


def medium_target(seed: int = 0xC1A57, scale: float = 1.0) -> SeqSet:
    """The target of the ``medium`` (and ``uneven``) workload alone."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return make_target(rng, int(100_000_000 * scale), n_contigs=max(1, int(200 * min(1.0, scale * 10))),
                       median=300_000 * scale, repeat_frac=0.10, n_families=max(1, int(500 * scale)))


def uneven_chunk(seed: int, k: int, n: int, scale: float = 1.0):
    """Chunk k of a chunked uneven read set (reads of 50 bp - 10 kbp, per-read
    error 1-12 %, as ``uneven``) on the medium target, from its own stream, so
    that chunks can be made in parallel processes.  Returns (bases, lengths)."""
    t = medium_target(seed, scale)
    rng = np.random.Generator(np.random.PCG64([seed, 7, k]))
    q = make_reads(rng, t, n, log_uniform=(50, 10_000), err_range=(0.01, 0.12), decoy_frac=0.0)
    return q.bases, np.diff(q.offsets)


def workload(name: str, seed: int = 0xC1A57, scale: float = 1.0, n_reads: int | None = None, first: int = 0):
    """(target, reads) for a named shape; ``scale`` shrinks sizes for tests,
    ``n_reads`` sets the read count; for ``medium`` and ``large`` the reads
    are reads [first, first + n_reads) of one fixed sequence."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if name == "small":
        t = make_target(rng, int(1_000_000 * scale))
        q = make_reads(rng, t, n_reads or max(1, int(1000 * scale)))
    elif name == "medium":
        t = make_target(rng, int(100_000_000 * scale), n_contigs=max(1, int(200 * min(1.0, scale * 10))),
                        median=300_000 * scale, repeat_frac=0.10, n_families=max(1, int(500 * scale)))
        q = make_reads_fixed(rng, t, n_reads or max(1, int(1_000_000 * scale)), first=first)
    elif name == "uneven":
        t = make_target(rng, int(100_000_000 * scale), n_contigs=max(1, int(200 * min(1.0, scale * 10))),
                        median=300_000 * scale, repeat_frac=0.10, n_families=max(1, int(500 * scale)))
        q = make_reads(rng, t, n_reads or max(1, int(200_000 * scale)), log_uniform=(50, 10_000),
                       err_range=(0.01, 0.12), decoy_frac=0.0)
    elif name == "large":
        lens = chromosome_lengths(rng, 24, int(3_000_000_000 * scale), int(50_000_000 * scale),
                                  int(250_000_000 * scale))
        t = make_target(rng, int(lens.sum()), lengths=lens, n_frac=0.01, n_run_mean=1000.0, repeat_frac=0.45,
                        n_families=max(1, int(1000 * scale)), fam_ident=(0.80, 0.99))
        t.labels = ["chr%d" % (i + 1) for i in range(len(t))]
        q = make_reads_fixed(rng, t, n_reads or max(1, int(5_000_000 * scale)), first=first)
    else:
        raise ValueError("unknown workload %r" % name)
    return t, q
