"""FASTA fixtures written at test time (seeded)."""
import os

import numpy as np

from clast_b200 import synth


def write_pair(tmp, seed, target_bp=60_000, n_contigs=4, n_reads=200, read_len=150, width=60, **kw):
    rng = np.random.Generator(np.random.PCG64(seed))
    t = synth.make_target(rng, target_bp, n_contigs=n_contigs, median=target_bp / max(1, n_contigs) * 0.8)
    q = synth.make_reads(rng, t, n_reads, length=read_len, **kw)
    tp, qp = os.path.join(tmp, "t%d.fa" % seed), os.path.join(tmp, "q%d.fa" % seed)
    t.to_fasta(tp, width=width)
    q.to_fasta(qp, width=width)
    return tp, qp, t, q


def write_quirky(tmp, seed):
    """Target and query files with the loader's special cases: '@startIdx'
    lines (preprocessDB output), lowercase, spaces, CRLF line ends, blank
    lines between records, a '>' inside a header and a second query file."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = synth.make_target(rng, 30_000, n_contigs=3, median=9000)
    q = synth.make_reads(rng, t, 80)
    tp = os.path.join(tmp, "tq%d.fa" % seed)
    with open(tp, "wb") as f:
        for i in range(len(t)):
            s = t.seq(i).tobytes()
            f.write(b">ctg%d some>description\n" % i)
            f.write(b"@%d\n" % (1000 * (i + 1)))
            for k in range(0, len(s), 70):
                line = s[k:k + 70]
                if k % 700 == 0:
                    line = line.lower()
                f.write(line + (b"\r\n" if (i == 1 and k % 140 == 0) else b"\n"))
            f.write(b"\n")
    q1, q2 = os.path.join(tmp, "qa%d.fa" % seed), os.path.join(tmp, "qb%d.fa" % seed)
    with open(q1, "wb") as f1, open(q2, "wb") as f2:
        for i in range(len(q)):
            f = f1 if i < len(q) // 2 else f2
            s = q.seq(i).tobytes()
            f.write(b">read%d\n" % i)
            f.write(s[:50] + b"\n" + s[50:100].replace(b"A", b"a", 3) + b" " + s[100:] + b"\n")
    return tp, [q1, q2]


def write_adversarial(tmp, seed):
    """Loader edge cases: '@' before the first header and between records,
    an empty header, sequence before any header, a blank line inside a
    record (the rest of that record is dropped), CR line ends, an over-long
    query record (skipped under a small -qRAM) and queries split over three
    files so that RAM loads span files."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = synth.make_target(rng, 40_000, n_contigs=4, median=9000)
    q = synth.make_reads(rng, t, 150)
    tp = os.path.join(tmp, "tadv%d.fa" % seed)
    with open(tp, "wb") as f:
        f.write(b"ACGTACGTACGTACGT\n@77\n")  # before any header: ignored / applies to record 0
        for i in range(len(t)):
            s = t.seq(i).tobytes()
            f.write(b">ctg%d\r\n" % i if i == 2 else b">ctg%d\n" % i)
            for k in range(0, len(s), 80):
                f.write(s[k:k + 80] + b"\n")
            if i == 1:
                f.write(b"@%d\n" % 4242)  # after the sequence: belongs to this record
        f.write(b">\nACGTACGTACGTACGTACGTACGTACGTACGT\n")  # empty header: dropped
    long_read = synth.make_reads(rng, t, 1, length=7000)
    qs = [os.path.join(tmp, "qadv%d_%d.fa" % (seed, k)) for k in range(3)]
    fs = [open(p, "wb") for p in qs]
    try:
        for i in range(len(q)):
            f = fs[min(2, i * 3 // len(q))]
            s = q.seq(i).tobytes()
            f.write(b">read%d\n" % i)
            if i % 17 == 5:  # a blank line inside the record: only the first half counts
                f.write(s[:80] + b"\n\n" + s[80:] + b"\n")
            else:
                f.write(s[:75] + b"\n" + s[75:] + b"\n")
            if i == len(q) // 2:
                f.write(b">long\n" + long_read.seq(0).tobytes() + b"\n")
    finally:
        for f in fs:
            f.close()
    return tp, qs
