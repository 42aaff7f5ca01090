"""Query sharding across GPUs with a replicated target index.

The path partitions naturally: given the window rules, every query window is
independent of the others (CHostSchedular.cu:12-23, 85-129).  Each rank maps
a contiguous run of whole query windows against its own copy of the target
indexes; the shards' results, concatenated in rank order inside every query
RAM load, are the single-GPU result (hits are ordered by read first, and a
shard that starts on a window boundary lays out the same windows as the whole
load does).  No device collective is involved: the results are gathered on
the host of rank 0.
"""
from __future__ import annotations

import numpy as np


def query_windows(lengths, load_sizes, lmer: int, q_vram: int):
    """Index of the first read of every query window (moveQueryWindow,
    CHostSchedular.cu:12-23): within each RAM load, a window grows while the
    bases of its strands, joints included (2 * (len + l - 1) per read), stay
    below q_vram.  Windows never cross a load boundary."""
    lengths = np.asarray(lengths, dtype=np.int64)
    starts = []
    r0 = 0
    for n in load_sizes:
        per = 2 * (lengths[r0:r0 + n] + lmer - 1)
        cum = np.concatenate([[0], np.cumsum(per)])
        qb = 0
        while qb < n:
            # the window [qb, qe) grows while cum[qe + 1] - cum[qb] < q_vram
            # and always holds at least one read
            qe = qb + 1
            lim = cum[qb] + q_vram
            j = int(np.searchsorted(cum, lim, side="left"))  # first index with cum >= lim
            qe = max(qe, min(n, j - 1))
            starts.append(r0 + qb)
            qb = qe
        r0 += n
    return starts


def shard_reads(lengths, load_sizes, lmer: int, q_vram: int, world: int):
    """Splits the reads into `world` contiguous shards that start on query
    window boundaries, balanced by bases.  Returns, per rank, (first read,
    end read, records per load inside the shard, index of each such load)."""
    lengths = np.asarray(lengths, dtype=np.int64)
    n = len(lengths)
    starts = query_windows(lengths, load_sizes, lmer, q_vram) + [n]
    cumb = np.concatenate([[0], np.cumsum(lengths)])
    total = cumb[-1]
    cuts = [0]
    for k in range(1, world):
        target = total * k / world
        # window start whose base offset is closest to the target, not before the previous cut
        cand = [s for s in starts if s >= cuts[-1]]
        best = min(cand, key=lambda s: abs(cumb[s] - target))
        cuts.append(best)
    cuts.append(n)
    load_first = np.concatenate([[0], np.cumsum(load_sizes)]).astype(np.int64)
    shards = []
    for k in range(world):
        a, b = cuts[k], cuts[k + 1]
        sizes, ids = [], []
        for li in range(len(load_sizes)):
            lo, hi = max(a, load_first[li]), min(b, load_first[li + 1])
            if hi > lo:
                sizes.append(int(hi - lo))
                ids.append(li)
        shards.append((int(a), int(b), sizes, ids))
    return shards


def merge_shards(results, shards, n_loads: int):
    """Concatenates per-rank map results (dicts of arrays with per-shard
    ``load_offsets`` and shard-relative ``read``) into the single-GPU layout."""
    fields = [k for k in results[0] if k != "load_offsets"]
    per_load = [[] for _ in range(n_loads)]
    for res, (a, _b, _sizes, ids) in zip(results, shards):
        lo = res["load_offsets"]
        for j, li in enumerate(ids):
            part = {f: res[f][lo[j]:lo[j + 1]] for f in fields}
            part["read"] = part["read"] + a
            per_load[li].append(part)
    out = {f: [] for f in fields}
    offs = [0]
    for li in range(n_loads):
        m = 0
        for part in per_load[li]:
            for f in fields:
                out[f].append(part[f])
            m += len(part["read"])
        offs.append(offs[-1] + m)
    merged = {f: (np.concatenate(v) if v else np.zeros(0)) for f, v in out.items()}
    merged["load_offsets"] = np.asarray(offs, dtype=np.int64)
    return merged


def map_sharded(map_fn, bases, offsets, load_sizes, lmer, q_vram, rank, world, group=None):
    """Maps this rank's shard with ``map_fn(bases, offsets, load_sizes)`` (for
    example ``lambda b, o, ls: engine.map(setting, targets, b, o, ls, q_vram)``
    on this rank's GPU) and gathers every shard on rank 0 over
    torch.distributed (host objects; gloo or NCCL).  Returns the merged result
    on rank 0 and None elsewhere."""
    import torch.distributed as dist
    from .api import MAP_FIELDS
    offsets = np.asarray(offsets, dtype=np.int64)
    lengths = np.diff(offsets)
    shards = shard_reads(lengths, load_sizes, lmer, q_vram, world)
    a, b, sizes, _ids = shards[rank]
    if b > a:
        sub_off = offsets[a:b + 1] - offsets[a]
        res = map_fn(np.asarray(bases[offsets[a]:offsets[b]]), sub_off, sizes)
    else:
        res = {f: np.zeros(0, np.float64 if f == "evalue" else np.int32) for f in MAP_FIELDS}
        res["load_offsets"] = np.zeros(1, np.int64)
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(res, gathered, dst=0, group=group)
    if rank != 0:
        return None
    return merge_shards(gathered, shards, len(load_sizes))
