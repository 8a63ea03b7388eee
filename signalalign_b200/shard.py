"""Read sharding across GPUs (one process per GPU).

Reads are independent, so a batch splits across ranks with no collective on the data path: every
rank computes the same assignment (largest band first, each read to the least-loaded rank, the
LPT rule), aligns its own reads, and rank 0 gathers the per-read results.  Band areas come from the
host band geometry (band_construct), so the assignment is known before any device work.
"""
import numpy as np


def band_areas(reads, p):
    """Band cells of each read (sum over its anti-diagonals of the band width)."""
    from signalalign_b200 import api
    out = []
    for r in reads:
        k = r.sm.kmer_length
        lX = max(len(r.reference) - (k - 1), 0)
        lo, hi = api.band_construct(r.anchors, lX, len(r.events), p.diagonal_expansion)
        out.append(int(np.sum((np.asarray(hi) - np.asarray(lo)) // 2 + 1)))
    return out


def assign(areas, world):
    """LPT assignment: read indices per rank, each rank's reads in ascending index order."""
    load = [0] * world
    shards = [[] for _ in range(world)]
    for i in sorted(range(len(areas)), key=lambda j: (-areas[j], j)):
        r = min(range(world), key=lambda q: (load[q], q))
        shards[r].append(i)
        load[r] += areas[i]
    return [sorted(s) for s in shards], load


def align_sharded(reads, p, rank, world, align=None, group=None, areas=None):
    """Align `reads` over `world` ranks; returns, on rank 0, a list with one (status, pairs,
    log_likelihood) per read in input order (None on the other ranks).  `align(reads, p)` returns
    the same triples for a list of reads (default: the batched FP32 form on this rank's GPU)."""
    import torch.distributed as dist
    if areas is None:
        areas = band_areas(reads, p)
    shards, _ = assign(areas, world)
    mine = shards[rank]
    if align is None:
        align = _align_batch
    results = align([reads[i] for i in mine], p) if mine else []
    local = list(zip(mine, results))
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(local, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(reads)
    for part in gathered:
        for i, res in part:
            out[i] = res
    return out


def _align_batch(reads, p):
    from signalalign_b200 import api
    b = api.align_batch(reads, p)
    return [(b.status(i), b.pairs(i), b.log_likelihood(i)) for i in range(len(reads))]
