"""Read sharding over several ranks (gloo, world size 2, on CPU).

Each rank aligns its LPT share of the reads and rank 0 gathers the results; here the aligner is the
FP64 CPU oracle, so the test runs without a GPU and covers the multi-rank host path: the assignment
is the same on every rank, covers every read exactly once, balances band area, and the gathered
results equal a single-process run in input order.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import oracle as orc
from signalalign_b200 import api, shard, synth
import workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _workload():
    cfg = synth.config1(seed=41, n_reads=7, span=(150, 600))
    m = W.gaussian_model(cfg)
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED)
    reads = [api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                           scale=rd["scale"], shift=rd["shift"]) for rd in cfg["reads"]]
    return cfg, m, reads


def _oracle_align(m):
    def align(reads, p):
        out = []
        for r in reads:
            om = orc.OracleModel(m, orc.EMIT_DESCALED, r.scale, r.shift, 1.0)
            pairs, tps = orc.aligned_pairs(om, r.reference, r.events, r.anchors,
                                           orc.params(threshold=p.threshold, expansion=p.diagonal_expansion),
                                           with_total_probs=True)
            out.append((0, pairs, float(tps[-1][1]) if len(tps) else 0.0))
        return out
    return align


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg, m, reads = _workload()
        p = api.pairwiseAlignmentBandingParameters_construct()
        areas = shard.band_areas(reads, p)
        shards, load = shard.assign(areas, world)
        np.save(os.path.join(outdir, "shards%d.npy" % rank), np.array([len(s) for s in shards] + sum(shards, [])))
        res = shard.align_sharded(reads, p, rank, world, align=_oracle_align(m), areas=areas)
        if rank == 0:
            np.save(os.path.join(outdir, "gathered.npy"),
                    np.array([(st, len(pr), ll) for st, pr, ll in res], dtype=np.float64))
            for i, (st, pr, ll) in enumerate(res):
                np.save(os.path.join(outdir, "pairs%d.npy" % i), pr)
    finally:
        dist.destroy_process_group()


def test_assignment_lpt():
    areas = [10, 9, 8, 1, 1, 1, 7, 3]
    shards, load = shard.assign(areas, 3)
    assert sorted(sum(shards, [])) == list(range(len(areas)))
    assert [sum(areas[i] for i in s) for s in shards] == load
    # the LPT bound: no rank more than one read above the least-loaded one
    assert max(load) - min(load) <= max(areas)


def test_two_ranks_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    # same assignment on both ranks, every read exactly once
    s0, s1 = np.load(tmp_path / "shards0.npy"), np.load(tmp_path / "shards1.npy")
    assert np.array_equal(s0, s1)
    idx = s0[world:]
    assert sorted(idx.tolist()) == list(range(len(idx)))
    # gathered results equal the single-process oracle, in input order
    cfg, m, reads = _workload()
    p = api.pairwiseAlignmentBandingParameters_construct()
    single = _oracle_align(m)(reads, p)
    got = np.load(tmp_path / "gathered.npy")
    assert len(got) == len(single)
    for i, (st, pr, ll) in enumerate(single):
        assert got[i][0] == st and got[i][1] == len(pr) and abs(got[i][2] - ll) <= 1e-12 * max(1.0, abs(ll))
        assert np.array_equal(np.load(tmp_path / ("pairs%d.npy" % i)), pr)
