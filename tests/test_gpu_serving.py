"""Serving loop (sa_server_*): reads submitted as they arrive, continuous batching.

A read's result must be the same alone and in a mix of concurrent reads (the FP32 form's tolerance:
posterior error <= 1e-4, log-likelihood 1e-3 relative), and the same as the batch entry point's.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from signalalign_b200 import synth
import workloads as W

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from signalalign_b200 import api as a
    return a


def _inputs(api, sm, reads):
    return [api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                          scale=rd["scale"], shift=rd["shift"]) for rd in reads]


def _same(api, a, b, thr):
    st_a, pa, lla, _ = a
    st_b, pb, llb, _ = b
    assert st_a == 0 and st_b == 0
    assert len(pa) > 0
    assert W.max_posterior_error(pa, pb, thr) <= FP32_TOL
    assert abs(lla - llb) <= 1e-3 * abs(lla)


def test_result_same_alone_and_in_mix(api):
    cfg = synth.config1(seed=31, n_reads=9, span=(500, 4000))
    sm = W.gpu_model(api, W.gaussian_model(cfg), orc.EMIT_DESCALED)
    reads = _inputs(api, sm, cfg["reads"])
    p = api.pairwiseAlignmentBandingParameters_construct()
    srv = api.Server(max_inflight_cells=50_000_000, max_batches=4)
    try:
        t = srv.submit(reads[0], p)
        srv.wait(t)
        alone = srv.result(t)
        # the same read again, submitted in the middle of a stream of others
        tickets = [srv.submit(r, p) for r in reads[1:5]] + [srv.submit(reads[0], p)] + \
                  [srv.submit(r, p) for r in reads[5:]]
        for tk in tickets:
            srv.wait(tk)
        mixed = [srv.result(tk) for tk in tickets]
    finally:
        srv.close()
    _same(api, alone, mixed[4], p.threshold)
    assert all(m[3] > 0 for m in mixed)
    # and each read as the batch entry point gives it
    batch = api.align_batch(reads, p)
    order = [1, 2, 3, 4, 0, 5, 6, 7, 8]
    for k, r in enumerate(order):
        _same(api, (batch.status(r), batch.pairs(r), batch.log_likelihood(r), 0.0), mixed[k], p.threshold)


def test_server_reports_per_read_errors(api):
    cfg = synth.config1(seed=32, n_reads=2, span=(500, 800))
    sm = W.gpu_model(api, W.gaussian_model(cfg), orc.EMIT_DESCALED)
    reads = _inputs(api, sm, cfg["reads"])
    bad = api.ReadInput(sm=sm, reference="ACGTNNACGTACGTACGT", events=reads[0].events[:20], anchors=np.zeros((0, 2)))
    p = api.pairwiseAlignmentBandingParameters_construct()
    srv = api.Server(max_inflight_cells=10_000_000, max_batches=2)
    try:
        # alone: a micro-batch whose only read fails planning launches no kernel
        t = srv.submit(bad, p)
        srv.wait(t)
        assert srv.result(t)[0] == 2
        tickets = [srv.submit(reads[0], p), srv.submit(bad, p), srv.submit(reads[1], p)]
        for tk in tickets:
            srv.wait(tk)
        res = [srv.result(tk) for tk in tickets]
    finally:
        srv.close()
    assert res[0][0] == 0 and res[2][0] == 0
    assert res[1][0] == 2    # SA_E_ALPHABET, the other reads unaffected


def test_reads_finish_as_the_kernel_publishes_them(api):
    """Every read of the FP32 form is finished from its published record (none waits for the end of
    its micro-batch), with the results of the batch entry point: windows one per warp (bands up to
    128 cells) and one per CTA (a wider band)."""
    for expansion, span in ((50, (500, 6000)), (200, (500, 3000))):
        cfg = synth.config1(seed=33 + expansion, n_reads=8, span=span)
        sm = W.gpu_model(api, W.gaussian_model(cfg), orc.EMIT_DESCALED)
        reads = _inputs(api, sm, cfg["reads"])
        p = api.pairwiseAlignmentBandingParameters_construct(diagonal_expansion=expansion)
        srv = api.Server(max_inflight_cells=500_000_000, max_batches=4)
        try:
            tickets = [srv.submit(r, p) for r in reads]
            for tk in tickets:
                srv.wait(tk)
            res = [srv.result(tk) for tk in tickets]
            stats = srv.stats()
        finally:
            srv.close()
        assert stats["reads_early"] == len(reads) and stats["reads_at_batch_end"] == 0
        batch = api.align_batch(reads, p)
        for r in range(len(reads)):
            _same(api, (batch.status(r), batch.pairs(r), batch.log_likelihood(r), 0.0), res[r], p.threshold)


def test_micro_batches_overlap_on_the_device(api):
    """A read submitted while another micro-batch runs starts its kernels before that one ends
    (device event times of the two micro-batches), and both results are right."""
    import time
    cfg = synth.config1(seed=35, n_reads=2, span=(30000, 40000))
    sm = W.gpu_model(api, W.gaussian_model(cfg), orc.EMIT_DESCALED)
    reads = _inputs(api, sm, cfg["reads"])
    p = api.pairwiseAlignmentBandingParameters_construct()
    # whole (unsegmented) forward sweeps, so the first micro-batch is still running when the second
    # is admitted
    saved = api.get_segment_policy()
    api.set_segment_policy(-1, saved[1])
    srv = api.Server(max_inflight_cells=1_000_000_000, max_batches=2)
    try:
        t0 = srv.submit(reads[0], p)
        time.sleep(0.003)
        t1 = srv.submit(reads[1], p)
        srv.wait(t0)
        srv.wait(t1)
        res = [srv.result(t0), srv.result(t1)]
        log = srv.batch_log()
    finally:
        srv.close()
        api.set_segment_policy(*saved)
    assert len(log) == 2 and all(b[2] == 1 for b in log), log
    (s0, e0, _), (s1, e1, _) = sorted(log)
    assert 0 <= s0 < e0 and 0 <= s1 < e1
    assert s1 < e0, "the second micro-batch started only after the first ended: %r" % (log,)
    batch = api.align_batch(reads, p)
    for r in range(2):
        _same(api, (batch.status(r), batch.pairs(r), batch.log_likelihood(r), 0.0), res[r], p.threshold)
