"""Forward segments of the batched FP32 form (sa_setSegmentPolicy).

A region's forward sweep is cut at traceback-window starts into segments swept at the same time;
each later segment warms up from a flat start and is checked where it meets the previous one (the
stitch).  What is checked here:

* segmented and unsegmented runs of the same reads give the same posteriors (within 1e-5: the two
  sweeps round differently) and the same log-likelihood (1e-7 relative), and both the oracle's
  within the FP32 form's 1e-4;
* every stitch agrees on these inputs, with its largest deviation far below the tolerance;
* a batch whose stitches are all made to disagree (negative tolerance scale) re-runs every
  segmented read unsegmented at download and returns exactly the unsegmented run's results;
* per-read completion (the serving path) counts the stitches of a read before publishing it.
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


@pytest.fixture
def policy(api):
    saved = api.get_segment_policy()
    yield
    api.set_segment_policy(*saved)


def _case(api, seed=61, n_reads=4, span=(4000, 9000)):
    cfg = synth.config1(seed=seed, n_reads=n_reads, span=span)
    m = W.gaussian_model(cfg)
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED)
    inputs = [api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                            scale=rd["scale"], shift=rd["shift"]) for rd in cfg["reads"]]
    return cfg, m, sm, inputs


def _run(api, inputs, p, segment_diags, tol_scale=None):
    api.set_segment_policy(segment_diags, 1024)
    b = api.Batch(inputs, p)
    b.upload()
    if tol_scale is not None:
        b.set_stitch_tolerance(tol_scale)
    b.run()
    b.download()
    return b


def test_segmented_equals_unsegmented_and_oracle(api, policy):
    cfg, m, sm, inputs = _case(api)
    p = api.pairwiseAlignmentBandingParameters_construct()
    seg = _run(api, inputs, p, 4096)
    whole = _run(api, inputs, p, -1)
    info = seg.segment_info()
    assert info["segments"] > 2 * len(inputs), info
    assert info["stitches"] == info["segments"] - len(inputs)
    assert info["redone"] == 0, info
    assert info["max_spread"] < 2e-5, info
    assert whole.segment_info()["segments"] == len(inputs)
    op = orc.params(threshold=p.threshold, expansion=p.diagonal_expansion)
    for i, rd in enumerate(cfg["reads"]):
        assert seg.status(i) == 0 and whole.status(i) == 0
        assert W.max_posterior_error(whole.pairs(i), seg.pairs(i), p.threshold) <= 1e-5
        assert abs(seg.log_likelihood(i) - whole.log_likelihood(i)) <= 1e-7 * abs(whole.log_likelihood(i))
        om = W.oracle_model(m, orc.EMIT_DESCALED, rd)
        want = orc.aligned_pairs(om, rd["reference"], rd["events"], rd["anchors"], op, True, True)
        assert W.max_posterior_error(want, seg.pairs(i), p.threshold) <= FP32_TOL


def test_disagreeing_stitches_rerun_unsegmented(api, policy):
    cfg, m, sm, inputs = _case(api, seed=62, n_reads=3, span=(3000, 7000))
    p = api.pairwiseAlignmentBandingParameters_construct()
    whole = _run(api, inputs, p, -1)
    forced = _run(api, inputs, p, 4096, tol_scale=-1.0)
    info = forced.segment_info()
    assert info["stitches"] > 0
    assert info["redone"] == len(inputs), info   # every read here has a stitch
    for i in range(len(inputs)):
        assert forced.status(i) == 0
        assert np.array_equal(forced.pairs(i), whole.pairs(i))
        assert forced.log_likelihood(i) == whole.log_likelihood(i)
    # the same batch run again with the default tolerance: no re-run, results within rounding
    forced.set_stitch_tolerance(1.0)
    forced.run()
    forced.download()
    assert forced.segment_info()["redone"] == 0
    for i in range(len(inputs)):
        assert W.max_posterior_error(whole.pairs(i), forced.pairs(i), p.threshold) <= 1e-5
        assert abs(forced.log_likelihood(i) - whole.log_likelihood(i)) <= 1e-7 * abs(whole.log_likelihood(i))


def test_served_reads_count_their_stitches(api, policy):
    """the serving path publishes a segmented read only after its stitches were checked, with the
    log-likelihood brought back to the first segment's frame"""
    cfg, m, sm, inputs = _case(api, seed=63, n_reads=3, span=(5000, 8000))
    p = api.pairwiseAlignmentBandingParameters_construct()
    api.set_segment_policy(4096, 1024)
    srv = api.Server(max_inflight_cells=500_000_000, max_batches=2)
    try:
        tickets = [srv.submit(r, p) for r in inputs]
        for tk in tickets:
            srv.wait(tk)
        res = [srv.result(tk) for tk in tickets]
        stats = srv.stats()
    finally:
        srv.close()
    assert stats["reads_early"] == len(inputs)
    whole = _run(api, inputs, p, -1)
    for i in range(len(inputs)):
        st, pairs, ll, _ = res[i]
        assert st == 0
        assert W.max_posterior_error(whole.pairs(i), pairs, p.threshold) <= 1e-5
        assert abs(ll - whole.log_likelihood(i)) <= 1e-7 * abs(whole.log_likelihood(i))


def test_segments_hdp_split_regions_and_wide_bands(api, policy):
    """Segmented against whole sweeps where the segment planner meets the other paths: an HDP machine
    (emissions in FP64 on the device), regions split by large anchor gaps, and a band wider than 128
    cells (two cells per thread, CTA-wide windows)."""
    from oracle import formats
    cfg = synth.config2(seed=64, n_reads=2, span=(5000, 7000))
    hdp = W.hdp_dict(cfg["hdp"], 5 ** 6)
    m = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["table"]).split("\n")[:3])
    sm_h = W.gpu_model(api, m, orc.EMIT_HDP, None, hdp)
    hdp_inputs = [api.ReadInput(sm=sm_h, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                                scale=rd["scale"], shift=rd["shift"]) for rd in cfg["reads"]]
    gcfg, _, sm_g, g_inputs = _case(api, seed=65, n_reads=2, span=(5000, 7000))
    # anchors dropped over 150 reference positions in the middle: that gap (about 200 x 320 cells)
    # is larger than the split limit (100 x 100), the others (about 50 x 80) are not, so each read
    # becomes two long regions
    split_inputs = []
    for rd in gcfg["reads"]:
        a = np.asarray(rd["anchors"]).reshape(-1, 2)
        L = len(rd["reference"])
        keep = (a[:, 0] < 0.5 * L - 75) | (a[:, 0] > 0.5 * L + 75)
        split_inputs.append(api.ReadInput(sm=sm_g, reference=rd["reference"], events=rd["events"], anchors=a[keep],
                                          scale=rd["scale"], shift=rd["shift"]))
    cases = [(hdp_inputs, api.pairwiseAlignmentBandingParameters_construct()),
             (split_inputs, api.pairwiseAlignmentBandingParameters_construct(split_matrix_bigger_than_this=100 * 100)),
             (g_inputs, api.pairwiseAlignmentBandingParameters_construct(diagonal_expansion=200))]
    for inputs, p in cases:
        seg = _run(api, inputs, p, 4096)
        whole = _run(api, inputs, p, -1)
        info = seg.segment_info()
        assert info["stitches"] > 0 and info["redone"] == 0, (p.diagonal_expansion, info)
        if p.split_matrix_bigger_than_this == 100 * 100:
            assert seg.regions > len(inputs)
        for i in range(len(inputs)):
            assert seg.status(i) == 0 and whole.status(i) == 0
            assert W.max_posterior_error(whole.pairs(i), seg.pairs(i), p.threshold) <= 1e-5
            assert abs(seg.log_likelihood(i) - whole.log_likelihood(i)) <= 1e-7 * abs(whole.log_likelihood(i))


def test_plain_form_segments(api, policy):
    """The plain FP64 form (the single-read entry and a batch's X reads) with forward segments: a
    long read with degenerate X (C or E) sites, two paths over each, against the whole sweep (FP64
    sweeps agree to rounding once the start is forgotten) and the oracle (1e-5); and a batch whose
    plain-form stitches are all made to disagree re-runs those regions whole, with the whole
    sweep's results exactly."""
    from oracle import formats
    cfg = synth.config3(seed=66, n_reads=1, span=(6000, 7000), grid_length=200, route="degenerate")
    rd = [a for a in cfg["alignments"] if a["model"] == "gauss"][0]
    m = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["gauss_table"]).split("\n")[:3])
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    p = api.pairwiseAlignmentBandingParameters_construct(diagonal_expansion=50)
    call = lambda: api.getAlignedPairsUsingAnchors(sm, rd["reference"], rd["events"], rd["anchors"], p,
                                                   degenerate=api.CYTOSINE_METHYLATION2, with_log_likelihood=True)
    api.set_segment_policy(4096, 1024)
    seg, ll_seg = call()
    api.set_segment_policy(-1, 1024)
    whole, ll_whole = call()
    assert len(whole) > 100
    assert W.max_posterior_error(whole, seg, p.threshold) <= 1e-7
    assert abs(ll_seg - ll_whole) <= 1e-9 * abs(ll_whole)
    om = W.oracle_model(m, orc.EMIT_DESCALED, rd)
    op = orc.params(threshold=p.threshold, expansion=p.diagonal_expansion)
    want = orc.aligned_pairs(om, rd["reference"], rd["events"], rd["anchors"], op, True, True, options="CE")
    assert W.max_posterior_error(want, seg, p.threshold) <= 1e-5
    # the same read inside a batch (routed to the plain form), stitches forced to disagree
    inp = [api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                         scale=rd["scale"], shift=rd["shift"], degenerate=api.CYTOSINE_METHYLATION2)]
    forced = _run(api, inp, p, 4096, tol_scale=-1.0)
    info = forced.segment_info()
    assert info["stitches"] > 0 and info["redone"] == 1, info
    assert forced.status(0) == 0
    assert np.array_equal(forced.pairs(0), whole)
    assert forced.log_likelihood(0) == ll_whole
    agreed = _run(api, inp, p, 4096)
    assert W.max_posterior_error(whole, agreed.pairs(0), p.threshold) <= 1e-7
    assert abs(agreed.log_likelihood(0) - ll_whole) <= 1e-9 * abs(ll_whole)
