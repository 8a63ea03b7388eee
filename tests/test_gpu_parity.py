"""GPU parity: both kernel forms against the FP64 CPU oracle on the same seeded inputs.

Tolerances:
* plain FP64 form: posterior error <= 1e-5 absolute; pair sets identical except pairs whose
  posterior lies within 1e-5 of the threshold.
* batched FP32 form: posterior error <= 1e-4 absolute (pairs missing on one side count with
  posterior 0 there, so a pair may only be missing if its posterior is within 1e-4 of the
  threshold); log-likelihood within 1e-3 relative.
"""
import numpy as np
import pytest

from oracle import formats
from oracle import oracle as orc
from signalalign_b200 import synth
import workloads as W

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-5
FP32_TOL = 1e-4


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from signalalign_b200 import api as a
    return a


@pytest.fixture(scope="module")
def cfg0():
    return synth.config0()


def _p(api, **kw):
    p = api.pairwiseAlignmentBandingParameters_construct()
    p.diagonal_expansion = kw.get("expansion", 50)
    p.threshold = kw.get("threshold", 0.01)
    if "split" in kw:
        p.split_matrix_bigger_than_this = kw["split"]
    if "min_diags" in kw:
        p.min_diags_between_traceback = kw["min_diags"]
    return p


def _op(p):
    return orc.params(threshold=p.threshold, expansion=p.diagonal_expansion, min_diags=p.min_diags_between_traceback,
                      traceback=p.traceback_diagonals, split=p.split_matrix_bigger_than_this)


DEGENERATE = {"CE": 0, "CEO": 1, "AI": 2}   # sa_degenerate codes of the options strings


def _fp64_case(api, m, emission, rd, p, ragged=(True, True), hdp=None, options="CEO"):
    om = W.oracle_model(m, emission, rd, hdp)
    sm = W.gpu_model(api, m, emission, rd, hdp)
    want = orc.aligned_pairs(om, rd["reference"], rd["events"], rd["anchors"], _op(p), ragged[0], ragged[1],
                             options=options)
    got = api.getAlignedPairsUsingAnchors(sm, rd["reference"], rd["events"], rd["anchors"], p, ragged[0], ragged[1],
                                          degenerate=DEGENERATE[options])
    return want, got


def _assert_fp64(want, got, thr):
    assert W.max_posterior_error(want, got, thr) <= FP64_TOL
    # away from the threshold the two pair lists are identical, in the same (reference) order
    keep_w = [tuple(r) for r in want[["x", "y", "kmer"]].tolist()]
    keep_g = [tuple(r) for r in got[["x", "y", "kmer"]].tolist()]
    if len(want) == len(got):
        assert keep_w == keep_g
    else:
        near = lambda s: abs(s / 1e7 - thr) <= FP64_TOL
        assert [k for k, s in zip(keep_w, want["score"]) if not near(s)] == \
               [k for k, s in zip(keep_g, got["score"]) if not near(s)]


def test_fp64_config0(api, cfg0):
    m = W.gaussian_model(cfg0)
    rd = cfg0["reads"][0]
    p = _p(api)
    want, got = _fp64_case(api, m, orc.EMIT_DESCALED, rd, p)
    assert len(want) > 500
    _assert_fp64(want, got, p.threshold)


@pytest.mark.parametrize("ragged", [(False, False), (True, False), (False, True)])
def test_fp64_ragged_ends(api, cfg0, ragged):
    m = W.gaussian_model(cfg0)
    rd = cfg0["reads"][0]
    p = _p(api, threshold=0.05)
    want, got = _fp64_case(api, m, orc.EMIT_DESCALED, rd, p, ragged=ragged)
    _assert_fp64(want, got, p.threshold)


def test_fp64_split_regions_and_windows(api, cfg0):
    """small split limit forces getSplitPoints regions; small traceback spacing forces many windows"""
    m = W.gaussian_model(cfg0)
    rd = cfg0["reads"][0]
    p = _p(api, split=2000, min_diags=120)
    assert len(api.getSplitPoints(rd["anchors"], len(rd["reference"]) - 5, len(rd["events"]),
                                  p.split_matrix_bigger_than_this, 1, 1)) > 1
    want, got = _fp64_case(api, m, orc.EMIT_DESCALED, rd, p)
    _assert_fp64(want, got, p.threshold)


def test_fp64_plain_scaled_model_zymo(api):
    """The Zymo read of the reference's tests, R7.3 model scaled with the read's parameters
    (emissions_signal_scaleModel), no anchors: the band is the full 892 x 799 matrix."""
    from golden_models import load_fixture, model_from_fixture
    fx = load_fixture("zymo")
    tp = fx["template_params"]
    m = formats.scale_model(model_from_fixture(fx), tp["scale"], tp["shift"], tp["var"], tp["scale_sd"],
                            tp["var_sd"])
    rd = dict(reference=fx["sequence"], events=np.array(fx["events"]), anchors=np.zeros((0, 2), np.int64),
              scale=1.0, shift=0.0)
    p = _p(api, expansion=2)
    want, got = _fp64_case(api, m, orc.EMIT_PLAIN, rd, p, ragged=(False, False))
    assert len(want) > 900
    _assert_fp64(want, got, p.threshold)


def test_fp64_hdp_small(api):
    cfg = W.small_hdp_config()
    n = len(cfg["alphabet"]) ** cfg["k"]
    hdp = W.hdp_dict(cfg["hdp"], n)
    text = synth.model_text(cfg["alphabet"], cfg["k"], cfg["table"])
    m = formats.parse_model_lines(*text.split("\n")[:3])
    p = _p(api)
    for rd in cfg["reads"]:
        want, got = _fp64_case(api, m, orc.EMIT_HDP, rd, p, hdp=hdp)
        assert len(want) > 50
        _assert_fp64(want, got, p.threshold)


def test_fp64_multipath_toy6(api):
    """Variable-order cells (hdCell_construct, pairwiseAligner.c:605-650): the toy 6-mer case of
    test_sm3_diagonalDPCalculations (stateMachineTests.c:443-560), reference "ACGATAXGGACAT" with
    X -> C/E/O, so the six columns over the X hold three paths each.  The banded routine with no
    anchors gives the golden 14 pairs, each (x, y) in the expected set, identical to the oracle."""
    from golden_models import load_fixture, model_from_fixture
    fx = load_fixture("toy6")
    m = model_from_fixture(fx)
    rd = dict(reference=fx["sequence"], events=np.array(fx["events"]), anchors=np.zeros((0, 2), np.int64),
              scale=1.0, shift=0.0)
    p = _p(api, expansion=2, threshold=fx["threshold"])
    want, got = _fp64_case(api, m, orc.EMIT_PLAIN, rd, p, ragged=(False, False), options="CEO")
    assert len(got) == fx["expected_pairs"]
    allowed = {tuple(a) for a in fx["allowed"]}
    assert all((int(q["x"]), int(q["y"])) in allowed for q in got)
    assert len({int(q["kmer"]) for q in got if (int(q["x"]), int(q["y"])) == (6, 5)}) == 3
    _assert_fp64(want, got, p.threshold)


@pytest.mark.parametrize("model", ["gauss", "hdp"])
def test_fp64_multipath_methylation_sites(api, model):
    """Methylation calling with degenerate positions (cytosine2: X -> C or E) at CCWGG sites on both
    strands, Gaussian and HDP machines: the cells over a site hold two paths and each emits its
    own posterior; FP64 GPU against the oracle."""
    cfg = synth.config3(seed=11, n_reads=2, span=(700, 1400), grid_length=200, route="degenerate")
    alphabet, k = cfg["alphabet"], cfg["k"]
    n = len(alphabet) ** k
    p = _p(api)
    site_bases = {"C": 0, "E": 0}
    for rd in cfg["alignments"]:
        if rd["model"] != model:
            continue
        assert "X" in rd["reference"] and rd["degenerate"] == "CE"
        table = cfg["hdp_table"] if model == "hdp" else cfg["gauss_table"]
        text = synth.model_text(cfg["alphabet"], cfg["k"], table)
        m = formats.parse_model_lines(*text.split("\n")[:3])
        hdp = W.hdp_dict(cfg["hdp"], n) if model == "hdp" else None
        emission = orc.EMIT_HDP if model == "hdp" else orc.EMIT_DESCALED
        want, got = _fp64_case(api, m, emission, rd, p, hdp=hdp, options="CE")
        assert len(want) > 50
        _assert_fp64(want, got, p.threshold)
        # the path each pair over a site took: the site's base in the pair's k-mer
        sites = [i for i, ch in enumerate(rd["reference"]) if ch == "X"]
        for q in got:
            x, kid = int(q["x"]), int(q["kmer"])
            kmer = "".join(alphabet[(kid // len(alphabet) ** (k - 1 - i)) % len(alphabet)] for i in range(k))
            for s_ in sites:
                if x <= s_ < x + k:
                    site_bases[kmer[s_ - x]] += 1
    assert site_bases["C"] > 0 and site_bases["E"] > 0


def test_fp64_edge_cases(api, cfg0):
    m = W.gaussian_model(cfg0)
    rd = cfg0["reads"][0]
    p = _p(api)
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    # no events: every cell is on y = 0, no pair can be emitted
    got = api.getAlignedPairsUsingAnchors(sm, rd["reference"], np.zeros((0, 4)), [], p)
    assert len(got) == 0
    # empty reference and no events: trivial
    got = api.getAlignedPairsUsingAnchors(sm, "", np.zeros((0, 4)), [], p)
    assert len(got) == 0
    # a reference shorter than k is rejected like sequence_correctSeqLength would make it negative
    with pytest.raises(api.SAError):
        api.getAlignedPairsUsingAnchors(sm, "ACG", rd["events"][:5], [], p)
    # out-of-alphabet character
    with pytest.raises(api.SAError) as ei:
        api.getAlignedPairsUsingAnchors(sm, "ACGTNACGTACGT", rd["events"][:10], [], p)
    assert ei.value.status == 2
    # non-monotone anchors
    with pytest.raises(api.SAError) as ei:
        api.getAlignedPairsUsingAnchors(sm, rd["reference"], rd["events"], [(50, 80), (40, 90)], p)
    assert ei.value.status == 3
    # tiny read without anchors matches the oracle
    small = dict(rd, reference=rd["reference"][:40], events=rd["events"][:50], anchors=np.zeros((0, 2), np.int64))
    want, got = _fp64_case(api, m, orc.EMIT_DESCALED, small, p)
    _assert_fp64(want, got, p.threshold)


# ------------------------------------------------------------------------------------------------
# batched FP32 form
# ------------------------------------------------------------------------------------------------
def _batch_vs_oracle(api, m, emission, reads, p, hdp=None):
    sms = [W.gpu_model(api, m, emission, None, hdp)]
    inputs = [api.ReadInput(sm=sms[0], reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                            scale=rd["scale"], shift=rd["shift"], var=rd.get("var", 1.0)) for rd in reads]
    b = api.align_batch(inputs, p)
    errs, llerr = [], []
    for i, rd in enumerate(reads):
        assert b.status(i) == 0
        om = W.oracle_model(m, emission, rd, hdp)
        want, tps = orc.aligned_pairs(om, rd["reference"], rd["events"], rd["anchors"], _op(p), True, True,
                                      with_total_probs=True)
        got = b.pairs(i)
        errs.append(W.max_posterior_error(want, got, p.threshold))
        top = [v for d, v in tps if d == len(rd["reference"]) - m["kmer_length"] + 1 + len(rd["events"])]
        if top:
            llerr.append(abs(b.log_likelihood(i) - top[0]) / abs(top[0]))
    return max(errs), (max(llerr) if llerr else 0.0), b


def test_fp32_config0(api, cfg0):
    m = W.gaussian_model(cfg0)
    p = _p(api)
    err, llerr, b = _batch_vs_oracle(api, m, orc.EMIT_DESCALED, cfg0["reads"], p)
    assert b.cells > 150000
    assert err <= FP32_TOL, err
    assert llerr <= 1e-3


def test_fp32_mixed_lengths(api):
    cfg = synth.config1(seed=11, n_reads=6, span=(200, 2500))
    m = W.gaussian_model(cfg)
    p = _p(api)
    err, llerr, _ = _batch_vs_oracle(api, m, orc.EMIT_DESCALED, cfg["reads"], p)
    assert err <= FP32_TOL, err
    assert llerr <= 1e-3


def test_fp32_hdp_small(api):
    cfg = W.small_hdp_config()
    n = len(cfg["alphabet"]) ** cfg["k"]
    hdp = W.hdp_dict(cfg["hdp"], n)
    text = synth.model_text(cfg["alphabet"], cfg["k"], cfg["table"])
    m = formats.parse_model_lines(*text.split("\n")[:3])
    err, llerr, _ = _batch_vs_oracle(api, m, orc.EMIT_HDP, cfg["reads"], _p(api), hdp=hdp)
    assert err <= FP32_TOL, err
    assert llerr <= 1e-3


def test_fp32_splits_and_windows(api, cfg0):
    m = W.gaussian_model(cfg0)
    p = _p(api, split=2000, min_diags=120)
    err, _, b = _batch_vs_oracle(api, m, orc.EMIT_DESCALED, cfg0["reads"], p)
    assert b.regions > 1
    assert err <= FP32_TOL, err


def test_fp32_result_independent_of_batch(api, cfg0):
    """a read's pairs are the same alone and inside a larger batch"""
    cfg = synth.config1(seed=12, n_reads=5, span=(300, 1500))
    m = W.gaussian_model(cfg)
    p = _p(api)
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED)
    mk = lambda rd: api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                                  scale=rd["scale"], shift=rd["shift"])
    alone = api.align_batch([mk(cfg["reads"][2])], p).pairs(0)
    mixed = api.align_batch([mk(rd) for rd in cfg["reads"]], p).pairs(2)
    assert np.array_equal(alone, mixed)


def test_fp32_config2_shape_hdp(api):
    """HDP machine with config 2's shape: 6-mer ACEGT (15,625 k-mers), 2000-point grid, methylated
    CpGs in the reference; short reads so the oracle is quick"""
    cfg = synth.config2(n_reads=2, span=(400, 700))
    hdp = W.hdp_dict(cfg["hdp"], 5 ** 6)
    m = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["table"]).split("\n")[:3])
    err, llerr, _ = _batch_vs_oracle(api, m, orc.EMIT_HDP, cfg["reads"], _p(api), hdp=hdp)
    assert err <= FP32_TOL, err
    assert llerr <= 1e-3


def test_fp32_config3_shape_mixed_models(api):
    """config 3's shape: template and complement streams, all-C and all-E hypotheses, Gaussian and
    HDP machines mixed in one batch; every alignment against the oracle"""
    cfg = synth.config3(n_reads=2, span=(400, 700), grid_length=400)
    gm = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["gauss_table"]).split("\n")[:3])
    hm = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["hdp_table"]).split("\n")[:3])
    hdp = W.hdp_dict(cfg["hdp"], 5 ** 6)
    sm_g = W.gpu_model(api, gm, orc.EMIT_DESCALED)
    sm_h = W.gpu_model(api, hm, orc.EMIT_HDP, None, hdp)
    als = cfg["alignments"]
    assert {a["hypothesis"] for a in als} == {"C", "E"} and {a["model"] for a in als} == {"gauss", "hdp"}
    inputs = [api.ReadInput(sm=sm_h if a["model"] == "hdp" else sm_g, reference=a["reference"], events=a["events"],
                            anchors=a["anchors"], scale=a["scale"], shift=a["shift"]) for a in als]
    p = _p(api)
    b = api.align_batch(inputs, p)
    for i, a in enumerate(als):
        assert b.status(i) == 0
        om = W.oracle_model(hm if a["model"] == "hdp" else gm, orc.EMIT_HDP if a["model"] == "hdp" else orc.EMIT_DESCALED,
                            a, hdp if a["model"] == "hdp" else None)
        want = orc.aligned_pairs(om, a["reference"], a["events"], a["anchors"], _op(p), True, True)
        assert len(want) > 50
        assert W.max_posterior_error(want, b.pairs(i), p.threshold) <= FP32_TOL


def test_batch_degenerate_reads_run_in_plain_form(api):
    """Reads with degenerate positions (route (ii) of methylation calling: 'X' at the CCWGG sites,
    cytosine2) in one batch with substituted-reference reads: the multi-path reads are aligned by
    the plain FP64 form inside the batch (FP64 tolerance against the oracle, and identical to the
    single-read entry), the others by the FP32 kernels (FP32 tolerance)."""
    sub = synth.config3(seed=5, n_reads=1, span=(500, 800), grid_length=300)["alignments"]
    deg_cfg = synth.config3(seed=5, n_reads=2, span=(500, 800), grid_length=300, route="degenerate")
    deg = deg_cfg["alignments"]
    gm = formats.parse_model_lines(*synth.model_text("ACEGT", 6, deg_cfg["gauss_table"]).split("\n")[:3])
    hm = formats.parse_model_lines(*synth.model_text("ACEGT", 6, deg_cfg["hdp_table"]).split("\n")[:3])
    hdp = W.hdp_dict(deg_cfg["hdp"], 5 ** 6)
    sm_g = W.gpu_model(api, gm, orc.EMIT_DESCALED)
    sm_h = W.gpu_model(api, hm, orc.EMIT_HDP, None, hdp)
    als = [a for pair in zip(deg, sub) for a in pair]   # interleaved
    inputs = [api.ReadInput(sm=sm_h if a["model"] == "hdp" else sm_g, reference=a["reference"], events=a["events"],
                            anchors=a["anchors"], scale=a["scale"], shift=a["shift"],
                            degenerate=DEGENERATE[a.get("degenerate", "CEO")]) for a in als]
    p = _p(api)
    b = api.align_batch(inputs, p)
    n_multi = 0
    for i, a in enumerate(als):
        assert b.status(i) == 0
        hd = a["model"] == "hdp"
        om = W.oracle_model(hm if hd else gm, orc.EMIT_HDP if hd else orc.EMIT_DESCALED, a, hdp if hd else None)
        options = a.get("degenerate", "CEO")
        want = orc.aligned_pairs(om, a["reference"], a["events"], a["anchors"], _op(p), True, True, options=options)
        assert len(want) > 50
        if "X" in a["reference"]:
            n_multi += 1
            _assert_fp64(want, b.pairs(i), p.threshold)
            sm = W.gpu_model(api, hm if hd else gm, orc.EMIT_HDP if hd else orc.EMIT_DESCALED, a, hdp if hd else None)
            alone = api.getAlignedPairsUsingAnchors(sm, a["reference"], a["events"], a["anchors"], p,
                                                    degenerate=DEGENERATE[options])
            assert np.array_equal(alone, b.pairs(i))
        else:
            assert W.max_posterior_error(want, b.pairs(i), p.threshold) <= FP32_TOL
    assert n_multi == len(deg)


def test_batch_only_degenerate_reads_and_empty_batch(api):
    """a batch whose every read has degenerate positions (no FP32 work: the plain form alone) gives
    the single-read entry's pairs; an empty batch plans, runs and downloads nothing"""
    cfg = synth.config3(seed=8, n_reads=1, span=(400, 600), grid_length=200, route="degenerate")
    gm = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["gauss_table"]).split("\n")[:3])
    als = [a for a in cfg["alignments"] if a["model"] == "gauss"]
    p = _p(api)
    inputs = []
    for a in als:
        sm = W.gpu_model(api, gm, orc.EMIT_DESCALED, a)
        inputs.append(api.ReadInput(sm=sm, reference=a["reference"], events=a["events"], anchors=a["anchors"],
                                    scale=a["scale"], shift=a["shift"], degenerate=DEGENERATE["CE"]))
    b = api.align_batch(inputs, p)
    for i, a in enumerate(als):
        assert b.status(i) == 0
        alone = api.getAlignedPairsUsingAnchors(inputs[i].sm, a["reference"], a["events"], a["anchors"], p,
                                                degenerate=DEGENERATE["CE"])
        assert len(alone) > 50 and np.array_equal(alone, b.pairs(i))
    empty = api.align_batch([], p)
    assert empty.cells == 0


def test_fp32_bounded_wait_runs_out(api):
    """Every device-side wait of the worker kernel is bounded (sa_batch_set_wait_limit).  With a
    bound of one clock cycle the warps waiting for traceback windows give up at once: the launch
    still ends normally, every read reports SA_E_TIMEOUT, and the context stays usable (the same
    batch run again with the default bound gives the oracle's pairs)."""
    cfg = synth.config1(seed=31, n_reads=2, span=(3000, 4000))
    m = W.gaussian_model(cfg)
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED)
    inputs = [api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                            scale=rd["scale"], shift=rd["shift"]) for rd in cfg["reads"]]
    p = _p(api)
    b = api.Batch(inputs, p)
    b.upload()
    b.set_wait_limit(1)
    b.run()
    b.download()
    assert [b.status(i) for i in range(2)] == [9, 9]        # SA_E_TIMEOUT
    b.set_wait_limit(20_000_000_000)
    b.run()
    b.download()
    for i, rd in enumerate(cfg["reads"]):
        assert b.status(i) == 0
        om = W.oracle_model(m, orc.EMIT_DESCALED, rd)
        want = orc.aligned_pairs(om, rd["reference"], rd["events"], rd["anchors"], _op(p), True, True)
        assert W.max_posterior_error(want, b.pairs(i), p.threshold) <= FP32_TOL


def test_fp32_launch_configurations(api):
    """Every launch configuration the tuner can choose gives the oracle's pairs: a traceback window
    per CTA instead of per warp (FP32 tolerance: different sweep code), and grid shapes (identical
    pairs: each window is computed the same way whichever CTA runs it).  Then the tuner itself on a
    small batch: it tries the candidates, sets the fastest for the device, and the batch's results
    after it are still the oracle's."""
    cfg = synth.config1(seed=41, n_reads=6, span=(800, 3000))
    m = W.gaussian_model(cfg)
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED)
    inputs = [api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                            scale=rd["scale"], shift=rd["shift"]) for rd in cfg["reads"]]
    p = _p(api)
    default = api.get_launch_config(0, 1)
    wants = []
    for rd in cfg["reads"]:
        om = W.oracle_model(m, orc.EMIT_DESCALED, rd)
        wants.append(orc.aligned_pairs(om, rd["reference"], rd["events"], rd["anchors"], _op(p), True, True))
    try:
        base = api.align_batch(inputs, p)
        for c in (dict(default, warp_windows=0), dict(default, ctas_per_sm=1, grid_per_region=2),
                  dict(default, grid_per_region=6, emission_ctas_per_sm=8)):
            api.set_launch_config(0, 1, c)
            b = api.align_batch(inputs, p)
            for i, want in enumerate(wants):
                assert b.status(i) == 0
                assert W.max_posterior_error(want, b.pairs(i), p.threshold) <= FP32_TOL, (c, i)
                if c["warp_windows"] == default["warp_windows"]:
                    assert np.array_equal(b.pairs(i), base.pairs(i)), (c, i)
        api.set_launch_config(0, 1, default)
        b = api.Batch(inputs, p)
        b.upload()
        best, ms, tried = api.tune_launch_config(b, None, 1)
        assert tried >= 8 and ms > 0
        assert api.get_launch_config(0, 1) == best
        b.download()
        for i, want in enumerate(wants):
            assert W.max_posterior_error(want, b.pairs(i), p.threshold) <= FP32_TOL
    finally:
        api.set_launch_config(0, 1, default)
