"""EM expectations (getExpectationsUsingAnchors with diagonalCalculation_Expectations,
pairwiseAligner.c:1255-1275, 1983-2003) on the plain FP64 form against the FP64 oracle: likelihood,
transition expectations and per-k-mer emission expectations.  The GPU evaluates the same terms in
the same order (the per-k-mer spread depends on the order), so agreement is to rounding of exp():
1e-9 relative."""
import numpy as np
import pytest

from oracle import oracle as orc
from signalalign_b200 import synth
import workloads as W

pytestmark = pytest.mark.gpu
RTOL = 1e-9


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from signalalign_b200 import api as a
    return a


def _p(api, **kw):
    p = api.pairwiseAlignmentBandingParameters_construct()
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _op(p):
    return orc.params(threshold=p.threshold, expansion=p.diagonal_expansion, min_diags=p.min_diags_between_traceback,
                      traceback=p.traceback_diagonals, split=p.split_matrix_bigger_than_this)


def _compare(got, want):
    assert got["likelihood"] == pytest.approx(want["likelihood"], rel=1e-12)
    np.testing.assert_allclose(got["transitions"], want["transitions"], rtol=RTOL)
    assert np.array_equal(got["observed"], want["observed"])
    obs = want["observed"] > 0
    assert obs.sum() > 100
    np.testing.assert_allclose(got["posteriors"], want["posteriors"], rtol=RTOL)
    np.testing.assert_allclose(got["event_expectations"][obs], want["event_expectations"][obs], rtol=RTOL, atol=1e-9)


@pytest.mark.parametrize("ragged", [(True, True), (False, False)])
def test_expectations_config0(api, ragged):
    cfg = synth.config0()
    m = W.gaussian_model(cfg)
    rd = cfg["reads"][0]
    p = _p(api)
    om = W.oracle_model(m, orc.EMIT_DESCALED, rd)
    want = orc.expectations(om, rd["reference"], rd["events"], rd["anchors"], _op(p), *ragged)
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    got = api.getExpectationsUsingAnchors(sm, rd["reference"], rd["events"], rd["anchors"], p, *ragged)
    _compare(got, want)
    # the transition expectations out of match sum to about the number of matches plus the gaps they open
    assert got["transitions"].sum() > 0.5 * len(rd["events"])


@pytest.mark.parametrize("split,min_diags", [(2000, 1000), (3000 * 3000, 150)])
def test_expectations_split_regions_short_windows_and_accumulation(api, split, min_diags):
    """forced split regions (processed in order in one CTA; 15-18 per read) or short traceback
    windows (the forward diagonals the reference has freed at each window's start), accumulated over
    two reads"""
    cfg = synth.config1(seed=21, n_reads=2, span=(600, 1200))
    m = W.gaussian_model(cfg)
    p = _p(api, split_matrix_bigger_than_this=split, min_diags_between_traceback=min_diags)
    got = want = None
    for rd in cfg["reads"]:
        om = W.oracle_model(m, orc.EMIT_DESCALED, rd)
        want = orc.expectations(om, rd["reference"], rd["events"], rd["anchors"], _op(p), state=want)
        sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
        got = api.getExpectationsUsingAnchors(sm, rd["reference"], rd["events"], rd["anchors"], p, state=got)
    _compare(got, want)


def test_expectations_unsupported_inputs(api):
    cfg = synth.config0()
    m = W.gaussian_model(cfg)
    rd = cfg["reads"][0]
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    # an 'X' in an ACGT reference cannot be expanded (its options C/E/O are outside the alphabet)
    ref = rd["reference"][:200] + "X" + rd["reference"][201:]
    with pytest.raises(api.SAError) as ei:
        api.getExpectationsUsingAnchors(sm, ref, rd["events"], rd["anchors"], _p(api))
    assert ei.value.status == 2   # SA_E_ALPHABET



@pytest.mark.parametrize("split", [3000 * 3000, 2000])
def test_expectations_hdp_assignments(api, split):
    """the HDP machine: transition expectations and, instead of emission expectations, the (k-mer,
    event) assignments of match transitions at or above the threshold, in the reference's order
    (cell_signal_updateExpectationsAndAssignments, pairwiseAligner.c:795-817); with split regions the
    event indices stay read-level"""
    from oracle import formats
    hc = W.small_hdp_config()
    hdp = W.hdp_dict(hc["hdp"], len(hc["alphabet"]) ** hc["k"])
    hm = formats.parse_model_lines(*synth.model_text(hc["alphabet"], hc["k"], hc["table"]).split("\n")[:3])
    p = _p(api, split_matrix_bigger_than_this=split)
    got = want = None
    for rd in hc["reads"][:2]:
        om = W.oracle_model(hm, orc.EMIT_HDP, rd, hdp)
        want = orc.expectations(om, rd["reference"], rd["events"], rd["anchors"], _op(p), state=want)
        smh = W.gpu_model(api, hm, orc.EMIT_HDP, rd, hdp)
        got = api.getExpectationsUsingAnchors(smh, rd["reference"], rd["events"], rd["anchors"], p, state=got)
    assert got["likelihood"] == pytest.approx(want["likelihood"], rel=1e-12)
    np.testing.assert_allclose(got["transitions"], want["transitions"], rtol=RTOL)
    assert len(want["assignments"]) > 500
    assert np.array_equal(got["assignments"], want["assignments"])


def test_em_iterations_match_oracle_and_batches_follow(api):
    """Three EM iterations on the device (expectations, continuousPairHmm_normalize, both loads into the
    machine, as test_continuousPairHmm_em runs them, stateMachineTests.c:1210-1260) against the same
    iterations on the oracle.  Re-estimated sds of k-mers seen once shrink by tens of orders of magnitude
    an iteration, so rounding differences grow: the oracle perturbed by 1e-9 moves 6e-8 after three
    iterations; rtol 1e-6.  Then a batch on the re-estimated machine, whose gap-Y table no longer follows
    its match table: its reads run in the plain FP64 form, identical to the single-read entry."""
    cfg = synth.config0()
    m = W.gaussian_model(cfg)
    rd = cfg["reads"][0]
    p = _p(api)
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    model = dict(m)
    for _ in range(3):
        want = orc.expectations(W.oracle_model(model, orc.EMIT_DESCALED, rd), rd["reference"], rd["events"],
                                rd["anchors"], _op(p), False, False)
        got = api.getExpectationsUsingAnchors(sm, rd["reference"], rd["events"], rd["anchors"], p, False, False)
        assert got["likelihood"] == pytest.approx(want["likelihood"], rel=1e-6)
        np.testing.assert_allclose(got["transitions"], want["transitions"], rtol=1e-6)
        api.loadExpectationsIntoStateMachine(sm, api.normalizeExpectations(got))
        model, _ = W.oracle_em_step(model, want, True)
    np.testing.assert_allclose(sm.tables()["t"], model["t"], rtol=1e-6)
    b = api.align_batch([api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                                       scale=rd["scale"], shift=rd["shift"])], p)
    assert b.status(0) == 0
    alone = api.getAlignedPairsUsingAnchors(sm, rd["reference"], rd["events"], rd["anchors"], p)
    assert len(alone) > 100 and np.array_equal(alone, b.pairs(0))


def test_hdp_em_transition_iterations_match_oracle(api):
    """test_hdpHmm_emTransitions (stateMachineTests.c:1262-1305) on the device: the HDP machine,
    transition pseudocount 0, transitions normalised and loaded each iteration, against the oracle"""
    from oracle import formats
    hc = W.small_hdp_config()
    hdp = W.hdp_dict(hc["hdp"], len(hc["alphabet"]) ** hc["k"])
    hm = formats.parse_model_lines(*synth.model_text(hc["alphabet"], hc["k"], hc["table"]).split("\n")[:3])
    rd = hc["reads"][0]
    p = _p(api)
    smh = W.gpu_model(api, hm, orc.EMIT_HDP, rd, hdp)
    model = dict(hm)
    lik = []
    for _ in range(4):
        want = orc.expectations(W.oracle_model(model, orc.EMIT_HDP, rd, hdp), rd["reference"], rd["events"],
                                rd["anchors"], _op(p), False, False, transition_pseudocount=0.0)
        got = api.getExpectationsUsingAnchors(smh, rd["reference"], rd["events"], rd["anchors"], p, False, False,
                                              transition_pseudocount=0.0)
        assert got["likelihood"] == pytest.approx(want["likelihood"], rel=1e-9)
        np.testing.assert_allclose(got["transitions"], want["transitions"], rtol=1e-8, atol=1e-12)
        assert np.array_equal(got["assignments"], want["assignments"])
        api.loadExpectationsIntoStateMachine(smh, api.normalizeExpectations(got, transitions_only=True),
                                             emissions=False)
        model, _ = W.oracle_em_step(model, want, False)
        lik.append(got["likelihood"])
    assert all(b >= a * (1 + 1e-7) for a, b in zip(lik, lik[1:]))   # negative: not lower, to 1e-7


def test_expectations_batch_matches_single_reads(api):
    """sa_getExpectationsBatch: Gaussian reads with split regions, HDP reads, a read whose 'X' the ACGT
    alphabet cannot expand and one with an empty reference, in one launch.  Each read's result is
    identical to its single-read call (one CTA walks its regions in the same order), the failing
    read gets its own status and the others are unaffected."""
    from oracle import formats
    cfg = synth.config1(seed=21, n_reads=4, span=(600, 1200))
    m = W.gaussian_model(cfg)
    p = _p(api, split_matrix_bigger_than_this=2000)
    hc = W.small_hdp_config()
    hdp = W.hdp_dict(hc["hdp"], len(hc["alphabet"]) ** hc["k"])
    hm = formats.parse_model_lines(*synth.model_text(hc["alphabet"], hc["k"], hc["table"]).split("\n")[:3])
    cases = [(rd, W.gpu_model(api, m, orc.EMIT_DESCALED, rd)) for rd in cfg["reads"]]
    cases += [(rd, W.gpu_model(api, hm, orc.EMIT_HDP, rd, hdp)) for rd in hc["reads"][:2]]
    reads, singles = [], []
    for rd, sm in cases:
        reads.append(api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                                   scale=rd["scale"], shift=rd["shift"], var=rd.get("var", 1.0)))
        singles.append(api.getExpectationsUsingAnchors(sm, rd["reference"], rd["events"], rd["anchors"], p))
    bad = cfg["reads"][0]
    reads.insert(2, api.ReadInput(sm=cases[0][1], reference=bad["reference"][:200] + "X" + bad["reference"][201:],
                                  events=bad["events"], anchors=bad["anchors"], scale=bad["scale"], shift=bad["shift"]))
    singles.insert(2, None)
    reads.append(api.ReadInput(sm=cases[0][1], reference="", events=bad["events"][:5], anchors=np.zeros((0, 2))))
    singles.append(api.getExpectationsUsingAnchors(cases[0][1], "", bad["events"][:5], np.zeros((0, 2)), p))
    got, status = api.getExpectationsBatch(reads, p)
    assert status[2] == 2                      # SA_E_ALPHABET, as the single call reports it
    for g, want, st in zip(got, singles, status):
        if want is None:
            continue
        assert st == 0
        for key in ("likelihood", "transitions", "event_expectations", "posteriors", "observed", "assignments"):
            np.testing.assert_array_equal(g[key], want[key])   # bit for bit (NaN where the single call has NaN)
    assert len(got[-2]["assignments"]) > 100   # the HDP reads' assignment lists
    rd = cfg["reads"][1]
    want = orc.expectations(W.oracle_model(m, orc.EMIT_DESCALED, rd), rd["reference"], rd["events"], rd["anchors"],
                            _op(p))
    _compare(got[1], want)
    empty, st = api.getExpectationsBatch([], p)
    assert empty == [] and st == []
