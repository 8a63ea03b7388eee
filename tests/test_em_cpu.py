"""The EM loop around the expectations path, on the CPU: the oracle's expectations (oracle/sa_oracle.c
orc_expectations) pinned by the properties the reference's own EM tests assert, and the library's
maximisation step and expectations file (sa_em.cpp) against the oracle restatement (oracle/io.py),
exactly.  No GPU needed: the library calls here are host code."""
import numpy as np
import pytest

from oracle import formats
from oracle import io as oio
from oracle import oracle as orc
from signalalign_b200 import synth
import workloads as W


@pytest.fixture(scope="module")
def api():
    from signalalign_b200 import api as a
    return a


def _oracle_em(model, read, emission, iterations, emissions, pseudocount, hdp=None):
    """iterations of E step (getExpectationsUsingAnchors, not ragged) and M step; the likelihoods and
    the last normalised transitions"""
    p = orc.params()
    lik = []
    T = None
    for _ in range(iterations):
        om = W.oracle_model(model, emission, read, hdp)
        ex = orc.expectations(om, read["reference"], read["events"], read["anchors"], p, False, False,
                              transition_pseudocount=pseudocount, emission_pseudocount=0.001)
        lik.append(ex["likelihood"])
        model, T = W.oracle_em_step(model, ex, emissions)
    return lik, T


def test_em_transitions_only_never_lowers_the_likelihood():
    """Baum-Welch on the transitions alone cannot lower the likelihood (up to the pseudocounts):
    the oracle's transition expectations are the posteriors of an EM step.  (The likelihood is the
    sum of the total probability over the posterior anti-diagonals, as the reference accumulates it.)"""
    cfg = synth.config0()
    lik, T = _oracle_em(W.gaussian_model(cfg), cfg["reads"][0], orc.EMIT_DESCALED, 6, False, 0.001)
    assert all(b >= a * (1 + 1e-9) for a, b in zip(lik, lik[1:])), lik   # negative: >= a(1+eps) is "not lower"
    assert lik[-1] > 0.8 * lik[0]         # the default transitions are far from this read's
    np.testing.assert_allclose(np.sum(T, axis=1), 1.0, rtol=1e-15)


def test_continuousPairHmm_em_property():
    """test_continuousPairHmm_em (tests/stateMachineTests.c:1210-1260): ten iterations of expectations
    (pseudocounts 0.001, not ragged), continuousPairHmm_normalize and both loads into the machine
    (the gap-Y means at the reference's i + 5 included); from the third iteration on the previous
    likelihood is at most 0.85 x the current one."""
    cfg = synth.config0()
    lik, _ = _oracle_em(W.gaussian_model(cfg), cfg["reads"][0], orc.EMIT_DESCALED, 10, True, 0.001)
    for it in range(2, 10):
        assert lik[it - 1] <= lik[it] * 0.85, (it, lik)


def test_hdpHmm_emTransitions_property():
    """test_hdpHmm_emTransitions (tests/stateMachineTests.c:1262-1305): the HDP machine, transition
    pseudocount 0, only the transitions normalised and loaded; every iteration's previous likelihood is
    at most 0.95 x the current one."""
    hc = W.small_hdp_config()
    hdp = W.hdp_dict(hc["hdp"], len(hc["alphabet"]) ** hc["k"])
    hm = formats.parse_model_lines(*synth.model_text(hc["alphabet"], hc["k"], hc["table"]).split("\n")[:3])
    lik, T = _oracle_em(hm, hc["reads"][0], orc.EMIT_HDP, 10, False, 0.0, hdp)
    prev = -np.inf
    for v in lik:
        assert prev <= v * 0.95, lik
        prev = v
    assert T[1][2] == 0.0   # gap-X -> gap-Y is never taken (stateMachine.c:1251-1252)


# ------------------------------------------------------------------------------------------------
# the library's maximisation step and expectations file against the restatement
# ------------------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def gauss_case():
    cfg = synth.config0()
    m = W.gaussian_model(cfg)
    rd = cfg["reads"][0]
    ex = orc.expectations(W.oracle_model(m, orc.EMIT_DESCALED, rd), rd["reference"], rd["events"], rd["anchors"],
                          orc.params(), False, False)
    return m, rd, ex


def _hmm(api, sm, ex):
    return dict(ex, event_model=sm.tables()["match"])


def test_normalize_and_load_match_oracle_exactly(api, gauss_case):
    m, rd, ex = gauss_case
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    hmm = api.normalizeExpectations(_hmm(api, sm, ex))
    want_T, want_em = oio.normalize_expectations(ex["transitions"], ex["event_expectations"], ex["posteriors"],
                                                 ex["observed"], np.asarray(m["match"]).reshape(-1, 5))
    assert np.array_equal(hmm["transitions"], np.array(want_T))
    assert np.array_equal(hmm["event_model"], np.array(want_em))
    assert (hmm["event_model"][:, 0] != np.asarray(m["match"]).reshape(-1, 5)[:, 0]).sum() > 100
    api.loadExpectationsIntoStateMachine(sm, hmm)
    got = sm.tables()
    t, match, gapy = oio.load_expectations(m["t"], m["match"], m["gapy"], want_T, want_em)
    assert np.array_equal(got["t"], np.array(t))
    assert got["t"][8] == -np.inf          # gap-X -> gap-Y switch is LOG_ZERO
    assert np.isfinite(got["t"][7])        # gap-Y -> gap-X now carries the expectation
    assert np.array_equal(got["match"].reshape(-1), np.asarray(match).reshape(-1))
    assert np.array_equal(got["gapy"].reshape(-1), np.asarray(gapy).reshape(-1))
    # transitions only: the tables stay
    sm2 = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    api.loadExpectationsIntoStateMachine(sm2, api.normalizeExpectations(_hmm(api, sm2, ex), transitions_only=True),
                                         emissions=False)
    got2 = sm2.tables()
    assert np.array_equal(got2["t"], np.array(t))
    assert np.array_equal(got2["match"].reshape(-1), np.asarray(m["match"]).reshape(-1))


def test_expectations_file_gaussian_bytes(api, gauss_case, tmp_path):
    """continuousPairHmm_writeToFile (continuousHmm.c:354-406): raw expectations as signalMachine writes
    them (signalMachine.c:648), and after normalisation"""
    m, rd, ex = gauss_case
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    for hmm in (_hmm(api, sm, ex), api.normalizeExpectations(_hmm(api, sm, ex))):
        got = api.formatExpectations(sm, hmm)
        want = oio.format_expectations(False, "ACGT", 6, hmm["transitions"], hmm["likelihood"],
                                       np.asarray(hmm["event_model"]).reshape(-1, 5), hmm["event_expectations"],
                                       hmm["posteriors"], hmm["observed"])
        assert got == want
        lines = got.split("\n")
        assert lines[0] == "3\t4\tACGT\t6\t" and len(lines) == 7 and lines[-1] == ""
        path = tmp_path / "expectations.tsv"
        api.writeExpectations(path, sm, hmm)
        api.writeExpectations(path, sm, hmm)       # opened with "w": replaced, not appended
        assert path.read_text() == want
    nan = dict(_hmm(api, sm, ex), transitions=np.full((3, 3), np.nan))
    assert api.formatExpectations(sm, nan) == ""   # hmmContinuous_checkTransitions


def test_expectations_file_hdp_bytes(api):
    """hdpHmm_writeToFile (continuousHmm.c:572-628): the assigned events' means and k-mers"""
    hc = W.small_hdp_config()
    hdp = W.hdp_dict(hc["hdp"], len(hc["alphabet"]) ** hc["k"])
    hm = formats.parse_model_lines(*synth.model_text(hc["alphabet"], hc["k"], hc["table"]).split("\n")[:3])
    rd = hc["reads"][0]
    ex = orc.expectations(W.oracle_model(hm, orc.EMIT_HDP, rd, hdp), rd["reference"], rd["events"], rd["anchors"],
                          orc.params(), transition_pseudocount=0.0)
    assert len(ex["assignments"]) > 100
    sm = W.gpu_model(api, hm, orc.EMIT_HDP, rd, hdp)
    hmm = api.normalizeExpectations(_hmm(api, sm, ex), transitions_only=True)
    got = api.formatExpectations(sm, hmm, rd["events"])
    ev = np.asarray(rd["events"]).reshape(-1, 4)
    want = oio.format_expectations(True, "ACGT", 4, hmm["transitions"], hmm["likelihood"],
                                   np.asarray(hm["match"]).reshape(-1, 5),
                                   assignment_kmers=ex["assignments"][:, 0],
                                   assignment_means=ev[ex["assignments"][:, 1], 0])
    assert got == want
    assert len(got.split("\n")[4].split("\t")) == len(ex["assignments"]) + 1
    with pytest.raises(api.SAError) as ei:      # an assignment's event outside the read
        api.formatExpectations(sm, hmm, rd["events"][:10])
    assert ei.value.status == 1
    with pytest.raises(api.SAError) as ei:      # emissions are loaded into Gaussian machines only
        api.loadExpectationsIntoStateMachine(sm, dict(hmm, event_model=sm.tables()["match"]))
    assert ei.value.status == 7


def test_expectations_batch_statuses_without_device_work(api):
    """sa_getExpectationsBatch: argument and parameter errors fail the call; reads that cannot run get
    their own status (an HDP machine without its tables, an 'X' the ACGT alphabet cannot expand) and,
    when no read runs, nothing touches the device"""
    import ctypes as C
    p = api.pairwiseAlignmentBandingParameters_construct()
    assert api.getExpectationsBatch([], p) == ([], [])
    assert api.lib().sa_getExpectationsBatch(None, -1, C.byref(p), None, None) == 1
    assert api.lib().sa_getExpectationsBatch(None, 2, C.byref(p), None, None) == 1
    cfg = synth.config0()
    m = W.gaussian_model(cfg)
    rd = cfg["reads"][0]
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    bad = api.pairwiseAlignmentBandingParameters_construct(diagonal_expansion=51)   # must be even
    with pytest.raises(api.SAError) as ei:
        api.getExpectationsBatch([api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"],
                                                anchors=rd["anchors"])], bad)
    assert ei.value.status == 1
    hdp_sm = api.StateMachine.from_tables("ACGT", 6, m["t"], m["match"], m["gapy"], m["gapx"], emission=api.EMIT_HDP)
    x_ref = rd["reference"][:100] + "X" + rd["reference"][101:]
    reads = [api.ReadInput(sm=hdp_sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"]),
             api.ReadInput(sm=sm, reference=x_ref, events=rd["events"], anchors=rd["anchors"])]
    got, status = api.getExpectationsBatch(reads, p)
    assert status == [7, 2]
    assert got[1]["likelihood"] == 0.0 and got[1]["transitions"][0, 0] == 0.001   # untouched accumulators


def test_expectations_file_loads_as_a_model(api, gauss_case, tmp_path):
    """The first three lines of an expectations file are a .model (stateMachine3_loadFromFile,
    stateMachine.c:1328-1426): the normalised transitions and the re-estimated event model written by
    sa_writeExpectations come back through the model reader at the file's six decimals (with the
    reader's own rules: gap-Y sd x 1.75, gap-Y -> gap-X into SWITCH_TO_Y)"""
    m, rd, ex = gauss_case
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    hmm = api.normalizeExpectations(_hmm(api, sm, ex))
    path = tmp_path / "trained.hmm"
    api.writeExpectations(path, sm, hmm)
    back = api.StateMachine.load(str(path)).tables()
    T = np.asarray(hmm["transitions"])
    want_p = [T[0][0], T[1][0], T[2][0], T[0][1], T[0][2], T[1][1], T[2][2], 0.0, T[2][1]]
    np.testing.assert_allclose(np.exp(back["t"]), want_p, rtol=0, atol=5e-7)   # "%f": six decimals
    assert back["t"][7] == -np.inf
    em = np.asarray(hmm["event_model"]).reshape(-1, 5)
    np.testing.assert_allclose(back["match"], em, rtol=0, atol=5e-7)
    np.testing.assert_allclose(back["gapy"][:, 1], 1.75 * back["match"][:, 1], rtol=1e-15)


def test_expectations_file_defaults_to_the_machines_match_table(api, gauss_case):
    """sa_formatExpectations with no event model writes the machine's match table (what
    continuousPairHmm_makeExpectationsHmm copies), so signalMachine's raw file needs only the machine"""
    m, rd, ex = gauss_case
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED, rd)
    with_model = api.formatExpectations(sm, _hmm(api, sm, ex))
    without = api.formatExpectations(sm, dict(ex, event_model=None))
    assert without == with_model and len(without) > 0
