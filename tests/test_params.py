"""Per-read scale / shift / drift / variance estimation (signalUtils_estimateNanoporeParams,
signalMachineUtils.c:186-223) against the oracle restatement (oracle/io.py): the 1D assignments and
the drift correction exactly (host), the weighted least-squares fits on the GPU within 1e-7
relative (the GPU sums in a different order than the reference's sequential loop)."""
import numpy as np
import pytest

from oracle import formats
from oracle import io as oio
from signalalign_b200 import synth


@pytest.fixture(scope="module")
def api():
    from signalalign_b200 import api as a
    return a


def make_strand(seed, table, alphabet="ACGT", k=6, length=3000, scale=1.03, shift=-4.0, drift=0.8, var=1.2,
                scale_sd=0.95):
    """a basecalled strand, its event map (a skipped position shares the previous event) and events
    drawn from the model under the given read parameters"""
    r = np.random.default_rng(seed)
    read = "".join(r.choice(list(alphabet), length))
    rows = length - (k - 1)
    steps = r.integers(0, 3, rows)   # 0 = the position shares its event with the previous one
    steps[0] = 0
    event_map = np.cumsum(steps > 0).astype(np.int64)
    n_events = int(event_map[-1]) + 1
    t = np.cumsum(r.exponential(0.02, n_events))
    events = np.zeros((n_events, 4))
    ids = synth.kmer_ids_of(read, alphabet, k)
    for i in range(rows):
        e = event_map[i]
        if events[e, 3] == 0.0 or i == 0:
            m = table[ids[i]]
            events[e, 0] = scale * m[0] + shift + drift * t[e] + r.normal(0, m[1] * var)
            events[e, 1] = m[2] * scale_sd + r.normal(0, 0.05)
            events[e, 2] = r.exponential(0.002)
            events[e, 3] = t[e]
    return read, event_map, events


@pytest.fixture(scope="module")
def model():
    table = synth.gaussian_table("ACGT", 6, 3)
    return formats.parse_model_lines(*synth.model_text("ACGT", 6, table).split("\n")[:3])


def _sm(api, m):
    return api.StateMachine.from_tables("ACGT", 6, m["t"], m["match"], m["gapy"], m["gapx"], emission=api.EMIT_DESCALED)


def test_one_d_assignments_match_oracle(api, model):
    sm = _sm(api, model)
    read, em, ev = make_strand(1, np.asarray(model["match"]).reshape(-1, 5))
    ids, ep = api.oneDAssignmentsFromRead(sm, read, em, ev)
    want = oio.one_d_assignments(read, [int(v) for v in em], ev.tolist(), "ACGT", 6)
    assert [int(v) for v in ids] == [w[0] for w in want]
    assert np.array_equal(ep, np.array([w[1:] for w in want]))
    assert len(ids) < len(read) - 5   # repeated events are collected once


def test_drift_adjustment_matches_oracle(api, model):
    _, _, ev = make_strand(2, np.asarray(model["match"]).reshape(-1, 5))
    got = api.adjustEventsForDrift(ev, 0.37)
    assert np.array_equal(got, np.array(oio.adjust_events_for_drift(ev.tolist(), 0.37)))


def test_assignments_reject_bad_input(api, model):
    sm = _sm(api, model)
    read, em, ev = make_strand(3, np.asarray(model["match"]).reshape(-1, 5), length=200)
    with pytest.raises(api.SAError):
        api.oneDAssignmentsFromRead(sm, read[:50] + "N" + read[51:], em, ev)
    bad = em.copy()
    bad[10] = len(ev) + 5
    with pytest.raises(api.SAError):
        api.oneDAssignmentsFromRead(sm, read, bad, ev)


@pytest.mark.gpu
def test_estimate_params_batch_matches_oracle(api, model):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    table = np.asarray(model["match"]).reshape(-1, 5)
    sm = _sm(api, model)
    truths = [dict(scale=1.03, shift=-4.0, drift=0.8, var=1.2, scale_sd=0.95),
              dict(scale=0.96, shift=3.0, drift=-0.5, var=0.9, scale_sd=1.05),
              dict(scale=1.0, shift=0.0, drift=0.0, var=1.0, scale_sd=1.0)]
    items, strands = [], []
    for i, tr in enumerate(truths):
        read, em, ev = make_strand(10 + i, table, length=4000 + 1000 * i, **tr)
        strands.append((read, em, ev))
        items.append((sm, read, em, ev, dict(var=1.0, scale_sd=1.0)))
    got = api.estimateNanoporeParams(items)
    for (st, p), (read, em, ev), tr in zip(got, strands, truths):
        assert st == 0
        want = oio.estimate_params(oio.one_d_assignments(read, [int(v) for v in em], ev.tolist(), "ACGT", 6), table)
        for k, v in want.items():
            assert p[k] == pytest.approx(v, rel=1e-7, abs=1e-9), k
        # and the fit recovers the parameters the events were drawn with
        assert p["scale"] == pytest.approx(tr["scale"], rel=0.02)
        assert p["shift"] == pytest.approx(tr["shift"], abs=1.5)
        assert p["drift"] == pytest.approx(tr["drift"], abs=0.2)


@pytest.mark.gpu
def test_estimate_params_read_without_assignments(api, model):
    """a strand shorter than one k-mer has no assignments: the reference aborts, the batch marks that
    read SA_E_ARG and still fits the others"""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    table = np.asarray(model["match"]).reshape(-1, 5)
    sm = _sm(api, model)
    read, em, ev = make_strand(30, table, length=2000)
    got = api.estimateNanoporeParams([(sm, read[:4], em, ev, {}), (sm, read, em, ev, dict(var=1.0))])
    assert got[0][0] == 1
    assert got[1][0] == 0 and got[1][1]["scale"] == pytest.approx(1.03, rel=0.02)
