"""The reference's banded known answers on the GPU: the Zymo read with its lastz anchors, machines
loaded by the product's own loaders from the reference's model files (tests/golden/*.xz).

Counts are the reference's (tests/stateMachineTests.c:823-960): 1076 pairs with the scaled and the
descaled R7.3 machines, 1076 with every C replaced by C, E or O, 7349 with every C replaced by X
(CEO paths), 1217 with the HDP machine at threshold 0.1.  Every case also matches the FP64 oracle
pair for pair:

* plain FP64 form (one read per launch): posterior error <= 1e-5, and the exact count;
* batched FP32 form: posterior error <= 1e-4; the count is the reference's except for pairs whose
  posterior lies within 1e-4 of the threshold.  The X case runs inside the batch in the plain FP64
  form (multi-path cells) and gives the exact count there too.
"""
import numpy as np
import pytest

from oracle import formats
from oracle import oracle as orc
from golden_models import golden_file, zymo_banded
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
def case(api):
    """(name, product machine, oracle model, reference, events, threshold, ragged, options, count)"""
    z = zymo_banded()
    tp, ex = z["template_params"], z["expected"]
    model = golden_file("testModelR73_acegot_template.model")
    nhdp = golden_file("templateSingleLevelFixed.nhdp")
    m = formats.load_model_file(model)
    # getStateMachine3 + emissions_signal_scaleModel (loadScaledStateMachine3, stateMachineTests.c:71-81)
    sm_scaled = api.getStateMachine3(model)
    sm_scaled.scaleModel(tp["scale"], tp["shift"], tp["var"], tp["scale_sd"], tp["var_sd"])
    om_scaled = orc.OracleModel(formats.scale_model(m, tp["scale"], tp["shift"], tp["var"], tp["scale_sd"],
                                                    tp["var_sd"]), orc.EMIT_PLAIN)
    # getStateMachine3_descaled with scaleNoise (loadDescaledStateMachine3, :83-90)
    sm_desc = api.getStateMachine3_descaled(model, tp["scale"], tp["shift"], tp["var"], tp["scale_sd"], tp["var_sd"],
                                            scale_noise=True)
    om_desc = orc.OracleModel(formats.scale_noise(m, tp["scale_sd"], tp["var_sd"]), orc.EMIT_DESCALED, tp["scale"],
                              tp["shift"], tp["var"])
    # getHdpStateMachine (loadStateMachineHdp, :124-130): the model's own level means
    sm_hdp = api.getHdpStateMachine(nhdp, model, tp["scale"], tp["shift"], tp["var"], set_expected_values=False)
    om_hdp = orc.OracleModel(m, orc.EMIT_HDP, tp["scale"], tp["shift"], tp["var"],
                             hdp=formats.parse_nhdp(nhdp))
    ref, ev = z["reference"], z["events"]
    rows = [("scaled", sm_scaled, om_scaled, ref, ev, 0.01, True, "CEO", ex["scaled"]),
            ("descaled", sm_desc, om_desc, ref, ev, 0.01, True, "CEO", ex["descaled"])]
    for base in "CEO":
        rows.append((base, sm_desc, om_desc, ref.replace("C", base), ev, 0.01, False, "CEO", ex[base]))
    rows.append(("X", sm_desc, om_desc, ref.replace("C", "X"), ev, 0.01, False, "CEO", ex["X"]))
    rows.append(("hdp", sm_hdp, om_hdp, ref, z["hdp_events"], 0.1, True, "CEO", ex["hdp_threshold_0_1"]))
    return dict(rows=rows, anchors=z["anchors"], expansion=z["expansion"], template_params=tp)


def _params(api, expansion, threshold):
    p = api.pairwiseAlignmentBandingParameters_construct()   # library defaults: expansion 20
    assert p.diagonal_expansion == expansion
    p.threshold = threshold
    return p


def _oracle(om, ref, ev, anc, expansion, thr, ragged, options):
    return orc.aligned_pairs(om, ref, ev, anc, orc.params(threshold=thr, expansion=expansion), ragged, ragged,
                             options=options)


def test_zymo_banded_plain_fp64(api, case):
    anc = case["anchors"]
    for name, sm, om, ref, ev, thr, ragged, options, count in case["rows"]:
        p = _params(api, case["expansion"], thr)
        got = api.getAlignedPairsUsingAnchors(sm, ref, ev, anc, p, ragged, ragged, degenerate=api.CYTOSINE_METHYLATION3)
        want = _oracle(om, ref, ev, anc, case["expansion"], thr, ragged, options)
        assert len(want) == count, name
        assert len(got) == count, (name, len(got))
        assert W.max_posterior_error(want, got, thr) <= FP64_TOL, name


def test_zymo_banded_batched_fp32(api, case):
    """every case in one batch; the X read runs in the batch's plain FP64 set"""
    anc = case["anchors"]
    rows = case["rows"]
    for thr in sorted({r[5] for r in rows}):
        sel = [r for r in rows if r[5] == thr]
        tp = case["template_params"]
        inputs = [api.ReadInput(sm=sm, reference=ref, events=ev, anchors=anc, scale=tp["scale"], shift=tp["shift"],
                                var=tp["var"], ragged_left=ragged, ragged_right=ragged,
                                degenerate=api.CYTOSINE_METHYLATION3)
                  for _, sm, _, ref, ev, _, ragged, _, _ in sel]
        b = api.align_batch(inputs, _params(api, case["expansion"], thr))
        for i, (name, sm, om, ref, ev, _, ragged, options, count) in enumerate(sel):
            assert b.status(i) == 0, name
            got = b.pairs(i)
            want = _oracle(om, ref, ev, anc, case["expansion"], thr, ragged, options)
            assert len(want) == count
            tol = FP64_TOL if name == "X" else FP32_TOL
            assert W.max_posterior_error(want, got, thr) <= tol, name
            near = int(np.sum(np.abs(want["score"] / 1e7 - thr) <= tol))
            assert abs(len(got) - count) <= near, (name, len(got), count, near)
