"""Pins the CPU oracle to the reference's own known-answer tests (no GPU needed).

Each test names the reference test it reproduces (tests/*.c in the signalAlign tree)."""
import math
import os

import numpy as np
import pytest

from oracle import formats
from oracle import oracle as orc
from oracle import anchors as A
from golden_models import golden_file, load_fixture, model_from_fixture, zymo_banded


def test_bands_golden():
    """test_bands (signalPairwiseAlignerTest.c:447-510): anchors (1,0),(2,1),(3,3), lX=6, lY=5, e=2."""
    L, R = orc.band([(1, 0), (2, 1), (3, 3)], 6, 5, 2)
    want = [(0, 0, 0), (1, -1, 1), (2, -2, 2), (3, -1, 3), (4, -2, 4), (5, -1, 3), (6, -2, 4), (7, -3, 3),
            (8, -2, 2), (9, -1, 3), (10, 0, 2), (11, 1, 1)]
    assert [(i, int(L[i]), int(R[i])) for i in range(12)] == want


def test_split_points_golden():
    """test_getSplitPoints (signalPairwiseAlignerTest.c:376-445)."""
    m = 2000 * 2000
    assert orc.split_points([], 3000, 1000, m, 0, 0) == [(0, 0, 3000, 1000)]
    assert orc.split_points([], 20000, 25000, m, 1, 1) == []
    assert orc.split_points([], 20000, 25000, m, 1, 0) == [(18000, 23000, 20000, 25000)]
    assert orc.split_points([], 20000, 25000, m, 0, 1) == [(0, 0, 2000, 2000)]
    assert orc.split_points([], 20000, 25000, m, 0, 0) == [(0, 0, 2000, 2000), (18000, 23000, 20000, 25000)]
    anchors = [(2000, 2000), (4002, 4001), (5000, 5000), (8000, 6000), (9000, 9000), (10000, 14000),
               (15000, 15000), (16000, 16000)]
    assert orc.split_points(anchors, 20000, 25000, m, 0, 0) == [
        (0, 0, 3001, 3001), (3002, 3001, 9500, 11001), (9501, 12000, 12001, 14500), (13000, 14501, 18000, 18001),
        (18001, 23000, 20000, 25000)]


def test_logadd_accuracy():
    """test_logAdd (signalPairwiseAlignerTest.c:121-131): 1e5 random pairs within 1e-3."""
    r = np.random.default_rng(5)
    for _ in range(100000 // 1000):
        i, j = r.random(1000), r.random(1000)
        got = np.array([math.exp(orc.log_add(math.log(a), math.log(b))) for a, b in zip(i, j)])
        assert np.all(np.abs(got - (i + j)) < 1e-3)
    assert orc.log_add(-math.inf, -math.inf) == -math.inf
    assert orc.log_add(-math.inf, -3.0) == -3.0
    assert orc.log_add(-3.0, -11.0) == -3.0   # difference >= 7.5 returns the max exactly


def test_emission_pdfs():
    """test_stateMachine3EmissionsPdfs (signalPairwiseAlignerTest.c:81-111)."""
    assert abs(orc.log_gauss_pdf(0, 0, 1) - math.log(1 / math.sqrt(2 * math.pi))) < 1e-3
    r = np.random.default_rng(5)
    for _ in range(200):
        sigma = r.uniform(0.1, 1.0)
        mu = r.uniform(0, 10)
        x = mu + r.uniform(-1, 1)
        ctrl = math.exp(-0.5 * ((x - mu) / sigma) ** 2) / (sigma * math.sqrt(2 * math.pi))
        assert abs(orc.log_gauss_pdf(x, mu, sigma) - math.log(ctrl)) < 1e-3
        lam = r.uniform(0.05, 1.0)
        xx = abs(x) + 0.1
        ig = math.sqrt(lam / (2 * math.pi * xx ** 3)) * math.exp(-lam * (xx - mu) ** 2 / (2 * mu * mu * xx))
        assert abs(orc.log_inv_gauss_pdf(xx, mu, lam) - math.log(ig)) < 1e-3
    assert orc.log_gauss_pdf(1.0, 0.0, 0.0) == -math.inf


def test_hdcell_expansion():
    """test_hdCellConstruct / test_hdCellConstructWorstCase (signalPairwiseAlignerTest.c:556-581) and
    test_substitutedKmers (variableOrderPairwiseAlignerTests.c:169-178)."""
    paths = orc.expand_kmer("ATGXAX", "CEO")
    assert len(paths) == 9 and paths[0] == "ATGCAC" and paths[8] == "ATGOAO"
    paths = orc.expand_kmer("XXXXXX", "CEO")
    assert len(paths) == 729 and paths[0] == "CCCCCC" and paths[728] == "OOOOOO"
    assert orc.expand_kmer("ATGXAX", "CE")[1] == "ATGCAE"
    assert orc.expand_kmer("ACGTAC", "CEO") == ["ACGTAC"]


def test_kmer_index_lexicographic():
    """test_getKmerIndex (variableOrderPairwiseAlignerTests.c:158-167): every ACEGOT 6-mer maps to its
    lexicographic index."""
    import itertools
    alpha = "ACEGOT"
    for i, t in enumerate(itertools.product(alpha, repeat=6)):
        if i % 97:
            continue
        km = "".join(t)
        assert orc.kmer_index(km, alpha) == i
        assert formats.kmer_id(km, alpha) == i
    assert orc.kmer_index("ACGTAN", alpha) == -1


@pytest.mark.parametrize("name", ["toy6", "toy5"])
def test_toy_dp(name):
    """test_sm3_diagonalDPCalculations / test_sm3_5merDiagonalDPCalculations (stateMachineTests.c:
    443-692): forward total == backward total (1e-3), every anti-diagonal's total within 1e-2, and
    exactly 14 / 7 pairs at threshold 0.2, all in the expected set."""
    fx = load_fixture(name)
    om = orc.OracleModel(model_from_fixture(fx), orc.EMIT_PLAIN)
    pairs, tf, tb, diag = orc.full_matrix(om, fx["sequence"], fx["events"], fx["threshold"], options="CEO",
                                          p_mode=1)
    assert abs(tf - tb) < 1e-3
    assert np.max(np.abs(diag - tf)) < 1e-2
    assert len(pairs) == fx["expected_pairs"]
    allowed = {tuple(a) for a in fx["allowed"]}
    assert all((int(p["x"]), int(p["y"])) in allowed for p in pairs)


def test_zymo_unbanded_1076():
    """Unbanded half of test_stateMachine3_getAlignedPairsWithBanding (stateMachineTests.c:823-851):
    the R7.3 model scaled by the read's template parameters (emissions_signal_scaleModel) gives 1076
    pairs at threshold 0.01 over the full 892 x 799 matrix."""
    fx = load_fixture("zymo")
    tp = fx["template_params"]
    m = formats.scale_model(model_from_fixture(fx), tp["scale"], tp["shift"], tp["var"], tp["scale_sd"],
                            tp["var_sd"])
    om = orc.OracleModel(m, orc.EMIT_PLAIN)
    pairs, tf, tb, _ = orc.full_matrix(om, fx["sequence"], fx["events"], 0.01, options="CEO", p_mode=0)
    assert len(pairs) == fx["expected_pairs"]
    xy = {(int(p["x"]), int(p["y"])) for p in pairs}
    assert len(xy) == len(pairs)                  # checkAlignedPairs: unique (x, y)
    assert np.all(pairs["score"] > 0) and np.all(pairs["score"] <= 10000000)
    assert abs(tf - tb) < 1e-3 * abs(tf)


def test_banded_matches_unbanded_on_toy():
    """With no anchors the band is the whole matrix and there is a single traceback window, so the
    banded routine's pairs match the full-matrix routine's except for the refresh schedule of the
    normaliser (here the normalisers agree to 1e-2)."""
    fx = load_fixture("toy5")
    om = orc.OracleModel(model_from_fixture(fx), orc.EMIT_PLAIN)
    banded = orc.aligned_pairs(om, fx["sequence"], fx["events"], [], orc.params(threshold=0.2, expansion=2),
                               ragged_left=False, ragged_right=False)
    full, _, _, _ = orc.full_matrix(om, fx["sequence"], fx["events"], 0.2, p_mode=0)
    assert {(int(p["x"]), int(p["y"])) for p in banded} == {(int(p["x"]), int(p["y"])) for p in full}


def test_parse_reference_nhdp():
    """deserialize_nhdp on the reference's HDP fixture: ACEGOT 6-mers over 46657 DPs, one observed
    ancestor chain per observed leaf; every k-mer resolves to an observed row or none."""
    h = formats.parse_nhdp(golden_file("templateSingleLevelFixed.nhdp"))
    assert h["alphabet"] == "ACEGOT" and h["kmer_length"] == 6
    assert len(h["parent"]) == 46657
    assert h["density"].shape[1] == h["grid_length"] and h["slope"].shape == h["density"].shape
    rows = h["kmer_row"]
    assert rows.shape == (46656,)
    assert np.all(rows < len(h["rows"]))


# ------------------------------------------------------------------------------------------------
# banded, anchored, multi-window known answers (lastz anchors)
# ------------------------------------------------------------------------------------------------
def _zymo_models(z):
    tp = z["template_params"]
    m = formats.load_model_file(golden_file("testModelR73_acegot_template.model"))
    scaled = formats.scale_model(m, tp["scale"], tp["shift"], tp["var"], tp["scale_sd"], tp["var_sd"])
    descaled = formats.scale_noise(m, tp["scale_sd"], tp["var_sd"])
    return m, scaled, descaled


def test_zymo_banded_known_answers():
    """The banded Zymo tests with the reference's own lastz anchors, default parameters (diagonal
    expansion 20; 892 k-mers x 799 events: two traceback windows and refreshes every 10th
    posterior anti-diagonal):
      test_stateMachine3_getAlignedPairsWithBanding (stateMachineTests.c:823-851, via
        test_stateMachine :694-717, ragged ends): 1076 pairs with the scaled machine
        (getStateMachine3 + emissions_signal_scaleModel) and with the descaled machine
        (getStateMachine3_descaled with scaleNoise);
      test_DegenerateNucleotides (:897-960, non-ragged ends, descaled machine): 1076 pairs with
        every C replaced by C, E or O, and 7349 with every C replaced by X (CEO paths);
      test_sm3Hdp_getAlignedPairsWithBanding (:881-895): 1217 pairs at threshold 0.1 with the HDP
        machine (getHdpStateMachine on templateSingleLevelFixed.nhdp, the model's level means, the
        read's scaling) on the events as nanopore_descaleNanoporeRead leaves them."""
    z = zymo_banded()
    tp, ex = z["template_params"], z["expected"]
    m, scaled, descaled = _zymo_models(z)
    ref, ev, anc = z["reference"], z["events"], z["anchors"]
    p = orc.params(threshold=0.01, expansion=z["expansion"])
    got = orc.aligned_pairs(orc.OracleModel(scaled, orc.EMIT_PLAIN), ref, ev, anc, p, True, True)
    assert len(got) == ex["scaled"]
    assert len({(int(r["x"]), int(r["y"])) for r in got}) == len(got)
    om = orc.OracleModel(descaled, orc.EMIT_DESCALED, tp["scale"], tp["shift"], tp["var"])
    assert len(orc.aligned_pairs(om, ref, ev, anc, p, True, True)) == ex["descaled"]
    for base in "CEO":
        assert len(orc.aligned_pairs(om, ref.replace("C", base), ev, anc, p, False, False)) == ex[base]
    deg = orc.aligned_pairs(om, ref.replace("C", "X"), ev, anc, p, False, False, options="CEO")
    assert len(deg) == ex["X"]
    h = formats.parse_nhdp(golden_file("templateSingleLevelFixed.nhdp"))
    omh = orc.OracleModel(m, orc.EMIT_HDP, tp["scale"], tp["shift"], tp["var"], hdp=h)
    ph = orc.params(threshold=0.1, expansion=z["expansion"])
    assert len(orc.aligned_pairs(omh, ref, z["hdp_events"], anc, ph, True, True)) == ex["hdp_threshold_0_1"]


@pytest.mark.skipif(not os.path.exists(A.LASTZ), reason="lastz not built (oracle/build_lastz.sh)")
def test_lastz_anchors_reproduce_fixture():
    """getRemappedAnchors (stateMachineTests.c:132-138) restated over the reference's own lastz gives
    the committed anchors: ZymoRef against the read's 2D sequence, remapped by its template event
    map, overlaps filtered."""
    z = zymo_banded()
    got = A.remapped_anchors(z["reference"], z["two_d_read"], z["template_event_map"])
    assert [list(a) for a in got] == z["anchors"].tolist()
    assert len(got) > 20
