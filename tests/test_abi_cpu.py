"""C-ABI checks that need no GPU: the library loads and exports every declared entry point; host
geometry (band, split points), model readers and table transforms match the oracle bit for bit."""
import math
import os
import re

import numpy as np
import pytest

from oracle import formats
from oracle import oracle as orc
from signalalign_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def api():
    from signalalign_b200 import api as a
    return a


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(sa_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol(api):
    lib = api.lib()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_band_golden_via_abi(api):
    L, R = api.band_construct([(1, 0), (2, 1), (3, 3)], 6, 5, 2)
    want = [(0, 0), (-1, 1), (-2, 2), (-1, 3), (-2, 4), (-1, 3), (-2, 4), (-3, 3), (-2, 2), (-1, 3), (0, 2), (1, 1)]
    assert list(zip(L.tolist(), R.tolist())) == want


def random_anchors(r, lX, lY, step, jitter):
    out = []
    for x in range(step, lX, step):
        y = int(x * lY / lX) + int(r.integers(-jitter, jitter + 1))
        xx = x + int(r.integers(-jitter, jitter + 1))
        if 0 <= xx < lX and 0 <= y < lY and (not out or (xx > out[-1][0] and y > out[-1][1])):
            out.append((xx, y))
    return np.array(out, dtype=np.int64).reshape(-1, 2)


@pytest.mark.parametrize("seed", range(8))
def test_band_matches_oracle_random(api, seed):
    r = np.random.default_rng(seed)
    lX, lY = int(r.integers(0, 3000)), int(r.integers(0, 4000))
    anchors = random_anchors(r, max(lX, 1), max(lY, 1), int(r.integers(5, 120)), int(r.integers(0, 20))) \
        if lX and lY else np.zeros((0, 2), np.int64)
    e = int(r.choice([0, 2, 20, 50, 100]))
    L1, R1 = api.band_construct(anchors, lX, lY, e)
    L2, R2 = orc.band(anchors, lX, lY, e)
    assert np.array_equal(L1, L2) and np.array_equal(R1, R2)


def test_band_rejects_bad_anchors(api):
    with pytest.raises(api.SAError) as ei:
        api.band_construct([(5, 5), (4, 6)], 10, 10, 2)
    assert ei.value.status == 3
    with pytest.raises(api.SAError):
        api.band_construct([(10, 3)], 10, 10, 2)   # x must stay below lX
    with pytest.raises(api.SAError):
        api.band_construct([], 5, 5, 3)            # odd expansion


def test_split_points_match_oracle(api):
    m = 2000 * 2000
    anchors = [(2000, 2000), (4002, 4001), (5000, 5000), (8000, 6000), (9000, 9000), (10000, 14000),
               (15000, 15000), (16000, 16000)]
    for rl in (0, 1):
        for rr in (0, 1):
            assert api.getSplitPoints(anchors, 20000, 25000, m, rl, rr) == orc.split_points(anchors, 20000, 25000,
                                                                                            m, rl, rr)
            assert api.getSplitPoints([], 20000, 25000, m, rl, rr) == orc.split_points([], 20000, 25000, m, rl, rr)
    r = np.random.default_rng(3)
    for _ in range(20):
        lX, lY = int(r.integers(1000, 40000)), int(r.integers(1000, 40000))
        a = random_anchors(r, lX, lY, int(r.integers(200, 6000)), 50)
        lim = int(r.choice([10 ** 5, 10 ** 6, 9 * 10 ** 6]))
        assert api.getSplitPoints(a, lX, lY, lim, 0, 1) == orc.split_points(a, lX, lY, lim, 0, 1)


def test_model_reader_matches_oracle_reader(api, tmp_path):
    cfg = synth.config0()
    text = synth.model_text("ACGT", 6, cfg["table"])
    path = tmp_path / "syn.model"
    path.write_text(text)
    sm = api.StateMachine.load(str(path), api.THREE_STATE, api.EMIT_DESCALED)
    got = sm.tables()
    want = formats.load_model_file(str(path))
    assert np.array_equal(got["match"], want["match"])
    assert np.array_equal(got["gapy"], want["gapy"])
    assert np.array_equal(got["gapx"], want["gapx"])
    assert np.array_equal(got["t"], np.array(want["t"]))
    assert sm.kmer_length == 6 and sm.n_kmers == 4096
    assert sm.kmer_string(0) == "AAAAAA" and sm.kmer_string(4095) == "TTTTTT"
    assert sm.kmer_id("ACGTAC") == formats.kmer_id("ACGTAC", "ACGT")
    assert sm.kmer_id("ACGTAE") == -1
    # emissions_signal_scaleModel on the C side equals the oracle's restatement
    sm.scaleModel(1.03, -2.5, 1.1, 0.9, 1.2)
    got = sm.tables()
    want2 = formats.scale_model(want, 1.03, -2.5, 1.1, 0.9, 1.2)
    for col in (0, 1, 2, 4):
        assert np.array_equal(got["match"][:, col], want2["match"][:, col])
        assert np.array_equal(got["gapy"][:, col], want2["gapy"][:, col])


def test_model_reader_errors(api, tmp_path):
    with pytest.raises(api.SAError) as ei:
        api.StateMachine.load(str(tmp_path / "missing.model"))
    assert ei.value.status == 8
    bad = tmp_path / "bad.model"
    bad.write_text("3\t4\tACGT\t2\n0.9 0.1\n1 2 3\n")
    with pytest.raises(api.SAError) as ei:
        api.StateMachine.load(str(bad))
    assert ei.value.status == 8


def write_nhdp(path, alphabet, k, grid_start, grid_stop, grid_length, observed_leaves, density, slope):
    """A minimal .nhdp in the layout serialize_nhdp / serialize_hdp write (nanopore_hdp.c:1060-1069,
    hdp.c:2914-3045): one base DP with every k-mer leaf as a child; `observed_leaves` get one data
    point each; density / slope rows for every observed DP (leaves and base)."""
    n_leaves = len(alphabet) ** k
    num_dps = n_leaves + 1
    base = n_leaves
    lines = [str(len(alphabet)), alphabet, str(k), "1", "1", "0", str(num_dps)]
    lines.append("\t".join("%.17g" % 80.0 for _ in observed_leaves))
    lines.append("\t".join(str(i) for i in observed_leaves))
    lines.append("80\t1\t2\t3")
    lines.append("%.17g\t%.17g\t%d" % (grid_start, grid_stop, grid_length))
    lines.append("1\t1")
    for i in range(n_leaves):
        lines.append("%d\t0" % base)
    lines.append("-\t0")
    obs = set(observed_leaves) | {base}
    for i in range(num_dps):
        lines.append("\t".join("%.17g" % v for v in density[i]) if i in obs else "")
    for i in range(num_dps):
        lines.append("\t".join("%.17g" % v for v in slope[i]) if i in obs else "")
    path.write_text("\n".join(lines) + "\n")


def test_nhdp_reader_matches_oracle_reader(api, tmp_path):
    alphabet, k, gl = "ACGT", 3, 50
    r = np.random.default_rng(1)
    dens = r.random((65, gl))
    slope = r.normal(size=(65, gl))
    observed = sorted(r.choice(64, 20, replace=False).tolist())
    p = tmp_path / "t.nhdp"
    write_nhdp(p, alphabet, k, 40.0, 120.0, gl, observed, dens, slope)
    mp = tmp_path / "t.model"
    table = np.tile([80.0, 2.0, 1.0, 0.3, 11.0], (64, 1))
    mp.write_text(synth.model_text(alphabet, k, table))
    h = formats.parse_nhdp(str(p))
    assert h["alphabet"] == "ACGT" and h["kmer_length"] == 3
    # unobserved leaves fall back to the base DP's row
    base_row = h["rows"].index(64)
    for kid in range(64):
        assert h["kmer_row"][kid] == (h["rows"].index(kid) if kid in observed else base_row)
    sm = api.StateMachine.load(str(mp), api.THREE_STATE_HDP, api.EMIT_HDP, nhdp_file=str(p),
                               set_hdp_expected_values=True)
    got = sm.tables()
    m = formats.load_model_file(str(mp))
    want = formats.hdp_expected_values(m, h)
    np.testing.assert_allclose(got["match"], want["match"], rtol=1e-13, atol=0)


def test_status_strings(api):
    lib = api.lib()
    for s in range(12):
        assert lib.sa_status_string(s).decode() == api.STATUS[s]


def test_batch_planning_with_degenerate_reads(api):
    """Host planning of a batch that mixes reads with degenerate ('X') positions, which go to the
    plain FP64 form, with ordinary reads: planning completes (on a host without a GPU the create
    call then stops at the first pinned or device allocation, the no-allocation entry at the
    models' device tables)."""
    cfg = synth.config3(seed=5, n_reads=1, span=(300, 400), grid_length=50, route="degenerate")
    sub = synth.config3(seed=5, n_reads=1, span=(300, 400), grid_length=50)["alignments"]
    m = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["gauss_table"]).split("\n")[:3])
    sm = api.StateMachine.from_tables("ACEGT", 6, m["t"], m["match"], m["gapy"], m["gapx"],
                                      emission=api.EMIT_DESCALED)
    als = cfg["alignments"] + sub
    reads = [api.ReadInput(sm=sm, reference=a["reference"], events=a["events"], anchors=a["anchors"],
                           scale=a["scale"], shift=a["shift"], degenerate=0) for a in als]
    assert sum("X" in a["reference"] for a in als) == 2
    p = api.pairwiseAlignmentBandingParameters_construct()
    try:
        b = api.Batch(reads, p)
    except api.SAError as e:
        assert e.status in (4, 5), e   # pinned staging or device step: no device here
    else:
        assert b.cells > 0
    # the no-allocation entry packs on the heap before it looks at the device: the packing runs here
    # and the call stops at the models' device tables
    try:
        api.align_batch_noalloc(reads, p)
    except api.SAError as e:
        assert e.status in (1, 4, 5), e


@pytest.mark.parametrize("name, alphabet, k", [("testModelR73_acegot_template.model", "ACEGOT", 6),
                                               ("testModelR9_5mer_acgt_template.model", "ACGT", 5)])
def test_reference_model_files_through_product_loader(api, name, alphabet, k):
    """stateMachine3_loadFromFile (stateMachine.c:1328-1426) on the reference's own model files
    (models/, kept byte for byte in tests/golden): the product's loader and the oracle's restated
    reader give identical tables, including the SWITCH_TO_X quirk (gap-Y -> gap-X stored in
    SWITCH_TO_Y, SWITCH_TO_X left at LOG_ZERO)."""
    from golden_models import golden_file
    path = golden_file(name)
    sm = api.StateMachine.load(path, api.THREE_STATE, api.EMIT_DESCALED)
    got = sm.tables()
    want = formats.load_model_file(path)
    assert want["alphabet"] == alphabet and sm.kmer_length == k and sm.n_kmers == len(alphabet) ** k
    for key in ("match", "gapy", "gapx"):
        assert np.array_equal(got[key], want[key]), key
    assert np.array_equal(got["t"], np.array(want["t"]))
    assert got["t"][7] == -math.inf                     # SWITCH_TO_X
    assert np.all(np.isfinite(got["match"]))


def test_reference_nhdp_through_product_loader(api):
    """deserialize_nhdp (nanopore_hdp.c:1071-1098) on the reference's templateSingleLevelFixed.nhdp
    through the product's HDP loader: grid, per-row posterior-predictive densities and knot slopes,
    and each k-mer's observed-ancestor row equal the oracle reader's; the R7.3 ACEGOT model's match
    table is untouched when the HDP expected values are not applied, and with them every observed
    k-mer's level mean and sd are the HDP's (stateMachine3_setModelToHdpExpectedValues)."""
    from golden_models import golden_file
    model, nhdp = golden_file("testModelR73_acegot_template.model"), golden_file("templateSingleLevelFixed.nhdp")
    want = formats.parse_nhdp(nhdp)
    sm = api.StateMachine.load(model, api.THREE_STATE_HDP, api.EMIT_HDP, nhdp_file=nhdp, set_hdp_expected_values=False)
    got = sm.hdp_tables()
    assert np.array_equal(got["grid"], want["grid"])
    assert np.array_equal(got["density"], want["density"])
    assert np.array_equal(got["slope"], want["slope"])
    assert np.array_equal(got["kmer_row"], want["kmer_row"])
    m = formats.load_model_file(model)
    assert np.array_equal(sm.tables()["match"], m["match"])
    sm2 = api.StateMachine.load(model, api.THREE_STATE_HDP, api.EMIT_HDP, nhdp_file=nhdp, set_hdp_expected_values=True)
    ev = formats.hdp_expected_values(m, want)
    assert np.allclose(sm2.tables()["match"], ev["match"], rtol=1e-12, atol=1e-12)


def test_launch_config_table(api, tmp_path):
    """sa_loadLaunchConfigs reads the tuner's table (tab-separated: device name, width class, four
    fields); malformed rows and missing files are SA_E_FILE; without a device (or for a device the
    table does not name) the defaults apply."""
    good = tmp_path / "cfg.tsv"
    good.write_text("# device\twidth\tcps\tgpr\tww\tecs\nNo Such GPU\t1\t1\t4\t0\t8\nNo Such GPU\t2\t1\t2\t0\t16\n")
    assert api.lib().sa_loadLaunchConfigs(str(good).encode()) == 0
    for bad in ("No Such GPU\t3\t1\t4\t0\t8\n", "No Such GPU\t1\t0\t4\t0\t8\n", "No Such GPU\t1\t1\t4\n",
                "No Such GPU\t1\tx\t4\t0\t8\n"):
        p = tmp_path / "bad.tsv"
        p.write_text(bad)
        assert api.lib().sa_loadLaunchConfigs(str(p).encode()) == 8
    assert api.lib().sa_loadLaunchConfigs(str(tmp_path / "missing.tsv").encode()) == 8
    with pytest.raises(api.SAError):
        api.get_launch_config(0, 3)
    import torch
    if not torch.cuda.is_available():
        assert api.get_launch_config(0, 1) == dict(ctas_per_sm=2, grid_per_region=3, warp_windows=1,
                                                   emission_ctas_per_sm=16)
