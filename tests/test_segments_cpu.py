"""Forward-segment planning on the host (sa_planForwardSegments), no GPU.

The batched FP32 form cuts a long region's forward sweep at traceback-window starts into segments
swept side by side; each later segment warms up over max(warm-up, 10 band widths) anti-diagonals.
Checked here against an independent restatement of where getPosteriorProbsWithBanding's windows
start (pairwiseAligner.c:1319-1333: a traceback at the first anti-diagonal at least
minDiagsBetweenTraceBack past the last one whose width is at most 2 * expansion + 1; the next window
starts traceBackDiagonals + 1 before it), with the band from the oracle:

* the segments of a region tile its anti-diagonals 0..lX+lY in order;
* every later segment starts at a window start, owns at least its warm-up, and its warm-up is
  2 mod 3 (so the stepping loop can stop at the segment's start) and at least 10 band widths;
* no segment's sweep (warm-up included) exceeds the cap by more than one window of snapping, and
  no last piece is shorter than half a piece;
* a negative cap keeps the region whole.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from signalalign_b200 import synth


@pytest.fixture(scope="module")
def api():
    from signalalign_b200 import api as a
    return a


def window_starts(anchors, lX, lY, expansion=50, min_diags=1000, traceback=40):
    L, R = orc.band(anchors, lX, lY, expansion)
    n = lX + lY
    starts, traced_back_to = [0], 0
    for d in range(1, n + 1):
        width = (R[d] - L[d]) // 2 + 1
        if d == n:
            break
        if d >= traced_back_to + min_diags and width <= 2 * expansion + 1:
            traced_back_to = d - (traceback + 1)
            starts.append(traced_back_to)
    return set(starts), int(np.max((R - L) // 2 + 1))


@pytest.mark.parametrize("cap", [4096, 8192, 20000])
def test_segments_tile_regions_at_window_starts(api, cap):
    cfg = synth.config1(seed=91, n_reads=4, span=(3000, 20000))
    p = api.pairwiseAlignmentBandingParameters_construct(diagonal_expansion=50)
    for rd in cfg["reads"]:
        lX, lY = len(rd["reference"]) - 5, len(rd["events"])
        segs = api.plan_forward_segments(rd["anchors"], lX, lY, p, cap, 1024)
        starts, maxw = window_starts(rd["anchors"], lX, lY, p.diagonal_expansion, p.min_diags_between_traceback,
                                     p.traceback_diagonals)
        assert (segs[:, 0] == 0).all()            # one region: no gap exceeds the split limit
        assert segs[0, 1] == 0 and segs[-1, 2] == lX + lY
        assert (segs[1:, 1] == segs[:-1, 2]).all()
        warm_min = max(1024, 10 * maxw)
        assert segs[0, 3] == 0
        for b, e, warm in segs[1:, 1:4]:
            assert b in starts, (b, sorted(starts)[:5])
            assert warm % 3 == 2 and warm_min <= warm <= warm_min + 2
            assert e - b >= warm_min
            assert b - warm >= 2
        if len(segs) > 1:
            piece = (lX + lY - warm_min) / len(segs)
            sweeps = [segs[0, 2]] + [e - b + w for b, e, w in segs[1:, 1:4]]
            assert max(sweeps) <= max(cap, piece + warm_min) + 1000 + 41 + 2
            assert segs[-1, 2] - segs[-1, 1] >= piece / 2


def test_short_regions_and_negative_cap_stay_whole(api):
    cfg = synth.config1(seed=92, n_reads=2, span=(600, 900))
    p = api.pairwiseAlignmentBandingParameters_construct()
    for rd in cfg["reads"]:
        lX, lY = len(rd["reference"]) - 5, len(rd["events"])
        assert len(api.plan_forward_segments(rd["anchors"], lX, lY, p, 4096)) == 1
    rd = synth.config1(seed=93, n_reads=1, span=(15000, 16000))["reads"][0]
    lX, lY = len(rd["reference"]) - 5, len(rd["events"])
    assert len(api.plan_forward_segments(rd["anchors"], lX, lY, p, 4096)) > 3
    whole = api.plan_forward_segments(rd["anchors"], lX, lY, p, -1)
    assert whole.shape[0] == 1 and whole[0, 1] == 0 and whole[0, 2] == lX + lY


def test_plan_arguments(api):
    rd = synth.config1(seed=94, n_reads=1, span=(15000, 16000))["reads"][0]
    lX, lY = len(rd["reference"]) - 5, len(rd["events"])
    p = api.pairwiseAlignmentBandingParameters_construct()
    with pytest.raises(api.SAError):
        api.plan_forward_segments(rd["anchors"], lX, lY, p, 0)        # 0 is the batch's automatic cap
    with pytest.raises(api.SAError):
        api.plan_forward_segments(rd["anchors"], lX, lY, p, 4096, 10)  # warm-up below 64


@pytest.mark.parametrize("expansion", [50, 200])
def test_flat_start_forgets_within_the_warmup(api, expansion):
    """What forward segments rest on, on the FP64 oracle: a forward sweep begun from a flat vector
    becomes the true sweep minus one constant (to 1e-9 on every finite cell, with the same -inf
    cells) well within the warm-up the planner gives a segment (max(1024, 10 band widths))."""
    import workloads as W
    cfg = synth.config1(seed=95 + expansion, n_reads=3, span=(3000, 5000))
    m = W.gaussian_model(cfg)
    worst = 0
    for rd in cfg["reads"]:
        om = W.oracle_model(m, orc.EMIT_DESCALED, rd)
        lX, lY = len(rd["reference"]) - 5, len(rd["events"])
        _, maxw = window_starts(rd["anchors"], lX, lY, expansion)
        warm = max(1024, 10 * maxw)
        starts = list(range(warm + 2, lX + lY - warm, 2500))
        steps = orc.flat_start_forgetting(om, rd["reference"], rd["events"], rd["anchors"], starts, expansion,
                                          horizon=warm + 500, tol=1e-9)
        assert (steps >= 0).all(), steps
        worst = max(worst, int(steps.max()) / warm)
    assert worst < 0.8, worst


def test_flat_start_forgets_with_two_path_cells(api):
    """The same with degenerate X (C or E) sites, whose cells hold two paths (the plain FP64 form's
    forward segments): every path slot of the flat-start sweep becomes the true one minus the
    constant within the warm-up."""
    from oracle import formats
    import workloads as W
    cfg = synth.config3(seed=97, n_reads=2, span=(3000, 4000), grid_length=200, route="degenerate")
    m = formats.parse_model_lines(*synth.model_text("ACEGT", 6, cfg["gauss_table"]).split("\n")[:3])
    worst, sites = 0, 0
    for rd in [a for a in cfg["alignments"] if a["model"] == "gauss"]:
        sites += rd["reference"].count("X")
        om = W.oracle_model(m, orc.EMIT_DESCALED, rd)
        lX, lY = len(rd["reference"]) - 5, len(rd["events"])
        _, maxw = window_starts(rd["anchors"], lX, lY)
        warm = max(1024, 10 * maxw)
        starts = list(range(warm + 2, lX + lY - warm, 2000))
        steps = orc.flat_start_forgetting(om, rd["reference"], rd["events"], rd["anchors"], starts, 50,
                                          horizon=warm + 500, tol=1e-9, options="CE")
        assert (steps >= 0).all(), steps
        worst = max(worst, int(steps.max()) / warm)
    assert sites > 10
    assert worst < 0.8, worst
