"""The host steps either side of the path, against the oracle restatement (oracle/io.py): anchor
pairs from a guide alignment, remapping to events, the overlap filter (before); ordering, score and
the three posterior file formats, byte for byte (after).  No GPU needed."""
import itertools

import numpy as np
import pytest

from oracle import formats
from oracle import io as oio
from signalalign_b200 import synth


@pytest.fixture(scope="module")
def api():
    from signalalign_b200 import api as a
    return a


def _random_sorted_pairs(r, lx, ly, accept):
    pairs = [(x, y) for x in range(lx) for y in range(ly) if r.random() > accept]
    return pairs


@pytest.mark.parametrize("seed", range(6))
def test_filter_matches_oracle_and_is_maximal(api, seed):
    """test_filterToRemoveOverlap (signalPairwiseAlignerTest.c:713-760, disabled there): the output is
    strictly increasing in both coordinates, and every pair that crosses no other pair is kept (the
    reference's check compares a pair with itself, which is why it never passed; it is restated here
    without that)."""
    r = np.random.default_rng(seed)
    pairs = _random_sorted_pairs(r, int(r.integers(0, 60)), int(r.integers(0, 60)), float(r.random()) * 0.9 + 0.1)
    if seed == 5:   # duplicates, equal x with rising y
        pairs = sorted(pairs + pairs[: len(pairs) // 3])
    got = api.filterToRemoveOverlap(pairs)
    assert got == oio.filter_to_remove_overlap(pairs)
    assert all(a[0] < b[0] and a[1] < b[1] for a, b in zip(got, got[1:]))
    uniq = sorted(set(pairs))
    free = [p for p in uniq if not any(q != p and ((q[0] <= p[0] and q[1] >= p[1]) or (q[0] >= p[0] and q[1] <= p[1]))
                                       for q in uniq)]
    assert set(free) <= set(got)


def test_filter_rejects_unsorted_input(api):
    with pytest.raises(api.SAError) as ei:
        api.filterToRemoveOverlap([(3, 4), (1, 2)])
    assert ei.value.status == 3


def _random_cigar(r, n_ops):
    ops = []
    for _ in range(n_ops):
        op = int(r.choice([0, 0, 0, 1, 2]))
        ops.append((op, int(r.integers(1, 40))))
    return ops


@pytest.mark.parametrize("seed", range(8))
def test_guide_alignment_anchor_pairs_match_oracle(api, seed):
    """signalUtils_guideAlignmentToRebasedAnchorPairs on random guide alignments, both reference
    strands, diagonal trims 0-14 (constraintDiagonalTrim defaults to 14)."""
    r = np.random.default_rng(100 + seed)
    ops = _random_cigar(r, int(r.integers(1, 30)))
    span1 = sum(l for o, l in ops if o != 2)
    span2 = sum(l for o, l in ops if o != 1)
    trim = int(r.integers(0, 15))
    start2 = int(r.integers(0, 500))
    if seed % 2 == 0:
        start1 = int(r.integers(0, 10000))
        s1, e1, st1 = start1, start1 + span1, 1
    else:   # reverse strand: start1 >= end1 before the rebase
        end1 = int(r.integers(0, 10000))
        s1, e1, st1 = end1 + span1, end1, 0
    got, rebased = api.guideAlignmentToRebasedAnchorPairs(s1, e1, st1, start2, start2 + span2, ops, trim)
    want, want_rebased = oio.guide_alignment_to_anchor_pairs(s1, e1, st1, start2, start2 + span2, ops, trim)
    assert got == want
    assert rebased == want_rebased
    assert rebased[0] == 0 and rebased[2] == 1


def test_guide_alignment_rejects_inconsistent_cigar(api):
    with pytest.raises(api.SAError) as ei:
        api.guideAlignmentToRebasedAnchorPairs(0, 10, 1, 0, 10, [(0, 9)], 0)
    assert ei.value.status == 1


@pytest.mark.parametrize("seed", range(4))
def test_remapped_anchor_pairs_match_oracle(api, seed):
    """signalUtils_getRemappedAnchorPairs: read positions through a monotone event map (several
    positions may share an event), shifted by the map at the alignment start, then filtered."""
    r = np.random.default_rng(200 + seed)
    n_pos = int(r.integers(50, 400))
    event_map = np.cumsum(r.integers(0, 3, n_pos)).astype(np.int64)
    xs = np.sort(r.choice(2000, size=60, replace=False))
    ys = np.sort(r.choice(n_pos, size=60, replace=False))
    anchors = [(int(x), int(y)) for x, y in zip(xs, ys)]
    offset = int(r.integers(0, n_pos))
    got = api.getRemappedAnchorPairs(anchors, event_map, offset)
    assert got == oio.remap_anchor_pairs(anchors, [int(v) for v in event_map], offset)


def test_sort_and_score(api):
    r = np.random.default_rng(3)
    pairs = [(int(r.integers(100000, 10000000)), int(r.integers(0, 50)), int(r.integers(0, 50)), int(r.integers(0, 99)))
             for _ in range(300)]
    got = api.sortByXPlusYCoordinate(pairs)
    assert [tuple(int(v) for v in p) for p in got] == oio.sort_by_x_plus_y(pairs)
    assert api.scoreByPosteriorProbabilityIgnoringGaps(pairs) == oio.posterior_score(pairs)


@pytest.fixture(scope="module")
def acegt():
    table = synth.gaussian_table("ACEGT", 6, 7)
    m = formats.parse_model_lines(*synth.model_text("ACEGT", 6, table).split("\n")[:3])
    return m


def _case(seed, m, n_pairs=200):
    r = np.random.default_rng(seed)
    L = 400
    target = "".join(r.choice(list("ACGT"), L))
    target = "".join("X" if (i % 37 == 5) else c for i, c in enumerate(target))   # degenerate sites
    n_events = 900
    events = np.column_stack([r.uniform(60, 120, n_events), r.uniform(0.5, 2, n_events), r.exponential(0.002, n_events),
                              np.cumsum(r.exponential(0.002, n_events))])
    event_offset = int(r.integers(0, 100))
    pairs = [(int(r.integers(100000, 10000001)), int(r.integers(0, L - 6 + 1)), int(r.integers(0, n_events - event_offset)),
              int(r.integers(0, 5 ** 6))) for _ in range(n_pairs)]
    return target, events, event_offset, pairs


@pytest.mark.parametrize("fmt,strand,forward", list(itertools.product([0, 1, 2], [0, 1], [True, False])))
def test_posterior_files_match_oracle_bytes(api, acegt, fmt, strand, forward, tmp_path):
    """writePosteriorProbsFull / writePosteriorProbsVC / writeAssignments (signalMachine.c:68-238) for
    every strand and guide direction: the same bytes as the restatement of the reference's printf
    calls; the file form appends exactly that text."""
    m = acegt
    sm = api.StateMachine.from_tables("ACEGT", 6, m["t"], m["match"], m["gapy"], m["gapx"], emission=api.EMIT_DESCALED)
    target, events, event_offset, pairs = _case(10 * fmt + 2 * strand + int(forward), m)
    kw = dict(target=target, strand=strand, forward=forward, event_offset=event_offset, reference_offset=1234,
              events=events, scale=1.02, shift=-3.5, var=1.1, scale_sd=0.97, read_label="read_7", contig="chr_test")
    got = api.formatAlignment(fmt, sm, pairs, **kw)
    match_table = np.asarray(m["match"]).reshape(-1, 5)
    want = oio.format_alignment(fmt, pairs, "ACEGT", 6, match_table, target, strand, forward, event_offset, 1234,
                                events, 1.02, -3.5, 1.1, 0.97, read_label="read_7", contig="chr_test")
    assert got == want
    assert len(got) > 0
    path = tmp_path / "posteriors.tsv"
    api.outputAlignment(fmt, path, sm, pairs, **kw)
    api.outputAlignment(fmt, path, sm, pairs, **kw)
    assert path.read_text() == want + want
