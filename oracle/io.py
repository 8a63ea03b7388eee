"""Oracle for the host steps either side of the path (test infrastructure only: the product never
imports this).  Plain-Python restatements of the reference, line for line:

* filterToRemoveOverlap (impl/pairwiseAligner.c:1575-1616)
* convertPairwiseForwardStrandAlignmentToAnchorPairs (impl/pairwiseAligner.c:1454-1478) behind
  signalUtils_guideAlignmentToRebasedAnchorPairs (impl/signalMachineUtils.c:130-164)
* nanopore_remapAnchorPairsWithOffset (impl/nanopore.c:438-450) behind
  signalUtils_getRemappedAnchorPairs (impl/signalMachineUtils.c:166-170)
* sortByXPlusYCoordinate2 (impl/pairwiseAligner.c:1434-1438), scoreByPosteriorProbabilityIgnoringGaps
  (signalMachine.c:317-331)
* writePosteriorProbsFull / writePosteriorProbsVC / writeAssignments (signalMachine.c:33-238), with
  the reference's printf formats.

The reverse complement is sonLib's stString_reverseComplementString (sonLib is not vendored in the
reference tree): A/C/G/T in either case complemented, other characters kept.
"""

MATCH, INDEL_X, INDEL_Y = 0, 1, 2
PAIR_PROB_1 = 10000000.0


def filter_to_remove_overlap(pairs):
    """pairs: list of (x, y) sorted by (x, y)."""
    keep = set()
    px = py = float("inf")
    for x, y in reversed(pairs):
        if x < px and y < py:
            keep.add((x, y))
        px, py = min(px, x), min(py, y)
    out = []
    px = py = float("-inf")
    for x, y in pairs:
        if x > px and y > py and (x, y) in keep:
            out.append((x, y))
        px, py = max(px, x), max(py, y)
    return out


def guide_alignment_to_anchor_pairs(start1, end1, strand1, start2, end2, ops, trim):
    """ops: list of (op, length).  Returns (anchors, (start1, end1, strand1)) after rebasing."""
    shift = start1 if strand1 else end1
    start1 -= shift
    end1 -= shift
    if not strand1:
        strand1 = 1
        start1, end1 = end1, start1
    pairs = []
    j, k = start1, start2
    for op, length in ops:
        if op == MATCH:
            for l in range(trim, length - trim):
                pairs.append((j + l, k + l))
        if op != INDEL_Y:
            j += length
        if op != INDEL_X:
            k += length
    assert j == end1 and k == end2
    return filter_to_remove_overlap(sorted(pairs)), (start1, end1, strand1)


def remap_anchor_pairs(anchors, event_map, map_offset):
    remapped = [(x, event_map[y] - event_map[map_offset]) for x, y in anchors]
    return filter_to_remove_overlap(remapped)


def sort_by_x_plus_y(pairs):
    """pairs: list of (score, x, y, kmer); stable for equal keys"""
    return sorted(pairs, key=lambda p: p[1] + p[2])


def posterior_score(pairs):
    total = 0.0
    for p in pairs:
        total += p[0]
    return 100.0 * total / (len(pairs) * PAIR_PROB_1) if pairs else float("nan")


_RC = {"A": "T", "C": "G", "G": "C", "T": "A", "a": "t", "c": "g", "g": "c", "t": "a"}


def reverse_complement(s):
    return "".join(_RC.get(c, c) for c in reversed(s))


def kmer_string(kmer_id, alphabet, k):
    out = []
    for _ in range(k):
        out.append(alphabet[kmer_id % len(alphabet)])
        kmer_id //= len(alphabet)
    return "".join(reversed(out))


def format_alignment(fmt, pairs, alphabet, k, match_table, target, strand, forward, event_offset, reference_offset,
                     events, scale, shift, var, scale_sd, read_label="", contig=""):
    """fmt 0 full, 1 variant caller, 2 assignments; pairs (score, x, y, kmer id); match_table rows of
    5 (mean, sd, noise mean, noise sd, lambda); events rows of 4.  Returns the text."""
    strand_label = "t" if strand == 0 else "c"
    as_given = (strand == 0 and forward) or (strand != 0 and not forward)
    ref_length = len(target)
    ref_length_kmers = ref_length - k
    lines = []
    for score, x_i, y0, kid in pairs:
        y = y0 + event_offset
        p = score / PAIR_PROB_1
        path_kmer = kmer_string(kid, alphabet, k)
        e_mean = match_table[kid][0]
        if fmt == 2:
            ev_mean = events[y][0]
            descaled = (ev_mean + var * e_mean - scale * e_mean - shift) / var
            lines.append("%s\t%s\t%f\t%f\n" % (path_kmer, strand_label, descaled, p))
            continue
        k_i = target[x_i:x_i + k]
        ref_kmer = k_i if as_given else reverse_complement(k_i)
        x_adj = x_i + reference_offset if as_given else ref_length_kmers - (x_i + (ref_length - reference_offset))
        if fmt == 0:
            ev = events[y]
            e_noise = match_table[kid][2]
            descaled = (ev[0] + var * e_mean - scale * e_mean - shift) / var
            lines.append("%s\t%d\t%s\t%s\t%s\t%d\t%f\t%f\t%f\t%s\t%f\t%f\t%f\t%f\t%f\t%s\n" % (
                contig, x_adj, ref_kmer, read_label, strand_label, y, ev[0], ev[1], ev[2], k_i,
                e_mean * scale + shift, e_noise * scale_sd, p, descaled, e_mean, path_kmer))
        else:
            forward_label = "forward" if forward else "backward"
            for q in range(k):
                if ref_kmer[q] != "X":
                    continue
                qpos = q if as_given else (k - 1) - q
                lines.append("%d\t%d\t%s\t%f\t%s\t%s\t%s\n" % (y, x_adj + q, path_kmer[qpos], p, strand_label,
                                                                forward_label, read_label))
    return "".join(lines)
