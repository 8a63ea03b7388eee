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
* nanopore_getOneDAssignmentsFromRead (impl/nanopore.c:503-533), nanopore_lineq_solve (:586-648),
  nanopore_compute_mean_scale_params with drift and variance (:650-781),
  nanopore_compute_noise_scale_params (:783-848), nanopore_adjustEventsForDriftP (:535-540): the
  fits of signalUtils_estimateNanoporeParams (impl/signalMachineUtils.c:186-223), sums in the
  reference's sequential order.
* continuousPairHmm_normalize / hmmDiscrete_normalizeTransitions, the two
  continuousPairHmm_load*IntoStateMachine calls and the expectations file writers
  (impl/continuousHmm.c:283-406, :572-628; impl/discreteHmm.c:125-137): the EM maximisation step.

The reverse complement is sonLib's stString_reverseComplementString (sonLib is not vendored in the
reference tree): A/C/G/T in either case complemented, other characters kept.
"""

import math

import numpy as np

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


# ------------------------------------------------------------------------------------------------
# per-read parameter estimation (impl/nanopore.c:503-540, :586-848)
# ------------------------------------------------------------------------------------------------
def one_d_assignments(read, event_map, events, alphabet, k):
    """nanopore_getOneDAssignmentsFromRead: [(kmer id, mean, sd, delta time)]"""
    out = []
    prev = -1
    for i in range(len(read) - (k - 1)):
        ev = event_map[i]
        kid = 0
        for c in read[i:i + k]:
            kid = kid * len(alphabet) + alphabet.index(c)
        if ev > prev:
            out.append((kid, events[ev][0], events[ev][1], events[ev][3]))
            prev = ev
    return out


def lineq_solve(a, b):
    """nanopore_lineq_solve (Gauss-Jordan, no pivoting needed for these systems)"""
    n = len(b)
    a = [row[:] for row in a]
    x = list(b)
    for i in range(n):
        f = 1.0 / a[i][i]
        x[i] *= f
        a[i] = [v * f for v in a[i]]
        for s in range(i + 1, n):
            g = a[s][i]
            x[s] -= g * x[i]
            a[s] = [a[s][j] - g * a[i][j] for j in range(n)]
    for i in range(n - 1, -1, -1):
        for s in range(i - 1, -1, -1):
            g = a[s][i]
            x[s] -= g * x[i]
            a[s] = [a[s][j] - g * a[i][j] for j in range(n)]
    return x


def estimate_params(assignments, model):
    """nanopore_compute_mean_scale_params (drift and var) + nanopore_compute_noise_scale_params:
    returns dict(shift, scale, drift, var, shift_sd, scale_sd, var_sd); model rows of 5"""
    xwx = [[0.0] * 3 for _ in range(3)]
    xwy = [0.0] * 3
    nwx = [[0.0] * 2 for _ in range(2)]
    nwy = [0.0] * 2
    for kid, mean, sd, dt in assignments:
        lm, lsd, nm, nsd = model[kid][0], model[kid][1], model[kid][2], model[kid][3]
        iv = 1.0 / (lsd * lsd)
        sm, st = lm * iv, dt * iv
        xwx[0][0] += iv; xwx[0][1] += sm; xwx[0][2] += st
        xwx[1][1] += sm * lm; xwx[1][2] += sm * dt; xwx[2][2] += st * dt
        xwy[0] += iv * mean; xwy[1] += sm * mean; xwy[2] += st * mean
        inv = 1.0 / (nsd * nsd)
        snm = nm * inv
        nwx[0][0] += inv; nwx[0][1] += snm; nwx[1][1] += snm * nm
        nwy[0] += inv * sd; nwy[1] += snm * sd
    xwx[1][0], xwx[2][0], xwx[2][1] = xwx[0][1], xwx[0][2], xwx[1][2]
    nwx[1][0] = nwx[0][1]
    beta = lineq_solve(xwx, xwy)
    gamma = lineq_solve(nwx, nwy)
    disp = disp_n = 0.0
    for kid, mean, sd, dt in assignments:
        lm, lsd, nm, nsd = model[kid][0], model[kid][1], model[kid][2], model[kid][3]
        r = mean - (beta[0] + beta[1] * lm + beta[2] * dt)
        disp += (r * r) / (lsd * lsd)
        rn = sd - (gamma[0] + gamma[1] * nm)
        disp_n += (rn * rn) / (nsd * nsd)
    n = len(assignments)
    return dict(shift=beta[0], scale=beta[1], drift=beta[2], var=(disp / n) ** 0.5, shift_sd=gamma[0],
                scale_sd=gamma[1], var_sd=(disp_n / n) ** 0.5)


def adjust_events_for_drift(events, drift):
    return [[e[0] - e[3] * drift, e[1], e[2], e[3]] for e in events]


# ------------------------------------------------------------------------------------------------
# EM maximisation step and the expectations file (impl/continuousHmm.c, impl/discreteHmm.c)
# ------------------------------------------------------------------------------------------------
LOG_ZERO = float("-inf")
# StateMachine3 transition fields, in the order of oracle models' "t" (inc/stateMachine.h:153-163)
T_MC, T_MFGX, T_MFGY, T_OX, T_OY, T_EX, T_EY, T_SX, T_SY = range(9)


def normalize_transitions(transitions):
    """hmmDiscrete_normalizeTransitions (discreteHmm.c:125-137): each row divided by its sum"""
    t = [[float(v) for v in row] for row in transitions]
    for f in range(3):
        total = 0.0
        for to in range(3):
            total += t[f][to]
        for to in range(3):
            t[f][to] = t[f][to] / total
    return t


def normalize_expectations(transitions, event_expectations, posteriors, observed, event_model):
    """continuousPairHmm_normalize (continuousHmm.c:283-306): the normalised transitions and the
    event model (n_kmers rows of 5, the machine's match table when the expectations were made) with
    each observed k-mer's level mean and sd replaced by the weighted mean and the root of the
    weighted spread (kept where either is exactly 0)."""
    em = [[float(v) for v in row] for row in event_model]
    for i in range(len(em)):
        if not observed[i]:
            continue
        w = float(posteriors[i])
        u = float(event_expectations[i][0]) / w
        o = (float(event_expectations[i][1]) / w) ** 0.5
        em[i][0] = em[i][0] if u == 0.0 else u
        em[i][1] = em[i][1] if o == 0.0 else o
    return normalize_transitions(transitions), em


def _log(v):
    return math.log(v) if v > 0.0 else LOG_ZERO


def load_expectations(model_t, match, gapy, transitions, event_model=None):
    """continuousPairHmm_loadTransitionsIntoStateMachine (continuousHmm.c:321-339) and, given an
    event model, continuousPairHmm_loadEmissionsIntoStateMachine (:341-352), which writes each
    k-mer's mean into the gap-Y table at [i + 5] (not [i * 5]) and its sd x 1.75 at [i * 5 + 1].
    Returns (t, match, gapy): a list and two arrays shaped like the inputs."""
    t = list(model_t)
    T = transitions
    t[T_MC], t[T_OX], t[T_OY] = _log(T[0][0]), _log(T[0][1]), _log(T[0][2])
    t[T_MFGX], t[T_EX], t[T_SY] = _log(T[1][0]), _log(T[1][1]), LOG_ZERO
    t[T_MFGY], t[T_EY], t[T_SX] = _log(T[2][0]), _log(T[2][2]), _log(T[2][1])
    shape = np.shape(match)
    match = np.array(match, dtype=np.float64).reshape(-1)
    gapy = np.array(gapy, dtype=np.float64).reshape(-1)
    if event_model is not None:
        for i, row in enumerate(event_model):
            match[i * 5] = row[0]
            match[i * 5 + 1] = row[1]
            gapy[i + 5] = row[0]
            gapy[i * 5 + 1] = row[1] * 1.75
    return t, match.reshape(shape), gapy.reshape(shape)


def format_expectations(hdp, alphabet, k, transitions, likelihood, event_model, event_expectations=None,
                        posteriors=None, observed=None, assignment_kmers=(), assignment_means=()):
    """continuousPairHmm_writeToFile (continuousHmm.c:354-406) / hdpHmm_writeToFile (:572-628): the
    text, or "" when a transition is NaN (hmmContinuous_checkTransitions, :12-22)."""
    flat_t = [float(v) for row in transitions for v in row]
    if any(v != v for v in flat_t):
        return ""
    out = ["3\t%d\t%s\t%d\t\n" % (len(alphabet), alphabet, k)]
    out.append("".join("%f\t" % v for v in flat_t) + "%f\n" % likelihood)
    out.append("".join("%f\t" % v for row in event_model for v in row) + "\n")
    if hdp:
        out.append("".join("%f\t" % v for v in assignment_means) + "\n")
        out.append("".join("%s\t" % kmer_string(int(kid), alphabet, k) for kid in assignment_kmers) + "\n")
    else:
        out.append("".join("%f\t" % v for row in event_expectations for v in row) + "\n")
        out.append("".join("%f\t" % v for v in posteriors) + "\n")
        out.append("".join("%d\t" % int(v) for v in observed) + "\n")
    return "".join(out)
