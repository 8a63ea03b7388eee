"""Readers for signalAlign's `.model` and `.nhdp` files and the host-side table transforms, as the
oracle sees them.

TEST INFRASTRUCTURE ONLY: these functions build the FP64 inputs of the CPU oracle.  The product
library has its own C++ readers (signalalign_b200/csrc/sa_model.cpp); tests compare the two.

Each function restates the reference routine it cites (paths inside the signalAlign tree).
"""
import math

import numpy as np

LOG_ZERO = -math.inf
MODEL_PARAMS = 5                       # inc/stateMachine.h:18
EXTRA_EVENT_NOISE_MULTIPLIER = 1.75    # inc/stateMachine.h:25
LOG_POINT_ONE = -2.3025850929940455    # stateMachine.c:1472-1474

# transition slot order shared with the C oracle (StateMachine3 fields, inc/stateMachine.h:153-163)
T_NAMES = ("MATCH_CONTINUE", "MATCH_FROM_GAP_X", "MATCH_FROM_GAP_Y", "GAP_OPEN_X", "GAP_OPEN_Y",
           "GAP_EXTEND_X", "GAP_EXTEND_Y", "GAP_SWITCH_TO_X", "GAP_SWITCH_TO_Y")


def sorted_alphabet(alphabet):
    """sequence_prepareAlphabet (pairwiseAligner.c:294-323): sorted copy, characters distinct."""
    if len(set(alphabet)) != len(alphabet):
        raise ValueError("Characters of alphabet must be distinct, got %r" % alphabet)
    return "".join(sorted(alphabet))


def nanopore_default_transitions():
    """stateMachine3_setTransitionsToNanoporeDefaults (stateMachine.c:1077-1088)."""
    return [-0.23552123624314988, -0.21880828092192281, -0.013406326748077823, -1.6269694202638481,
            -4.3187242127300092, -1.6269694202638481, -4.3187242127239411, LOG_ZERO, LOG_ZERO]


def _clog(v):
    """C's log(): log(0) = -inf, log(negative) = nan."""
    if v == 0.0:
        return LOG_ZERO
    if v < 0.0 or v != v:
        return math.nan
    return math.log(v)


def transitions_from_tokens(tokens):
    """stateMachine3_loadTransitionsFromFile (stateMachine.c:1090-1146).  Token 7 (gapY->gapX) goes to
    GAP_SWITCH_TO_Y, so GAP_SWITCH_TO_X keeps its nanopore default (LOG_ZERO)."""
    t = nanopore_default_transitions()
    v = [float(s) for s in tokens]
    t[0] = _clog(v[0])   # match->match
    t[3] = _clog(v[1])   # match->gapX
    t[4] = _clog(v[2])   # match->gapY
    t[1] = _clog(v[3])   # gapX->match
    t[5] = _clog(v[4])   # gapX->gapX
    t[2] = _clog(v[6])   # gapY->match
    t[8] = _clog(v[7])   # gapY->gapX, stored in SWITCH_TO_Y
    t[6] = _clog(v[8])   # gapY->gapY
    return t


def parse_model_lines(line0, line1, line2):
    """stateMachine3_loadFromFile (stateMachine.c:1328-1426) on the three text lines of a .model."""
    tok0 = line0.split()
    if len(tok0) != 4:
        raise ValueError("model line 0 needs 4 tokens, got %d" % len(tok0))
    state_number, alphabet_size, alphabet, k = int(tok0[0]), int(tok0[1]), tok0[2], int(tok0[3])
    if state_number != 3:
        raise ValueError("only 3-state models are supported, got %d" % state_number)
    if len(alphabet) != alphabet_size:
        raise ValueError("alphabet size mismatch")
    alpha = sorted_alphabet(alphabet)
    n = alphabet_size ** k
    tok1 = line1.split()
    if len(tok1) != state_number * state_number + 1:
        raise ValueError("transitions line needs %d tokens" % (state_number * state_number + 1))
    t = transitions_from_tokens(tok1)
    vals = np.array([float(s) for s in line2.split()], dtype=np.float64)
    if vals.size != n * MODEL_PARAMS:
        raise ValueError("emission line has %d values, want %d" % (vals.size, n * MODEL_PARAMS))
    match = vals.reshape(n, MODEL_PARAMS).copy()
    gapy = match.copy()
    gapy[:, 1] *= EXTRA_EVENT_NOISE_MULTIPLIER
    gapx = np.full(n, LOG_POINT_ONE)
    return dict(alphabet=alpha, alphabet_size=alphabet_size, kmer_length=k, n_kmers=n, t=t,
                match=match, gapy=gapy, gapx=gapx)


def load_model_file(path):
    with open(path) as fh:
        lines = [fh.readline() for _ in range(3)]
    return parse_model_lines(*lines)


def scale_model(model, scale, shift, var, scale_sd, var_sd):
    """emissions_signal_scaleModel (stateMachine.c:630-668), on copies of the tables."""
    m = dict(model)
    match, gapy = model["match"].copy(), model["gapy"].copy()
    match[:, 0] = match[:, 0] * scale + shift
    match[:, 1] = match[:, 1] * var
    gapy[:, 0] = gapy[:, 0] * scale + shift
    gapy[:, 1] = gapy[:, 1] * var
    match[:, 2] = match[:, 2] * scale_sd
    match[:, 4] = match[:, 4] * var_sd
    match[:, 3] = np.sqrt(np.power(match[:, 2], 3.0) / match[:, 4])
    gapy[:, 2] = gapy[:, 2] * scale_sd
    gapy[:, 4] = gapy[:, 4] * var_sd
    gapy[:, 3] = np.sqrt(np.power(gapy[:, 2], 3.0) / match[:, 4])
    m["match"], m["gapy"] = match, gapy
    return m


def scale_noise(model, scale_sd, var_sd):
    """emissions_signal_scaleNoise (stateMachine.c:607-628), on copies of the tables."""
    m = dict(model)
    match, gapy = model["match"].copy(), model["gapy"].copy()
    match[:, 2] *= scale_sd
    match[:, 4] *= var_sd
    match[:, 3] = np.sqrt(np.power(match[:, 2], 3.0) / match[:, 4])
    gapy[:, 2] *= scale_sd
    gapy[:, 4] *= var_sd
    gapy[:, 3] = np.sqrt(np.power(gapy[:, 2], 3.0) / match[:, 4])
    m["match"], m["gapy"] = match, gapy
    return m


def kmer_id(kmer, alphabet):
    """kmer_id (nanopore_hdp.c:360-393) over the sorted alphabet; raises on characters outside it."""
    a = len(alphabet)
    v = 0
    for ch in kmer:
        j = alphabet.find(ch)
        if j < 0:
            raise ValueError("K-mer contains character outside alphabet: %r" % kmer)
        v = v * a + j
    return v


def linspace_ref(start, stop, length):
    """linspace (hdp_math_utils.c:497-509): start + i*dx for i < n, last point exactly stop."""
    n = length - 1
    dx = (stop - start) / float(n)
    lin = np.empty(length, dtype=np.float64)
    lin[:n] = start + np.arange(n, dtype=np.float64) * dx
    lin[n] = stop
    return lin


def parse_nhdp(path):
    """deserialize_nhdp (nanopore_hdp.c:1071-1098) + deserialize_hdp (hdp.c:3047-3316), keeping what the
    density query needs: grid, per-DP posterior predictive and slopes, the observed marks
    (mark_observed_dps, hdp.c:1127-1155) and, per k-mer, the row of its nearest observed ancestor
    (dir_proc_density, hdp.c:2594-2597)."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    it = iter(lines)
    alphabet_size = int(next(it).split()[0])
    alphabet = next(it).split()[0][:alphabet_size]
    k = int(next(it).split()[0])
    splines_finalized = bool(int(next(it)))
    has_data = bool(int(next(it)))
    sample_gamma = bool(int(next(it)))
    num_dps = int(next(it))
    dp_ids = None
    if has_data:
        next(it)  # data values
        dp_ids = [int(s) for s in next(it).split()]
    next(it)  # base params
    g = next(it).split()
    grid_start, grid_stop, grid_length = float(g[0]), float(g[1]), int(g[2])
    next(it)  # gamma
    if sample_gamma:
        for _ in range(4):
            next(it)
    parent = np.full(num_dps, -1, dtype=np.int64)
    for i in range(num_dps):
        tok = next(it).split()
        if tok[0] != "-":
            parent[i] = int(tok[0])
    observed = np.zeros(num_dps, dtype=bool)
    density = {}
    slope = {}
    if has_data:
        for d in dp_ids:
            while d >= 0 and not observed[d]:
                observed[d] = True
                density[d] = np.zeros(grid_length)
                d = parent[d]
        for i in range(num_dps):
            tok = next(it).split()
            if tok:
                density[i] = np.array([float(s) for s in tok], dtype=np.float64)
    if splines_finalized:
        for i in range(num_dps):
            tok = next(it).split()
            if tok:
                slope[i] = np.array([float(s) for s in tok], dtype=np.float64)
    alpha = sorted_alphabet(alphabet)
    n_kmers = alphabet_size ** k
    rows = sorted(d for d in density if observed[d])
    row_of = {d: r for r, d in enumerate(rows)}
    kmer_row = np.full(n_kmers, -1, dtype=np.int64)
    for kid in range(min(n_kmers, num_dps)):
        d = kid
        while d >= 0 and not observed[d]:
            d = parent[d]
        if d >= 0:
            kmer_row[kid] = row_of[d]
    dens = np.stack([density[d] for d in rows]) if rows else np.zeros((0, grid_length))
    slp = np.stack([slope.get(d, np.zeros(grid_length)) for d in rows]) if rows else np.zeros((0, grid_length))
    return dict(alphabet=alpha, alphabet_size=alphabet_size, kmer_length=k, grid_start=grid_start,
                grid_stop=grid_stop, grid_length=grid_length, grid=linspace_ref(grid_start, grid_stop, grid_length),
                density=dens, slope=slp, kmer_row=kmer_row, observed=observed, parent=parent, rows=rows)


def hdp_expected_values(model, hdp):
    """stateMachine3_setModelToHdpExpectedValues (stateMachine.c:1163-1192) with dir_proc_expected_val /
    dir_proc_variance (hdp.c:2772-2800): observed k-mers get the HDP mean and sd in the match table."""
    m = dict(model)
    match = model["match"].copy()
    grid = hdp["grid"]
    dx = grid[1:] - grid[:-1]
    for kid in range(model["n_kmers"]):
        if not hdp["observed"][kid]:
            continue
        distr = hdp["density"][hdp["kmer_row"][kid]]
        ev = 0.0
        for i in range(1, len(grid)):
            ev += grid[i] * distr[i] * dx[i - 1]
        var = 0.0
        for i in range(1, len(grid)):
            dev = grid[i] - ev
            var += dev * dev * distr[i] * dx[i - 1]
        match[kid, 0] = ev
        match[kid, 1] = math.sqrt(var)
    m["match"] = match
    return m
