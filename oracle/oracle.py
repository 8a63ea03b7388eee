"""ctypes front end of the CPU oracle (oracle/sa_oracle.c).

TEST INFRASTRUCTURE ONLY: tests, the smoke check and the CPU-baseline leg of bench.py use this
module as the checker.  It is never on the product path.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

EMIT_PLAIN, EMIT_DESCALED, EMIT_HDP = 0, 1, 2

_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)


class _Model(C.Structure):
    _fields_ = [("emission", C.c_int32), ("alphabet_size", C.c_int32), ("kmer_length", C.c_int32),
                ("pad", C.c_int32), ("alphabet", C.c_char_p), ("n_kmers", C.c_int64), ("t", C.c_double * 9),
                ("match", _f64p), ("gapy", _f64p), ("gapx", _f64p),
                ("scale", C.c_double), ("shift", C.c_double), ("var", C.c_double),
                ("grid_length", C.c_int64), ("grid", _f64p), ("density", _f64p), ("slope", _f64p),
                ("kmer_row", _i64p)]


class _Params(C.Structure):
    _fields_ = [("threshold", C.c_double), ("min_diags_between_traceback", C.c_int64),
                ("traceback_diagonals", C.c_int64), ("diagonal_expansion", C.c_int64),
                ("split_matrix_bigger_than_this", C.c_int64)]


PAIR_DTYPE = np.dtype([("score", np.int64), ("x", np.int64), ("y", np.int64), ("kmer", np.int64)])


def build(force=False):
    """Compile liboracle.so with -O2 and no floating-point contraction (deterministic FP64)."""
    src = os.path.join(_HERE, "sa_oracle.c")
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src):
        return LIB_PATH
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=gnu11", "-Wall",
                           "-o", LIB_PATH, src, "-lm"])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_logAdd.restype = C.c_double
        L.orc_logAdd.argtypes = [C.c_double, C.c_double]
        L.orc_band.restype = C.c_int
        L.orc_band.argtypes = [_i64p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _i64p, _i64p]
        L.orc_split_points.restype = C.c_int64
        L.orc_split_points.argtypes = [_i64p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_int,
                                       _i64p, C.c_int64]
        L.orc_aligned_pairs.restype = C.c_int
        L.orc_aligned_pairs.argtypes = [C.POINTER(_Model), C.c_char_p, C.c_int64, _f64p, C.c_int64, _i64p,
                                        C.c_int64, C.POINTER(_Params), C.c_int, C.c_int, C.c_char_p,
                                        C.c_void_p, C.c_int64, _i64p, _f64p, C.c_int64, _i64p]
        L.orc_flat_start_forgetting.restype = C.c_int
        L.orc_flat_start_forgetting.argtypes = [C.POINTER(_Model), C.c_char_p, C.c_int64, _f64p, C.c_int64, _i64p,
                                                C.c_int64, C.c_int64, C.c_int, C.c_char_p, _i64p, C.c_int64,
                                                C.c_int64, C.c_double, _i64p]
        L.orc_full_matrix.restype = C.c_int
        L.orc_full_matrix.argtypes = [C.POINTER(_Model), C.c_char_p, C.c_int64, _f64p, C.c_int64, C.c_double,
                                      C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_void_p, C.c_int64, _i64p,
                                      _f64p, _f64p, _f64p]
        L.orc_expectations.restype = C.c_int
        L.orc_expectations.argtypes = [C.POINTER(_Model), C.c_char_p, C.c_int64, _f64p, C.c_int64, _i64p,
                                       C.c_int64, C.POINTER(_Params), C.c_int, C.c_int, _f64p, _f64p, _f64p, _f64p,
                                       C.POINTER(C.c_uint8), _i64p, _i64p, C.c_int64, _i64p]
        L.orc_emission.restype = C.c_double
        L.orc_emission.argtypes = [C.POINTER(_Model), C.c_int64, C.c_double, C.c_double, C.c_int]
        L.orc_log_gauss_pdf.restype = C.c_double
        L.orc_log_gauss_pdf.argtypes = [C.c_double] * 3
        L.orc_log_inv_gauss_pdf.restype = C.c_double
        L.orc_log_inv_gauss_pdf.argtypes = [C.c_double] * 3
        L.orc_kmer_index.restype = C.c_int64
        L.orc_kmer_index.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_int]
        L.orc_expand_kmer.restype = C.c_int64
        L.orc_expand_kmer.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_char_p, C.c_int64]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class OracleModel:
    """FP64 state machine for the oracle: a parsed .model dict (oracle.formats) plus emission kind,
    the per-read scale/shift/var and, for HDP, the parsed .nhdp dict."""

    def __init__(self, model, emission, scale=1.0, shift=0.0, var=1.0, hdp=None):
        self.model = model
        self.match = np.ascontiguousarray(model["match"], dtype=np.float64)
        self.gapy = np.ascontiguousarray(model["gapy"], dtype=np.float64)
        self.gapx = np.ascontiguousarray(model["gapx"], dtype=np.float64)
        self.alphabet = model["alphabet"].encode()
        s = _Model()
        s.emission = emission
        s.alphabet_size = model["alphabet_size"]
        s.kmer_length = model["kmer_length"]
        s.alphabet = self.alphabet
        s.n_kmers = model["n_kmers"]
        for i, v in enumerate(model["t"]):
            s.t[i] = v
        s.match, s.gapy, s.gapx = _p(self.match, C.c_double), _p(self.gapy, C.c_double), _p(self.gapx, C.c_double)
        s.scale, s.shift, s.var = scale, shift, var
        if hdp is not None:
            self.grid = np.ascontiguousarray(hdp["grid"], dtype=np.float64)
            self.density = np.ascontiguousarray(hdp["density"], dtype=np.float64)
            self.slope = np.ascontiguousarray(hdp["slope"], dtype=np.float64)
            self.kmer_row = np.ascontiguousarray(hdp["kmer_row"], dtype=np.int64)
            s.grid_length = len(self.grid)
            s.grid, s.density = _p(self.grid, C.c_double), _p(self.density, C.c_double)
            s.slope, s.kmer_row = _p(self.slope, C.c_double), _p(self.kmer_row, C.c_int64)
        self.s = s


def params(threshold=0.01, expansion=50, min_diags=1000, traceback=40, split=3000 * 3000):
    """PairwiseAlignmentParameters (inc/pairwiseAligner.h:123-134); library defaults at
    pairwiseAligner.c:1843-1856, signalMachine overrides expansion to 50 (signalMachine.c:397)."""
    return dict(threshold=threshold, diagonal_expansion=expansion, min_diags_between_traceback=min_diags,
                traceback_diagonals=traceback, split_matrix_bigger_than_this=split)


def _params_struct(p):
    s = _Params()
    s.threshold = p["threshold"]
    s.min_diags_between_traceback = p["min_diags_between_traceback"]
    s.traceback_diagonals = p["traceback_diagonals"]
    s.diagonal_expansion = p["diagonal_expansion"]
    s.split_matrix_bigger_than_this = p["split_matrix_bigger_than_this"]
    return s


class OracleError(RuntimeError):
    pass


def log_add(x, y):
    return lib().orc_logAdd(x, y)


def band(anchors, lX, lY, expansion):
    a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 2))
    n = lX + lY + 1
    L, R = np.zeros(n, np.int64), np.zeros(n, np.int64)
    rc = lib().orc_band(_p(a, C.c_int64), len(a), lX, lY, expansion, _p(L, C.c_int64), _p(R, C.c_int64))
    if rc:
        raise OracleError("orc_band rc=%d" % rc)
    return L, R


def split_points(anchors, lX, lY, limit, ragged_left, ragged_right):
    a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 2))
    out = np.zeros((len(a) + 2, 4), np.int64)
    n = lib().orc_split_points(_p(a, C.c_int64), len(a), lX, lY, limit, int(ragged_left), int(ragged_right),
                               _p(out, C.c_int64), len(out))
    if n < 0:
        raise OracleError("orc_split_points rc=%d" % -n)
    return [tuple(int(v) for v in r) for r in out[:n]]


def aligned_pairs(om, ref, events, anchors, p, ragged_left=True, ragged_right=True, options="CEO",
                  max_pairs=None, with_total_probs=False):
    """getAlignedPairsUsingAnchors (pairwiseAligner.c:1871-1899) on the oracle.  ref: nucleotide string;
    events: (lY, 4) float64; anchors: (n, 2) int64.  Returns a structured array of pairs
    (score, x, y, kmer id) in the reference's emission order (and the refresh total probabilities)."""
    k = om.model["kmer_length"]
    lX = max(len(ref) - (k - 1), 0) if len(ref) > 0 else 0
    ev = np.ascontiguousarray(np.asarray(events, dtype=np.float64).reshape(-1, 4))
    a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 2))
    cap = max_pairs or (8 * (lX + len(ev)) + 64)
    out = np.zeros(cap, PAIR_DTYPE)
    n_out = C.c_int64(0)
    tp = np.zeros((max(1, (lX + len(ev)) // 5 + 64), 2), np.float64)
    n_tp = C.c_int64(0)
    ps = _params_struct(p)
    rc = lib().orc_aligned_pairs(C.byref(om.s), ref.encode(), lX, _p(ev, C.c_double), len(ev), _p(a, C.c_int64),
                                 len(a), C.byref(ps), int(ragged_left), int(ragged_right), options.encode(),
                                 out.ctypes.data, cap, C.byref(n_out), _p(tp, C.c_double), len(tp), C.byref(n_tp))
    if rc:
        raise OracleError("orc_aligned_pairs rc=%d" % rc)
    pairs = out[:n_out.value].copy()
    if with_total_probs:
        return pairs, tp[:n_tp.value].copy()
    return pairs


def expectations(om, ref, events, anchors, p, ragged_left=True, ragged_right=True, transition_pseudocount=0.001,
                 emission_pseudocount=0.001, state=None):
    """getExpectationsUsingAnchors (pairwiseAligner.c:1983-2003) with diagonalCalculation_Expectations
    into a continuous pair HMM (continuousPairHmm_construct's pseudocounts, continuousHmm.c:84-141).
    state: a previous result to accumulate into.  Returns dict(likelihood, transitions (3x3),
    event_expectations (n_kmers x 2), posteriors (n_kmers), observed (n_kmers), assignments ((k-mer id,
    event index) rows: the HDP machine's instead of the emission expectations,
    cell_signal_updateExpectationsAndAssignments, pairwiseAligner.c:795-817))."""
    k = om.model["kmer_length"]
    n = om.model["n_kmers"]
    lX = max(len(ref) - (k - 1), 0) if len(ref) > 0 else 0
    ev = np.ascontiguousarray(np.asarray(events, dtype=np.float64).reshape(-1, 4))
    a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 2))
    if state is None:
        state = dict(likelihood=0.0, transitions=np.full((3, 3), transition_pseudocount),
                     event_expectations=np.zeros((n, 2)), posteriors=np.full(n, emission_pseudocount),
                     observed=np.zeros(n, np.uint8), assignments=np.zeros((0, 2), np.int64))
    st = {key: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for key, v in state.items()}
    cap = len(st["assignments"]) + 4 * (lX + len(ev)) + 64
    ak = np.zeros(cap, np.int64)
    ae = np.zeros(cap, np.int64)
    ak[:len(st["assignments"])] = st["assignments"][:, 0]
    ae[:len(st["assignments"])] = st["assignments"][:, 1]
    na = C.c_int64(len(st["assignments"]))
    ll = np.array([st["likelihood"]], np.float64)
    tr = np.ascontiguousarray(st["transitions"], dtype=np.float64)
    ee = np.ascontiguousarray(st["event_expectations"], dtype=np.float64)
    po = np.ascontiguousarray(st["posteriors"], dtype=np.float64)
    ob = np.ascontiguousarray(st["observed"], dtype=np.uint8)
    ps = _params_struct(p)
    rc = lib().orc_expectations(C.byref(om.s), ref.encode(), lX, _p(ev, C.c_double), len(ev), _p(a, C.c_int64), len(a),
                                C.byref(ps), int(ragged_left), int(ragged_right), _p(ll, C.c_double),
                                _p(tr, C.c_double), _p(ee, C.c_double), _p(po, C.c_double), _p(ob, C.c_uint8),
                                _p(ak, C.c_int64), _p(ae, C.c_int64), cap, C.byref(na))
    if rc:
        raise OracleError("orc_expectations rc=%d" % rc)
    if na.value > cap:
        raise OracleError("orc_expectations: assignment capacity")
    return dict(likelihood=float(ll[0]), transitions=tr, event_expectations=ee, posteriors=po, observed=ob,
                assignments=np.column_stack([ak[:na.value], ae[:na.value]]))


def full_matrix(om, ref, events, threshold, ragged_left=False, ragged_right=False, options="CEO", p_mode=0):
    """getAlignedPairsWithoutBanding (pairwiseAligner.c:1923-1981) (p_mode 0) or the toy DP of
    stateMachineTests.c:443-563 (p_mode 1).  Returns (pairs, forward total, backward total,
    per-diagonal total probabilities)."""
    k = om.model["kmer_length"]
    lX = len(ref) - (k - 1)
    ev = np.ascontiguousarray(np.asarray(events, dtype=np.float64).reshape(-1, 4))
    cap = 16 * (lX + len(ev)) + 64
    out = np.zeros(cap, PAIR_DTYPE)
    n_out = C.c_int64(0)
    tf, tb = C.c_double(0), C.c_double(0)
    diag = np.zeros(lX + len(ev) + 1, np.float64)
    rc = lib().orc_full_matrix(C.byref(om.s), ref.encode(), lX, _p(ev, C.c_double), len(ev), threshold,
                               int(ragged_left), int(ragged_right), options.encode(), p_mode, out.ctypes.data, cap,
                               C.byref(n_out), C.byref(tf), C.byref(tb), _p(diag, C.c_double))
    if rc:
        raise OracleError("orc_full_matrix rc=%d" % rc)
    return out[:n_out.value].copy(), tf.value, tb.value, diag


def emission(om, kmer_id, mean, noise, match=True):
    return lib().orc_emission(C.byref(om.s), kmer_id, mean, noise, int(match))


def log_gauss_pdf(x, mu, sigma):
    return lib().orc_log_gauss_pdf(x, mu, sigma)


def log_inv_gauss_pdf(x, mu, lam):
    return lib().orc_log_inv_gauss_pdf(x, mu, lam)


def kmer_index(kmer, alphabet):
    return lib().orc_kmer_index(kmer.encode(), len(kmer), alphabet.encode(), len(alphabet))


def expand_kmer(kmer, options, max_paths=100000):
    buf = C.create_string_buffer(max_paths * len(kmer))
    n = lib().orc_expand_kmer(kmer.encode(), len(kmer), options.encode(), buf, max_paths)
    raw = buf.raw
    return [raw[i * len(kmer):(i + 1) * len(kmer)].decode() for i in range(n)]


def flat_start_forgetting(om, ref, events, anchors, starts, expansion=50, horizon=4000, tol=1e-9, ragged_left=True,
                          options="CEO"):
    """orc_flat_start_forgetting: per start, the anti-diagonals after which a forward sweep begun
    there from a flat vector equals the true forward sweep minus one constant (within tol), or -1"""
    k = om.model["kmer_length"]
    lX = max(len(ref) - (k - 1), 0)
    ev = np.ascontiguousarray(np.asarray(events, dtype=np.float64).reshape(-1, 4))
    a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 2))
    st = np.ascontiguousarray(np.asarray(starts, dtype=np.int64))
    out = np.zeros(len(st), np.int64)
    rc = lib().orc_flat_start_forgetting(C.byref(om.s), ref.encode(), lX, _p(ev, C.c_double), len(ev),
                                         _p(a, C.c_int64), len(a), expansion, int(ragged_left), options.encode(),
                                         _p(st, C.c_int64), len(st), horizon, tol, _p(out, C.c_int64))
    if rc:
        raise OracleError("orc_flat_start_forgetting rc=%d" % rc)
    return out

