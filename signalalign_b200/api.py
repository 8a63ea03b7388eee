"""Python mirror of signalAlign's alignment interface over the C ABI of libsa_b200.so.

Names follow the reference (getStateMachine3, getStateMachine3_descaled, getHdpStateMachine,
pairwiseAlignmentBandingParameters_construct, band_construct, getSplitPoints,
getAlignedPairsUsingAnchors); errors that the reference turns into an abort raise SAError here.
There is no CPU fallback: every alignment runs on the GPU through the library, and importing this
module fails if the library has not been built.
"""
import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsa_b200.so")
# launch configurations chosen by the tuner (python -m signalalign_b200.tune), read when the library loads
LAUNCH_CONFIGS = os.path.join(_HERE, "launch_configs.tsv")

THREE_STATE, THREE_STATE_HDP = 2, 7
EMIT_PLAIN, EMIT_DESCALED, EMIT_HDP = 0, 1, 2
CYTOSINE_METHYLATION2, CYTOSINE_METHYLATION3, ADENOSINE_METHYLATION, CANONICAL_VARIANTS = 0, 1, 2, 3
PAIR_ALIGNMENT_PROB_1 = 10000000

STATUS = {0: "ok", 1: "bad argument", 2: "k-mer character outside the model alphabet",
          3: "anchors not strictly increasing or outside the matrix", 4: "out of memory", 5: "CUDA error",
          6: "pair output buffer too small", 7: "unsupported state machine or input",
          8: "model file missing or malformed", 9: "device wait timed out", 10: "device consistency check failed",
          11: "request exceeds a fixed capacity"}


class SAError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = int(status)
        super().__init__("%s: %s (status %d)" % (where, STATUS.get(self.status, "unknown"), self.status))


class LaunchConfig(C.Structure):
    """sa_launch_config: launch choices of the batched FP32 kernels"""
    _fields_ = [("ctas_per_sm", C.c_int32), ("grid_per_region", C.c_int32), ("warp_windows", C.c_int32),
                ("emission_ctas_per_sm", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Params(C.Structure):
    _fields_ = [("threshold", C.c_double), ("min_diags_between_traceback", C.c_int64),
                ("traceback_diagonals", C.c_int64), ("diagonal_expansion", C.c_int64),
                ("constraint_diagonal_trim", C.c_int64), ("split_matrix_bigger_than_this", C.c_int64)]


class AlignedPair(C.Structure):
    _fields_ = [("score", C.c_int64), ("x", C.c_int64), ("y", C.c_int64), ("kmer", C.c_int64)]


PAIR_DTYPE = np.dtype([("score", np.int64), ("x", np.int64), ("y", np.int64), ("kmer", np.int64)])


class Read(C.Structure):
    _fields_ = [("sm", C.c_void_p), ("reference", C.c_char_p), ("reference_length", C.c_int64),
                ("events", C.POINTER(C.c_double)), ("n_events", C.c_int64),
                ("anchors", C.POINTER(C.c_int64)), ("n_anchors", C.c_int64),
                ("scale", C.c_double), ("shift", C.c_double), ("var", C.c_double),
                ("ragged_left", C.c_int32), ("ragged_right", C.c_int32), ("degenerate", C.c_int32),
                ("pad", C.c_int32)]


_lib = None
class CigarOp(C.Structure):
    _fields_ = [("op", C.c_int32), ("pad", C.c_int32), ("length", C.c_int64)]


class GuideAlignment(C.Structure):
    _fields_ = [("start1", C.c_int64), ("end1", C.c_int64), ("strand1", C.c_int32), ("pad1", C.c_int32),
                ("start2", C.c_int64), ("end2", C.c_int64), ("strand2", C.c_int32), ("pad2", C.c_int32)]


class ReadParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("scale", "shift", "var", "shift_sd", "scale_sd", "var_sd", "drift")]


class ParamRead(C.Structure):
    _fields_ = [("sm", C.c_void_p), ("read", C.c_char_p), ("read_length", C.c_int64),
                ("event_map", C.POINTER(C.c_int64)), ("events", C.POINTER(C.c_double)), ("n_events", C.c_int64)]


class Expectations(C.Structure):
    _fields_ = [("likelihood", C.c_double), ("transitions", C.c_double * 9),
                ("event_expectations", C.POINTER(C.c_double)), ("posteriors", C.POINTER(C.c_double)),
                ("observed", C.POINTER(C.c_uint8)), ("assignment_kmers", C.POINTER(C.c_int64)),
                ("assignment_events", C.POINTER(C.c_int64)), ("assignment_capacity", C.c_int64),
                ("n_assignments", C.c_int64)]


class OutputRead(C.Structure):
    _fields_ = [("read_label", C.c_char_p), ("contig", C.c_char_p), ("target", C.c_char_p), ("target_length", C.c_int64),
                ("strand", C.c_int32), ("forward", C.c_int32), ("event_offset", C.c_int64),
                ("reference_offset", C.c_int64), ("events", C.POINTER(C.c_double)), ("n_events", C.c_int64),
                ("scale", C.c_double), ("shift", C.c_double), ("var", C.c_double), ("scale_sd", C.c_double)]


CIGAR_MATCH, CIGAR_INDEL_X, CIGAR_INDEL_Y = 0, 1, 2
OUTPUT_FULL, OUTPUT_VARIANT_CALLER, OUTPUT_ASSIGNMENTS = 0, 1, 2
TEMPLATE, COMPLEMENT = 0, 1

_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)


def _bind(L):
    vp = C.c_void_p
    sig = {
        "sa_stateMachine_loadFromFile": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_int32, C.c_int32,
                                                   C.POINTER(vp)]),
        "sa_stateMachine_fromTables": (C.c_int, [C.c_int, C.c_int, C.c_char_p, C.c_int32, C.c_int32, _f64p, _f64p,
                                                 _f64p, _f64p, C.c_int32, C.POINTER(vp)]),
        "sa_stateMachine_setHdp": (C.c_int, [vp, C.c_double, C.c_double, C.c_int64, C.c_int64, _f64p, _f64p, _i64p]),
        "sa_stateMachine_setScaling": (C.c_int, [vp, C.c_double, C.c_double, C.c_double]),
        "sa_stateMachine_scaleModel": (C.c_int, [vp] + [C.c_double] * 5),
        "sa_stateMachine_scaleNoise": (C.c_int, [vp, C.c_double, C.c_double]),
        "sa_stateMachine_kmerLength": (C.c_int32, [vp]),
        "sa_stateMachine_numberOfKmers": (C.c_int64, [vp]),
        "sa_stateMachine_kmerString": (C.c_char_p, [vp, C.c_int64]),
        "sa_stateMachine_kmerId": (C.c_int64, [vp, C.c_char_p]),
        "sa_stateMachine_getTables": (C.c_int, [vp, _f64p, _f64p, _f64p, _f64p]),
        "sa_stateMachine_getHdpTables": (C.c_int, [vp, _i64p, _i64p, _f64p, _f64p, _f64p, _i64p]),
        "sa_stateMachine_destruct": (None, [vp]),
        "sa_params_default": (None, [C.POINTER(Params)]),
        "sa_band_construct": (C.c_int, [_i64p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _i64p, _i64p]),
        "sa_getSplitPoints": (C.c_int, [_i64p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int32, C.c_int32,
                                        _i64p, C.c_int64, _i64p]),
        "sa_getAlignedPairsUsingAnchors": (C.c_int, [vp, C.c_char_p, C.c_int64, C.c_int, _f64p, C.c_int64, _i64p,
                                                     C.c_int64, C.POINTER(Params), C.c_int32, C.c_int32,
                                                     C.POINTER(C.POINTER(AlignedPair)), _i64p, _f64p]),
        "sa_free_pairs": (None, [vp]),
        "sa_batch_create": (C.c_int, [C.POINTER(Read), C.c_int64, C.POINTER(Params), C.POINTER(vp)]),
        "sa_batch_upload": (C.c_int, [vp, vp]),
        "sa_batch_run": (C.c_int, [vp, vp]),
        "sa_batch_download": (C.c_int, [vp, vp]),
        "sa_align_batch": (C.c_int, [C.POINTER(Read), C.c_int64, C.POINTER(Params), vp, C.POINTER(vp)]),
        "sa_batch_read_status": (C.c_int, [vp, C.c_int64]),
        "sa_batch_pair_count": (C.c_int64, [vp, C.c_int64]),
        "sa_batch_pairs": (C.POINTER(AlignedPair), [vp, C.c_int64]),
        "sa_batch_log_likelihood": (C.c_double, [vp, C.c_int64]),
        "sa_batch_cells": (C.c_int64, [vp]),
        "sa_batch_regions": (C.c_int64, [vp]),
        "sa_batch_kernel_ms": (C.c_int, [vp, _f64p, _f64p, _f64p]),
        "sa_batch_transfer_bytes": (C.c_int, [vp, _i64p, _i64p]),
        "sa_batch_set_wait_limit": (C.c_int, [vp, C.c_int64]),
        "sa_setSegmentPolicy": (C.c_int, [C.c_int32, C.c_int32]),
        "sa_getSegmentPolicy": (C.c_int, [C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
        "sa_batch_segment_info": (C.c_int, [vp, _i64p, _i64p, _i64p, _f64p]),
        "sa_planForwardSegments": (C.c_int, [_i64p, C.c_int64, C.c_int64, C.c_int64, C.POINTER(Params), C.c_int32,
                                             C.c_int32, _i64p, C.c_int64, _i64p]),
        "sa_batch_set_stitch_tolerance": (C.c_int, [vp, C.c_double]),
        "sa_getLaunchConfig": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(LaunchConfig)]),
        "sa_setLaunchConfig": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(LaunchConfig)]),
        "sa_tuneLaunchConfig": (C.c_int, [vp, vp, C.c_int32, C.POINTER(LaunchConfig), _f64p, C.POINTER(C.c_int32)]),
        "sa_loadLaunchConfigs": (C.c_int, [C.c_char_p]),
        "sa_batch_destroy": (None, [vp]),
        "sa_align_batch_noalloc": (C.c_int, [C.POINTER(Read), C.c_int64, C.POINTER(Params), vp,
                                             C.POINTER(AlignedPair), C.c_int64, _i64p, C.POINTER(C.c_int32), _f64p,
                                             _i64p]),
        "sa_server_create": (C.c_int, [C.c_int32, C.c_int64, C.c_int32, C.POINTER(vp)]),
        "sa_server_submit": (C.c_int, [vp, C.POINTER(Read), C.POINTER(Params), _i64p]),
        "sa_server_wait": (C.c_int, [vp, C.c_int64, C.c_double]),
        "sa_server_result": (C.c_int, [vp, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.POINTER(AlignedPair)), _i64p,
                                       _f64p, _f64p]),
        "sa_server_release": (C.c_int, [vp, C.c_int64]),
        "sa_server_destroy": (None, [vp]),
        "sa_server_stats": (C.c_int, [vp, C.POINTER(ServerCounters)]),
        "sa_server_read_timing": (C.c_int, [vp, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "sa_server_batch_log": (C.c_int, [vp, C.POINTER(C.c_double), C.c_int64, _i64p]),
        "sa_filterToRemoveOverlap": (C.c_int, [_i64p, C.c_int64, _i64p, _i64p]),
        "sa_guideAlignmentToRebasedAnchorPairs": (C.c_int, [C.POINTER(GuideAlignment), C.POINTER(CigarOp), C.c_int64,
                                                            C.c_int64, _i64p, C.c_int64, _i64p]),
        "sa_getRemappedAnchorPairs": (C.c_int, [_i64p, C.c_int64, _i64p, C.c_int64, C.c_int64, _i64p, _i64p]),
        "sa_sortByXPlusYCoordinate": (None, [C.POINTER(AlignedPair), C.c_int64]),
        "sa_scoreByPosteriorProbabilityIgnoringGaps": (C.c_double, [C.POINTER(AlignedPair), C.c_int64]),
        "sa_formatAlignment": (C.c_int, [C.c_int, vp, C.POINTER(OutputRead), C.POINTER(AlignedPair), C.c_int64,
                                         C.POINTER(C.c_void_p), _i64p]),
        "sa_outputAlignment": (C.c_int, [C.c_int, C.c_char_p, vp, C.POINTER(OutputRead), C.POINTER(AlignedPair),
                                         C.c_int64]),
        "sa_free_text": (None, [C.c_void_p]),
        "sa_oneDAssignmentsFromRead": (C.c_int, [C.POINTER(ParamRead), _i64p, _f64p, C.c_int64, _i64p]),
        "sa_estimateNanoporeParams": (C.c_int, [C.POINTER(ParamRead), C.c_int64, C.POINTER(ReadParams),
                                                C.POINTER(C.c_int32), vp]),
        "sa_adjustEventsForDrift": (C.c_int, [_f64p, C.c_int64, C.c_double]),
        "sa_getExpectationsUsingAnchors": (C.c_int, [vp, C.c_char_p, C.c_int64, _f64p, C.c_int64, _i64p, C.c_int64,
                                                     C.POINTER(Params), C.c_int32, C.c_int32,
                                                     C.POINTER(Expectations)]),
        "sa_getExpectationsBatch": (C.c_int, [C.POINTER(Read), C.c_int64, C.POINTER(Params), C.POINTER(Expectations),
                                              C.POINTER(C.c_int32)]),
        "sa_normalizeExpectations": (C.c_int, [C.POINTER(Expectations), C.c_int64, _f64p]),
        "sa_stateMachine_loadExpectations": (C.c_int, [vp, _f64p, _f64p]),
        "sa_formatExpectations": (C.c_int, [vp, C.POINTER(Expectations), _f64p, _f64p, C.c_int64,
                                            C.POINTER(C.c_void_p), _i64p]),
        "sa_writeExpectations": (C.c_int, [C.c_char_p, vp, C.POINTER(Expectations), _f64p, _f64p, C.c_int64]),
        "sa_status_string": (C.c_char_p, [C.c_int]),
        "sa_kernel_launch_count": (C.c_int64, []),
        "sa_allocation_count": (C.c_int64, []),
        "sa_allocation_ms": (C.c_double, []),
        "sa_measure_fp32_peak": (C.c_int, [C.c_int32, _f64p]),
    }
    for name, (res, args) in sig.items():
        if not hasattr(L, name):
            continue
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


def lib():
    """The loaded C-ABI library.  Raises if it was not built: there is no fallback path."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libsa_b200.so is not built (run `python -m signalalign_b200.build` or "
                              "__graft_entry__.build())")
        _lib = _bind(C.CDLL(LIB_PATH))
        if os.path.exists(LAUNCH_CONFIGS):
            _check(_lib.sa_loadLaunchConfigs(LAUNCH_CONFIGS.encode()), "loadLaunchConfigs")
    return _lib


def _check(st, where):
    if st:
        raise SAError(st, where)


def _f64(a, cols=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if cols is not None:
        a = a.reshape(-1, cols)
    return a


def _anchors(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64).reshape(-1, 2))


def pairwiseAlignmentBandingParameters_construct(**overrides):
    """pairwiseAlignmentBandingParameters_construct (pairwiseAligner.c:1843-1856)."""
    p = Params()
    lib().sa_params_default(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


class StateMachine:
    """A 3-state signal state machine whose emission tables live on the GPU."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)

    @property
    def handle(self):
        return self._h

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.sa_stateMachine_destruct(self._h)
            self._h = C.c_void_p(0)

    @classmethod
    def load(cls, model_file, machine_type=THREE_STATE, emission=EMIT_DESCALED, nhdp_file=None,
             set_hdp_expected_values=True, device=0):
        h = C.c_void_p()
        st = lib().sa_stateMachine_loadFromFile(model_file.encode(), machine_type, emission,
                                                nhdp_file.encode() if nhdp_file else None,
                                                int(set_hdp_expected_values), device, C.byref(h))
        _check(st, "stateMachine3_loadFromFile(%s)" % model_file)
        sm = cls(h.value)
        sm.emission = emission
        return sm

    @classmethod
    def from_tables(cls, alphabet, kmer_length, transitions, match, gap_y, gap_x, emission=EMIT_DESCALED,
                    device=0):
        machine_type = THREE_STATE_HDP if emission == EMIT_HDP else THREE_STATE
        t = _f64(transitions)
        m, y, x = _f64(match, 5), _f64(gap_y, 5), _f64(gap_x)
        h = C.c_void_p()
        st = lib().sa_stateMachine_fromTables(machine_type, emission, alphabet.encode(), len(alphabet), kmer_length,
                                              t.ctypes.data_as(_f64p), m.ctypes.data_as(_f64p),
                                              y.ctypes.data_as(_f64p), x.ctypes.data_as(_f64p), device, C.byref(h))
        _check(st, "stateMachine_fromTables")
        sm = cls(h.value)
        sm.emission = emission
        return sm

    def set_hdp(self, grid_start, grid_stop, grid_length, density, slope, kmer_row):
        d, s = _f64(density, grid_length), _f64(slope, grid_length)
        r = np.ascontiguousarray(np.asarray(kmer_row, dtype=np.int64))
        st = lib().sa_stateMachine_setHdp(self._h, grid_start, grid_stop, grid_length, len(d),
                                          d.ctypes.data_as(_f64p), s.ctypes.data_as(_f64p), r.ctypes.data_as(_i64p))
        _check(st, "stateMachine_setHdp")

    def set_scaling(self, scale, shift, var):
        _check(lib().sa_stateMachine_setScaling(self._h, scale, shift, var), "stateMachine_setScaling")

    def scaleModel(self, scale, shift, var, scale_sd, var_sd):
        _check(lib().sa_stateMachine_scaleModel(self._h, scale, shift, var, scale_sd, var_sd), "scaleModel")

    def scaleNoise(self, scale_sd, var_sd):
        _check(lib().sa_stateMachine_scaleNoise(self._h, scale_sd, var_sd), "scaleNoise")

    @property
    def kmer_length(self):
        return lib().sa_stateMachine_kmerLength(self._h)

    @property
    def n_kmers(self):
        return lib().sa_stateMachine_numberOfKmers(self._h)

    def kmer_string(self, kmer_id):
        s = lib().sa_stateMachine_kmerString(self._h, int(kmer_id))
        return s.decode() if s is not None else None

    def kmer_id(self, kmer):
        return lib().sa_stateMachine_kmerId(self._h, kmer.encode())

    def tables(self):
        n = self.n_kmers
        m, y, x, t = np.zeros((n, 5)), np.zeros((n, 5)), np.zeros(n), np.zeros(9)
        _check(lib().sa_stateMachine_getTables(self._h, m.ctypes.data_as(_f64p), y.ctypes.data_as(_f64p),
                                               x.ctypes.data_as(_f64p), t.ctypes.data_as(_f64p)), "getTables")
        return dict(match=m, gapy=y, gapx=x, t=t)

    def hdp_tables(self):
        """the HDP grid, densities, slopes and k-mer rows as loaded (sa_stateMachine_getHdpTables)"""
        gl, nr = C.c_int64(0), C.c_int64(0)
        _check(lib().sa_stateMachine_getHdpTables(self._h, C.byref(gl), C.byref(nr), None, None, None, None),
               "getHdpTables")
        g, d, s = np.zeros(gl.value), np.zeros((nr.value, gl.value)), np.zeros((nr.value, gl.value))
        r = np.zeros(self.n_kmers, np.int64)
        _check(lib().sa_stateMachine_getHdpTables(self._h, C.byref(gl), C.byref(nr), g.ctypes.data_as(_f64p),
                                                  d.ctypes.data_as(_f64p), s.ctypes.data_as(_f64p),
                                                  r.ctypes.data_as(_i64p)), "getHdpTables")
        return dict(grid=g, density=d, slope=s, kmer_row=r)


def getStateMachine3(model_file, device=0):
    """getStateMachine3 (stateMachine.c:1645-1653): plain (not descaled) emissions."""
    return StateMachine.load(model_file, THREE_STATE, EMIT_PLAIN, device=device)


def getStateMachine3_descaled(model_file, scale, shift, var, scale_sd=1.0, var_sd=1.0, scale_noise=False, device=0):
    """getStateMachine3_descaled (stateMachine.c:1627-1643)."""
    sm = StateMachine.load(model_file, THREE_STATE, EMIT_DESCALED, device=device)
    sm.set_scaling(scale, shift, var)
    if scale_noise:
        sm.scaleNoise(scale_sd, var_sd)
    return sm


def getHdpStateMachine(nhdp_file, model_file, scale, shift, var, set_expected_values=True, device=0):
    """getHdpStateMachine (stateMachine.c:1655-1669), optionally followed by
    stateMachine3_setModelToHdpExpectedValues as signalMachine does (signalMachine.c:709-711)."""
    sm = StateMachine.load(model_file, THREE_STATE_HDP, EMIT_HDP, nhdp_file=nhdp_file,
                           set_hdp_expected_values=set_expected_values, device=device)
    sm.set_scaling(scale, shift, var)
    return sm


def band_construct(anchors, lX, lY, expansion):
    """band_construct (pairwiseAligner.c:131-182): (xmyL, xmyR) for xay = 0..lX+lY."""
    a = _anchors(anchors)
    L, R = np.zeros(lX + lY + 1, np.int64), np.zeros(lX + lY + 1, np.int64)
    _check(lib().sa_band_construct(a.ctypes.data_as(_i64p), len(a), lX, lY, expansion, L.ctypes.data_as(_i64p),
                                   R.ctypes.data_as(_i64p)), "band_construct")
    return L, R


def getSplitPoints(anchors, lX, lY, split_matrix_bigger_than_this, ragged_left, ragged_right):
    """getSplitPoints (pairwiseAligner.c:1730-1757): list of (x1, y1, x2, y2)."""
    a = _anchors(anchors)
    cap = len(a) + 2
    out = np.zeros((cap, 4), np.int64)
    n = C.c_int64(0)
    _check(lib().sa_getSplitPoints(a.ctypes.data_as(_i64p), len(a), lX, lY, split_matrix_bigger_than_this,
                                   int(ragged_left), int(ragged_right), out.ctypes.data_as(_i64p), cap, C.byref(n)),
           "getSplitPoints")
    return [tuple(int(v) for v in r) for r in out[:n.value]]


def getAlignedPairsUsingAnchors(sm, reference, events, anchors, p, ragged_left=True, ragged_right=True,
                                degenerate=CYTOSINE_METHYLATION3, as_tuples=False, with_log_likelihood=False):
    """getAlignedPairsUsingAnchors (pairwiseAligner.c:1871-1899) on the plain FP64 GPU form.

    Returns a structured array (score, x, y, kmer id) in the reference's emission order, or a list
    of (score, x, y, path k-mer string) tuples like the reference's stIntTuple list."""
    ev = _f64(events, 4)
    a = _anchors(anchors)
    out = C.POINTER(AlignedPair)()
    n = C.c_int64(0)
    ll = C.c_double(0)
    ref = reference.encode()
    st = lib().sa_getAlignedPairsUsingAnchors(sm.handle, ref, len(ref), degenerate, ev.ctypes.data_as(_f64p), len(ev),
                                              a.ctypes.data_as(_i64p), len(a), C.byref(p), int(ragged_left),
                                              int(ragged_right), C.byref(out), C.byref(n), C.byref(ll))
    _check(st, "getAlignedPairsUsingAnchors")
    try:
        arr = np.ctypeslib.as_array(C.cast(out, C.POINTER(C.c_int64)), shape=(n.value * 4,)).copy() \
            if n.value else np.zeros(0, np.int64)
    finally:
        lib().sa_free_pairs(C.cast(out, C.c_void_p))
    pairs = arr.view(PAIR_DTYPE).reshape(-1)
    if as_tuples:
        pairs = [(int(r["score"]), int(r["x"]), int(r["y"]), sm.kmer_string(r["kmer"])) for r in pairs]
    if with_log_likelihood:
        return pairs, ll.value
    return pairs


@dataclass
class ReadInput:
    """One read of a batch (the inputs of performSignalAlignment, signalMachine.c:333-354)."""
    sm: StateMachine
    reference: str
    events: np.ndarray
    anchors: np.ndarray
    scale: float = 1.0
    shift: float = 0.0
    var: float = 1.0
    ragged_left: bool = True
    ragged_right: bool = True
    degenerate: int = CYTOSINE_METHYLATION3


def _read_array(reads, keep):
    """sa_read array of ReadInputs; the numpy / bytes buffers it points into are appended to keep."""
    arr = (Read * len(reads))()
    for i, r in enumerate(reads):
        ev = _f64(r.events, 4)
        a = _anchors(r.anchors)
        ref = r.reference.encode()
        keep += [ev, a, ref]
        arr[i].sm = r.sm.handle.value
        arr[i].reference = ref
        arr[i].reference_length = len(ref)
        arr[i].events = ev.ctypes.data_as(_f64p)
        arr[i].n_events = len(ev)
        arr[i].anchors = a.ctypes.data_as(_i64p)
        arr[i].n_anchors = len(a)
        arr[i].scale, arr[i].shift, arr[i].var = r.scale, r.shift, r.var
        arr[i].ragged_left, arr[i].ragged_right = int(r.ragged_left), int(r.ragged_right)
        arr[i].degenerate = r.degenerate
    return arr


class Batch:
    """A planned batch on the device: upload / run / download, or all at once with align()."""

    def __init__(self, reads, p):
        self._keep = []
        arr = _read_array(reads, self._keep)
        self._reads = arr
        self.n = len(reads)
        self._sms = [r.sm for r in reads]
        h = C.c_void_p()
        _check(lib().sa_batch_create(arr, len(reads), C.byref(p), C.byref(h)), "batch_create")
        self._h = h
        self._keep = []   # the library copied the inputs

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.sa_batch_destroy(self._h)
            self._h = C.c_void_p(0)

    def upload(self, stream=None):
        _check(lib().sa_batch_upload(self._h, stream), "batch_upload")

    def run(self, stream=None):
        _check(lib().sa_batch_run(self._h, stream), "batch_run")

    def download(self, stream=None):
        _check(lib().sa_batch_download(self._h, stream), "batch_download")

    def set_wait_limit(self, cycles):
        """bound (SM clock cycles) of the worker kernel's device-side waits (sa_batch_set_wait_limit)"""
        _check(lib().sa_batch_set_wait_limit(self._h, int(cycles)), "batch_set_wait_limit")

    def set_stitch_tolerance(self, scale):
        """scale of the forward-segment stitch tolerance (negative: every stitch disagrees and every
        segmented read is re-run unsegmented at download)"""
        _check(lib().sa_batch_set_stitch_tolerance(self._h, float(scale)), "batch_set_stitch_tolerance")

    def segment_info(self):
        """dict: forward segments, stitches, reads re-run unsegmented, largest stitch deviation"""
        a, b, c, d = C.c_int64(0), C.c_int64(0), C.c_int64(0), C.c_double(0)
        _check(lib().sa_batch_segment_info(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)),
               "batch_segment_info")
        return dict(segments=a.value, stitches=b.value, redone=c.value, max_spread=d.value)

    @property
    def cells(self):
        return lib().sa_batch_cells(self._h)

    @property
    def regions(self):
        return lib().sa_batch_regions(self._h)

    def kernel_ms(self):
        """(emission, worker, gather) device milliseconds of the last run"""
        e, w, g = C.c_double(0), C.c_double(0), C.c_double(0)
        _check(lib().sa_batch_kernel_ms(self._h, C.byref(e), C.byref(w), C.byref(g)), "batch_kernel_ms")
        return e.value, w.value, g.value

    def transfer_bytes(self):
        h, d = C.c_int64(0), C.c_int64(0)
        _check(lib().sa_batch_transfer_bytes(self._h, C.byref(h), C.byref(d)), "batch_transfer_bytes")
        return h.value, d.value

    def status(self, i):
        return lib().sa_batch_read_status(self._h, i)

    def log_likelihood(self, i):
        return lib().sa_batch_log_likelihood(self._h, i)

    def pairs(self, i):
        n = lib().sa_batch_pair_count(self._h, i)
        if n <= 0:
            return np.zeros(0, PAIR_DTYPE)
        ptr = lib().sa_batch_pairs(self._h, i)
        arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int64)), shape=(n * 4,)).copy()
        return arr.view(PAIR_DTYPE).reshape(-1)


def align_batch(reads, p, stream=None):
    """Batched FP32 form: plan, upload, one persistent launch, download."""
    b = Batch(reads, p)
    b.upload(stream)
    b.run(stream)
    b.download(stream)
    return b


# size of the static device array behind sa_align_batch_noalloc (SA_NOALLOC_SCRATCH_BYTES)
NOALLOC_SCRATCH_BYTES = 64 << 20


class NoallocResult:
    """Host results of one sa_align_batch_noalloc call."""

    def __init__(self, pairs, offsets, status, loglik, scratch_bytes):
        self._pairs, self._off = pairs, offsets
        self._status, self._ll = status, loglik
        self.scratch_bytes = scratch_bytes

    def status(self, i):
        return int(self._status[i])

    def log_likelihood(self, i):
        return float(self._ll[i])

    def pairs(self, i):
        return self._pairs[self._off[i]:self._off[i + 1]].copy()


def align_batch_noalloc(reads, p, stream=None, pair_capacity=None):
    """Batched FP32 form without device allocation (sa_align_batch_noalloc).  The reads' state
    machines must already hold device tables (any earlier allocating alignment with them)."""
    keep = []
    arr = _read_array(reads, keep)
    n = len(reads)
    if pair_capacity is None:
        pair_capacity = sum(4 * (len(r.reference) + len(r.events)) + 256 for r in reads)
    for _ in range(2):
        pairs = np.zeros(max(pair_capacity, 1), PAIR_DTYPE)
        off = np.zeros(n + 1, np.int64)
        status = np.zeros(max(n, 1), np.int32)
        ll = np.zeros(max(n, 1), np.float64)
        need = C.c_int64(0)
        st = lib().sa_align_batch_noalloc(arr, n, C.byref(p), stream, pairs.ctypes.data_as(C.POINTER(AlignedPair)),
                                          pair_capacity, off.ctypes.data_as(_i64p),
                                          status.ctypes.data_as(C.POINTER(C.c_int32)), ll.ctypes.data_as(_f64p),
                                          C.byref(need))
        if st == 6 and off[n] > pair_capacity:   # SA_E_OUTPUT: size the pair array from pair_offsets
            pair_capacity = int(off[n])
            continue
        _check(st, "align_batch_noalloc")
        return NoallocResult(pairs, off, status, ll, need.value)
    raise SAError(6, "align_batch_noalloc")


class ServerCounters(C.Structure):
    _fields_ = [("reads_early", C.c_int64), ("reads_at_batch_end", C.c_int64), ("batches", C.c_int64),
                ("admit_ms", C.c_double), ("fetch_ms", C.c_double), ("finish_ms", C.c_double),
                ("plan_ms", C.c_double), ("upload_ms", C.c_double)]


class Server:
    """Continuous-batching serving loop (sa_server_*): submit reads as they arrive, wait for each."""

    def __init__(self, device=0, max_inflight_cells=200_000_000, max_batches=8):
        h = C.c_void_p()
        _check(lib().sa_server_create(device, max_inflight_cells, max_batches, C.byref(h)), "server_create")
        self._h = h

    def submit(self, read, p):
        keep = []
        arr = _read_array([read], keep)
        t = C.c_int64(0)
        _check(lib().sa_server_submit(self._h, arr, C.byref(p), C.byref(t)), "server_submit")
        return t.value

    def wait(self, ticket, timeout_ms=60000.0):
        _check(lib().sa_server_wait(self._h, ticket, timeout_ms), "server_wait")

    def result(self, ticket, release=True):
        """(status, pairs, log_likelihood, latency_ms) of a finished read"""
        st = C.c_int32(0)
        ptr = C.POINTER(AlignedPair)()
        n = C.c_int64(0)
        ll, lat = C.c_double(0), C.c_double(0)
        _check(lib().sa_server_result(self._h, ticket, C.byref(st), C.byref(ptr), C.byref(n), C.byref(ll),
                                      C.byref(lat)), "server_result")
        if n.value > 0:
            pairs = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int64)), shape=(n.value * 4,)).copy()
            pairs = pairs.view(PAIR_DTYPE).reshape(-1)
        else:
            pairs = np.zeros(0, PAIR_DTYPE)
        if release:
            lib().sa_server_release(self._h, ticket)
        return st.value, pairs, ll.value, lat.value

    def stats(self):
        """sa_server_counters as a dict: reads finished on publication / at their micro-batch's end,
        micro-batches, and the dispatcher's time admitting, fetching and finishing (ms)"""
        c = ServerCounters()
        _check(lib().sa_server_stats(self._h, C.byref(c)), "server_stats")
        return {f: getattr(c, f) for f, _ in ServerCounters._fields_}

    def timing(self, ticket):
        """(queue_ms, launch_ms) of a finished read not yet released"""
        q, l = C.c_double(0), C.c_double(0)
        _check(lib().sa_server_read_timing(self._h, ticket, C.byref(q), C.byref(l)), "server_read_timing")
        return q.value, l.value

    def release(self, ticket):
        _check(lib().sa_server_release(self._h, ticket), "server_release")

    def batch_log(self):
        """per finished micro-batch (start_ms, worker_end_ms, reads): device times from the server's
        creation, in finishing order"""
        n = C.c_int64(0)
        _check(lib().sa_server_batch_log(self._h, None, 0, C.byref(n)), "server_batch_log")
        out = np.zeros(3 * max(n.value, 1), np.float64)
        _check(lib().sa_server_batch_log(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), n.value, C.byref(n)),
               "server_batch_log")
        return [tuple(out[3 * i: 3 * i + 3]) for i in range(n.value)]

    def close(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.sa_server_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        self.close()


def allocation_count():
    """device and pinned-host allocations the library has made in this process (sa_allocation_count)"""
    return lib().sa_allocation_count()


def allocation_ms():
    """host time the library's device and pinned-host allocations took, in ms (sa_allocation_ms)"""
    return lib().sa_allocation_ms()


def set_segment_policy(segment_diags=0, warmup_diags=1024):
    """forward segments of later batches: segment_diags < 0 keeps regions whole, > 0 caps a segment's
    sweep, 0 picks the cap from the batch (sa_setSegmentPolicy)"""
    _check(lib().sa_setSegmentPolicy(int(segment_diags), int(warmup_diags)), "setSegmentPolicy")


def plan_forward_segments(anchors, lX, lY, p, segment_diags, warmup_diags=1024):
    """sa_planForwardSegments: (n, 6) int64 rows (region, first anti-diagonal, last, warm-up, first
    window, region's widest anti-diagonal) for one read, host only"""
    a = _anchors(anchors)
    cap = 4 + (lX + lY) // 64
    out = np.zeros((cap, 6), np.int64)
    n = C.c_int64(0)
    _check(lib().sa_planForwardSegments(a.ctypes.data_as(_i64p), len(a), lX, lY, C.byref(p), int(segment_diags),
                                        int(warmup_diags), out.ctypes.data_as(_i64p), cap, C.byref(n)),
           "planForwardSegments")
    return out[:n.value].copy()


def get_segment_policy():
    a, b = C.c_int32(0), C.c_int32(0)
    _check(lib().sa_getSegmentPolicy(C.byref(a), C.byref(b)), "getSegmentPolicy")
    return a.value, b.value


def get_launch_config(device=0, width_class=1):
    """the launch configuration sa_batch_run uses on `device` for a band-width class (1, 2, 4)"""
    c = LaunchConfig()
    _check(lib().sa_getLaunchConfig(device, width_class, C.byref(c)), "getLaunchConfig")
    return c.as_dict()


def set_launch_config(device, width_class, cfg):
    c = LaunchConfig(**cfg)
    _check(lib().sa_setLaunchConfig(device, width_class, C.byref(c)), "setLaunchConfig")


def tune_launch_config(batch, stream=None, repeats=3):
    """sa_tuneLaunchConfig on an uploaded Batch: (best configuration, its mean ms, candidates tried)"""
    c, ms, n = LaunchConfig(), C.c_double(0), C.c_int32(0)
    _check(lib().sa_tuneLaunchConfig(batch._h, stream, repeats, C.byref(c), C.byref(ms), C.byref(n)),
           "tuneLaunchConfig")
    return c.as_dict(), ms.value, n.value


def kernel_launch_count():
    return lib().sa_kernel_launch_count()


def measure_fp32_peak(device=0):
    """FP32 FMA issue rate of the device in TFLOP/s (probe kernel)."""
    v = C.c_double(0)
    _check(lib().sa_measure_fp32_peak(device, C.byref(v)), "measure_fp32_peak")
    return v.value


# ------------------------------------------------------------------------------------------------
# before the path: anchor pairs (signalMachine.c:615, :343-344)
# ------------------------------------------------------------------------------------------------
def filterToRemoveOverlap(pairs):
    """filterToRemoveOverlap (pairwiseAligner.c:1575-1616) on (x, y) pairs sorted by (x, y)."""
    a = _anchors(pairs)
    out = np.zeros((max(len(a), 1), 2), np.int64)
    n = C.c_int64(0)
    _check(lib().sa_filterToRemoveOverlap(a.ctypes.data_as(_i64p), len(a), out.ctypes.data_as(_i64p), C.byref(n)),
           "filterToRemoveOverlap")
    return [tuple(int(v) for v in r) for r in out[:n.value]]


def guideAlignmentToRebasedAnchorPairs(start1, end1, strand1, start2, end2, ops, trim, strand2=1):
    """signalUtils_guideAlignmentToRebasedAnchorPairs (signalMachineUtils.c:142-164).  ops: (op, length)
    cigar operations (CIGAR_MATCH / CIGAR_INDEL_X / CIGAR_INDEL_Y).  Returns (anchor pairs, rebased
    (start1, end1, strand1))."""
    ga = GuideAlignment(start1, end1, int(strand1), 0, start2, end2, int(strand2), 0)
    arr = (CigarOp * max(len(ops), 1))()
    for i, (op, length) in enumerate(ops):
        arr[i].op, arr[i].length = op, length
    cap = sum(l for o, l in ops if o == CIGAR_MATCH) + 1
    out = np.zeros((cap, 2), np.int64)
    n = C.c_int64(0)
    _check(lib().sa_guideAlignmentToRebasedAnchorPairs(C.byref(ga), arr, len(ops), trim, out.ctypes.data_as(_i64p),
                                                       cap, C.byref(n)), "guideAlignmentToRebasedAnchorPairs")
    return [tuple(int(v) for v in r) for r in out[:n.value]], (ga.start1, ga.end1, ga.strand1)


def getRemappedAnchorPairs(anchors, event_map, map_offset):
    """signalUtils_getRemappedAnchorPairs (signalMachineUtils.c:166-170)."""
    a = _anchors(anchors)
    em = np.ascontiguousarray(event_map, dtype=np.int64)
    out = np.zeros((max(len(a), 1), 2), np.int64)
    n = C.c_int64(0)
    _check(lib().sa_getRemappedAnchorPairs(a.ctypes.data_as(_i64p), len(a), em.ctypes.data_as(_i64p), len(em),
                                           map_offset, out.ctypes.data_as(_i64p), C.byref(n)), "getRemappedAnchorPairs")
    return [tuple(int(v) for v in r) for r in out[:n.value]]


# ------------------------------------------------------------------------------------------------
# after the path: ordering, score and posterior files (signalMachine.c:68-260, :715-728)
# ------------------------------------------------------------------------------------------------
def _pair_array(pairs):
    a = np.ascontiguousarray(np.asarray(pairs, dtype=PAIR_DTYPE) if not isinstance(pairs, np.ndarray) or
                             pairs.dtype != PAIR_DTYPE else pairs)
    return a


def sortByXPlusYCoordinate(pairs):
    """stList_sort(..., sortByXPlusYCoordinate2): ascending x + y (equal keys keep their order)."""
    a = _pair_array(pairs).copy()
    lib().sa_sortByXPlusYCoordinate(a.ctypes.data_as(C.POINTER(AlignedPair)), len(a))
    return a


def scoreByPosteriorProbabilityIgnoringGaps(pairs):
    a = _pair_array(pairs)
    return lib().sa_scoreByPosteriorProbabilityIgnoringGaps(a.ctypes.data_as(C.POINTER(AlignedPair)), len(a))


def _output_read(target, strand, forward, event_offset, reference_offset, events, scale, shift, var, scale_sd,
                 read_label, contig, keep):
    ev = _f64(events, 4)
    t = target.encode()
    lab, con = read_label.encode(), contig.encode()
    keep += [ev, t, lab, con]
    return OutputRead(lab, con, t, len(t), int(strand), int(forward), event_offset, reference_offset,
                      ev.ctypes.data_as(_f64p), len(ev), scale, shift, var, scale_sd)


def formatAlignment(fmt, sm, pairs, target, strand, forward, event_offset, reference_offset, events, scale=1.0,
                    shift=0.0, var=1.0, scale_sd=1.0, read_label="", contig=""):
    """The text outputAlignment (signalMachine.c:240-260) appends for one strand of one read."""
    keep = []
    rd = _output_read(target, strand, forward, event_offset, reference_offset, events, scale, shift, var, scale_sd,
                      read_label, contig, keep)
    a = _pair_array(pairs)
    text = C.c_void_p()
    n = C.c_int64(0)
    _check(lib().sa_formatAlignment(fmt, sm.handle, C.byref(rd), a.ctypes.data_as(C.POINTER(AlignedPair)), len(a),
                                    C.byref(text), C.byref(n)), "formatAlignment")
    try:
        return C.string_at(text, n.value).decode() if n.value else ""
    finally:
        lib().sa_free_text(text)


def outputAlignment(fmt, path, sm, pairs, target, strand, forward, event_offset, reference_offset, events, scale=1.0,
                    shift=0.0, var=1.0, scale_sd=1.0, read_label="", contig=""):
    """outputAlignment: the lines appended to the posterior file at `path`."""
    keep = []
    rd = _output_read(target, strand, forward, event_offset, reference_offset, events, scale, shift, var, scale_sd,
                      read_label, contig, keep)
    a = _pair_array(pairs)
    _check(lib().sa_outputAlignment(fmt, str(path).encode(), sm.handle, C.byref(rd),
                                    a.ctypes.data_as(C.POINTER(AlignedPair)), len(a)), "outputAlignment")


# ------------------------------------------------------------------------------------------------
# before the path: per-read scale / shift / drift / variance (signalMachineUtils.c:186-223)
# ------------------------------------------------------------------------------------------------
def _param_read(sm, read, event_map, events, keep):
    em = np.ascontiguousarray(event_map, dtype=np.int64)
    ev = _f64(events, 4)
    rb = read.encode()
    keep += [em, ev, rb]
    return ParamRead(sm.handle, rb, len(rb), em.ctypes.data_as(_i64p), ev.ctypes.data_as(_f64p), len(ev))


def oneDAssignmentsFromRead(sm, read, event_map, events):
    """nanopore_getOneDAssignmentsFromRead: (k-mer ids, [(mean, noise, delta time)])"""
    keep = []
    pr = _param_read(sm, read, event_map, events, keep)
    cap = max(len(read), 1)
    ids = np.zeros(cap, np.int64)
    ep = np.zeros((cap, 3), np.float64)
    n = C.c_int64(0)
    _check(lib().sa_oneDAssignmentsFromRead(C.byref(pr), ids.ctypes.data_as(_i64p), ep.ctypes.data_as(_f64p), cap,
                                            C.byref(n)), "oneDAssignmentsFromRead")
    return ids[:n.value], ep[:n.value]


def estimateNanoporeParams(items, stream=None):
    """Batched fits on the GPU.  items: [(sm, read, event_map, events, initial params dict)].
    Returns [(status, params dict)]."""
    keep = []
    arr = (ParamRead * max(len(items), 1))()
    prm = (ReadParams * max(len(items), 1))()
    for i, (sm, read, em, ev, init) in enumerate(items):
        arr[i] = _param_read(sm, read, em, ev, keep)
        for k, v in (init or {}).items():
            setattr(prm[i], k, v)
    status = (C.c_int32 * max(len(items), 1))()
    _check(lib().sa_estimateNanoporeParams(arr, len(items), prm, status, stream), "estimateNanoporeParams")
    names = [f[0] for f in ReadParams._fields_]
    return [(status[i], {k: getattr(prm[i], k) for k in names}) for i in range(len(items))]


def adjustEventsForDrift(events, drift):
    """nanopore_adjustEventsForDriftP on a copy of the event table"""
    ev = _f64(events, 4).copy()
    _check(lib().sa_adjustEventsForDrift(ev.ctypes.data_as(_f64p), len(ev), drift), "adjustEventsForDrift")
    return ev


# ------------------------------------------------------------------------------------------------
# EM expectations (getExpectationsUsingAnchors, pairwiseAligner.c:1983-2003)
# ------------------------------------------------------------------------------------------------
def getExpectationsUsingAnchors(sm, reference, events, anchors, p, ragged_left=True, ragged_right=True, state=None,
                                transition_pseudocount=0.001, emission_pseudocount=0.001):
    """Expectations of one read on the plain FP64 form, accumulated into `state` (a previous result)
    or into fresh accumulators with the given pseudocounts (hmmContinuous_getExpectationsHmm).
    Returns dict(likelihood, transitions (3x3), event_expectations (n_kmers x 2), posteriors,
    observed, assignments ((k-mer id, event index) rows, the HDP machine's))."""
    if state is None:
        state = makeExpectationsHmm(sm, transition_pseudocount, emission_pseudocount)
    ee = np.ascontiguousarray(state["event_expectations"], dtype=np.float64).copy()
    po = np.ascontiguousarray(state["posteriors"], dtype=np.float64).copy()
    ob = np.ascontiguousarray(state["observed"], dtype=np.uint8).copy()
    ex, _ = _expectations_struct(dict(state, event_expectations=ee, posteriors=po, observed=ob, assignments=None))
    cap = 4 * (len(reference) + len(events)) + 64
    ak = np.zeros(cap, np.int64)
    ae = np.zeros(cap, np.int64)
    ex.assignment_kmers = ak.ctypes.data_as(_i64p)
    ex.assignment_events = ae.ctypes.data_as(_i64p)
    ex.assignment_capacity = cap
    ev = _f64(events, 4)
    a = _anchors(anchors)
    ref = reference.encode()
    _check(lib().sa_getExpectationsUsingAnchors(sm.handle, ref, len(ref), ev.ctypes.data_as(_f64p), len(ev),
                                                a.ctypes.data_as(_i64p), len(a), C.byref(p), int(ragged_left),
                                                int(ragged_right), C.byref(ex)), "getExpectationsUsingAnchors")
    got = np.column_stack([ak[:ex.n_assignments], ae[:ex.n_assignments]])
    return dict(likelihood=ex.likelihood, transitions=np.array(list(ex.transitions)).reshape(3, 3),
                event_expectations=ee, posteriors=po, observed=ob,
                assignments=np.concatenate([np.asarray(state.get("assignments", np.zeros((0, 2), np.int64)),
                                                       dtype=np.int64).reshape(-1, 2), got]),
                event_model=state.get("event_model"))


def getExpectationsBatch(reads, p, states=None, transition_pseudocount=0.001, emission_pseudocount=0.001):
    """Expectations of many reads (ReadInputs) in one launch (sa_getExpectationsBatch), each read into
    its own accumulators (states[i], or fresh ones).  Returns (list of result dicts as
    getExpectationsUsingAnchors returns, list of per-read statuses)."""
    n = len(reads)
    if states is None:
        states = [makeExpectationsHmm(r.sm, transition_pseudocount, emission_pseudocount) for r in reads]
    keep = []
    arr = _read_array(reads, keep)
    exs = (Expectations * max(n, 1))()
    bufs = []
    for i, (r, st) in enumerate(zip(reads, states)):
        ee = np.ascontiguousarray(st["event_expectations"], dtype=np.float64).copy()
        po = np.ascontiguousarray(st["posteriors"], dtype=np.float64).copy()
        ob = np.ascontiguousarray(st["observed"], dtype=np.uint8).copy()
        ex, _ = _expectations_struct(dict(st, event_expectations=ee, posteriors=po, observed=ob, assignments=None))
        # assignment lists: the HDP machine's only
        cap = 4 * (len(r.reference) + len(r.events)) + 64 if getattr(r.sm, "emission", EMIT_HDP) == EMIT_HDP else 0
        ak, ae = np.zeros(max(cap, 1), np.int64), np.zeros(max(cap, 1), np.int64)
        ex.assignment_kmers, ex.assignment_events = ak.ctypes.data_as(_i64p), ae.ctypes.data_as(_i64p)
        ex.assignment_capacity = cap
        exs[i] = ex
        bufs.append((ee, po, ob, ak, ae))
    status = np.zeros(max(n, 1), np.int32)
    _check(lib().sa_getExpectationsBatch(arr, n, C.byref(p), exs, status.ctypes.data_as(C.POINTER(C.c_int32))),
           "getExpectationsBatch")
    out = []
    for i, st in enumerate(states):
        ee, po, ob, ak, ae = bufs[i]
        ex = exs[i]
        got = np.column_stack([ak[:min(ex.n_assignments, len(ak))], ae[:min(ex.n_assignments, len(ae))]])
        out.append(dict(likelihood=ex.likelihood, transitions=np.array(list(ex.transitions)).reshape(3, 3),
                        event_expectations=ee, posteriors=po, observed=ob,
                        assignments=np.concatenate([np.asarray(st.get("assignments", np.zeros((0, 2), np.int64)),
                                                               dtype=np.int64).reshape(-1, 2), got]),
                        event_model=st.get("event_model")))
    return out, [int(v) for v in status[:n]]


def makeExpectationsHmm(sm, transition_pseudocount=0.001, emission_pseudocount=0.001):
    """continuousPairHmm_makeExpectationsHmm / hdpHmm_makeExpectationsHmm (continuousHmm.c:201-212,
    :788-795): empty accumulators with the pseudocounts, and the machine's match table as the event
    model."""
    n = sm.n_kmers
    return dict(likelihood=0.0, transitions=np.full((3, 3), float(transition_pseudocount)),
                event_expectations=np.zeros((n, 2)), posteriors=np.full(n, float(emission_pseudocount)),
                observed=np.zeros(n, np.uint8), assignments=np.zeros((0, 2), np.int64),
                event_model=sm.tables()["match"])


def _expectations_struct(hmm):
    """sa_expectations over the arrays of an expectations dict; returns (struct, arrays to keep alive)"""
    ex = Expectations()
    ex.likelihood = hmm["likelihood"]
    for i, v in enumerate(np.asarray(hmm["transitions"], dtype=np.float64).reshape(-1)):
        ex.transitions[i] = v
    keep = []
    for name, field, dt, ct in (("event_expectations", "event_expectations", np.float64, C.c_double),
                                ("posteriors", "posteriors", np.float64, C.c_double),
                                ("observed", "observed", np.uint8, C.c_uint8)):
        if hmm.get(name) is not None:
            a = np.ascontiguousarray(hmm[name], dtype=dt)
            keep.append(a)
            setattr(ex, field, a.ctypes.data_as(C.POINTER(ct)))
    if hmm.get("assignments") is not None:
        asg = np.asarray(hmm["assignments"], dtype=np.int64).reshape(-1, 2)
        ak, ae = np.ascontiguousarray(asg[:, 0]), np.ascontiguousarray(asg[:, 1])
        keep += [ak, ae]
        ex.assignment_kmers, ex.assignment_events = ak.ctypes.data_as(_i64p), ae.ctypes.data_as(_i64p)
        ex.assignment_capacity = ex.n_assignments = len(asg)
    return ex, keep


def normalizeExpectations(hmm, transitions_only=False):
    """continuousPairHmm_normalize (continuousHmm.c:283-306), or hmmDiscrete_normalizeTransitions alone
    (discreteHmm.c:125-137, the HDP machine's step) with transitions_only: a new dict with normalised
    transitions and, for the Gaussian machine, the re-estimated event model."""
    out = dict(hmm)
    em = None if transitions_only else np.array(hmm["event_model"], dtype=np.float64).reshape(-1, 5)
    ex, keep = _expectations_struct(hmm)
    n = len(em) if em is not None else 0
    _check(lib().sa_normalizeExpectations(C.byref(ex), n, em.ctypes.data_as(_f64p) if em is not None else None),
           "normalizeExpectations")
    out["transitions"] = np.array(list(ex.transitions)).reshape(3, 3)
    if em is not None:
        out["event_model"] = em
    return out


def loadExpectationsIntoStateMachine(sm, hmm, emissions=True):
    """continuousPairHmm_loadTransitionsIntoStateMachine and, with emissions,
    continuousPairHmm_loadEmissionsIntoStateMachine (continuousHmm.c:321-352) from a normalised
    expectations dict."""
    t = np.ascontiguousarray(hmm["transitions"], dtype=np.float64).reshape(-1)
    em = np.ascontiguousarray(hmm["event_model"], dtype=np.float64).reshape(-1) if emissions else None
    _check(lib().sa_stateMachine_loadExpectations(sm.handle, t.ctypes.data_as(_f64p),
                                                  em.ctypes.data_as(_f64p) if em is not None else None),
           "loadExpectationsIntoStateMachine")


def formatExpectations(sm, hmm, events=None):
    """The text hmmContinuous_writeToFile (continuousHmm.c:872-884) writes for an expectations dict;
    events (rows of 4) give the HDP machine's assigned event means."""
    ex, keep = _expectations_struct(hmm)
    em = hmm.get("event_model")
    em = np.ascontiguousarray(em, dtype=np.float64) if em is not None else None
    ev = _f64(events, 4) if events is not None else np.zeros((0, 4))
    text = C.c_void_p()
    n = C.c_int64(0)
    _check(lib().sa_formatExpectations(sm.handle, C.byref(ex), em.ctypes.data_as(_f64p) if em is not None else None,
                                       ev.ctypes.data_as(_f64p), len(ev), C.byref(text), C.byref(n)),
           "formatExpectations")
    try:
        return C.string_at(text, n.value).decode() if n.value else ""
    finally:
        lib().sa_free_text(text)


def writeExpectations(path, sm, hmm, events=None):
    """hmmContinuous_writeToFile: the expectations file at `path` (replaced)."""
    ex, keep = _expectations_struct(hmm)
    em = hmm.get("event_model")
    em = np.ascontiguousarray(em, dtype=np.float64) if em is not None else None
    ev = _f64(events, 4) if events is not None else np.zeros((0, 4))
    _check(lib().sa_writeExpectations(str(path).encode(), sm.handle, C.byref(ex),
                                      em.ctypes.data_as(_f64p) if em is not None else None,
                                      ev.ctypes.data_as(_f64p), len(ev)), "writeExpectations")
