"""sa_align_batch_noalloc: the batched FP32 form with its device buffers in one static device array.

Collected last (file name) so that it also runs after every other test has used the library; it
needs nothing they leave behind.  The GPU test compares two calls in a row with sa_align_batch on
the same reads, at the FP32 form's tolerance (posterior error <= 1e-4, log-likelihood 1e-3
relative).  The CPU tests cover the checks made before any device work.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import oracle as orc
from signalalign_b200 import api, synth
import workloads as W

FP32_TOL = 1e-4
HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "sa_b200.h")


def _inputs(sm, reads):
    return [api.ReadInput(sm=sm, reference=rd["reference"], events=rd["events"], anchors=rd["anchors"],
                          scale=rd["scale"], shift=rd["shift"], var=rd.get("var", 1.0)) for rd in reads]


def _params(expansion=50, threshold=0.01):
    p = api.pairwiseAlignmentBandingParameters_construct()
    p.diagonal_expansion = expansion
    p.threshold = threshold
    return p


def test_scratch_size_matches_header():
    text = open(HEADER).read()
    m = re.search(r"#define\s+SA_NOALLOC_SCRATCH_BYTES\s+\((\d+)ll\s*<<\s*(\d+)\)", text)
    assert m, "SA_NOALLOC_SCRATCH_BYTES not found"
    assert int(m.group(1)) << int(m.group(2)) == api.NOALLOC_SCRATCH_BYTES


def test_rejects_batch_larger_than_scratch():
    """two 15 kb reads need more than the scratch array: SA_E_CAPACITY before any device work, with
    the bytes needed reported"""
    cfg = synth.config1(seed=21, n_reads=2, span=(15000, 15000))
    sm = W.gpu_model(api, W.gaussian_model(cfg), orc.EMIT_DESCALED)
    with pytest.raises(api.SAError) as ei:
        api.align_batch_noalloc(_inputs(sm, cfg["reads"]), _params())
    assert ei.value.status == 11   # SA_E_CAPACITY
    keep = []
    arr = api._read_array(_inputs(sm, cfg["reads"]), keep)
    off = np.zeros(3, np.int64)
    status = np.zeros(2, np.int32)
    need = C.c_int64(0)
    p = _params()
    st = api.lib().sa_align_batch_noalloc(arr, 2, C.byref(p), None, None, 0, off.ctypes.data_as(api._i64p),
                                          status.ctypes.data_as(C.POINTER(C.c_int32)), None, C.byref(need))
    assert st == 11
    assert need.value > api.NOALLOC_SCRATCH_BYTES


def test_requires_resident_device_tables():
    """a machine that no allocating call has used yet has no device tables: SA_E_ARG, and the scratch
    size is still reported (a small read fits)"""
    cfg = synth.config0()
    sm = W.gpu_model(api, W.gaussian_model(cfg), orc.EMIT_DESCALED)
    keep = []
    arr = api._read_array(_inputs(sm, cfg["reads"]), keep)
    off = np.zeros(2, np.int64)
    status = np.zeros(1, np.int32)
    need = C.c_int64(0)
    p = _params()
    st = api.lib().sa_align_batch_noalloc(arr, 1, C.byref(p), None, None, 0, off.ctypes.data_as(api._i64p),
                                          status.ctypes.data_as(C.POINTER(C.c_int32)), None, C.byref(need))
    assert st == 1   # SA_E_ARG
    assert 0 < need.value <= api.NOALLOC_SCRATCH_BYTES


@pytest.mark.gpu
def test_noalloc_matches_align_batch_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cfg0 = synth.config0()
    cfg1 = synth.config1(seed=12, n_reads=5, span=(300, 1500))
    sm = W.gpu_model(api, W.gaussian_model(cfg1), orc.EMIT_DESCALED)
    reads = cfg0["reads"] + cfg1["reads"]
    inputs = _inputs(sm, reads)
    p = _params()
    ref = api.align_batch(inputs, p)         # allocating entry point; also makes the tables resident
    allocations = api.allocation_count()
    for call in range(2):
        got = api.align_batch_noalloc(inputs, p)
        assert api.allocation_count() == allocations    # no cudaMalloc / cudaHostAlloc on this path
        assert 0 < got.scratch_bytes <= api.NOALLOC_SCRATCH_BYTES
        for i in range(len(reads)):
            assert got.status(i) == 0 and ref.status(i) == 0
            want_pairs, got_pairs = ref.pairs(i), got.pairs(i)
            assert len(want_pairs) > 0
            err = W.max_posterior_error(want_pairs, got_pairs, p.threshold)
            assert err <= FP32_TOL, (call, i, err)
            ll_w, ll_g = ref.log_likelihood(i), got.log_likelihood(i)
            assert abs(ll_g - ll_w) <= 1e-3 * abs(ll_w), (call, i, ll_w, ll_g)


@pytest.mark.gpu
def test_noalloc_leaves_plain_form_reads_unsupported():
    """Reads only the plain FP64 form runs get SA_E_UNSUPPORTED from the no-allocation entry (it
    allocates nothing for that form): a reference with an 'X' position, and a read of a machine
    whose gap-Y table no longer follows its match table (after the EM emission load).  The other
    reads of the call are aligned as sa_align_batch aligns them."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cfg = synth.config1(seed=13, n_reads=3, span=(300, 900))
    m = W.gaussian_model(cfg)
    sm = W.gpu_model(api, m, orc.EMIT_DESCALED)
    em_sm = W.gpu_model(api, m, orc.EMIT_DESCALED)
    table = em_sm.tables()
    api.loadExpectationsIntoStateMachine(em_sm, dict(transitions=np.full((3, 3), 1.0 / 3.0),
                                                     event_model=table["match"]))
    reads = _inputs(sm, cfg["reads"])
    rd = cfg["reads"][1]
    reads[1] = api.ReadInput(sm=sm, reference=rd["reference"][:50] + "X" + rd["reference"][51:], events=rd["events"],
                             anchors=rd["anchors"], scale=rd["scale"], shift=rd["shift"],
                             degenerate=api.CANONICAL_VARIANTS)   # X -> A, C, G, T: four paths
    reads[2] = _inputs(em_sm, [cfg["reads"][2]])[0]
    p = _params()
    ref = api.align_batch(reads, p)          # allocating: every read runs; tables resident
    got = api.align_batch_noalloc(reads, p)
    assert [got.status(i) for i in range(3)] == [0, 7, 7]
    assert ref.status(1) == 0 and ref.status(2) == 0 and len(ref.pairs(2)) > 0
    err = W.max_posterior_error(ref.pairs(0), got.pairs(0), p.threshold)
    assert err <= FP32_TOL
