"""The batched FP32 form on reads at the long end of each configuration, against the FP64 oracle.

Long reads are where the FP32 form's lagged renormalisation and its refresh folds run the longest
chains (a 20 kb reference with ~32k events gives ~52k anti-diagonals and ~50 traceback windows),
so the accuracy bound is checked there, not only on short reads:

* config 1 shape: two reads of 18-20 kb (6-mer ACGT Gaussian table), >= 45k anti-diagonals each;
* config 2 shape: one HDP read of 12-15 kb (6-mer ACEGT, 2000-point grid);
* config 3 shape: one read of 28-30 kb, template and complement, all-C and all-E hypotheses
  (about 75k anti-diagonals per alignment),
all in one batch, so Gaussian and HDP machines and short and long chains share the launch.

Tolerances as in test_gpu_parity: posterior error <= 1e-4 absolute over the union of the pair sets
(a pair on one side only counts as its posterior minus the threshold), log-likelihood <= 1e-3
relative.  The oracle runs on the host threads, one alignment per thread.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import formats
from oracle import oracle as orc
from signalalign_b200 import synth
import workloads as W

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4
LL_REL_TOL = 1e-3


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from signalalign_b200 import api as a
    return a


def _params(api):
    return api.pairwiseAlignmentBandingParameters_construct(diagonal_expansion=50, threshold=0.01)


def _oracle_all(jobs):
    """jobs: (oracle model, alignment dict); returns (pairs, final total probability) per job"""
    p = orc.params(threshold=0.01, expansion=50)

    def one(job):
        om, a = job
        want, tps = orc.aligned_pairs(om, a["reference"], a["events"], a["anchors"], p, True, True,
                                      with_total_probs=True)
        n = len(a["reference"]) - 5 + len(a["events"])
        top = [v for d, v in tps if d == n]
        return want, (top[0] if top else None)

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        return list(ex.map(one, jobs))


def test_long_reads_all_configs_one_batch(api):
    # config 1 shape
    c1 = synth.config1(seed=21, n_reads=2, span=(18000, 20000))
    g1 = W.gaussian_model(c1)
    sm1 = W.gpu_model(api, g1, orc.EMIT_DESCALED)
    # config 2 shape
    c2 = synth.config2(seed=22, n_reads=1, span=(12000, 15000))
    hdp2 = W.hdp_dict(c2["hdp"], 5 ** 6)
    m2 = formats.parse_model_lines(*synth.model_text("ACEGT", 6, c2["table"]).split("\n")[:3])
    sm2 = W.gpu_model(api, m2, orc.EMIT_HDP, None, hdp2)
    # config 3 shape
    c3 = synth.config3(seed=23, n_reads=1, span=(28000, 30000), grid_length=2000)
    hdp3 = W.hdp_dict(c3["hdp"], 5 ** 6)
    gm3 = formats.parse_model_lines(*synth.model_text("ACEGT", 6, c3["gauss_table"]).split("\n")[:3])
    hm3 = formats.parse_model_lines(*synth.model_text("ACEGT", 6, c3["hdp_table"]).split("\n")[:3])
    sm3g = W.gpu_model(api, gm3, orc.EMIT_DESCALED)
    sm3h = W.gpu_model(api, hm3, orc.EMIT_HDP, None, hdp3)

    als, jobs = [], []
    for rd in c1["reads"]:
        als.append((sm1, rd))
        jobs.append((W.oracle_model(g1, orc.EMIT_DESCALED, rd), rd))
    for rd in c2["reads"]:
        als.append((sm2, rd))
        jobs.append((W.oracle_model(m2, orc.EMIT_HDP, rd, hdp2), rd))
    for a in c3["alignments"]:
        hd = a["model"] == "hdp"
        als.append((sm3h if hd else sm3g, a))
        jobs.append((W.oracle_model(hm3 if hd else gm3, orc.EMIT_HDP if hd else orc.EMIT_DESCALED, a,
                                    hdp3 if hd else None), a))
    n_anti = [len(a["reference"]) - 5 + len(a["events"]) for _, a in als]
    assert min(n_anti[:2]) >= 45000            # config-1 reads near the 20 kb end
    assert max(n_anti) >= 70000                # the 30 kb config-3 alignment

    inputs = [api.ReadInput(sm=sm, reference=a["reference"], events=a["events"], anchors=a["anchors"],
                            scale=a["scale"], shift=a["shift"], var=a.get("var", 1.0)) for sm, a in als]
    b = api.align_batch(inputs, _params(api))
    want = _oracle_all(jobs)
    for i, (w, top) in enumerate(want):
        assert b.status(i) == 0
        assert len(w) > 1000
        err = W.max_posterior_error(w, b.pairs(i), 0.01)
        assert err <= FP32_TOL, (i, n_anti[i], err)
        assert top is not None
        assert abs(b.log_likelihood(i) - top) <= LL_REL_TOL * abs(top), (i, b.log_likelihood(i), top)
