"""Builds full FP64 model dicts (oracle.formats layout) from the cut-down golden fixtures."""
import json
import os

import numpy as np

from oracle import formats

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_fixture(name):
    with open(os.path.join(GOLDEN, name + ".json")) as fh:
        return json.load(fh)


def model_from_fixture(fx):
    """Rebuild what stateMachine3_loadFromFile would hold, with NaN for k-mers the fixture omits."""
    head = fx["header"]
    asz, k = int(head[1]), int(head[3])
    alpha = formats.sorted_alphabet(head[2])
    n = asz ** k
    vals = np.full((n, 5), np.nan)
    for km, row in fx["table"].items():
        vals[formats.kmer_id(km, alpha)] = [float(v) for v in row]
    line2 = None
    m = dict(alphabet=alpha, alphabet_size=asz, kmer_length=k, n_kmers=n,
             t=formats.transitions_from_tokens(fx["transitions"]))
    m["match"] = vals
    gapy = vals.copy()
    gapy[:, 1] *= formats.EXTRA_EVENT_NOISE_MULTIPLIER
    m["gapy"] = gapy
    m["gapx"] = np.full(n, formats.LOG_POINT_ONE)
    del line2
    return m
