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


_unpacked = {}


def golden_file(name):
    """Path of a reference model file kept as `name`.xz in tests/golden, unpacked once per process
    into a temporary directory (the product's loaders read paths)."""
    if name not in _unpacked:
        import lzma
        import tempfile
        d = _unpacked.setdefault("_dir", tempfile.mkdtemp(prefix="sa_golden_"))
        path = os.path.join(d, name)
        with open(os.path.join(GOLDEN, name + ".xz"), "rb") as fh:
            data = lzma.decompress(fh.read())
        with open(path, "wb") as fh:
            fh.write(data)
        _unpacked[name] = path
    return _unpacked[name]


def descale_events_as_reference(events, scale, shift):
    """nanopore_descaleEvents (impl/nanopore.c:71-75) as nanopore_descaleNanoporeRead calls it: the
    loop steps through the flat (mean, noise, duration, start) array by 4 but stops at the event
    count, not at 4x the event count, so only the first ceil(n / 4) event means become
    (mean - shift) / scale.  The HDP banded known-answer test (tests/stateMachineTests.c:881-895)
    runs on the events as this leaves them."""
    ev = np.array(events, dtype=np.float64).reshape(-1, 4).copy()
    flat = ev.reshape(-1)
    for i in range(0, len(ev), 4):
        flat[i] = (flat[i] - shift) / scale
    return ev


def zymo_banded():
    """The banded Zymo known-answer case: reference, template events (as loaded, and as the HDP test
    descales them), lastz anchors, template scaling and the reference's expected pair counts."""
    zy = load_fixture("zymo")
    bd = load_fixture("zymo_banded")
    tp = zy["template_params"]
    events = np.array(zy["events"], dtype=np.float64)
    return dict(reference=zy["sequence"], events=events,
                hdp_events=descale_events_as_reference(events, tp["scale"], tp["shift"]),
                anchors=np.array(bd["anchors"], dtype=np.int64), template_params=tp,
                expansion=bd["diagonal_expansion"], expected=bd["expected"], two_d_read=bd["two_d_read"],
                template_event_map=bd["template_event_map"])
