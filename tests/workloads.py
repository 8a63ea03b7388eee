"""Shared builders: the same synthetic model and reads for the oracle and for the GPU library."""
import numpy as np

from oracle import formats
from oracle import io as oio
from oracle import oracle as orc
from signalalign_b200 import synth


def gaussian_model(cfg):
    """The .model the synthetic config would be stored as, read back as the reference loader would."""
    text = synth.model_text(cfg["alphabet"], cfg["k"], cfg["table"])
    l0, l1, l2 = text.split("\n")[:3]
    return formats.parse_model_lines(l0, l1, l2)


def oracle_model(m, emission, read=None, hdp=None):
    scale, shift, var = (read["scale"], read["shift"], read.get("var", 1.0)) if read else (1.0, 0.0, 1.0)
    return orc.OracleModel(m, emission, scale, shift, var, hdp=hdp)


def gpu_model(api, m, emission, read=None, hdp=None):
    sm = api.StateMachine.from_tables(m["alphabet"], m["kmer_length"], m["t"], m["match"], m["gapy"], m["gapx"],
                                      emission=emission)
    if hdp is not None:
        sm.set_hdp(hdp["grid_start"], hdp["grid_stop"], hdp["grid_length"], hdp["density"], hdp["slope"],
                   hdp["kmer_row"])
    if read is not None:
        sm.set_scaling(read["scale"], read["shift"], read.get("var", 1.0))
    return sm


def hdp_dict(tables, n_kmers):
    """oracle/GPU HDP inputs from synth.hdp_tables: every k-mer observed with its own row."""
    return dict(grid_start=tables["grid_start"], grid_stop=tables["grid_stop"], grid_length=tables["grid_length"],
                grid=formats.linspace_ref(tables["grid_start"], tables["grid_stop"], tables["grid_length"]),
                density=tables["density"], slope=tables["slope"], kmer_row=np.arange(n_kmers, dtype=np.int64))


def small_hdp_config(seed=7, n_reads=3, span=(300, 900), grid_length=200):
    """A small HDP workload (4-mer ACGT) that the oracle finishes in well under a second."""
    alphabet, k = "ACGT", 4
    tables = synth.hdp_tables(alphabet, k, seed, grid_length=grid_length)
    n = len(alphabet) ** k
    r = np.random.Generator(np.random.PCG64(seed))
    table = np.zeros((n, 5))
    table[:, 0] = tables["mean"]
    table[:, 1] = tables["sd"]
    table[:, 2] = r.uniform(0.5, 2.0, n)
    table[:, 3] = 0.3 * table[:, 2]
    table[:, 4] = table[:, 2] ** 3 / table[:, 3] ** 2
    reads = []
    for _ in range(n_reads):
        L = int(r.integers(span[0], span[1] + 1))
        seq = synth.random_reference(L, r)
        reads.append(synth.make_read(seq, alphabet, k, table[:, 0], table[:, 1], table[:, 2], table[:, 3], r))
    return dict(alphabet=alphabet, k=k, table=table, hdp=tables, reads=reads)


def pair_map(pairs):
    return {(int(p["x"]), int(p["y"]), int(p["kmer"])): int(p["score"]) for p in pairs}


def max_posterior_error(a, b, threshold):
    """Largest |posterior difference| over the union of two pair sets; a pair missing on one side
    counts as posterior 0 there.  Returns (max error, pairs missing on either side whose present
    posterior is more than `slack` above the threshold)."""
    ma, mb = pair_map(a), pair_map(b)
    err = 0.0
    for key in set(ma) | set(mb):
        pa = ma.get(key, 0) / 1e7
        pb = mb.get(key, 0) / 1e7
        if key in ma and key in mb:
            err = max(err, abs(pa - pb))
        else:
            present = pa if key in ma else pb
            err = max(err, present - threshold)
    return err


def oracle_em_step(model, ex, emissions):
    """The oracle's maximisation step on a model dict: continuousPairHmm_normalize and both loads
    (emissions) or the transitions alone.  Returns (model, normalised transitions)."""
    em0 = np.asarray(model["match"], dtype=np.float64).reshape(-1, 5)
    if emissions:
        T, em = oio.normalize_expectations(ex["transitions"], ex["event_expectations"], ex["posteriors"],
                                           ex["observed"], em0)
    else:
        T, em = oio.normalize_transitions(ex["transitions"]), None
    t, match, gapy = oio.load_expectations(model["t"], model["match"], model["gapy"], T, em)
    return dict(model, t=t, match=match, gapy=gapy), T
