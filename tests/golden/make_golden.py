"""Regenerate the golden fixtures in this directory from the signalAlign source tree.

Usage:  python tests/golden/make_golden.py /path/to/signalAlign
        (or with the tree's path in the SIGNALALIGN_SRC environment variable)

The fixtures hold only the inputs of the reference's own known-answer tests, cut down to what
those tests touch, so the test suite runs without the source tree:

* toy6.json  -- inputs of test_sm3_diagonalDPCalculations (tests/stateMachineTests.c:443-563):
  reference "ACGATAXGGACAT", 7 events, testModelR73_acegot_template.model entries for the
  k-mers the X expansions (CEO) reach.  Expected: 14 pairs at threshold 0.2, inside an 8-pair set.
* toy5.json  -- inputs of test_sm3_5merDiagonalDPCalculations (:565-692) with
  testModelR9_5mer_acgt_template.model.  Expected: 7 pairs.
* zymo.json  -- inputs of the unbanded half of test_stateMachine3_getAlignedPairsWithBanding
  (:823-851): tests/test_npReads/ZymoRef.txt, the template events and template scaling of
  tests/test_npReads/ZymoC_ch_1_file1.npRead, and the R7.3 ACEGOT template model entries for the
  k-mers of ZymoRef.  Expected: 1076 pairs.
* zymo_banded.json -- the anchors of the banded Zymo tests (getRemappedAnchors,
  tests/stateMachineTests.c:132-138): lastz (the reference's vendored copy, built by
  oracle/build_lastz.sh) on ZymoRef against the read's 2D sequence, through
  oracle/anchors.py's restatement of getBlastPairsForPairwiseAlignmentParameters, remapped by the
  template 2D event map and filtered; with the 2D sequence and the event map themselves, so the
  anchors can be regenerated from the fixture alone.  Expected counts (default parameters:
  diagonal expansion 20): 1076 pairs with the scaled and the descaled R7.3 machines
  (test_stateMachine3_getAlignedPairsWithBanding, :823-851, ragged ends); 1076 with every C of
  the reference replaced by C, E or O and 7349 with it replaced by X (CEO paths)
  (test_DegenerateNucleotides, :897-960, non-ragged ends); 1217 with the HDP machine at threshold
  0.1 on the read's events as nanopore_descaleNanoporeRead leaves them
  (test_sm3Hdp_getAlignedPairsWithBanding, :881-895).
* testModelR73_acegot_template.model.xz, testModelR9_5mer_acgt_template.model.xz,
  templateSingleLevelFixed.nhdp.xz -- the reference's model files (models/), compressed, byte for
  byte: the product's loaders are tested on them and the banded tests load their machines from
  them.
"""
import itertools
import json
import lzma
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def read_model(path):
    with open(path) as fh:
        l0, l1, l2 = fh.readline(), fh.readline(), fh.readline()
    return l0.split(), l1.split(), l2.split()


def kmer_id(kmer, alphabet):
    v = 0
    for ch in kmer:
        v = v * len(alphabet) + alphabet.index(ch)
    return v


def subset(model_path, kmers):
    tok0, tok1, vals = read_model(model_path)
    alpha = "".join(sorted(tok0[2]))
    table = {}
    for km in sorted(set(kmers)):
        i = kmer_id(km, alpha)
        table[km] = vals[5 * i:5 * i + 5]
    return dict(header=tok0, transitions=tok1, table=table)


def expand(seq, k, options):
    out = []
    for i in range(len(seq) - k + 1):
        km = seq[i:i + k]
        pos = [j for j, c in enumerate(km) if c == "X"]
        for pat in itertools.product(options, repeat=len(pos)):
            s = list(km)
            for j, c in zip(pos, pat):
                s[j] = c
            out.append("".join(s))
    return out


def main(src):
    models = os.path.join(src, "models")
    # toy 6-mer DP (stateMachineTests.c:443-563)
    seq6 = "ACGATAXGGACAT"
    ev6 = [[58.743435, 0.887833, 0.0571, 0.0], [53.604965, 0.816836, 0.0571, 0.1],
           [58.432015, 0.735143, 0.0571, 0.2], [63.684352, 0.795437, 0.0571, 0.3],
           [58.921430, 0.812959, 0.0571, 0.4], [59.895882, 0.740952, 0.0571, 0.5],
           [61.684303, 0.722332, 0.0571, 0.67]]
    toy6 = subset(os.path.join(models, "testModelR73_acegot_template.model"), expand(seq6, 6, "CEO"))
    toy6.update(sequence=seq6, events=ev6, threshold=0.2, expected_pairs=14,
                allowed=[[0, 0], [1, 1], [2, 2], [3, 3], [4, 3], [5, 4], [6, 5], [7, 6]],
                source="tests/stateMachineTests.c:443-563")
    # toy 5-mer DP (stateMachineTests.c:565-692)
    seq5 = "ACGATATGGACAT"
    ev5 = [[70.0423375640843, 2.1070814631739, 0.0571, 0.0], [73.7087073662952, 1.90162684687837, 0.0571, 0.1],
           [105.375581864011, 2.87252862011704, 0.0571, 0.2], [82.9620934477158, 2.38320603353748, 0.0571, 0.3],
           [84.6977645711335, 3.08486975249442, 0.0571, 0.4], [58.0551144225027, 2.52297561817531, 0.0571, 0.5],
           [94.337668063878, 1.9731952395105, 0.0571, 0.67]]
    toy5 = subset(os.path.join(models, "testModelR9_5mer_acgt_template.model"), expand(seq5, 5, "CEO"))
    toy5.update(sequence=seq5, events=ev5, threshold=0.2, expected_pairs=7,
                allowed=[[0, 0], [1, 1], [2, 2], [3, 3], [5, 4], [6, 5], [8, 6]],
                source="tests/stateMachineTests.c:565-692")
    # Zymo read, unbanded (stateMachineTests.c:823-851)
    with open(os.path.join(src, "tests", "test_npReads", "ZymoRef.txt")) as fh:
        zref = fh.readline().strip()
    with open(os.path.join(src, "tests", "test_npReads", "ZymoC_ch_1_file1.npRead")) as fh:
        lines = fh.read().split("\n")
    head = lines[0].split()
    n_t = int(head[1])
    ev = [float(v) for v in lines[7].split()]
    assert len(ev) == 4 * n_t
    zy = subset(os.path.join(models, "testModelR73_acegot_template.model"), expand(zref, 6, "CEO"))
    zy.update(sequence=zref, events=[ev[4 * i:4 * i + 4] for i in range(n_t)],
              template_params=dict(scale=float(head[5]), shift=float(head[6]), var=float(head[7]),
                                   scale_sd=float(head[8]), var_sd=float(head[9])),
              threshold=0.01, expected_pairs=1076, source="tests/stateMachineTests.c:823-851")
    # banded Zymo anchors (lastz must have been built: oracle/build_lastz.sh)
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import anchors as A
    npr = A.parse_np_read(os.path.join(src, "tests", "test_npReads", "ZymoC_ch_1_file1.npRead"))
    anchors = A.remapped_anchors(zref, npr["two_d_read"], npr["template_event_map"])
    banded = dict(anchors=[list(a) for a in anchors], two_d_read=npr["two_d_read"],
                  template_event_map=npr["template_event_map"], diagonal_expansion=20,
                  expected=dict(scaled=1076, descaled=1076, C=1076, E=1076, O=1076, X=7349, hdp_threshold_0_1=1217),
                  source="tests/stateMachineTests.c:132-138, :694-717, :823-895, :897-960")
    with open(os.path.join(HERE, "zymo_banded.json"), "w") as fh:
        json.dump(banded, fh, separators=(",", ":"))
    print("wrote zymo_banded", len(anchors), "anchors")
    for fn in ("testModelR73_acegot_template.model", "testModelR9_5mer_acgt_template.model",
               "templateSingleLevelFixed.nhdp"):
        with open(os.path.join(models, fn), "rb") as fh:
            data = fh.read()
        with open(os.path.join(HERE, fn + ".xz"), "wb") as fh:
            fh.write(lzma.compress(data, preset=9))
        print("wrote", fn + ".xz")
    for name, obj in (("toy6", toy6), ("toy5", toy5), ("zymo", zy)):
        with open(os.path.join(HERE, name + ".json"), "w") as fh:
            json.dump(obj, fh, separators=(",", ":"))
        print("wrote", name, len(obj["table"]), "k-mers")


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIGNALALIGN_SRC")
    if not src:
        sys.exit("usage: make_golden.py /path/to/signalAlign (or set SIGNALALIGN_SRC)")
    main(src)
