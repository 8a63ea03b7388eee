"""Test infrastructure: the lastz anchoring of signalAlign's known-answer tests, restated.

The reference's banded known-answer tests (tests/stateMachineTests.c:694-717, :823-960) take their
anchors from lastz through getBlastPairsForPairwiseAlignmentParameters and getRemappedAnchors.  This
module restates that pipeline so the anchors can be regenerated here (tests/golden/make_golden.py)
and committed as fixtures; the product never anchors reads itself (its inputs are anchor pairs).

* lastz itself is the reference's vendored copy (externalTools/lastz-distrib-1.03.54, installed as
  cPecanLastz by externalTools/Makefile:4-7), built from its own sources by oracle/build_lastz.sh
  into oracle/_ref/cPecanLastz and run with the reference's exact arguments
  (impl/pairwiseAligner.c:1509-1521).
* sonLib's cigarRead (un-vendored submodule) is restated from the format lastz writes
  (README.lastz.html, "CIGAR": `cigar: <query> <qstart> <qend> <qstrand> <target> <tstart> <tend>
  <tstrand> <score> <op> <len> ...`, zero-based half-open starts).  The reference asserts that the
  record's first sequence (sonLib's contig1) is the target "a" and its second the query "b"
  (pairwiseAligner.c:1529-1530), so the query fields are sequence 2.  M advances both sequences,
  D (target base not in the query) advances sequence 1 only (PAIRWISE_INDEL_X), I advances
  sequence 2 only (PAIRWISE_INDEL_Y); the restatement checks that the operations end exactly at
  both end coordinates, which is what convertPairwiseForwardStrandAlignmentToAnchorPairs asserts
  (pairwiseAligner.c:1475-1476).
"""
import os
import subprocess
import tempfile

from oracle import io as oio

HERE = os.path.dirname(os.path.abspath(__file__))
LASTZ = os.path.join(HERE, "_ref", "cPecanLastz")
LASTZ_ARGS = ["--hspthresh=1800", "--chain", "--strand=plus", "--gapped", "--format=cigar", "--gap=100,100",
              "--ambiguous=iupac,100,100"]
MATCH, INDEL_X, INDEL_Y = 0, 1, 2


def parse_np_read(path):
    """nanopore_loadNanoporeReadFromFile (impl/nanopore.c:98-370): the fields the tests use."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    head = lines[0].split()
    assert len(head) == 18
    read_length, n_t, n_c, t_len, c_len = (int(v) for v in head[:5])
    keys = ["scale", "shift", "var", "scale_sd", "var_sd", "drift"]
    tp = {k: float(v) for k, v in zip(keys, head[5:11])}
    cp = {k: float(v) for k, v in zip(keys, head[11:17])}
    two_d = int(head[17])
    two_d_read = lines[1].split()[0][:read_length] if two_d else ""
    template_read = lines[2].split()[0][:t_len]
    template_strand_map = [int(v) for v in lines[3].split()]
    template_event_map = [int(v) for v in lines[6].split()]
    ev = [float(v) for v in lines[7].split()]
    assert len(template_strand_map) == t_len and len(template_event_map) == read_length and len(ev) == 4 * n_t
    return dict(read_length=read_length, n_template_events=n_t, n_complement_events=n_c,
                template_params=tp, complement_params=cp, two_d_read=two_d_read, template_read=template_read,
                template_strand_event_map=template_strand_map, template_event_map=template_event_map,
                template_events=[ev[4 * i:4 * i + 4] for i in range(n_t)])


def parse_cigar_line(line):
    """one `cigar:` record -> dict(start1, end1, start2, end2, ops=[(op, length)])"""
    tok = line.split()
    assert tok[0] == "cigar:"
    name2, s2, e2, st2, name1, s1, e1, st1 = tok[1:9]
    assert name1 == "a" and name2 == "b" and st1 == "+" and st2 == "+"
    ops = []
    kind = {"M": MATCH, "D": INDEL_X, "I": INDEL_Y}
    for c, n in zip(tok[10::2], tok[11::2]):
        ops.append((kind[c], int(n)))
    return dict(start1=int(s1), end1=int(e1), start2=int(s2), end2=int(e2), ops=ops)


def cigar_to_anchor_pairs(al, trim):
    """convertPairwiseForwardStrandAlignmentToAnchorPairs (pairwiseAligner.c:1454-1478)"""
    out = []
    j, k = al["start1"], al["start2"]
    for op, n in al["ops"]:
        if op == MATCH:
            out.extend((j + q, k + q) for q in range(trim, n - trim))
        if op != INDEL_Y:
            j += n
        if op != INDEL_X:
            k += n
    assert j == al["end1"] and k == al["end2"]
    return out


def run_lastz(s_x, s_y, lastz=LASTZ):
    """The lastz call of getBlastPairs (pairwiseAligner.c:1501-1523): sX written to a FASTA file as
    "a"; sY to a second file as "b" when longer than 1000, else piped on stdin.  Returns the cigar
    records in output order."""
    with tempfile.TemporaryDirectory() as tmp:
        fa = os.path.join(tmp, "a.fa")
        with open(fa, "w") as fh:
            fh.write(">a\n%s\n" % s_x)
        if len(s_y) > 1000:
            fb = os.path.join(tmp, "b.fa")
            with open(fb, "w") as fh:
                fh.write(">b\n%s\n" % s_y)
            res = subprocess.run([lastz] + LASTZ_ARGS + [fa, fb], capture_output=True, text=True, check=True)
        else:
            res = subprocess.run([lastz] + LASTZ_ARGS + [fa], input=">b\n%s\n\n" % s_y, capture_output=True,
                                 text=True, check=True)
    return [parse_cigar_line(ln) for ln in res.stdout.splitlines() if ln.startswith("cigar:")]


def blast_pairs(s_x, s_y, trim, repeat_mask, lastz=LASTZ):
    """getBlastPairs (pairwiseAligner.c:1480-1558), returned sorted by (x, y) as both of its callers
    re-sort it (:1632, :1659)"""
    if not s_x or not s_y:
        return []
    if not repeat_mask:
        s_x, s_y = s_x.upper(), s_y.upper()
    pairs = []
    for al in run_lastz(s_x, s_y, lastz):
        pairs.extend(cigar_to_anchor_pairs(al, trim))
    return sorted(pairs)


def blast_pairs_for_params(s_x, s_y, trim=14, anchor_matrix=500 * 500, repeat_mask_matrix=500 * 500, lastz=LASTZ):
    """getBlastPairsForPairwiseAlignmentParameters (pairwiseAligner.c:1646-1697) with
    getBlastPairsForPairwiseAlignmentParametersP (:1618-1644): top-level pairs (filtered), and in
    every gap between consecutive ones whose area exceeds repeat_mask_matrix, the filtered pairs of
    a second lastz run on the upper-cased slices."""
    l_x, l_y = len(s_x), len(s_y)
    if l_x * l_y <= anchor_matrix:
        return []
    top = oio.filter_to_remove_overlap(blast_pairs(s_x, s_y, trim, True, lastz))
    combined = []

    def gap(px, py, x, y):
        if (x - px) * (y - py) > repeat_mask_matrix:
            sub = oio.filter_to_remove_overlap(blast_pairs(s_x[px:x], s_y[py:y], trim, False, lastz))
            combined.extend((a + px, b + py) for a, b in sub)

    px = py = 0
    for x, y in top:
        assert 0 <= x < l_x and 0 <= y < l_y and x >= px and y >= py
        gap(px, py, x, y)
        combined.append((x, y))
        px, py = x + 1, y + 1
    gap(px, py, l_x, l_y)
    return combined


def remapped_anchors(reference, read, event_map, trim=14, lastz=LASTZ):
    """getRemappedAnchors / get1dRemappedAnchors (tests/stateMachineTests.c:132-146): read-coordinate
    anchors through the event map (nanopore_remapAnchorPairs, impl/nanopore.c:426-436), then
    filterToRemoveOverlap."""
    pairs = blast_pairs_for_params(reference, read, trim, lastz=lastz)
    return oio.filter_to_remove_overlap([(x, event_map[y]) for x, y in pairs])
