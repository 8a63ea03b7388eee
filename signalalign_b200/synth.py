"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is involved: every read is drawn from numpy's PCG64 with a fixed seed.

* Gaussian k-mer tables: level_mean ~ U(60, 120) pA, level_sd ~ U(1, 3), noise mean ~ U(0.5, 2),
  noise sd = 0.3 x noise mean x U(0.8, 1.2), lambda = mean^3 / sd^2 (the inverse-Gaussian shape
  matching that mean and sd), transitions = signalAlign's nanopore defaults.
* Reads: a uniform random reference; per reference k-mer 0 events with probability 0.1, else a
  geometric count (overall mean 1.6); event mean ~ N(scale * level_mean + shift, level_sd) with
  scale = 1 +- 0.05 and shift ~ U(-5, 5); event sd ~ Gamma(mean noise_mean, sd noise_sd);
  duration ~ Exp(mean 2 ms); start = running sum of durations.
* Anchors: every 50th reference position of the true path, x jittered by up to +-3, then reduced
  to a strictly increasing chain.
* HDP tables: per k-mer mixtures of 1-8 normals (means within +-3 pA of a base level ~ U(60, 120),
  sd ~ U(1, 3), Dirichlet(1) weights) tabulated on a uniform grid, with knot slopes from the
  natural cubic spline condition that signalAlign's spline_knot_slopes solves.
"""
import math

import numpy as np

NANOPORE_TRANSITION_TOKENS = ["0.790158882824", "0.196524254983", "0.0133168621928", "0.803475745017",
                              "0.196524254983", "0.0", "0.986683137807", "1e-09", "0.0133168621929", "0.0"]


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def kmer_strings(alphabet, k):
    """All k-mers in k-mer-id order (lexicographic over the sorted alphabet)."""
    alpha = "".join(sorted(alphabet))
    a = len(alpha)
    n = a ** k
    ids = np.arange(n)
    chars = np.empty((n, k), dtype="<U1")
    for pos in range(k - 1, -1, -1):
        chars[:, pos] = np.array(list(alpha))[ids % a]
        ids = ids // a
    return ["".join(r) for r in chars]


def gaussian_table(alphabet, k, seed):
    """n_kmers x 5 table [level_mean, level_sd, noise_mean, noise_sd, noise_lambda]."""
    r = _rng(seed)
    n = len(alphabet) ** k
    mu = r.uniform(60.0, 120.0, n)
    sd = r.uniform(1.0, 3.0, n)
    nu = r.uniform(0.5, 2.0, n)
    nu_sd = 0.3 * nu * r.uniform(0.8, 1.2, n)
    lam = nu ** 3 / nu_sd ** 2
    return np.stack([mu, sd, nu, nu_sd, lam], axis=1)


def model_text(alphabet, k, table, transition_tokens=NANOPORE_TRANSITION_TOKENS):
    """The three lines of a signalAlign .model file (format of stateMachine.c:1328-1426)."""
    l0 = "3\t%d\t%s\t%d\n" % (len(alphabet), alphabet, k)
    l1 = "\t".join(transition_tokens) + "\n"
    l2 = "\t".join(repr(float(v)) for v in table.reshape(-1)) + "\n"
    return l0 + l1 + l2


def kmer_ids_of(seq, alphabet, k):
    alpha = "".join(sorted(alphabet))
    lut = np.full(256, -1, dtype=np.int64)
    for i, ch in enumerate(alpha):
        lut[ord(ch)] = i
    codes = lut[np.frombuffer(seq.encode(), dtype=np.uint8)]
    n = len(seq) - k + 1
    ids = np.zeros(max(n, 0), dtype=np.int64)
    for j in range(k):
        ids = ids * len(alpha) + codes[j:j + n]
    return ids


def make_read(seq, alphabet, k, level_mean, level_sd, noise_mean, noise_sd, r, anchor_every=50, jitter=3,
              skip_prob=0.1, mean_events=1.6, drawer=None):
    """Events for one reference, plus anchors and the scaling used.  `drawer(ids, r)` may override the
    per-event level draw (used for HDP mixtures); it returns the unscaled level per event."""
    ids = kmer_ids_of(seq, alphabet, k)
    lX = len(ids)
    p_geo = 1.0 / (mean_events / (1.0 - skip_prob))
    counts = np.where(r.random(lX) < skip_prob, 0, r.geometric(p_geo, lX))
    ev_kmer = np.repeat(ids, counts)
    ev_pos = np.repeat(np.arange(lX), counts)
    lY = len(ev_kmer)
    scale = 1.0 + r.uniform(-0.05, 0.05)
    shift = r.uniform(-5.0, 5.0)
    if drawer is None:
        level = r.normal(level_mean[ev_kmer], level_sd[ev_kmer])
    else:
        level = drawer(ev_kmer, r)
    mean = scale * level + shift if drawer is not None else scale * level_mean[ev_kmer] + shift + \
        (level - level_mean[ev_kmer])
    nm, ns = noise_mean[ev_kmer], noise_sd[ev_kmer]
    shape = (nm / ns) ** 2
    noise = r.gamma(shape, nm / shape)
    noise = np.maximum(noise, 1e-3)
    dur = r.exponential(0.002, lY)
    start = np.concatenate([[0.0], np.cumsum(dur)[:-1]]) if lY else np.zeros(0)
    events = np.stack([mean, noise, dur, start], axis=1) if lY else np.zeros((0, 4))
    # anchors every `anchor_every` reference positions on the true path
    first_event = np.full(lX, -1, dtype=np.int64)
    if lY:
        starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
        first_event = np.where(counts > 0, starts, -1)
    anchors = []
    for x in range(anchor_every, lX, anchor_every):
        xx = x
        while xx < lX and first_event[xx] < 0:
            xx += 1
        if xx >= lX:
            break
        ax = min(max(xx + int(r.integers(-jitter, jitter + 1)), 0), lX - 1)
        anchors.append((ax, int(first_event[xx])))
    chain = []
    for a in anchors:
        if not chain or (a[0] > chain[-1][0] and a[1] > chain[-1][1]):
            chain.append(a)
    anc = np.array(chain, dtype=np.int64).reshape(-1, 2)
    return dict(reference=seq, events=events, anchors=anc, scale=scale, shift=shift, var=1.0,
                true_pos=ev_pos)


def random_reference(length, r, alphabet="ACGT"):
    return "".join(np.array(list(alphabet))[r.integers(0, len(alphabet), length)])


def config0(seed=0):
    """One read: 1,000 bp uniform ACGT reference, 6-mer ACGT Gaussian table, about 1,600 events."""
    table = gaussian_table("ACGT", 6, seed + 1000)
    r = _rng(seed)
    seq = random_reference(1000, r)
    read = make_read(seq, "ACGT", 6, table[:, 0], table[:, 1], table[:, 2], table[:, 3], r)
    return dict(alphabet="ACGT", k=6, table=table, reads=[read])


def config1(seed=1, n_reads=256, span=(2000, 20000)):
    """256 reads with reference spans ~ U(2 kb, 20 kb) over the same 6-mer ACGT table."""
    table = gaussian_table("ACGT", 6, 1000)
    r = _rng(seed)
    reads = []
    for _ in range(n_reads):
        L = int(r.integers(span[0], span[1] + 1))
        seq = random_reference(L, r)
        reads.append(make_read(seq, "ACGT", 6, table[:, 0], table[:, 1], table[:, 2], table[:, 3], r))
    return dict(alphabet="ACGT", k=6, table=table, reads=reads)


def spline_knot_slopes(x, y):
    """Knot slopes of the natural cubic spline through (x, y): the tridiagonal system that
    hdp_math_utils.c:400-442 (spline_knot_slopes) solves, written as a Thomas sweep."""
    n = len(x)
    h = np.diff(x)
    a = np.zeros(n)
    b = np.zeros(n)
    c = np.zeros(n)
    d = np.zeros(n)
    b[0] = 2.0 / h[0]
    c[0] = 1.0 / h[0]
    d[0] = 3.0 * (y[1] - y[0]) / h[0] ** 2
    for i in range(1, n - 1):
        a[i] = 1.0 / h[i - 1]
        b[i] = 2.0 * (1.0 / h[i - 1] + 1.0 / h[i])
        c[i] = 1.0 / h[i]
        d[i] = 3.0 * ((y[i] - y[i - 1]) / h[i - 1] ** 2 + (y[i + 1] - y[i]) / h[i] ** 2)
    a[n - 1] = 1.0 / h[n - 2]
    b[n - 1] = 2.0 / h[n - 2]
    d[n - 1] = 3.0 * (y[n - 1] - y[n - 2]) / h[n - 2] ** 2
    cp = np.zeros(n)
    dp = np.zeros(n)
    cp[0] = c[0] / b[0]
    dp[0] = d[0] / b[0]
    for i in range(1, n):
        m = b[i] - a[i] * cp[i - 1]
        cp[i] = c[i] / m if i < n - 1 else 0.0
        dp[i] = (d[i] - a[i] * dp[i - 1]) / m
    k = np.zeros(n)
    k[n - 1] = dp[n - 1]
    for i in range(n - 2, -1, -1):
        k[i] = dp[i] - cp[i] * k[i + 1]
    return k


def spline_knot_slopes_batch(x, Y):
    """Row-wise spline_knot_slopes for a (rows, n) array of knot values on one grid."""
    n = len(x)
    h = np.diff(x)
    a = np.zeros(n); b = np.zeros(n); c = np.zeros(n)
    b[0] = 2.0 / h[0]; c[0] = 1.0 / h[0]
    a[1:n - 1] = 1.0 / h[:-1]
    b[1:n - 1] = 2.0 * (1.0 / h[:-1] + 1.0 / h[1:])
    c[1:n - 1] = 1.0 / h[1:]
    a[n - 1] = 1.0 / h[n - 2]; b[n - 1] = 2.0 / h[n - 2]
    D = np.zeros_like(Y)
    D[:, 0] = 3.0 * (Y[:, 1] - Y[:, 0]) / h[0] ** 2
    D[:, 1:n - 1] = 3.0 * ((Y[:, 1:n - 1] - Y[:, :n - 2]) / h[:-1] ** 2 + (Y[:, 2:] - Y[:, 1:n - 1]) / h[1:] ** 2)
    D[:, n - 1] = 3.0 * (Y[:, n - 1] - Y[:, n - 2]) / h[n - 2] ** 2
    cp = np.zeros(n)
    DP = np.zeros_like(Y)
    cp[0] = c[0] / b[0]
    DP[:, 0] = D[:, 0] / b[0]
    for i in range(1, n):
        m = b[i] - a[i] * cp[i - 1]
        cp[i] = c[i] / m if i < n - 1 else 0.0
        DP[:, i] = (D[:, i] - a[i] * DP[:, i - 1]) / m
    K = np.zeros_like(Y)
    K[:, n - 1] = DP[:, n - 1]
    for i in range(n - 2, -1, -1):
        K[:, i] = DP[:, i] - cp[i] * K[:, i + 1]
    return K


def hdp_tables(alphabet, k, seed, grid_start=30.0, grid_stop=150.0, grid_length=2000):
    """Per-k-mer mixture densities on the grid, their knot slopes, mixture means/sds and components."""
    r = _rng(seed)
    n = len(alphabet) ** k
    n_comp = r.integers(1, 9, n)
    base = r.uniform(60.0, 120.0, n)
    maxc = 8
    means = base[:, None] + r.uniform(-3.0, 3.0, (n, maxc))
    sds = r.uniform(1.0, 3.0, (n, maxc))
    w = r.gamma(1.0, 1.0, (n, maxc))
    w[np.arange(maxc)[None, :] >= n_comp[:, None]] = 0.0
    w /= w.sum(axis=1, keepdims=True)
    n_pts = grid_length - 1
    dx = (grid_stop - grid_start) / float(n_pts)
    grid = np.empty(grid_length)
    grid[:n_pts] = grid_start + np.arange(n_pts) * dx
    grid[n_pts] = grid_stop
    dens = np.zeros((n, grid_length))
    for c in range(maxc):
        z = (grid[None, :] - means[:, c:c + 1]) / sds[:, c:c + 1]
        dens += w[:, c:c + 1] * np.exp(-0.5 * z * z) / (sds[:, c:c + 1] * math.sqrt(2 * math.pi))
    slopes = spline_knot_slopes_batch(grid, dens)
    mix_mean = (w * means).sum(axis=1)
    mix_var = (w * (sds ** 2 + means ** 2)).sum(axis=1) - mix_mean ** 2
    return dict(grid_start=grid_start, grid_stop=grid_stop, grid_length=grid_length, grid=grid, density=dens,
                slope=slopes, mean=mix_mean, sd=np.sqrt(mix_var), comp_means=means, comp_sds=sds, weights=w)


def config2(seed=2, n_reads=128, span=(5000, 15000), grid_length=2000):
    """HDP emissions over 6-mer ACEGT (15,625 k-mers); 128 reads of 5-15 kb."""
    alphabet = "ACEGT"
    hdp = hdp_tables(alphabet, 6, seed + 500, grid_length=grid_length)
    n = len(alphabet) ** 6
    r = _rng(seed)
    table = np.zeros((n, 5))
    table[:, 0] = hdp["mean"]
    table[:, 1] = hdp["sd"]
    table[:, 2] = r.uniform(0.5, 2.0, n)
    table[:, 3] = 0.3 * table[:, 2]
    table[:, 4] = table[:, 2] ** 3 / table[:, 3] ** 2

    def drawer(ev_kmer, rr):
        w = hdp["weights"][ev_kmer]
        u = rr.random(len(ev_kmer))[:, None]
        comp = (np.cumsum(w, axis=1) < u).sum(axis=1)
        comp = np.minimum(comp, 7)
        return rr.normal(hdp["comp_means"][ev_kmer, comp], hdp["comp_sds"][ev_kmer, comp])

    reads = []
    for _ in range(n_reads):
        L = int(r.integers(span[0], span[1] + 1))
        seq = list(random_reference(L, r))
        # methylate half of the CpG cytosines
        for i in range(L - 1):
            if seq[i] == "C" and seq[i + 1] == "G" and r.random() < 0.5:
                seq[i] = "E"
        seq = "".join(seq)
        reads.append(make_read(seq, alphabet, 6, table[:, 0], table[:, 1], table[:, 2], table[:, 3], r,
                               drawer=drawer))
    return dict(alphabet=alphabet, k=6, table=table, hdp=hdp, reads=reads)


def _hdp_drawer(hdp):
    def drawer(ev_kmer, rr):
        w = hdp["weights"][ev_kmer]
        u = rr.random(len(ev_kmer))[:, None]
        comp = np.minimum((np.cumsum(w, axis=1) < u).sum(axis=1), 7)
        return rr.normal(hdp["comp_means"][ev_kmer, comp], hdp["comp_sds"][ev_kmer, comp])
    return drawer


_COMPLEMENT = str.maketrans("ACGT", "TGCA")


def config3(seed=3, n_reads=512, span=(1000, 30000), grid_length=2000, route="substitute"):
    """Methylation hypotheses with 2D reads: per read a template and a complement event stream (each
    with its own scale/shift), CCWGG motifs placed about once per 256 bp and their second C
    methylated (E) with probability 1/2 on each strand.  With route "substitute" every stream is
    aligned under the all-C and the all-E hypothesis (substituted references, 4 alignments per
    read); with route "degenerate" each stream is aligned once against a reference with 'X' at the
    sites and degenerate type cytosine2 (C or E), so the cells over a site hold two paths (2
    alignments per read, each with "degenerate": "CE").  Half of the reads use the 6-mer ACEGT
    Gaussian table, half the 6-mer ACEGT HDP tables."""
    assert route in ("substitute", "degenerate")
    alphabet, k = "ACEGT", 6
    n = len(alphabet) ** k
    r = _rng(seed)
    gauss = gaussian_table(alphabet, k, seed + 100)
    hdp = hdp_tables(alphabet, k, seed + 500, grid_length=grid_length)
    htable = np.zeros((n, 5))
    htable[:, 0], htable[:, 1] = hdp["mean"], hdp["sd"]
    htable[:, 2] = r.uniform(0.5, 2.0, n)
    htable[:, 3] = 0.3 * htable[:, 2]
    htable[:, 4] = htable[:, 2] ** 3 / htable[:, 3] ** 2
    drawer = _hdp_drawer(hdp)
    motifs = ("CCAGG", "CCTGG")
    alignments = []
    for ri in range(n_reads):
        L = int(r.integers(span[0], span[1] + 1))
        seq = list(random_reference(L, r))
        sites = []
        for pos in range(int(r.integers(0, 256)), L - 5, 256):
            seq[pos:pos + 5] = list(motifs[int(r.integers(0, 2))])
            sites.append(pos + 1)
        canon = "".join(seq)
        use_hdp = ri % 2 == 1
        table = htable if use_hdp else gauss
        for strand in ("template", "complement"):
            base = canon if strand == "template" else canon.translate(_COMPLEMENT)[::-1]
            pos_s = sites if strand == "template" else [L - s - 3 for s in sites]
            truth = list(base)
            for q in pos_s:
                if truth[q] == "C" and r.random() < 0.5:
                    truth[q] = "E"
            rd = make_read("".join(truth), alphabet, k, table[:, 0], table[:, 1], table[:, 2], table[:, 3], r,
                           drawer=drawer if use_hdp else None)
            for hyp in (("C", "E") if route == "substitute" else ("X",)):
                ref = list(base)
                for q in pos_s:
                    if ref[q] == "C":
                        ref[q] = hyp
                extra = dict(degenerate="CE") if hyp == "X" else {}
                alignments.append(dict(rd, reference="".join(ref), read=ri, strand=strand, hypothesis=hyp,
                                       model="hdp" if use_hdp else "gauss", **extra))
    return dict(alphabet=alphabet, k=k, gauss_table=gauss, hdp_table=htable, hdp=hdp, alignments=alignments)


def band_cells(xmyL, xmyR):
    """DP cells of a band: sum over anti-diagonals of the width."""
    return int(np.sum((np.asarray(xmyR) - np.asarray(xmyL)) // 2 + 1))
