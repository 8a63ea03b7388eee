/*
 * sa_oracle.c -- CPU restatement (FP64, single thread per call) of signalAlign's banded,
 * anchored 3-state pair-HMM forward-backward and its posterior aligned-pair output.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is compared against:
 * only tests, the smoke check and the CPU-baseline leg of the benchmark load it.  The product
 * library never links, loads or falls back to it.
 *
 * It follows the reference algorithm step by step (same recursion order, same logAdd
 * polynomial, same windowed traceback schedule, same every-10th-diagonal total-probability
 * refresh), because the posterior set depends on those details.  Every function cites the
 * reference file:line it restates (paths relative to the signalAlign source tree).
 *
 * Parity pins (see tests/test_oracle_golden.py): band tuples of test_bands, split tuples of
 * test_getSplitPoints, logAdd accuracy of test_logAdd, the 14-pair / 7-pair toy DPs of
 * test_sm3_diagonalDPCalculations / test_sm3_5merDiagonalDPCalculations, and the 1076-pair
 * unbanded Zymo alignment of test_stateMachine3_getAlignedPairsWithBanding.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#define ORC_LOG_ZERO (-INFINITY)
#define ORC_NB_EVENT_PARAMS 4          /* inc/nanopore.h:4 */
#define ORC_PAIR_PROB_1 10000000.0      /* inc/pairwiseAligner.h:27 */
#define ORC_MAX_K 16

enum { ORC_OK = 0, ORC_E_ARG = 1, ORC_E_ALPHABET = 2, ORC_E_ANCHORS = 3, ORC_E_NOMEM = 4,
       ORC_E_OVERFLOW = 5, ORC_E_PATHS = 6 };

/* emission kinds: how the reference's StateMachine function pointers are set up */
enum { ORC_EMIT_PLAIN = 0,     /* getStateMachine3: strawManGetKmerEventMatchProb (stateMachine.c:547) */
       ORC_EMIT_DESCALED = 1,  /* getStateMachine3_descaled: ...WithDescaling (stateMachine.c:498) */
       ORC_EMIT_HDP = 2 };     /* getHdpStateMachine: getHdpKmerDensity (stateMachine.c:468) */

/* transition slots, named after StateMachine3 (inc/stateMachine.h:153-163) */
enum { T_MATCH_CONTINUE = 0, T_MATCH_FROM_GAP_X, T_MATCH_FROM_GAP_Y, T_GAP_OPEN_X, T_GAP_OPEN_Y,
       T_GAP_EXTEND_X, T_GAP_EXTEND_Y, T_GAP_SWITCH_TO_X, T_GAP_SWITCH_TO_Y };

enum { S_MATCH = 0, S_GAPX = 1, S_GAPY = 2 };   /* inc/stateMachine.h:42-44 */

typedef struct {
    int32_t emission;
    int32_t alphabet_size;
    int32_t kmer_length;
    int32_t pad;
    const char *alphabet;         /* sorted, as sequence_prepareAlphabet leaves it */
    int64_t n_kmers;
    double t[9];
    const double *match;          /* n_kmers x 5: level_mean, level_sd, noise_mean, noise_sd, lambda */
    const double *gapy;           /* n_kmers x 5, level_sd already x1.75 (stateMachine.c:1418-1420) */
    const double *gapx;           /* n_kmers, log(0.1) unless changed (stateMachine.c:1472-1474) */
    double scale, shift, var;
    /* HDP densities, only for ORC_EMIT_HDP */
    int64_t grid_length;
    const double *grid;           /* linspace grid (hdp_math_utils.c:497-509) */
    const double *density;        /* rows x grid_length posterior predictive */
    const double *slope;          /* rows x grid_length spline knot slopes */
    const int64_t *kmer_row;      /* kmer id -> row of its nearest observed ancestor (hdp.c:2594-2597) */
} orc_model;

typedef struct {
    double threshold;
    int64_t min_diags_between_traceback;
    int64_t traceback_diagonals;
    int64_t diagonal_expansion;
    int64_t split_matrix_bigger_than_this;
} orc_params;

typedef struct {
    int64_t score;     /* floor(p * 1e7) */
    int64_t x;         /* reference k-mer index */
    int64_t y;         /* event index */
    int64_t kmer;      /* k-mer id of the path k-mer */
} orc_pair;

/* ------------------------------------------------------------------------------------------
 * log-space add: pairwiseAligner.c:234-254 (4-piece cubic for log(1+e^d), cut at 7.5)
 * ---------------------------------------------------------------------------------------- */
static inline double orc_lookup(double d) {
    if (d <= 1.00f)
        return ((-0.009350833524763f * d + 0.130659527668286f) * d + 0.498799810682272f) * d + 0.693203116424741f;
    if (d <= 2.50f)
        return ((-0.014532321752540f * d + 0.139942324101744f) * d + 0.495635523139337f) * d + 0.692140569840976f;
    if (d <= 4.50f)
        return ((-0.004605031767994f * d + 0.063427417320019f) * d + 0.695956496475118f) * d + 0.514272634594009f;
    return ((-0.000458661602210f * d + 0.009695946122598f) * d + 0.930734667215156f) * d + 0.168037164329057f;
}

double orc_logAdd(double x, double y) {
    if (x < y)
        return (x == ORC_LOG_ZERO || y - x >= 7.5) ? y : orc_lookup(y - x) + x;
    return (y == ORC_LOG_ZERO || x - y >= 7.5) ? x : orc_lookup(x - y) + y;
}

/* ------------------------------------------------------------------------------------------
 * band geometry: pairwiseAligner.c:97-182 (band_avoidOffByOne, band_setCurrentDiagonal,
 * band_boundCoordinate, band_construct).  Output: xmyL/xmyR for xay = 0..lX+lY.
 * ---------------------------------------------------------------------------------------- */
static inline int64_t orc_xcoord(int64_t xay, int64_t xmy) { return (xay + xmy) / 2; }
static inline int64_t orc_ycoord(int64_t xay, int64_t xmy) { return (xay - xmy) / 2; }

static inline int64_t orc_parity_fix(int64_t xay, int64_t xmy) { return (xay + xmy) % 2 == 0 ? xmy : xmy + 1; }

static inline int64_t orc_clamp(int64_t z, int64_t lz) { return z < 0 ? 0 : (z > lz ? lz : z); }

int orc_band(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY, int64_t expansion,
             int64_t *out_xmyL, int64_t *out_xmyR) {
    if (lX < 0 || lY < 0 || expansion % 2 != 0) return ORC_E_ARG;
    int64_t n = lX + lY, ai = 0;
    int64_t pxay = 0, pxmy = 0, nxay = 0, nxmy = 0;
    int64_t xL = 0, yL = 0, xU = 0, yU = 0;
    for (int64_t xay = 0; xay <= n; ) {
        /* intersect the anti-diagonal with the box [xL,xU] x [yL,yU] */
        int64_t l = orc_parity_fix(xay, xL - yL), r = orc_parity_fix(xay, xU - yU);
        int64_t xl = orc_xcoord(xay, l);
        if (xl < xL) l += 2 * (xL - xl);
        int64_t yl = orc_ycoord(xay, l);      /* y of the left end after the x fix */
        if (yL < yl) l += 2 * (yl - yL);
        int64_t xr = orc_xcoord(xay, r);
        if (xU < xr) r -= 2 * (xr - xU);
        int64_t yr = orc_ycoord(xay, r);
        if (yr < yU) r -= 2 * (yU - yr);
        if (l > r || (xay + l) % 2 != 0) return ORC_E_ANCHORS;
        out_xmyL[xay] = l;
        out_xmyR[xay] = r;
        if (nxay == xay++) {
            pxay = nxay;
            pxmy = nxmy;
            int64_t x = lX, y = lY;
            if (ai < n_anchors) {
                x = anchors[2 * ai] + 1;
                y = anchors[2 * ai + 1] + 1;
                ai++;
                if (!(x > orc_xcoord(pxay, pxmy) && y > orc_ycoord(pxay, pxmy) && x <= lX && y <= lY))
                    return ORC_E_ANCHORS;
            }
            nxay = x + y;
            nxmy = x - y;
            xL = orc_clamp(orc_xcoord(pxay, pxmy - expansion), lX);
            yL = orc_clamp(orc_ycoord(nxay, nxmy - expansion), lY);
            xU = orc_clamp(orc_xcoord(nxay, nxmy + expansion), lX);
            yU = orc_clamp(orc_ycoord(pxay, pxmy + expansion), lY);
        }
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------------
 * split points: pairwiseAligner.c:1706-1757 (getSplitPointsP, getSplitPoints).
 * out: 4 int64 per region (x1, y1, x2, y2).  Returns the number of regions, or -error.
 * ---------------------------------------------------------------------------------------- */
static int orc_split_p(int64_t *x1, int64_t *y1, int64_t x2, int64_t y2, int64_t x3, int64_t y3,
                       int64_t *out, int64_t *n_out, int64_t max_out, int64_t limit, int skip) {
    int64_t lX2 = x3 - x2, lY2 = y3 - y2;
    if (lX2 * lY2 > limit) {
        int64_t maxLen = (int64_t) sqrt((double) limit);
        int64_t hX = lX2 / 2 > maxLen ? maxLen : lX2 / 2;
        int64_t hY = lY2 / 2 > maxLen ? maxLen : lY2 / 2;
        if (!skip) {
            if (*n_out >= max_out) return -ORC_E_OVERFLOW;
            int64_t *o = out + 4 * (*n_out)++;
            o[0] = *x1; o[1] = *y1; o[2] = x2 + hX; o[3] = y2 + hY;
        }
        *x1 = x3 - hX;
        *y1 = y3 - hY;
        return 1;
    }
    return 0;
}

int64_t orc_split_points(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY, int64_t limit,
                         int ragged_left, int ragged_right, int64_t *out, int64_t max_out) {
    int64_t x1 = 0, y1 = 0, x2 = 0, y2 = 0, n_out = 0;
    for (int64_t i = 0; i < n_anchors; i++) {
        int64_t x3 = anchors[2 * i], y3 = anchors[2 * i + 1];
        int r = orc_split_p(&x1, &y1, x2, y2, x3, y3, out, &n_out, max_out, limit, ragged_left && i == 0);
        if (r < 0) return r;
        if (x3 < x2 || y3 < y2 || x3 >= lX || y3 >= lY) return -ORC_E_ANCHORS;
        x2 = x3 + 1;
        y2 = y3 + 1;
    }
    int r = orc_split_p(&x1, &y1, x2, y2, lX, lY, out, &n_out, max_out, limit, ragged_left && n_anchors == 0);
    if (r < 0) return r;
    if (!r || !ragged_right) {
        if (n_out >= max_out) return -ORC_E_OVERFLOW;
        int64_t *o = out + 4 * n_out++;
        o[0] = x1; o[1] = y1; o[2] = lX; o[3] = lY;
    }
    return n_out;
}

/* ------------------------------------------------------------------------------------------
 * k-mer paths: a reference k-mer with 'X' expands to nbOptions^(#X) paths, first 'X'
 * position varying slowest (pairwiseAligner.c:537-650: path_findDegeneratePositions,
 * path_permutePattern, hdCell_construct, hdCell_getSubstitutedKmer).
 * ---------------------------------------------------------------------------------------- */
typedef struct {
    int64_t n_paths;
    int64_t first;      /* index into the flat path arrays */
} orc_pos;

typedef struct {
    int64_t lX;
    orc_pos *pos;        /* lX + 1 entries; pos[x] describes matrix column x (k-mer x-1); pos[0] = NULL k-mer */
    char *kmers;         /* n_paths_total x k chars (NULL path stores nothing meaningful) */
    int64_t *ids;        /* k-mer id per path, -1 for the NULL path */
    int64_t total;
    int k;
} orc_paths;

static int64_t orc_kmer_id(const char *kmer, int k, const char *alphabet, int asz) {
    /* nanopore_hdp.c:360-393 (word_id, kmer_to_word, kmer_id) */
    int64_t id = 0;
    for (int i = 0; i < k; i++) {
        int j = 0;
        while (j < asz && alphabet[j] != kmer[i]) j++;
        if (j == asz) return -1;
        id = id * asz + j;
    }
    return id;
}

static void orc_paths_free(orc_paths *P) {
    free(P->pos); free(P->kmers); free(P->ids);
}

static int orc_paths_build(orc_paths *P, const char *seq, int64_t lX, int k, const char *options, int nopt,
                           const orc_model *m) {
    P->lX = lX; P->k = k;
    P->pos = (orc_pos *) calloc((size_t) lX + 1, sizeof(orc_pos));
    if (!P->pos) return ORC_E_NOMEM;
    int64_t total = 1, cap = lX + 16;
    P->kmers = (char *) malloc((size_t) cap * k);
    P->ids = (int64_t *) malloc((size_t) cap * sizeof(int64_t));
    if (!P->kmers || !P->ids) return ORC_E_NOMEM;
    P->pos[0].n_paths = 1; P->pos[0].first = 0; P->ids[0] = -1;
    memset(P->kmers, 0, (size_t) k);
    for (int64_t x = 1; x <= lX; x++) {
        const char *km = seq + (x - 1);
        int degen[ORC_MAX_K], nd = 0;
        for (int i = 0; i < k; i++) if (km[i] == 'X') degen[nd++] = i;
        int64_t np = 1;
        for (int i = 0; i < nd; i++) np *= nopt;
        if (total + np > cap) {
            cap = 2 * (total + np);
            P->kmers = (char *) realloc(P->kmers, (size_t) cap * k);
            P->ids = (int64_t *) realloc(P->ids, (size_t) cap * sizeof(int64_t));
            if (!P->kmers || !P->ids) return ORC_E_NOMEM;
        }
        P->pos[x].n_paths = np; P->pos[x].first = total;
        for (int64_t p = 0; p < np; p++) {
            char *dst = P->kmers + (total + p) * k;
            memcpy(dst, km, (size_t) k);
            int64_t rem = p;
            for (int i = nd - 1; i >= 0; i--) { dst[degen[i]] = options[rem % nopt]; rem /= nopt; }
            int64_t id = orc_kmer_id(dst, k, m->alphabet, m->alphabet_size);
            if (id < 0) return ORC_E_ALPHABET;
            P->ids[total + p] = id;
        }
        total += np;
    }
    P->total = total;
    return ORC_OK;
}

/* path_checkLegal (pairwiseAligner.c:527-552): NULL on either side is legal; otherwise the
 * (k-1)-suffix of the from-k-mer must equal the (k-1)-prefix of the to-k-mer */
static inline int orc_legal(const orc_paths *P, int64_t from, int64_t to) {
    if (P->ids[from] < 0 || P->ids[to] < 0) return 1;
    const char *a = P->kmers + from * P->k, *b = P->kmers + to * P->k;
    for (int i = 0; i < P->k - 1; i++) if (a[i + 1] != b[i]) return 0;
    return 1;
}

/* stString_eq on path k-mers, NULL == NULL */
static inline int orc_same(const orc_paths *P, int64_t a, int64_t b) {
    if (P->ids[a] < 0 || P->ids[b] < 0) return P->ids[a] < 0 && P->ids[b] < 0;
    return memcmp(P->kmers + a * P->k, P->kmers + b * P->k, (size_t) P->k) == 0;
}

/* ------------------------------------------------------------------------------------------
 * emissions: stateMachine.c:226-289 (logInvGaussPdf, logGaussPdf, descaleEventMean_JordanStyle),
 * :498-589 (strawMan match probs), :155-172 (k-mer gap prob), :468-495 + hdp.c:2583-2607 +
 * hdp_math_utils.c:471-495 (HDP density with grid cubic-Hermite interpolation).
 * ---------------------------------------------------------------------------------------- */
static inline double orc_log_gauss(double x, double mu, double sigma) {
    if (sigma == 0.0) return ORC_LOG_ZERO;
    double ls = log(sigma);
    double a = (x - mu) / sigma;
    return -0.91893853320467267 - ls + (-0.5 * a * a);
}

static inline double orc_log_inv_gauss(double n, double mu, double lambda) {
    double ln = log(n);
    double a = (n - mu) / mu;
    double ll = log(lambda);
    return (ll - 1.8378770664093453 - 3 * ln - lambda * a * a / n) / 2;
}

static inline double orc_descale(double e, double mu, double scale, double shift, double var) {
    return (e + var * mu - scale * mu - shift) / var;
}

static double orc_grid_spline(const orc_model *m, const double *y, const double *s, double q) {
    const double *x = m->grid;
    int64_t len = m->grid_length;
    if (q <= x[0]) return y[0] - s[0] * (x[0] - q);
    if (q >= x[len - 1]) return y[len - 1] + s[len - 1] * (q - x[len - 1]);
    double dx = x[1] - x[0];
    int64_t il = (int64_t) ((q - x[0]) / dx);
    if (il > len - 2) il = len - 2;   /* q just below the last knot can round onto it */
    if (il < 0) il = 0;
    int64_t ir = il + 1;
    double dy = y[ir] - y[il];
    double a = s[il] * dx - dy;
    double b = dy - s[ir] * dx;
    double tl = (q - x[il]) / dx;
    double tr = 1.0 - tl;
    return tr * y[il] + tl * y[ir] + tl * tr * (a * tr + b * tl);
}

/* match (match!=0) or extra-event (match==0) emission of event ev for k-mer id */
static double orc_emit_event(const orc_model *m, int64_t id, const double *ev, int match) {
    if (id < 0) return ORC_LOG_ZERO;
    if (m->emission == ORC_EMIT_HDP) {
        double mu = m->match[id * 5];
        double u = orc_descale(ev[0], mu, m->scale, m->shift, m->var);
        int64_t row = m->kmer_row[id];
        double d = row < 0 ? 0.0 : orc_grid_spline(m, m->density + row * m->grid_length,
                                                   m->slope + row * m->grid_length, u);
        if (!(d > 0.0)) d = 0.0;
        return log((1 / m->var) * d);
    }
    const double *tab = (match ? m->match : m->gapy) + id * 5;
    double mean = ev[0], noise = ev[1];
    double mu = tab[0], sd = tab[1];
    if (m->emission == ORC_EMIT_DESCALED) mean = orc_descale(mean, mu, m->scale, m->shift, m->var);
    double lm = orc_log_gauss(mean, mu, sd);
    double ln = orc_log_inv_gauss(noise, tab[2], tab[4]);
    return lm + ln;
}

static inline double orc_emit_gapx(const orc_model *m, int64_t id) {
    if (m->emission == ORC_EMIT_HDP) return -2.3025850929940455;   /* stateMachine.c:1282 */
    if (id < 0) return ORC_LOG_ZERO;
    return m->gapx[id];
}

/* ------------------------------------------------------------------------------------------
 * DP diagonals: one per anti-diagonal, cells in ascending xmy, each cell holding its paths,
 * each path 3 state values (pairwiseAligner.c:837-1012 stores the same in heap HDCells).
 * ---------------------------------------------------------------------------------------- */
typedef struct {
    int64_t xmyL, xmyR, ncell;
    int64_t *poff;      /* ncell + 1 path offsets */
    double *v;          /* 3 doubles per path */
    int live;
} orc_diag;

typedef struct {
    const orc_model *m;
    const orc_paths *P;
    const double *events;
    int64_t lY;
    orc_diag *F, *B;
    int64_t n;          /* diagonal count - 1 */
} orc_dp;

static int orc_diag_alloc(orc_diag *d, int64_t xay, int64_t l, int64_t r, const orc_paths *P) {
    d->xmyL = l; d->xmyR = r; d->ncell = (r - l) / 2 + 1;
    d->poff = (int64_t *) malloc((size_t) (d->ncell + 1) * sizeof(int64_t));
    if (!d->poff) return ORC_E_NOMEM;
    int64_t acc = 0;
    for (int64_t c = 0; c < d->ncell; c++) {
        int64_t x = orc_xcoord(xay, l + 2 * c);
        d->poff[c] = acc;
        acc += P->pos[x].n_paths;
    }
    d->poff[d->ncell] = acc;
    d->v = (double *) malloc((size_t) acc * 3 * sizeof(double));
    if (!d->v) return ORC_E_NOMEM;
    d->live = 0;
    return ORC_OK;
}

static void orc_diag_fill(orc_diag *d, double a, double b, double c) {
    int64_t np = d->poff[d->ncell];
    for (int64_t i = 0; i < np; i++) { d->v[3 * i] = a; d->v[3 * i + 1] = b; d->v[3 * i + 2] = c; }
}

static inline double *orc_cell(orc_diag *d, int64_t xmy) {
    if (!d || !d->live || xmy < d->xmyL || xmy > d->xmyR) return NULL;
    return d->v + 3 * d->poff[(xmy - d->xmyL) / 2];
}

static inline void orc_start_probs(const orc_model *m, int ragged, double *s) {
    /* stateMachine.c:1022-1032 */
    if (ragged) { s[0] = ORC_LOG_ZERO; s[1] = 0; s[2] = 0; }
    else { s[0] = 0; s[1] = ORC_LOG_ZERO; s[2] = ORC_LOG_ZERO; }
}

static inline void orc_end_probs(const orc_model *m, int ragged, double *s) {
    /* stateMachine.c:1034-1061 */
    if (ragged) {
        s[0] = (m->t[T_GAP_OPEN_X] + m->t[T_GAP_OPEN_Y]) / 2.0;
        s[1] = m->t[T_GAP_EXTEND_X];
        s[2] = m->t[T_GAP_EXTEND_Y];
    } else {
        s[0] = m->t[T_MATCH_CONTINUE];
        s[1] = m->t[T_MATCH_FROM_GAP_X];
        s[2] = m->t[T_MATCH_FROM_GAP_Y];
    }
}

/* doTransitionForward / doTransitionBackward (pairwiseAligner.c:701-720) */
#define ORC_TRANS(fromv, tov, sf, st, e, t, fwd) do { \
        if (fwd) (tov)[st] = orc_logAdd((tov)[st], (fromv)[sf] + ((e) + (t))); \
        else (fromv)[sf] = orc_logAdd((fromv)[sf], (tov)[st] + ((e) + (t))); } while (0)

/* stateMachine3_cellCalculate / stateMachine3HDP_cellCalculate (stateMachine.c:1194-1325):
 * current cell at column x with event ev; lower/middle/upper are neighbour cell value blocks
 * (NULL if absent); paths of the current column are pc, of the previous column pp. */
static void orc_cell_calc(const orc_dp *dp, int64_t x, const double *ev,
                          double *cur, double *lower, double *middle, double *upper, int fwd) {
    const orc_model *m = dp->m;
    const orc_paths *P = dp->P;
    const double *t = m->t;
    int64_t c0 = P->pos[x].first, nc = P->pos[x].n_paths;
    if (lower) {
        int64_t l0 = P->pos[x - 1].first, nl = P->pos[x - 1].n_paths;
        for (int64_t p = 0; p < nc; p++) {
            for (int64_t q = 0; q < nl; q++) {
                if (!orc_legal(P, l0 + q, c0 + p)) continue;
                double *lv = lower + 3 * q, *cv = cur + 3 * p;
                double e = orc_emit_gapx(m, P->ids[c0 + p]);
                ORC_TRANS(lv, cv, S_MATCH, S_GAPX, e, t[T_GAP_OPEN_X], fwd);
                ORC_TRANS(lv, cv, S_GAPX, S_GAPX, e, t[T_GAP_EXTEND_X], fwd);
                ORC_TRANS(lv, cv, S_GAPY, S_GAPX, e, t[T_GAP_SWITCH_TO_X], fwd);
            }
        }
    }
    if (middle) {
        int64_t m0 = P->pos[x - 1].first, nm = P->pos[x - 1].n_paths;
        for (int64_t p = 0; p < nc; p++) {
            for (int64_t q = 0; q < nm; q++) {
                if (!orc_legal(P, m0 + q, c0 + p)) continue;
                double *mv = middle + 3 * q, *cv = cur + 3 * p;
                double e = orc_emit_event(m, P->ids[c0 + p], ev, 1);
                ORC_TRANS(mv, cv, S_MATCH, S_MATCH, e, t[T_MATCH_CONTINUE], fwd);
                ORC_TRANS(mv, cv, S_GAPX, S_MATCH, e, t[T_MATCH_FROM_GAP_X], fwd);
                ORC_TRANS(mv, cv, S_GAPY, S_MATCH, e, t[T_MATCH_FROM_GAP_Y], fwd);
            }
        }
    }
    if (upper) {
        for (int64_t p = 0; p < nc; p++) {
            for (int64_t q = 0; q < nc; q++) {
                if (!orc_same(P, c0 + q, c0 + p)) continue;
                double *uv = upper + 3 * q, *cv = cur + 3 * p;
                double e = orc_emit_event(m, P->ids[c0 + p], ev, 0);
                ORC_TRANS(uv, cv, S_MATCH, S_GAPY, e, t[T_GAP_OPEN_Y], fwd);
                ORC_TRANS(uv, cv, S_GAPY, S_GAPY, e, t[T_GAP_EXTEND_Y], fwd);
            }
        }
    }
}

static double orc_null_event[2] = { -INFINITY, 0 };   /* NULLEVENT, pairwiseAligner.c:261 */

static inline const double *orc_event(const orc_dp *dp, int64_t y) {
    /* sequence_getEvent (pairwiseAligner.c:442-445): negative index gives NULLEVENT */
    return y - 1 >= 0 ? dp->events + (y - 1) * ORC_NB_EVENT_PARAMS : orc_null_event;
}

/* diagonalCalculation (pairwiseAligner.c:1127-1158) over `cur` at xay, neighbours m1 (xay-1) and
 * m2 (xay-2) */
static void orc_diag_calc(const orc_dp *dp, int64_t xay, orc_diag *cur, orc_diag *m1, orc_diag *m2, int fwd) {
    for (int64_t xmy = cur->xmyL; xmy <= cur->xmyR; xmy += 2) {
        int64_t x = orc_xcoord(xay, xmy), y = orc_ycoord(xay, xmy);
        double *c = orc_cell(cur, xmy);
        double *lo = orc_cell(m1, xmy - 1), *mi = orc_cell(m2, xmy), *up = orc_cell(m1, xmy + 1);
        orc_cell_calc(dp, x, orc_event(dp, y), c, lo, mi, up, fwd);
    }
}

/* cell_dotProduct / hdCell_totalProbability / dpDiagonal_dotProduct (pairwiseAligner.c:677-742,
 * 1014-1027) */
static double orc_diag_dot(const orc_dp *dp, int64_t xay, orc_diag *a, orc_diag *b) {
    const orc_paths *P = dp->P;
    double total = ORC_LOG_ZERO;
    for (int64_t xmy = a->xmyL; xmy <= a->xmyR; xmy += 2) {
        int64_t x = orc_xcoord(xay, xmy);
        int64_t c0 = P->pos[x].first, nc = P->pos[x].n_paths;
        double *va = orc_cell(a, xmy), *vb = orc_cell(b, xmy);
        double cellTotal = ORC_LOG_ZERO;
        for (int64_t p = 0; p < nc; p++) {
            for (int64_t q = 0; q < nc; q++) {
                if (!orc_same(P, c0 + p, c0 + q)) continue;
                double *u = va + 3 * p, *w = vb + 3 * q;
                double s = u[0] + w[0];
                s = orc_logAdd(s, u[1] + w[1]);
                s = orc_logAdd(s, u[2] + w[2]);
                cellTotal = orc_logAdd(cellTotal, s);
            }
        }
        total = orc_logAdd(total, cellTotal);
    }
    return total;
}

/* diagonalCalculationTotalProbability (pairwiseAligner.c:1182-1200): the dot product on xay plus
 * the matches that jump from xay-1 over xay into xay+1 */
static double orc_total_prob(orc_dp *dp, int64_t xay, int have_b_next, orc_diag *scratch) {
    double total = orc_diag_dot(dp, xay, &dp->F[xay], &dp->B[xay]);
    if (xay >= 1 && have_b_next && dp->F[xay - 1].live) {
        orc_diag *bn = &dp->B[xay + 1];
        /* scratch has the geometry of B[xay+1] */
        orc_diag_fill(scratch, ORC_LOG_ZERO, ORC_LOG_ZERO, ORC_LOG_ZERO);
        scratch->live = 1;
        orc_diag_calc(dp, xay + 1, scratch, NULL, &dp->F[xay - 1], 1);
        total = orc_logAdd(total, orc_diag_dot(dp, xay + 1, scratch, bn));
    }
    return total;
}

/* diagonalCalculationPosteriorMatchProbs (pairwiseAligner.c:1202-1253) */
static int orc_posteriors(orc_dp *dp, int64_t xay, double total, double threshold, orc_pair *out,
                          int64_t *n_out, int64_t max_out, int64_t ox, int64_t oy) {
    const orc_paths *P = dp->P;
    orc_diag *f = &dp->F[xay], *b = &dp->B[xay];
    for (int64_t xmy = f->xmyL; xmy <= f->xmyR; xmy += 2) {
        int64_t x = orc_xcoord(xay, xmy), y = orc_ycoord(xay, xmy);
        if (!(x > 0 && y > 0)) continue;
        int64_t c0 = P->pos[x].first, nc = P->pos[x].n_paths;
        double *vf = orc_cell(f, xmy), *vb = orc_cell(b, xmy);
        for (int64_t p = 0; p < nc; p++) {
            for (int64_t q = 0; q < nc; q++) {
                if (!orc_same(P, c0 + p, c0 + q)) continue;
                double pp = exp((vf[3 * p + S_MATCH] + vb[3 * q + S_MATCH]) - total);
                if (pp >= threshold) {
                    if (pp > 1.0) pp = 1.0;
                    if (*n_out >= max_out) return ORC_E_OVERFLOW;
                    orc_pair *o = out + (*n_out)++;
                    o->score = (int64_t) floor(pp * ORC_PAIR_PROB_1);
                    o->x = x - 1 + ox;
                    o->y = y - 1 + oy;
                    o->kmer = P->ids[c0 + p];
                }
            }
        }
    }
    return ORC_OK;
}

/* Expectations of a continuous pair HMM (continuousPairHmm_construct, continuousHmm.c:84-141):
 * transition expectations (from * 3 + to), per k-mer weighted event sums (mean, spread) and weights;
 * the caller initialises them (pseudocounts) */
typedef struct {
    double likelihood;
    double transitions[9];
    double *event_exp;          /* n_kmers x 2 */
    double *posteriors;         /* n_kmers */
    unsigned char *observed;    /* n_kmers */
    /* HDP machine (hdpHmm_makeExpectationsHmm, continuousHmm.c:788-795): instead of the emission
     * expectations, the (k-mer, event) of every match transition with posterior >= threshold */
    int hdp;
    double threshold;
    int64_t *assign_kmer, *assign_event, assign_cap, n_assign;
} orc_expect;

/* cell_signal_updateExpectations (pairwiseAligner.c:763-793): one transition of the cell's
 * calculation, its posterior added to the transition expectations and, into match, to the k-mer's
 * emission expectation (continuousPairHmm_addToEmissionExpectation, continuousHmm.c:160-169: the
 * spread uses the running mean, so the order of the updates matters) */
static void orc_expect_update(const orc_model *m, orc_expect *ex, double from_v, double to_v, int from, int to,
                              double e, double t, double total, int64_t kmer, const double *ev, int64_t event) {
    double p = exp(from_v + to_v + (e + t) - total);
    ex->transitions[from * 3 + to] += p;
    if (to == S_MATCH && ex->hdp) {
        /* cell_signal_updateExpectationsAndAssignments (pairwiseAligner.c:795-817) */
        if (p >= ex->threshold) {
            if (ex->n_assign < ex->assign_cap) {
                ex->assign_kmer[ex->n_assign] = kmer;
                ex->assign_event[ex->n_assign] = event;
            }
            ex->n_assign++;
        }
    } else if (to == S_MATCH) {
        double mu = m->match[kmer * 5];
        double x = (ev[0] + m->var * mu - m->scale * mu - m->shift) / m->var;
        ex->event_exp[2 * kmer] += p * x;
        ex->posteriors[kmer] += p;
        double uk = ex->event_exp[2 * kmer] / ex->posteriors[kmer];
        ex->event_exp[2 * kmer + 1] += p * (x - uk) * (x - uk);
        ex->observed[kmer] = 1;
    }
}

/* diagonalCalculation_Expectations (pairwiseAligner.c:1255-1275): the likelihood takes the diagonal's
 * total; the cells of B[xay] in ascending xmy are recalculated against the forward neighbours
 * (lower and upper F[xay-1], middle F[xay-2]) in stateMachine3_cellCalculate's order, each
 * transition reported to orc_expect_update.  The reference frees a forward diagonal after its last
 * posterior use (pairwiseAligner.c:1384-1387), so in a window traced back to T the middle
 * neighbours of xay = T+1 (F[T-1]) are gone and their transitions are skipped.  Single-path cells
 * only. */
static void orc_expect_diag(orc_dp *dp, int64_t xay, double total, orc_expect *ex, int64_t traced_back_to,
                            int64_t oy) {
    const orc_model *m = dp->m;
    const orc_paths *P = dp->P;
    const double *t = m->t;
    ex->likelihood += total;
    orc_diag *b = &dp->B[xay];
    for (int64_t xmy = b->xmyL; xmy <= b->xmyR; xmy += 2) {
        int64_t x = orc_xcoord(xay, xmy), y = orc_ycoord(xay, xmy);
        double *cur = orc_cell(b, xmy);
        double *lo = xay >= 1 ? orc_cell(&dp->F[xay - 1], xmy - 1) : NULL;
        double *mi = xay - 2 >= traced_back_to ? orc_cell(&dp->F[xay - 2], xmy) : NULL;
        double *up = xay >= 1 ? orc_cell(&dp->F[xay - 1], xmy + 1) : NULL;
        int64_t kid = P->ids[P->pos[x].first];
        const double *ev = orc_event(dp, y);
        if (lo) {
            double e = orc_emit_gapx(m, kid);
            orc_expect_update(m, ex, lo[S_MATCH], cur[S_GAPX], S_MATCH, S_GAPX, e, t[T_GAP_OPEN_X], total, kid, ev, y - 1 + oy);
            orc_expect_update(m, ex, lo[S_GAPX], cur[S_GAPX], S_GAPX, S_GAPX, e, t[T_GAP_EXTEND_X], total, kid, ev, y - 1 + oy);
            orc_expect_update(m, ex, lo[S_GAPY], cur[S_GAPX], S_GAPY, S_GAPX, e, t[T_GAP_SWITCH_TO_X], total, kid, ev, y - 1 + oy);
        }
        if (mi) {
            double e = orc_emit_event(m, kid, ev, 1);
            orc_expect_update(m, ex, mi[S_MATCH], cur[S_MATCH], S_MATCH, S_MATCH, e, t[T_MATCH_CONTINUE], total, kid, ev, y - 1 + oy);
            orc_expect_update(m, ex, mi[S_GAPX], cur[S_MATCH], S_GAPX, S_MATCH, e, t[T_MATCH_FROM_GAP_X], total, kid, ev, y - 1 + oy);
            orc_expect_update(m, ex, mi[S_GAPY], cur[S_MATCH], S_GAPY, S_MATCH, e, t[T_MATCH_FROM_GAP_Y], total, kid, ev, y - 1 + oy);
        }
        if (up) {
            double e = orc_emit_event(m, kid, ev, 0);
            orc_expect_update(m, ex, up[S_MATCH], cur[S_GAPY], S_MATCH, S_GAPY, e, t[T_GAP_OPEN_Y], total, kid, ev, y - 1 + oy);
            orc_expect_update(m, ex, up[S_GAPY], cur[S_GAPY], S_GAPY, S_GAPY, e, t[T_GAP_EXTEND_Y], total, kid, ev, y - 1 + oy);
        }
    }
}

static void orc_dp_free(orc_dp *dp) {
    if (dp->F) for (int64_t i = 0; i <= dp->n; i++) { free(dp->F[i].poff); free(dp->F[i].v); }
    if (dp->B) for (int64_t i = 0; i <= dp->n; i++) { free(dp->B[i].poff); free(dp->B[i].v); }
    free(dp->F); free(dp->B);
}

static int orc_dp_init(orc_dp *dp, const orc_model *m, const orc_paths *P, const double *events, int64_t lY,
                       const int64_t *xmyL, const int64_t *xmyR) {
    memset(dp, 0, sizeof(*dp));
    dp->m = m; dp->P = P; dp->events = events; dp->lY = lY; dp->n = P->lX + lY;
    dp->F = (orc_diag *) calloc((size_t) dp->n + 1, sizeof(orc_diag));
    dp->B = (orc_diag *) calloc((size_t) dp->n + 1, sizeof(orc_diag));
    if (!dp->F || !dp->B) return ORC_E_NOMEM;
    for (int64_t d = 0; d <= dp->n; d++) {
        int rc = orc_diag_alloc(&dp->F[d], d, xmyL[d], xmyR[d], P);
        if (rc) return rc;
        rc = orc_diag_alloc(&dp->B[d], d, xmyL[d], xmyR[d], P);
        if (rc) return rc;
    }
    return ORC_OK;
}

/* getPosteriorProbsWithBanding (pairwiseAligner.c:1282-1420) for one region.  Optional outputs:
 * the total probability of every refresh as (xay, P) pairs. */
static int orc_banded_region(const orc_model *m, const char *seq, int64_t lX, const double *events, int64_t lY,
                             const int64_t *anchors, int64_t n_anchors, const orc_params *p,
                             int ragged_left, int ragged_right, const char *options, int nopt,
                             orc_pair *out, int64_t *n_out, int64_t max_out, int64_t ox, int64_t oy,
                             double *tp_out, int64_t *n_tp, int64_t max_tp, orc_expect *ex) {
    int64_t n = lX + lY;
    if (n == 0) return ORC_OK;
    if (p->traceback_diagonals < 1 || p->diagonal_expansion < 0 || p->diagonal_expansion % 2 != 0 ||
        p->min_diags_between_traceback < 2 || !(p->traceback_diagonals + 1 < p->min_diags_between_traceback))
        return ORC_E_ARG;
    int64_t *xl = (int64_t *) malloc((size_t) (n + 1) * sizeof(int64_t));
    int64_t *xr = (int64_t *) malloc((size_t) (n + 1) * sizeof(int64_t));
    if (!xl || !xr) { free(xl); free(xr); return ORC_E_NOMEM; }
    int rc = orc_band(anchors, n_anchors, lX, lY, p->diagonal_expansion, xl, xr);
    orc_paths P; memset(&P, 0, sizeof(P));
    orc_dp dp; memset(&dp, 0, sizeof(dp));
    orc_diag scratch; memset(&scratch, 0, sizeof(scratch));
    if (rc) goto done;
    rc = orc_paths_build(&P, seq, lX, m->kmer_length, options, nopt, m);
    if (rc) goto done;
    rc = orc_dp_init(&dp, m, &P, events, lY, xl, xr);
    if (rc) goto done;

    double s[3];
    orc_start_probs(m, ragged_left, s);
    orc_diag_fill(&dp.F[0], s[0], s[1], s[2]);
    dp.F[0].live = 1;
    int64_t traced_back_to = 0;
    for (int64_t d = 1; d <= n; d++) {
        orc_diag *f = &dp.F[d];
        orc_diag_fill(f, ORC_LOG_ZERO, ORC_LOG_ZERO, ORC_LOG_ZERO);
        f->live = 1;
        orc_diag_calc(&dp, d, f, &dp.F[d - 1], d >= 2 ? &dp.F[d - 2] : NULL, 1);
        int at_end = d == n;
        int tb = d >= traced_back_to + p->min_diags_between_traceback &&
                 f->ncell <= p->diagonal_expansion * 2 + 1;
        if (!(at_end || tb)) continue;
        /* backward matrix for this window: B[d] is an end point, B[traced_back_to+1 .. d-1] start at zero,
         * B[traced_back_to] and below do not exist */
        orc_end_probs(m, at_end && ragged_right, s);
        orc_diag_fill(&dp.B[d], s[0], s[1], s[2]);
        dp.B[d].live = 1;
        for (int64_t j = traced_back_to + 1; j < d; j++) {
            orc_diag_fill(&dp.B[j], ORC_LOG_ZERO, ORC_LOG_ZERO, ORC_LOG_ZERO);
            dp.B[j].live = 1;
        }
        for (int64_t j = 0; j <= traced_back_to; j++) dp.B[j].live = 0;
        int64_t traced_back_from = d - (at_end ? 0 : p->traceback_diagonals + 1);
        double total = ORC_LOG_ZERO;
        int64_t k = 0;
        for (int64_t d2 = d; d2 > traced_back_to; d2--) {
            if (d2 > traced_back_to + 1)
                orc_diag_calc(&dp, d2, &dp.B[d2], &dp.B[d2 - 1], d2 - 2 > traced_back_to ? &dp.B[d2 - 2] : NULL, 0);
            if (d2 <= traced_back_from) {
                if (k++ % 10 == 0) {
                    int have_next = d2 < d;
                    if (have_next) {
                        free(scratch.poff); free(scratch.v);
                        rc = orc_diag_alloc(&scratch, d2 + 1, dp.B[d2 + 1].xmyL, dp.B[d2 + 1].xmyR, &P);
                        if (rc) goto done;
                    }
                    total = orc_total_prob(&dp, d2, have_next, &scratch);
                    if (tp_out && *n_tp < max_tp) {
                        tp_out[2 * *n_tp] = (double) (d2 + ox + oy);
                        tp_out[2 * *n_tp + 1] = total;
                        (*n_tp)++;
                    }
                }
                if (ex) orc_expect_diag(&dp, d2, total, ex, traced_back_to, oy);
                else rc = orc_posteriors(&dp, d2, total, p->threshold, out, n_out, max_out, ox, oy);
                if (rc) goto done;
            }
        }
        for (int64_t j = traced_back_to + 1; j <= d; j++) dp.B[j].live = 0;
        traced_back_to = traced_back_from;
        if (at_end) break;
    }
done:
    free(scratch.poff); free(scratch.v);
    orc_dp_free(&dp);
    orc_paths_free(&P);
    free(xl); free(xr);
    return rc;
}

/* getAlignedPairsUsingAnchors -> getPosteriorProbsWithBandingSplittingAlignmentsByLargeGaps
 * (pairwiseAligner.c:1773-1837, 1871-1899).  seq is the reference nucleotide string, lX the
 * number of k-mers in it.  Returns ORC_OK and fills out[0..*n_out). */
static int orc_split_run(const orc_model *m, const char *seq, int64_t lX, const double *events, int64_t lY,
                         const int64_t *anchors, int64_t n_anchors, const orc_params *p,
                         int ragged_left, int ragged_right, const char *options,
                         orc_pair *out, int64_t max_out, int64_t *n_out,
                         double *tp_out, int64_t max_tp, int64_t *n_tp, orc_expect *ex);

int orc_aligned_pairs(const orc_model *m, const char *seq, int64_t lX, const double *events, int64_t lY,
                      const int64_t *anchors, int64_t n_anchors, const orc_params *p,
                      int ragged_left, int ragged_right, const char *options,
                      orc_pair *out, int64_t max_out, int64_t *n_out,
                      double *tp_out, int64_t max_tp, int64_t *n_tp) {
    return orc_split_run(m, seq, lX, events, lY, anchors, n_anchors, p, ragged_left, ragged_right, options, out,
                         max_out, n_out, tp_out, max_tp, n_tp, NULL);
}

/* getExpectationsUsingAnchors (pairwiseAligner.c:1983-2003): the banded routine with
 * diagonalCalculation_Expectations in place of the posterior callback.  The expectation arrays are
 * the caller's (initialised with its pseudocounts); canonical references only (no 'X'). */
int orc_expectations(const orc_model *m, const char *seq, int64_t lX, const double *events, int64_t lY,
                     const int64_t *anchors, int64_t n_anchors, const orc_params *p, int ragged_left,
                     int ragged_right, double *likelihood, double *transitions, double *event_exp,
                     double *posteriors, unsigned char *observed, int64_t *assign_kmer, int64_t *assign_event,
                     int64_t assign_cap, int64_t *n_assign) {
    orc_expect ex;
    ex.hdp = m->emission == ORC_EMIT_HDP;
    ex.threshold = p->threshold;
    ex.assign_kmer = assign_kmer;
    ex.assign_event = assign_event;
    ex.assign_cap = assign_cap;
    ex.n_assign = *n_assign;
    ex.likelihood = *likelihood;
    for (int i = 0; i < 9; i++) ex.transitions[i] = transitions[i];
    ex.event_exp = event_exp;
    ex.posteriors = posteriors;
    ex.observed = observed;
    int64_t n_out = 0;
    int rc = orc_split_run(m, seq, lX, events, lY, anchors, n_anchors, p, ragged_left, ragged_right, "CEO", NULL, 0,
                           &n_out, NULL, 0, NULL, &ex);
    *likelihood = ex.likelihood;
    for (int i = 0; i < 9; i++) transitions[i] = ex.transitions[i];
    *n_assign = ex.n_assign;
    return rc;
}

static int orc_split_run(const orc_model *m, const char *seq, int64_t lX, const double *events, int64_t lY,
                         const int64_t *anchors, int64_t n_anchors, const orc_params *p,
                         int ragged_left, int ragged_right, const char *options,
                         orc_pair *out, int64_t max_out, int64_t *n_out,
                         double *tp_out, int64_t max_tp, int64_t *n_tp, orc_expect *ex) {
    *n_out = 0;
    if (n_tp) *n_tp = 0;
    int64_t n_tp_local = 0;
    int nopt = (int) strlen(options);
    int64_t max_split = n_anchors + 2;
    int64_t *splits = (int64_t *) malloc((size_t) max_split * 4 * sizeof(int64_t));
    if (!splits) return ORC_E_NOMEM;
    int64_t ns = orc_split_points(anchors, n_anchors, lX, lY, p->split_matrix_bigger_than_this,
                                  ragged_left, ragged_right, splits, max_split);
    if (ns < 0) { free(splits); return (int) -ns; }
    int64_t j = 0;
    int rc = ORC_OK;
    int64_t *sub = (int64_t *) malloc((size_t) (n_anchors + 1) * 2 * sizeof(int64_t));
    if (!sub) { free(splits); return ORC_E_NOMEM; }
    for (int64_t i = 0; i < ns && rc == ORC_OK; i++) {
        int64_t x1 = splits[4 * i], y1 = splits[4 * i + 1], x2 = splits[4 * i + 2], y2 = splits[4 * i + 3];
        int64_t nsub = 0;
        while (j < n_anchors) {
            int64_t x = anchors[2 * j], y = anchors[2 * j + 1];
            if (x + y >= x2 + y2) break;
            if (!(x >= x1 && x < x2 && y >= y1 && y < y2)) { rc = ORC_E_ANCHORS; break; }
            sub[2 * nsub] = x - x1; sub[2 * nsub + 1] = y - y1; nsub++;
            j++;
        }
        if (rc) break;
        rc = orc_banded_region(m, seq + x1, x2 - x1, events + y1 * ORC_NB_EVENT_PARAMS, y2 - y1, sub, nsub, p,
                               ragged_left || i > 0, ragged_right || i < ns - 1, options, nopt,
                               out, n_out, max_out, x1, y1, tp_out, n_tp ? n_tp : &n_tp_local, max_tp, ex);
    }
    if (rc == ORC_OK && j != n_anchors) rc = ORC_E_ANCHORS;
    free(sub);
    free(splits);
    return rc;
}

/* getAlignedPairsWithoutBanding (pairwiseAligner.c:1923-1981) and the toy full-matrix DP of
 * stateMachineTests.c:443-563.  p_mode 0: posteriors normalised by the total probability of the
 * last diagonal (the library routine); p_mode 1: by the forward total at the end cell (the toy
 * test).  Also returns the forward total, the backward total and the total probability of every
 * diagonal (diag_tp, n+1 values, may be NULL). */
int orc_full_matrix(const orc_model *m, const char *seq, int64_t lX, const double *events, int64_t lY,
                    double threshold, int ragged_left, int ragged_right, const char *options, int p_mode,
                    orc_pair *out, int64_t max_out, int64_t *n_out,
                    double *fwd_total, double *bwd_total, double *diag_tp) {
    *n_out = 0;
    int64_t n = lX + lY;
    int64_t *xl = (int64_t *) malloc((size_t) (n + 1) * sizeof(int64_t));
    int64_t *xr = (int64_t *) malloc((size_t) (n + 1) * sizeof(int64_t));
    orc_paths P; memset(&P, 0, sizeof(P));
    orc_dp dp; memset(&dp, 0, sizeof(dp));
    orc_diag scratch; memset(&scratch, 0, sizeof(scratch));
    int rc = (!xl || !xr) ? ORC_E_NOMEM : orc_band(NULL, 0, lX, lY, 2, xl, xr);
    if (rc) goto done;
    rc = orc_paths_build(&P, seq, lX, m->kmer_length, options, (int) strlen(options), m);
    if (rc) goto done;
    rc = orc_dp_init(&dp, m, &P, events, lY, xl, xr);
    if (rc) goto done;
    for (int64_t d = 0; d <= n; d++) {
        orc_diag_fill(&dp.F[d], ORC_LOG_ZERO, ORC_LOG_ZERO, ORC_LOG_ZERO); dp.F[d].live = 1;
        orc_diag_fill(&dp.B[d], ORC_LOG_ZERO, ORC_LOG_ZERO, ORC_LOG_ZERO); dp.B[d].live = 1;
    }
    double s[3];
    orc_start_probs(m, ragged_left, s);
    orc_diag_fill(&dp.F[0], s[0], s[1], s[2]);
    orc_end_probs(m, ragged_right, s);
    orc_diag_fill(&dp.B[n], s[0], s[1], s[2]);
    for (int64_t d = 1; d <= n; d++)
        orc_diag_calc(&dp, d, &dp.F[d], &dp.F[d - 1], d >= 2 ? &dp.F[d - 2] : NULL, 1);
    for (int64_t d = n; d > 0; d--)
        orc_diag_calc(&dp, d, &dp.B[d], &dp.B[d - 1], d >= 2 ? &dp.B[d - 2] : NULL, 0);
    /* forward total at the end cell, backward total at the start cell (cell_dotProduct2) */
    {
        double e[3], st[3];
        orc_end_probs(m, 0, e);
        orc_start_probs(m, 0, st);
        double tf = ORC_LOG_ZERO, tb = ORC_LOG_ZERO;
        double *cf = orc_cell(&dp.F[n], lX - lY);
        int64_t nc = P.pos[lX].n_paths;
        for (int64_t q = 0; q < nc; q++) {
            double *v = cf + 3 * q;
            double s2 = v[0] + e[0];
            s2 = orc_logAdd(s2, v[1] + e[1]);
            s2 = orc_logAdd(s2, v[2] + e[2]);
            tf = orc_logAdd(tf, s2);
        }
        double *cb = orc_cell(&dp.B[0], 0);
        double s2 = cb[0] + st[0];
        s2 = orc_logAdd(s2, cb[1] + st[1]);
        s2 = orc_logAdd(s2, cb[2] + st[2]);
        tb = orc_logAdd(tb, s2);
        if (fwd_total) *fwd_total = tf;
        if (bwd_total) *bwd_total = tb;
    }
    if (diag_tp) {
        for (int64_t d = 0; d <= n; d++) {
            int have_next = d < n;
            if (have_next) {
                free(scratch.poff); free(scratch.v);
                rc = orc_diag_alloc(&scratch, d + 1, dp.B[d + 1].xmyL, dp.B[d + 1].xmyR, &P);
                if (rc) goto done;
            }
            diag_tp[d] = orc_total_prob(&dp, d, have_next, &scratch);
        }
    }
    double total;
    if (p_mode == 1) total = *fwd_total;
    else total = orc_total_prob(&dp, n, 0, &scratch);
    for (int64_t d = (p_mode == 1 ? 1 : 0); d <= n && rc == ORC_OK; d++)
        rc = orc_posteriors(&dp, d, total, threshold, out, n_out, max_out, 0, 0);
done:
    free(scratch.poff); free(scratch.v);
    orc_dp_free(&dp);
    orc_paths_free(&P);
    free(xl); free(xr);
    return rc;
}

/* exported helpers for tests */
double orc_emission(const orc_model *m, int64_t kmer_id, double mean, double noise, int match) {
    double ev[2] = { mean, noise };
    return orc_emit_event(m, kmer_id, ev, match);
}

double orc_log_gauss_pdf(double x, double mu, double sigma) { return orc_log_gauss(x, mu, sigma); }
double orc_log_inv_gauss_pdf(double x, double mu, double lambda) { return orc_log_inv_gauss(x, mu, lambda); }

int64_t orc_kmer_index(const char *kmer, int k, const char *alphabet, int asz) {
    return orc_kmer_id(kmer, k, alphabet, asz);
}

/* hdCell path expansion for one k-mer (test_hdCellConstruct): writes n_paths x k chars */
int64_t orc_expand_kmer(const char *kmer, int k, const char *options, char *out, int64_t max_paths) {
    int nopt = (int) strlen(options), degen[ORC_MAX_K], nd = 0;
    for (int i = 0; i < k; i++) if (kmer[i] == 'X') degen[nd++] = i;
    int64_t np = 1;
    for (int i = 0; i < nd; i++) np *= nopt;
    if (np > max_paths) return -1;
    for (int64_t p = 0; p < np; p++) {
        char *dst = out + p * k;
        memcpy(dst, kmer, (size_t) k);
        int64_t rem = p;
        for (int i = nd - 1; i >= 0; i--) { dst[degen[i]] = options[rem % nopt]; rem /= nopt; }
    }
    return np;
}

/* Forgetting of the forward start (test infrastructure for the GPU form's forward segments): the
 * forward sweep of getPosteriorProbsWithBanding (pairwiseAligner.c:1310-1325) from anti-diagonal 0,
 * and, for each start s in starts, the same sweep begun at s from a flat vector (anti-diagonals
 * s-2 and s-1 all 0 in every state of every band cell).  logAdd depends only on the difference of
 * its arguments, so a sweep's values shifted by a constant stay shifted by it.  steps_out[k] is the
 * number of anti-diagonals after s from which on, up to s + horizon (or the end), both sweeps have
 * the same -inf cells and every finite difference lies within tol of the others on the same
 * anti-diagonal; -1 if that never holds. */
int orc_flat_start_forgetting(const orc_model *m, const char *seq, int64_t lX, const double *events, int64_t lY,
                              const int64_t *anchors, int64_t n_anchors, int64_t expansion, int ragged_left,
                              const char *options, const int64_t *starts, int64_t n_starts, int64_t horizon,
                              double tol, int64_t *steps_out) {
    int64_t n = lX + lY;
    int64_t *xl = (int64_t *) malloc((size_t) (n + 1) * sizeof(int64_t));
    int64_t *xr = (int64_t *) malloc((size_t) (n + 1) * sizeof(int64_t));
    orc_paths P; memset(&P, 0, sizeof(P));
    orc_dp dp; memset(&dp, 0, sizeof(dp));
    int rc = !xl || !xr ? ORC_E_NOMEM : orc_band(anchors, n_anchors, lX, lY, expansion, xl, xr);
    if (!rc) rc = orc_paths_build(&P, seq, lX, m->kmer_length, options, (int) strlen(options), m);
    if (!rc) rc = orc_dp_init(&dp, m, &P, events, lY, xl, xr);
    if (rc) goto done;
    double s0[3];
    orc_start_probs(m, ragged_left, s0);
    orc_diag_fill(&dp.F[0], s0[0], s0[1], s0[2]);
    dp.F[0].live = 1;
    for (int64_t d = 1; d <= n; d++) {
        orc_diag_fill(&dp.F[d], ORC_LOG_ZERO, ORC_LOG_ZERO, ORC_LOG_ZERO);
        dp.F[d].live = 1;
        orc_diag_calc(&dp, d, &dp.F[d], &dp.F[d - 1], d >= 2 ? &dp.F[d - 2] : NULL, 1);
    }
    /* the flat-start sweeps use the backward store */
    for (int64_t k = 0; k < n_starts; k++) {
        int64_t st = starts[k], last_bad = -1, end = st + horizon < n ? st + horizon : n;
        steps_out[k] = -1;
        if (st < 2 || st > n) continue;
        orc_diag_fill(&dp.B[st - 2], 0, 0, 0); dp.B[st - 2].live = 1;
        orc_diag_fill(&dp.B[st - 1], 0, 0, 0); dp.B[st - 1].live = 1;
        for (int64_t d = st; d <= end; d++) {
            orc_diag_fill(&dp.B[d], ORC_LOG_ZERO, ORC_LOG_ZERO, ORC_LOG_ZERO);
            dp.B[d].live = 1;
            orc_diag_calc(&dp, d, &dp.B[d], &dp.B[d - 1], &dp.B[d - 2], 1);
            int64_t nv = 3 * dp.F[d].poff[dp.F[d].ncell];
            double lo = INFINITY, hi = -INFINITY;
            int bad = 0;
            for (int64_t i = 0; i < nv; i++) {
                double a = dp.F[d].v[i], b = dp.B[d].v[i];
                int fa = a > -1e300, fb = b > -1e300;
                if (fa != fb) { bad = 1; break; }
                if (!fa) continue;
                lo = a - b < lo ? a - b : lo;
                hi = a - b > hi ? a - b : hi;
            }
            if (bad || hi - lo > tol) last_bad = d;
        }
        steps_out[k] = last_bad < end ? last_bad + 1 - st : -1;
        for (int64_t d = st - 2; d <= end; d++) dp.B[d].live = 0;
    }
done:
    orc_dp_free(&dp);
    orc_paths_free(&P);
    free(xl); free(xr);
    return rc;
}
