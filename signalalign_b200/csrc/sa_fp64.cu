// Plain FP64 form: one region (read, or split sub-region) per CTA, sweeping the
// band anti-diagonal by anti-diagonal in log space with the reference's logAdd, windowed traceback
// and every-10th-anti-diagonal total-probability refresh (getPosteriorProbsWithBanding,
// pairwiseAligner.c:1282-1420).  It is the parity anchor of the engine: results agree with
// signalAlign's CPU code to rounding.  Compiled with -fmad=false.
//
// Plain sets: every region of every read of a set is one CTA of one launch.  Device layout of a
// region (all global memory).  A matrix column x holds one path per k-mer its reference window can
// spell (one, unless the window has 'X' positions: hdCell_construct, pairwiseAligner.c:605-650); a
// band cell holds one slot of 3 states per path of its column.
//   xl[d], xr[d]     band of anti-diagonal d (xmy range), d = 0..n
//   pfirst[x]        first path of column x (x = 0 is the empty prefix, one NULL path), lX+2 entries
//   pid[q]           k-mer id of path q (-1 for NULL); ppre[q] = id / |alphabet|, psuf[q] =
//                    id mod |alphabet|^(k-1): path q -> r is legal iff psuf[q] == ppre[r] (path_checkLegal)
//   ev[y]            (mean, noise) of event y, lY entries
//   F, B             3 doubles per slot (match, gap-X, gap-Y), forward and backward, in rings of
//                    `ring` anti-diagonals of `stride` slots: a traceback window [T, D] reads F and B
//                    on T .. D only, and ring > D - T for every window (the reference also keeps only
//                    the current window's forward diagonals, pairwiseAligner.c:1390-1410).  The
//                    paths of one anti-diagonal are consecutive (x rises by one from cell to cell).
//   row[d]           (d mod ring) * stride - first path of anti-diagonal d: slot of path q on d is
//                    row[d] + q
//   E                2 doubles per slot (match and extra-event emissions), a ring like F, written by
//                    the forward sweep where it needs them and read back by the backward sweep, the
//                    refresh totals and the expectations
//   P                refresh total probabilities, indexed by anti-diagonal
//   out, tag         the set's pairs (shared, appended by atomics) and each pair's region
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "sa_dp64.cuh"
#include "sa_internal.h"

namespace sa {
namespace {

using namespace dp64;

enum { S_M = 0, S_X = 1, S_Y = 2 };
enum { T_MC = 0, T_MFGX, T_MFGY, T_OX, T_OY, T_EX, T_EY, T_SX, T_SY };

struct Region64 {
    int32_t lX, lY, n, n_windows;
    int32_t ragged_left, ragged_right;
    int32_t model, ring, stride, pad;
    // Forward segments of a long region (alignment runs): this task sweeps from anti-diagonal s0
    // (1 for the region's first segment, which starts from the start probabilities; a later
    // segment starts from a flat vector, every cell 0, on s0-2 and s0-1) and runs windows w0 .. w1-1;
    // stitches where it meets its neighbours (-1: none); pairs are tagged with region `tag`
    int32_t s0, w0, w1, tag, st_in, st_out;
    int64_t ev_base;              // the region's first event in the read (split regions start later)
    const int32_t *xl, *xr;
    const int32_t *pfirst, *pid, *ppre, *psuf;
    const int32_t *row;           // per anti-diagonal d: (d mod ring) * stride - its first path slot
    const double2 *ev;
    const Window *win;
    double *F, *B, *P;
    double *E;                    // ring like F: per path slot the match and extra-event emissions
                                  // the forward sweep computed (the backward sweep reuses them)
    double threshold;
    double *loglik;
    int32_t *status;
};

// where two forward segments of a region meet, at anti-diagonal b (the later one's first window's T):
// the values of every path slot of b-1 and b, from both sides (4 blocks of stride x 3 doubles:
// later b-1, later b, earlier b-1, earlier b), and the read it belongs to
struct Stitch64 {
    double *vals;
    int32_t b, region, stride, pad;
};
struct Stitch64Res {        // cleared before every run
    double delta;           // earlier-side value - later-side value (the constant)
    double spread;          // largest deviation from it over the slots
    int32_t arrive, result; // sides that wrote their values; 1 agreed, 2 disagreed
};

struct SetOut {
    sa_aligned_pair *out;
    int32_t *tag;
    unsigned long long *count;
    int64_t cap;
    const Stitch64 *stitch;   // alignment runs with forward segments
    Stitch64Res *stres;
    int32_t *fail;            // per region: a stitch disagreed
    double stitch_tol;        // tolerance scale (negative: every stitch disagrees)
};

// Expectations mode (getExpectationsUsingAnchors, pairwiseAligner.c:1983-2003): one CTA walks the
// read's regions in order and folds every transition posterior into a continuous pair HMM's
// accumulators in the reference's order (their emission spreads depend on it).
constexpr int kExpectScratch = 9;   // doubles of expectations scratch per cell

struct ExpectOut {
    int32_t on, n_regions;
    int32_t first_region, pad0;   // the read's regions: first_region .. first_region + n_regions - 1
    double *scratch;            // per cell of the anti-diagonal at hand: 8 transition posteriors and
                                // the descaled event mean
    int32_t *mask;              // per cell: lower / middle / upper neighbour present, k-mer id + 1
    double *acc;                // likelihood, then the 3 x 3 transition expectations
    double *event_exp;          // per k-mer: weighted mean sum, weighted spread sum
    double *posteriors;         // per k-mer: weight
    unsigned char *observed;    // per k-mer
    // HDP machine: (k-mer, event) of each match transition with posterior >= threshold instead
    int32_t hdp, pad;
    double threshold;
    int64_t *assign_kmer, *assign_event, *n_assign;
    int64_t assign_cap;
};

// the 3 states of path q in the cell of anti-diagonal d (q must belong to that cell's column)
__device__ __forceinline__ double *slot(double *base, const Region64 &R, int32_t d, int32_t q) {
    return base + 3 * ((int64_t) R.row[d] + q);
}

// the match and extra-event emissions of path q's cell on anti-diagonal d, as the forward sweep
// computed them (only where it needed them: a middle or an upper neighbour present)
__device__ __forceinline__ double *eslot(const Region64 &R, int32_t d, int32_t q) {
    return R.E + 2 * ((int64_t) R.row[d] + q);
}

__device__ __forceinline__ bool in_band(const Region64 &R, int32_t d, int32_t xmy) {
    return d >= 0 && d <= R.n && xmy >= R.xl[d] && xmy <= R.xr[d];
}

// path_checkLegal (pairwiseAligner.c:527-552): NULL on either side, or the (k-1)-suffix of q equal
// to the (k-1)-prefix of r
__device__ __forceinline__ bool legal(const Region64 &R, int32_t q, int32_t r) {
    return R.pid[q] < 0 || R.pid[r] < 0 || R.psuf[q] == R.ppre[r];
}

// forward cell by pull: the reference's push order (lower -> gap-X, middle -> match, upper -> gap-Y,
// stateMachine3_cellCalculate, stateMachine.c:1194-1257) with each state accumulated from LOG_ZERO;
// path r of the cell takes every legal path q of the neighbour in ascending order, the upper
// neighbour (same column) only its own path
__device__ void forward_cell(const Model64 &M, const Region64 &R, int32_t d, int32_t xmy) {
    const int32_t x = (d + xmy) >> 1, y = (d - xmy) >> 1;
    const bool lo = in_band(R, d - 1, xmy - 1), mi = d >= 2 && in_band(R, d - 2, xmy), up = in_band(R, d - 1, xmy + 1);
    const int32_t q0 = R.pfirst[x - (x > 0)], q1 = R.pfirst[x];
    for (int32_t r = R.pfirst[x]; r < R.pfirst[x + 1]; ++r) {
        const int32_t kid = R.pid[r];
        double vM = kNegInf, vX = kNegInf, vY = kNegInf;
        if (lo) {
            const double e = emit_gapx(M, kid);
            for (int32_t q = q0; q < q1; ++q) {
                if (!legal(R, q, r)) continue;
                const double *l = slot(R.F, R, d - 1, q);
                vX = log_add(vX, l[S_M] + (e + M.t[T_OX]));
                vX = log_add(vX, l[S_X] + (e + M.t[T_EX]));
                vX = log_add(vX, l[S_Y] + (e + M.t[T_SX]));
            }
        }
        double *es = eslot(R, d, r);
        if (mi) {
            const double2 ev = R.ev[y - 1];
            const double e = emit_event(M, kid, ev.x, ev.y, true);
            es[0] = e;
            for (int32_t q = q0; q < q1; ++q) {
                if (!legal(R, q, r)) continue;
                const double *m = slot(R.F, R, d - 2, q);
                vM = log_add(vM, m[S_M] + (e + M.t[T_MC]));
                vM = log_add(vM, m[S_X] + (e + M.t[T_MFGX]));
                vM = log_add(vM, m[S_Y] + (e + M.t[T_MFGY]));
            }
        }
        if (up) {
            const double *u = slot(R.F, R, d - 1, r);
            const double2 ev = R.ev[y - 1];
            const double e = emit_event(M, kid, ev.x, ev.y, false);
            es[1] = e;
            vY = log_add(vY, u[S_M] + (e + M.t[T_OY]));
            vY = log_add(vY, u[S_Y] + (e + M.t[T_EY]));
        }
        double *c = slot(R.F, R, d, r);
        c[S_M] = vM;
        c[S_X] = vX;
        c[S_Y] = vY;
    }
}

// backward cell by pull.  The reference pushes from later cells into earlier ones
// (doTransitionBackward, pairwiseAligner.c:715-720); a cell on anti-diagonal d receives, in time
// order, the middle contribution of (x+1, y+1) on d+2, then the upper-role contribution of (x, y+1)
// and the lower-role contribution of (x+1, y), both on d+1 (cells there are walked in ascending xmy).
// Path r of the cell receives from every path p of the pushing cell that r may precede, in
// ascending p, each with p's emission.
__device__ void backward_cell(const Model64 &M, const Region64 &R, int32_t d, int32_t xmy, int32_t top) {
    const int32_t x = (d + xmy) >> 1;
    const bool mi = d + 2 <= top && in_band(R, d + 2, xmy), up = in_band(R, d + 1, xmy - 1),
               lo = in_band(R, d + 1, xmy + 1);
    // column x+1 exists whenever a cell of it is in the band
    const int32_t p0 = (mi || lo) ? R.pfirst[x + 1] : 0, p1 = (mi || lo) ? R.pfirst[x + 2] : 0;
    for (int32_t r = R.pfirst[x]; r < R.pfirst[x + 1]; ++r) {
        double vM = kNegInf, vX = kNegInf, vY = kNegInf;
        if (mi) {
            for (int32_t p = p0; p < p1; ++p) {
                if (!legal(R, r, p)) continue;
                const double *m = slot(R.B, R, d + 2, p);
                const double e = eslot(R, d + 2, p)[0];   // the forward sweep's match emission of p
                vM = log_add(vM, m[S_M] + (e + M.t[T_MC]));
                vX = log_add(vX, m[S_M] + (e + M.t[T_MFGX]));
                vY = log_add(vY, m[S_M] + (e + M.t[T_MFGY]));
            }
        }
        if (up) {
            const double *u = slot(R.B, R, d + 1, r);
            const double e = eslot(R, d + 1, r)[1];   // its extra-event emission
            vM = log_add(vM, u[S_Y] + (e + M.t[T_OY]));
            vY = log_add(vY, u[S_Y] + (e + M.t[T_EY]));
        }
        if (lo) {
            for (int32_t p = p0; p < p1; ++p) {
                if (!legal(R, r, p)) continue;
                const double *l = slot(R.B, R, d + 1, p);
                const double e = emit_gapx(M, R.pid[p]);
                vM = log_add(vM, l[S_X] + (e + M.t[T_OX]));
                vX = log_add(vX, l[S_X] + (e + M.t[T_EX]));
                vY = log_add(vY, l[S_X] + (e + M.t[T_SX]));
            }
        }
        double *c = slot(R.B, R, d, r);
        c[S_M] = vM;
        c[S_X] = vX;
        c[S_Y] = vY;
    }
}

// diagonalCalculationTotalProbability (pairwiseAligner.c:1182-1200), sequential in the reference's
// order: dot product of F and B on d in ascending xmy (a cell's paths folded first,
// hdCell_totalProbability), then the matches that jump from d-1 over d into d+1, dotted with B[d+1].
__device__ double total_probability(const Model64 &M, const Region64 &R, int32_t d, bool have_next) {
    double total = kNegInf;
    for (int32_t xmy = R.xl[d]; xmy <= R.xr[d]; xmy += 2) {
        const int32_t x = (d + xmy) >> 1;
        double cell_total = kNegInf;
        for (int32_t r = R.pfirst[x]; r < R.pfirst[x + 1]; ++r) {
            const double *f = slot(R.F, R, d, r), *b = slot(R.B, R, d, r);
            double s = f[S_M] + b[S_M];
            s = log_add(s, f[S_X] + b[S_X]);
            s = log_add(s, f[S_Y] + b[S_Y]);
            cell_total = log_add(cell_total, s);
        }
        total = log_add(total, cell_total);
    }
    if (d >= 1 && have_next) {
        const int32_t dn = d + 1;
        double through = kNegInf;
        for (int32_t xmy = R.xl[dn]; xmy <= R.xr[dn]; xmy += 2) {
            const int32_t x = (dn + xmy) >> 1;
            const bool mi = in_band(R, d - 1, xmy);
            double cell_total = kNegInf;
            for (int32_t r = R.pfirst[x]; r < R.pfirst[x + 1]; ++r) {
                double m = kNegInf;
                if (mi) {
                    const double e = eslot(R, dn, r)[0];   // the forward sweep's match emission
                    for (int32_t q = R.pfirst[x - 1]; q < R.pfirst[x]; ++q) {
                        if (!legal(R, q, r)) continue;
                        const double *f = slot(R.F, R, d - 1, q);
                        m = log_add(m, f[S_M] + (e + M.t[T_MC]));
                        m = log_add(m, f[S_X] + (e + M.t[T_MFGX]));
                        m = log_add(m, f[S_Y] + (e + M.t[T_MFGY]));
                    }
                }
                const double *b = slot(R.B, R, dn, r);
                double s = m + b[S_M];
                s = log_add(s, kNegInf + b[S_X]);
                s = log_add(s, kNegInf + b[S_Y]);
                cell_total = log_add(cell_total, s);
            }
            through = log_add(through, cell_total);
        }
        total = log_add(total, through);
    }
    return total;
}

// diagonalCalculation_Expectations (pairwiseAligner.c:1255-1275) on anti-diagonal d2 of a window
// traced back to T: the cells of B[d2] against their forward neighbours (the reference has freed
// F[T-1] by then, so the middle neighbours of d2 = T+1 are absent), each transition's posterior
// exp(F[from] + B[to] + (e + t) - total) (cell_signal_updateExpectations, :763-793), computed in
// parallel.  Then thread 0 adds the transition posteriors in stateMachine3_cellCalculate's order, cell
// by cell (and, for the HDP machine, appends the assignments in that order), while the other threads
// fold the match posteriors into the per-k-mer emission expectations
// (continuousPairHmm_addToEmissionExpectation, continuousHmm.c:160-169): k-mers are independent, and
// one k-mer's updates (a running mean, so order matters) are made by one thread in cell order.  The
// cells of an anti-diagonal lie in distinct columns, so a k-mer recurs on it only where the reference
// repeats it within the band; the first such cell's thread makes the updates of all of them.
__device__ void expect_diagonal(const Model64 &M, const Region64 &R, const ExpectOut &X, int32_t d2, int32_t T,
                                double total, double (&acc)[10]) {
    const int tid = threadIdx.x, nt = blockDim.x;
    double *const scratch = X.scratch;
    int32_t *const mask = X.mask;
    for (int32_t xmy = R.xl[d2] + 2 * tid; xmy <= R.xr[d2]; xmy += 2 * nt) {
        const int32_t c = (xmy - R.xl[d2]) >> 1;
        const int32_t x = (d2 + xmy) >> 1, y = (d2 - xmy) >> 1;
        const int32_t r = R.pfirst[x], kid = R.pid[r];
        const double *cur = slot(R.B, R, d2, r);
        const bool lo = in_band(R, d2 - 1, xmy - 1), mi = d2 - 2 >= T && in_band(R, d2 - 2, xmy),
                   up = in_band(R, d2 - 1, xmy + 1);
        double *ps = scratch + kExpectScratch * (int64_t) c;
        if (lo) {
            const double *l = slot(R.F, R, d2 - 1, R.pfirst[x - 1]);
            const double e = emit_gapx(M, kid);
            ps[0] = exp(l[S_M] + cur[S_X] + (e + M.t[T_OX]) - total);
            ps[1] = exp(l[S_X] + cur[S_X] + (e + M.t[T_EX]) - total);
            ps[2] = exp(l[S_Y] + cur[S_X] + (e + M.t[T_SX]) - total);
        }
        if (mi) {
            const double *m = slot(R.F, R, d2 - 2, R.pfirst[x - 1]);
            const double2 ev = R.ev[y - 1];
            const double e = eslot(R, d2, r)[0];   // the forward sweep's emissions of the cell
            ps[3] = exp(m[S_M] + cur[S_M] + (e + M.t[T_MC]) - total);
            ps[4] = exp(m[S_X] + cur[S_M] + (e + M.t[T_MFGX]) - total);
            ps[5] = exp(m[S_Y] + cur[S_M] + (e + M.t[T_MFGY]) - total);
            // the descaled event mean (emissions_signal_descaleEventMean_JordanStyle) with the
            // k-mer's level mean from the machine's match table
            const double mu = M.match[(int64_t) kid * 5];
            ps[8] = (ev.x + M.var * mu - M.scale * mu - M.shift) / M.var;
        }
        if (up) {
            const double *u = slot(R.F, R, d2 - 1, r);
            const double e = eslot(R, d2, r)[1];
            ps[6] = exp(u[S_M] + cur[S_Y] + (e + M.t[T_OY]) - total);
            ps[7] = exp(u[S_Y] + cur[S_Y] + (e + M.t[T_EY]) - total);
        }
        // neighbour flags in the low 3 bits, k-mer id + 1 above them (ids are below 2^27)
        mask[c] = (lo ? 1 : 0) | (mi ? 2 : 0) | (up ? 4 : 0) | ((kid + 1) << 3);
    }
    __syncthreads();
    const int32_t w = (R.xr[d2] - R.xl[d2]) / 2 + 1;
    if (tid == 0) {
        // the accumulators in registers for the pass; a cell's posteriors are loaded whether or not
        // its neighbours exist (unused values are never added), so loads of later cells need not
        // wait for earlier cells' branches
        double t[9];
        for (int i = 0; i < 9; ++i) t[i] = acc[1 + i];
        acc[0] += total;   // hmmExpectations->likelihood += totalProbability, once per diagonal
#pragma unroll 4
        for (int32_t c = 0; c < w; ++c) {
            const int32_t mk = mask[c];
            const double *ps = scratch + kExpectScratch * (int64_t) c;
            const double p0 = ps[0], p1 = ps[1], p2 = ps[2], p3 = ps[3], p4 = ps[4], p5 = ps[5], p6 = ps[6],
                         p7 = ps[7];
            if (mk & 1) {   // lower: M, X, Y -> X
                t[S_M * 3 + S_X] += p0;
                t[S_X * 3 + S_X] += p1;
                t[S_Y * 3 + S_X] += p2;
            }
            if (mk & 2) {   // middle: M, X, Y -> M
                t[S_M * 3 + S_M] += p3;
                t[S_X * 3 + S_M] += p4;
                t[S_Y * 3 + S_M] += p5;
            }
            if (mk & 4) {   // upper: M, Y -> Y
                t[S_M * 3 + S_Y] += p6;
                t[S_Y * 3 + S_Y] += p7;
            }
        }
        for (int i = 0; i < 9; ++i) acc[1 + i] = t[i];
        // cell_signal_updateExpectationsAndAssignments (pairwiseAligner.c:795-817): the HDP
        // machine's assignments, in cell order and, within a cell, from match, gap-X, gap-Y
        if (X.hdp) {
            for (int32_t c = 0; c < w; ++c) {
                const int32_t mk = mask[c];
                if (!(mk & 2)) continue;
                const double *ps = scratch + kExpectScratch * (int64_t) c;
                const int32_t xmy = R.xl[d2] + 2 * c;
                const int32_t y = (d2 - xmy) >> 1;
                const int64_t kid = (mk >> 3) - 1;
                for (int j = 0; j < 3; ++j) {
                    if (ps[3 + j] >= X.threshold) {
                        const int64_t at = *X.n_assign;
                        if (at < X.assign_cap) {
                            X.assign_kmer[at] = kid;
                            X.assign_event[at] = R.ev_base + y - 1;
                        }
                        *X.n_assign = at + 1;
                    }
                }
            }
        }
    } else if (!X.hdp) {
        for (int32_t c = tid - 1; c < w; c += nt - 1) {
            const int32_t mk = mask[c];
            if (!(mk & 2)) continue;
            const int32_t key = mk >> 3;
            // an earlier cell of the anti-diagonal with the same k-mer makes this cell's updates
            // (no early exit: the loads do not wait on one another)
            bool dup = false;
#pragma unroll 4
            for (int32_t c2 = 0; c2 < c; ++c2) {
                const int32_t m2 = mask[c2];
                dup |= (m2 & 2) != 0 && (m2 >> 3) == key;
            }
            if (dup) continue;
            const int64_t kid = key - 1;
            double e0 = X.event_exp[2 * kid], e1 = X.event_exp[2 * kid + 1], po = X.posteriors[kid];
            for (int32_t c2 = c; c2 < w; ++c2) {
                const int32_t m2 = mask[c2];
                if (!((m2 & 2) && (m2 >> 3) == key)) continue;
                const double *ps = scratch + kExpectScratch * (int64_t) c2;
                const double xe = ps[8];
                for (int j = 0; j < 3; ++j) {
                    const double p = ps[3 + j];
                    e0 += p * xe;
                    po += p;
                    const double uk = e0 / po;
                    e1 += p * (xe - uk) * (xe - uk);
                }
            }
            X.event_exp[2 * kid] = e0;
            X.event_exp[2 * kid + 1] = e1;
            X.posteriors[kid] = po;
            X.observed[kid] = 1;
        }
    }
    __syncthreads();
}

// One region: forward sweep, windowed traceback, and per traceback window either the posterior
// pairs or (expectations mode) the expectation updates.
// path slots of anti-diagonal d: the first slot (of its first cell) and their number
__device__ __forceinline__ void diag_slots(const Region64 &R, int32_t d, int32_t &first, int32_t &count) {
    first = R.pfirst[(d + R.xl[d]) >> 1];
    count = R.pfirst[((d + R.xr[d]) >> 1) + 1] - first;
}

// every path slot of anti-diagonal d set to `v` in all three states (whole CTA)
__device__ void fill_diag(double *ring, const Region64 &R, int32_t d, double v) {
    int32_t first, count;
    diag_slots(R, d, first, count);
    for (int32_t k = threadIdx.x; k < count; k += blockDim.x) {
        double *c = slot(ring, R, d, first + k);
        c[S_M] = v;
        c[S_X] = v;
        c[S_Y] = v;
    }
}

// the forward values of anti-diagonal d into block `blk` of stitch st's values (whole CTA)
__device__ void stitch_copy64(const Region64 &R, const SetOut &O, int32_t st, int32_t d, int blk) {
    const Stitch64 S = O.stitch[st];
    double *dst = S.vals + (int64_t) blk * 3 * S.stride;
    int32_t first, count;
    diag_slots(R, d, first, count);
    for (int32_t k = threadIdx.x; k < count; k += blockDim.x) {
        const double *c = slot(R.F, R, d, first + k);
        dst[3 * k] = c[S_M];
        dst[3 * k + 1] = c[S_X];
        dst[3 * k + 2] = c[S_Y];
    }
}

// Stitch st once both sides wrote their values (whole CTA, the side that arrives second): the same
// -inf slots, and every difference (earlier - later) within 1e-9 + 1e-11 x (its distance below the
// largest earlier value) of the difference at that value, which becomes the stitch's constant.
// FP64 sweeps from different starts agree to rounding once the start is forgotten.
__device__ void stitch_check64(const Region64 &R, const SetOut &O, int32_t st) {
    __shared__ double red_a[32], red_d[32];
    __shared__ int red_ok;
    const Stitch64 S = O.stitch[st];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = (blockDim.x + 31) >> 5;
    int32_t f0, c0, f1, c1;
    diag_slots(R, S.b - 1, f0, c0);
    diag_slots(R, S.b, f1, c1);
    const int64_t stride3 = 3 * (int64_t) S.stride;
    const double *later = S.vals, *earlier = S.vals + 2 * stride3;
    auto at = [&](const double *base, int32_t q, double &v) {   // q over both anti-diagonals
        v = q < 3 * c0 ? __ldcg(base + q) : __ldcg(base + stride3 + (q - 3 * c0));
    };
    const int32_t nq = 3 * (c0 + c1);
    double amax = -INFINITY, dref = 0.0;
    for (int32_t q = tid; q < nq; q += blockDim.x) {
        double a, b;
        at(earlier, q, a);
        at(later, q, b);
        if (a > kNegInf && b > kNegInf && a > amax) {
            amax = a;
            dref = a - b;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double a2 = __shfl_xor_sync(0xffffffffu, amax, o), d2 = __shfl_xor_sync(0xffffffffu, dref, o);
        if (a2 > amax || (a2 == amax && d2 < dref)) { amax = a2; dref = d2; }
    }
    if (lane == 0) { red_a[warp] = amax; red_d[warp] = dref; }
    if (tid == 0) red_ok = 1;
    __syncthreads();
    amax = red_a[0];
    dref = red_d[0];
    for (int w = 1; w < nw; ++w)
        if (red_a[w] > amax || (red_a[w] == amax && red_d[w] < dref)) { amax = red_a[w]; dref = red_d[w]; }
    bool ok = O.stitch_tol >= 0.0;
    double spread = 0.0;
    for (int32_t q = tid; q < nq; q += blockDim.x) {
        double a, b;
        at(earlier, q, a);
        at(later, q, b);
        const bool fa = a > kNegInf, fb = b > kNegInf;
        if (fa != fb) {
            ok = false;
        } else if (fa) {
            const double dev = fabs((a - b) - dref);
            spread = fmax(spread, dev);
            if (!(dev <= O.stitch_tol * (1e-9 + 1e-11 * (amax - a)))) ok = false;
        }
    }
    __syncthreads();   // red_a / red_d read by every thread
    if (!ok) red_ok = 0;
    for (int o = 16; o > 0; o >>= 1) spread = fmax(spread, __shfl_xor_sync(0xffffffffu, spread, o));
    if (lane == 0) red_a[warp] = spread;
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < nw; ++w) spread = fmax(spread, red_a[w]);
        Stitch64Res &res = O.stres[st];
        res.delta = dref;
        res.spread = spread;
        res.result = red_ok ? 1 : 2;
        if (!red_ok) atomicExch(O.fail + S.region, 1);
        __threadfence();
    }
    __syncthreads();
}

// one side of stitch st has written its values (whole CTA): the second to arrive checks it
__device__ void stitch_arrive64(const Region64 &R, const SetOut &O, int32_t st) {
    __shared__ int second;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        second = atomicAdd(&O.stres[st].arrive, 1) == 1;
        __threadfence();
    }
    __syncthreads();
    if (second) stitch_check64(R, O, st);
    __syncthreads();
}

__device__ void run_region(const Model64 &M, const Region64 &R, int32_t region, const SetOut &O, const ExpectOut &X,
                           double (&acc)[10]) {
    const int tid = threadIdx.x, nt = blockDim.x;
    if (R.s0 <= 1) {
        // startStateProb / raggedStartStateProb (stateMachine.c:1022-1032) on anti-diagonal 0
        if (tid == 0) {
            double *c = slot(R.F, R, 0, 0);
            c[S_M] = R.ragged_left ? kNegInf : 0.0;
            c[S_X] = R.ragged_left ? 0.0 : kNegInf;
            c[S_Y] = R.ragged_left ? 0.0 : kNegInf;
        }
    } else {
        // a later forward segment: a flat start two anti-diagonals before its sweep
        fill_diag(R.F, R, R.s0 - 2, 0.0);
        fill_diag(R.F, R, R.s0 - 1, 0.0);
    }
    __syncthreads();
    // anti-diagonals whose forward values go to a stitch: b-1 and b of each
    const int32_t b_in = R.st_in >= 0 ? O.stitch[R.st_in].b : -10, b_out = R.st_out >= 0 ? O.stitch[R.st_out].b : -10;
    int32_t wi = R.w0;
    Window W = R.win[wi];
    for (int32_t d = R.s0 <= 1 ? 1 : R.s0; d <= R.n; ++d) {
        for (int32_t xmy = R.xl[d] + 2 * tid; xmy <= R.xr[d]; xmy += 2 * nt) forward_cell(M, R, d, xmy);
        __syncthreads();
        if (d == b_in - 1 || d == b_in) {
            stitch_copy64(R, O, R.st_in, d, d - (b_in - 1));
            __syncthreads();
        }
        if (d == b_out - 1 || d == b_out) {
            stitch_copy64(R, O, R.st_out, d, 2 + d - (b_out - 1));
            __syncthreads();
        }
        if (d != W.D) continue;
        // endStateProb / raggedEndStateProb (stateMachine.c:1034-1061) on the traceback anti-diagonal
        const bool ragged_end = W.at_end && R.ragged_right;
        const double e0 = ragged_end ? (M.t[T_OX] + M.t[T_OY]) / 2.0 : M.t[T_MC];
        const double e1 = ragged_end ? M.t[T_EX] : M.t[T_MFGX];
        const double e2 = ragged_end ? M.t[T_EY] : M.t[T_MFGY];
        for (int32_t xmy = R.xl[d] + 2 * tid; xmy <= R.xr[d]; xmy += 2 * nt) {
            const int32_t x = (d + xmy) >> 1;
            for (int32_t r = R.pfirst[x]; r < R.pfirst[x + 1]; ++r) {
                double *c = slot(R.B, R, d, r);
                c[S_M] = e0;
                c[S_X] = e1;
                c[S_Y] = e2;
            }
        }
        __syncthreads();
        for (int32_t d2 = W.D - 1; d2 > W.T; --d2) {
            for (int32_t xmy = R.xl[d2] + 2 * tid; xmy <= R.xr[d2]; xmy += 2 * nt) backward_cell(M, R, d2, xmy, W.D);
            __syncthreads();
        }
        // refresh anti-diagonals from, from-10, ... (> T): independent, one thread each
        for (int32_t j = tid;; j += nt) {
            const int32_t dr = W.from - 10 * j;
            if (dr <= W.T) break;
            R.P[dr] = total_probability(M, R, dr, dr < W.D);
        }
        __syncthreads();
        if (X.on) {
            for (int32_t d2 = W.from; d2 > W.T; --d2)
                expect_diagonal(M, R, X, d2, W.T, R.P[W.from - 10 * ((W.from - d2) / 10)], acc);
            if (W.at_end) break;
            W = R.win[++wi];
            continue;
        }
        // diagonalCalculationPosteriorMatchProbs (pairwiseAligner.c:1202-1253) on (T, from]
        for (int32_t d2 = W.from; d2 > W.T; --d2) {
            const double total = R.P[W.from - 10 * ((W.from - d2) / 10)];
            for (int32_t xmy = R.xl[d2] + 2 * tid; xmy <= R.xr[d2]; xmy += 2 * nt) {
                const int32_t x = (d2 + xmy) >> 1, y = (d2 - xmy) >> 1;
                if (!(x > 0 && y > 0)) continue;
                for (int32_t r = R.pfirst[x]; r < R.pfirst[x + 1]; ++r) {
                    const double *f = slot(R.F, R, d2, r), *b = slot(R.B, R, d2, r);
                    double p = exp((f[S_M] + b[S_M]) - total);
                    if (p >= R.threshold) {
                        if (p > 1.0) p = 1.0;
                        unsigned long long o_at = atomicAdd(O.count, 1ULL);
                        if ((int64_t) o_at < O.cap) {
                            sa_aligned_pair o;
                            o.score = (int64_t) floor(p * 10000000.0);
                            o.x = x - 1;
                            o.y = y - 1;
                            o.kmer = R.pid[r];
                            O.out[o_at] = o;
                            O.tag[o_at] = R.tag;
                        } else {
                            atomicExch(R.status, (int32_t) SA_E_OUTPUT);
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (W.at_end || wi + 1 >= R.w1) break;
        W = R.win[++wi];
    }
    // the total probability of the last anti-diagonal is the region's log-likelihood (in the last
    // segment's frame: the host adds the stitches' constants)
    if (tid == 0 && R.w1 >= R.n_windows) *R.loglik = R.P[R.n];
    __syncthreads();
    if (R.st_in >= 0) stitch_arrive64(R, O, R.st_in);
    if (R.st_out >= 0) stitch_arrive64(R, O, R.st_out);
}

// Expectations mode (XS: one ExpectOut per read): CTA b walks read b's regions in order.
__global__ void __launch_bounds__(128) region_kernel(const Model64 *models, const Region64 *regions, SetOut O,
                                                     const ExpectOut *XS) {
    double acc[10];
    if (XS) {
        // the read's regions in order (the reference's split wrapper loops over them), one CTA
        const ExpectOut X = XS[blockIdx.x];
        for (int i = 0; i < 10; ++i) acc[i] = X.acc[i];
        for (int32_t r = X.first_region; r < X.first_region + X.n_regions; ++r) {
            const Region64 R = regions[r];
            run_region(models[R.model], R, r, O, X, acc);
        }
        if (threadIdx.x == 0)
            for (int i = 0; i < 10; ++i) X.acc[i] = acc[i];
        return;
    }
    const ExpectOut X{};
    const Region64 R = regions[blockIdx.x];
    run_region(models[R.model], R, (int32_t) blockIdx.x, O, X, acc);
}

// the per-k-mer logs the FP64 emissions use, with the same device log as an inline call
__global__ void kmer_logs_kernel(const double *match, const double *gapy, int64_t n, double *out) {
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        out[4 * i + 0] = log(match[5 * i + 1]);
        out[4 * i + 1] = log(gapy[5 * i + 1]);
        out[4 * i + 2] = log(match[5 * i + 4]);
        out[4 * i + 3] = log(gapy[5 * i + 4]);
    }
}

}  // namespace

// Called with the machine's device current and its tables resident; synchronous, so the table is
// ready for launches on any stream.
sa_status compute_kmer_logs(sa_state_machine *sm) {
    const int64_t n = sm->n_kmers;
    DeviceModel &d = sm->dev;
    if (device_malloc(reinterpret_cast<void **>(&d.klog), sizeof(double) * 4 * (size_t) std::max<int64_t>(n, 1)) !=
        cudaSuccess) {
        d.klog = nullptr;
        return SA_E_NOMEM;
    }
    if (n > 0) {
        const int64_t blocks = std::min<int64_t>((n + 255) / 256, 4096);
        kmer_logs_kernel<<<(unsigned) blocks, 256>>>(d.match, d.gapy, n, d.klog);
        count_launch();
    }
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return SA_E_CUDA;
    return SA_OK;
}

// ------------------------------------------------------------------------------------------------
// plain sets: host side
// ------------------------------------------------------------------------------------------------
namespace {

// host plan of one region: geometry (band, windows) and its paths
struct PlainRegion {
    int32_t read = 0, model = 0;
    Region rg;
    std::vector<int32_t> xl, xr, pfirst, pid, ppre, psuf, row;
    int32_t ring = 3, stride = 1, max_paths = 1;
    size_t ev_off = 0;   // first event of the region in the set's event array
    std::vector<int32_t> cuts;   // windows that start a later forward segment
    int32_t warm = 0;            // their warm-up
};

}  // namespace

struct PlainSet {
    struct ReadModel {
        sa_state_machine *sm;
        double scale, shift, var;
    };
    int device = 0;
    std::vector<ReadModel> models;   // one per read: the machine and the read's scaling
    std::vector<int32_t> read_status;
    std::vector<int64_t> read_first, read_count;   // regions of each read
    std::vector<PlainRegion> regs;
    std::vector<double2> events;
    int64_t cells = 0, cap = 0;
    double threshold = 0.01;
    // forward segments (alignment runs): per region its first task and first stitch
    int64_t n_tasks = 0, n_stitch = 0, n_redone = 0;
    std::vector<int64_t> task_first, stitch_first;
    double stitch_tol = 1.0;
    size_t res_stres = 0, res_fail = 0;
    size_t o_redo = 0;
    Region64 *d_tasks = nullptr, *d_redo = nullptr;
    Stitch64 *d_stitch = nullptr;
    Stitch64Res *d_stres = nullptr;
    int32_t *d_fail = nullptr;
    std::vector<Region64> whole;   // host copies of the regions' whole-sweep descriptors (re-runs)
    // device block: inputs (staged in `host_in` with the same layout), results, work
    MemBlock host_in, host_res, dev;
    size_t in_bytes = 0, res_off = 0, res_bytes = 0, dev_bytes = 0;
    size_t res_status = 0, res_count = 0;   // offsets in the results block
    Region64 *d_regions = nullptr;
    Model64 *d_models = nullptr;
    double *d_loglik = nullptr;
    int32_t *d_status = nullptr;
    unsigned long long *d_count = nullptr;
    sa_aligned_pair *d_out = nullptr;
    int32_t *d_tag = nullptr;
    double *d_P = nullptr;
    size_t p_bytes = 0;
    // results
    std::vector<std::vector<sa_aligned_pair>> pairs;
    std::vector<double> ll;
    std::vector<int32_t> status;

    ~PlainSet() {
        mem_put(host_in);
        mem_put(host_res);
        mem_put(dev);
    }
};

namespace {

size_t align256(size_t v) { return (v + 255) & ~(size_t) 255; }

// Places every buffer of the set; with non-null bases writes the staged inputs and the Region64 /
// Model64 descriptors (device addresses).  Returns the device bytes.
size_t plain_layout(PlainSet *s, unsigned char *host, unsigned char *dev) {
    size_t at = 0;
    auto take = [&](size_t bytes) {
        at = align256(at);
        const size_t o = at;
        at += std::max<size_t>(bytes, 1);
        return o;
    };
    const size_t nreg = s->regs.size();
    const size_t o_regions = take(nreg * sizeof(Region64));
    const size_t o_models = take(s->models.size() * sizeof(Model64));
    const size_t o_tasks = take((size_t) s->n_tasks * sizeof(Region64));
    const size_t o_stitch = take((size_t) s->n_stitch * sizeof(Stitch64));
    std::vector<Region64> R(nreg);
    struct Off { size_t xl, xr, pfirst, pid, ppre, psuf, row, win; };
    std::vector<Off> off(nreg);
    for (size_t i = 0; i < nreg; ++i) {
        const PlainRegion &pr = s->regs[i];
        off[i].xl = take(pr.xl.size() * sizeof(int32_t));
        off[i].xr = take(pr.xr.size() * sizeof(int32_t));
        off[i].pfirst = take(pr.pfirst.size() * sizeof(int32_t));
        off[i].pid = take(pr.pid.size() * sizeof(int32_t));
        off[i].ppre = take(pr.ppre.size() * sizeof(int32_t));
        off[i].psuf = take(pr.psuf.size() * sizeof(int32_t));
        off[i].row = take(pr.row.size() * sizeof(int32_t));
        off[i].win = take(pr.rg.windows.size() * sizeof(Window));
    }
    const size_t o_events = take(s->events.size() * sizeof(double2));
    s->in_bytes = align256(at);
    at = s->in_bytes;
    s->res_off = at;
    const size_t o_loglik = take(nreg * sizeof(double));
    const size_t o_status = take(nreg * sizeof(int32_t));
    const size_t o_count = take(sizeof(unsigned long long));
    const size_t o_stres = take((size_t) s->n_stitch * sizeof(Stitch64Res));
    const size_t o_fail = take(nreg * sizeof(int32_t));
    s->res_bytes = align256(at) - s->res_off;
    s->res_status = o_status - s->res_off;
    s->res_count = o_count - s->res_off;
    s->res_stres = o_stres - s->res_off;
    s->res_fail = o_fail - s->res_off;
    at = s->res_off + s->res_bytes;
    size_t p_total = 0;
    for (const PlainRegion &pr : s->regs) p_total += (size_t) (pr.rg.lX + pr.rg.lY + 1);
    const size_t o_P = take(p_total * sizeof(double));
    s->p_bytes = p_total * sizeof(double);
    // rings per task: a region's first segment (or its whole sweep) uses the region's, every later
    // segment its own; stitch values 4 x stride x 3 doubles each
    std::vector<size_t> o_F(s->n_tasks), o_B(s->n_tasks), o_E(s->n_tasks), o_sv(s->n_stitch);
    for (size_t i = 0; i < nreg; ++i) {
        const size_t ring_bytes = 3 * sizeof(double) * (size_t) s->regs[i].ring * (size_t) s->regs[i].stride;
        for (size_t q = 0; q <= s->regs[i].cuts.size(); ++q) {
            const size_t t = (size_t) s->task_first[i] + q;
            o_F[t] = take(ring_bytes);
            o_B[t] = take(ring_bytes);
            o_E[t] = take(ring_bytes / 3 * 2);
        }
        for (size_t q = 0; q < s->regs[i].cuts.size(); ++q)
            o_sv[(size_t) s->stitch_first[i] + q] = take(4 * 3 * sizeof(double) * (size_t) s->regs[i].stride);
    }
    s->o_redo = take(nreg * sizeof(Region64));
    const size_t o_out = take((size_t) s->cap * sizeof(sa_aligned_pair));
    const size_t o_tag = take((size_t) s->cap * sizeof(int32_t));
    s->dev_bytes = align256(at);
    if (dev) {
        s->d_regions = reinterpret_cast<Region64 *>(dev + o_regions);
        s->d_models = reinterpret_cast<Model64 *>(dev + o_models);
        s->d_tasks = reinterpret_cast<Region64 *>(dev + o_tasks);
        s->d_stitch = reinterpret_cast<Stitch64 *>(dev + o_stitch);
        s->d_stres = reinterpret_cast<Stitch64Res *>(dev + o_stres);
        s->d_fail = reinterpret_cast<int32_t *>(dev + o_fail);
        s->d_redo = reinterpret_cast<Region64 *>(dev + s->o_redo);
        s->d_loglik = reinterpret_cast<double *>(dev + o_loglik);
        s->d_status = reinterpret_cast<int32_t *>(dev + o_status);
        s->d_count = reinterpret_cast<unsigned long long *>(dev + o_count);
        s->d_P = reinterpret_cast<double *>(dev + o_P);
        s->d_out = reinterpret_cast<sa_aligned_pair *>(dev + o_out);
        s->d_tag = reinterpret_cast<int32_t *>(dev + o_tag);
    }
    if (host && dev) {
        size_t p_at = 0;
        for (size_t i = 0; i < nreg; ++i) {
            const PlainRegion &pr = s->regs[i];
            auto put = [&](size_t o, const void *src, size_t bytes) {
                if (bytes) std::memcpy(host + o, src, bytes);
            };
            put(off[i].xl, pr.xl.data(), pr.xl.size() * sizeof(int32_t));
            put(off[i].xr, pr.xr.data(), pr.xr.size() * sizeof(int32_t));
            put(off[i].pfirst, pr.pfirst.data(), pr.pfirst.size() * sizeof(int32_t));
            put(off[i].pid, pr.pid.data(), pr.pid.size() * sizeof(int32_t));
            put(off[i].ppre, pr.ppre.data(), pr.ppre.size() * sizeof(int32_t));
            put(off[i].psuf, pr.psuf.data(), pr.psuf.size() * sizeof(int32_t));
            put(off[i].row, pr.row.data(), pr.row.size() * sizeof(int32_t));
            put(off[i].win, pr.rg.windows.data(), pr.rg.windows.size() * sizeof(Window));
            Region64 &r = R[i];
            std::memset(&r, 0, sizeof(r));
            r.lX = (int32_t) pr.rg.lX;
            r.lY = (int32_t) pr.rg.lY;
            r.n = (int32_t) (pr.rg.lX + pr.rg.lY);
            r.n_windows = (int32_t) pr.rg.windows.size();
            r.ragged_left = pr.rg.ragged_left;
            r.ragged_right = pr.rg.ragged_right;
            r.model = pr.model;
            r.ev_base = pr.rg.y1;
            r.threshold = s->threshold;
            r.ring = pr.ring;
            r.stride = pr.stride;
            r.xl = reinterpret_cast<const int32_t *>(dev + off[i].xl);
            r.xr = reinterpret_cast<const int32_t *>(dev + off[i].xr);
            r.pfirst = reinterpret_cast<const int32_t *>(dev + off[i].pfirst);
            r.pid = reinterpret_cast<const int32_t *>(dev + off[i].pid);
            r.ppre = reinterpret_cast<const int32_t *>(dev + off[i].ppre);
            r.psuf = reinterpret_cast<const int32_t *>(dev + off[i].psuf);
            r.row = reinterpret_cast<const int32_t *>(dev + off[i].row);
            r.ev = reinterpret_cast<const double2 *>(dev + o_events) + pr.ev_off;
            r.win = reinterpret_cast<const Window *>(dev + off[i].win);
            const size_t t0 = (size_t) s->task_first[i];
            r.F = reinterpret_cast<double *>(dev + o_F[t0]);
            r.B = reinterpret_cast<double *>(dev + o_B[t0]);
            r.E = reinterpret_cast<double *>(dev + o_E[t0]);
            r.s0 = 1;
            r.w0 = 0;
            r.w1 = r.n_windows;
            r.tag = (int32_t) i;
            r.st_in = r.st_out = -1;
            r.P = s->d_P + p_at;
            p_at += (size_t) r.n + 1;
            r.loglik = s->d_loglik + i;
            r.status = s->d_status + i;
        }
        std::memcpy(host + o_regions, R.data(), nreg * sizeof(Region64));
        s->whole = R;
        // tasks: per region its segments (one, the whole sweep, when it has no cuts), and the stitches
        std::vector<Region64> T((size_t) s->n_tasks);
        std::vector<Stitch64> ST((size_t) s->n_stitch);
        for (size_t i = 0; i < nreg; ++i) {
            const PlainRegion &pr = s->regs[i];
            const std::vector<int32_t> &cuts = pr.cuts;
            for (size_t q = 0; q <= cuts.size(); ++q) {
                const size_t t = (size_t) s->task_first[i] + q;
                Region64 r = R[i];
                r.F = reinterpret_cast<double *>(dev + o_F[t]);
                r.B = reinterpret_cast<double *>(dev + o_B[t]);
                r.E = reinterpret_cast<double *>(dev + o_E[t]);
                r.w0 = q == 0 ? 0 : cuts[q - 1];
                r.w1 = q == cuts.size() ? r.n_windows : cuts[q];
                r.s0 = q == 0 ? 1 : pr.rg.windows[cuts[q - 1]].T - pr.warm;
                r.st_in = q == 0 ? -1 : (int32_t) (s->stitch_first[i] + (int64_t) q - 1);
                r.st_out = q == cuts.size() ? -1 : (int32_t) (s->stitch_first[i] + (int64_t) q);
                T[t] = r;
            }
            for (size_t q = 0; q < cuts.size(); ++q) {
                Stitch64 &st = ST[(size_t) s->stitch_first[i] + q];
                std::memset(&st, 0, sizeof(st));
                st.vals = reinterpret_cast<double *>(dev + o_sv[(size_t) s->stitch_first[i] + q]);
                st.b = pr.rg.windows[cuts[q]].T;
                st.region = (int32_t) i;
                st.stride = pr.stride;
            }
        }
        if (!T.empty()) std::memcpy(host + o_tasks, T.data(), T.size() * sizeof(Region64));
        if (!ST.empty()) std::memcpy(host + o_stitch, ST.data(), ST.size() * sizeof(Stitch64));
        for (size_t m = 0; m < s->models.size(); ++m) {
            const sa_state_machine *sm = s->models[m].sm;
            Model64 M;
            std::memset(&M, 0, sizeof(M));
            M.emission = sm->emission;
            for (int i = 0; i < 9; ++i) M.t[i] = sm->t[i];
            M.match = sm->dev.match;
            M.gapy = sm->dev.gapy;
            M.gapx = sm->dev.gapx;
            M.klog = sm->dev.klog;
            M.scale = s->models[m].scale;
            M.shift = s->models[m].shift;
            M.var = s->models[m].var;
            if (sm->emission == SA_EMIT_HDP) {
                M.grid_length = sm->hdp.grid_length;
                M.grid = sm->dev.hdp_grid;
                M.density = sm->dev.hdp_density;
                M.slope = sm->dev.hdp_slope;
                M.kmer_row = sm->dev.hdp_kmer_row;
            }
            std::memcpy(host + o_models + m * sizeof(Model64), &M, sizeof(M));
        }
        if (!s->events.empty()) std::memcpy(host + o_events, s->events.data(), s->events.size() * sizeof(double2));
    }
    return s->dev_bytes;
}

}  // namespace

namespace {

// reference emission order of a region's pairs: window by window, anti-diagonals descending, xmy
// ascending, a cell's paths in order (diagonalCalculationPosteriorMatchProbs, pairwiseAligner.c:1202-1253)
struct Emitted {
    sa_aligned_pair pair;
    int64_t key_window, key_diag, key_xmy, key_path;
};

// Plans one region of the set: band, paths, ring geometry.
void plan_region(const PathTable &pt, int32_t asz, int64_t kpow, PlainRegion &pr) {
    const Region &rg = pr.rg;
    const int32_t n = (int32_t) (rg.lX + rg.lY);
    pr.xl.assign(rg.xmy_l.begin(), rg.xmy_l.end());
    pr.xr.assign(rg.xmy_r.begin(), rg.xmy_r.end());
    // column 0 is the NULL path, column x the reference column x1 + x
    pr.pfirst.assign(rg.lX + 2, 0);
    pr.pid.assign(1, -1);
    for (int64_t x = 1; x <= rg.lX; ++x) {
        pr.pfirst[x] = (int32_t) pr.pid.size();
        for (int32_t q = pt.first[rg.x1 + x]; q < pt.first[rg.x1 + x + 1]; ++q) pr.pid.push_back(pt.ids[q]);
    }
    pr.pfirst[rg.lX + 1] = (int32_t) pr.pid.size();
    pr.ppre.resize(pr.pid.size());
    pr.psuf.resize(pr.pid.size());
    for (size_t q = 0; q < pr.pid.size(); ++q) {
        pr.ppre[q] = pr.pid[q] < 0 ? -1 : pr.pid[q] / asz;
        pr.psuf[q] = pr.pid[q] < 0 ? -1 : (int32_t) (pr.pid[q] % kpow);
    }
    pr.stride = 1;
    for (int32_t d = 0; d <= n; ++d) {
        const int64_t x0 = (d + rg.xmy_l[d]) / 2, x1 = (d + rg.xmy_r[d]) / 2;
        pr.stride = std::max<int32_t>(pr.stride, pr.pfirst[x1 + 1] - pr.pfirst[x0]);
    }
    pr.max_paths = 1;
    for (int64_t x = 0; x <= rg.lX; ++x) pr.max_paths = std::max(pr.max_paths, pr.pfirst[x + 1] - pr.pfirst[x]);
    int32_t span = 0;
    for (const Window &w : rg.windows) span = std::max(span, w.D - w.T + 1);
    pr.ring = std::max(3, span) + 1;
    // ring row of each anti-diagonal, so a slot lookup is one load instead of a modulo and two
    // dependent loads
    pr.row.resize((size_t) n + 1);
    for (int32_t d = 0; d <= n; ++d)
        pr.row[d] = (int32_t) ((int64_t) (d % pr.ring) * pr.stride - pr.pfirst[(d + rg.xmy_l[d]) / 2]);
}

}  // namespace

// Plans a set of reads for the plain form.  Reads that fail planning keep their status and get no
// regions.  `max_bytes` bounds the device block (SA_E_CAPACITY above it).
sa_status plain_create(const sa_read *reads, int64_t n_reads, const sa_params &p, size_t max_bytes, PlainSet **out,
                       bool segments) {
    *out = nullptr;
    auto *s = new (std::nothrow) PlainSet();
    if (!s) return SA_E_NOMEM;
    s->threshold = p.threshold;
    s->read_status.assign(n_reads, SA_OK);
    s->read_first.assign(n_reads, 0);
    s->read_count.assign(n_reads, 0);
    int device = -1;
    int64_t cap = 0;
    for (int64_t r = 0; r < n_reads; ++r) {
        const sa_read &rd = reads[r];
        auto *sm = const_cast<sa_state_machine *>(rd.sm);
        s->models.push_back(PlainSet::ReadModel{sm, rd.scale, rd.shift, rd.var});
        s->read_first[r] = (int64_t) s->regs.size();
        sa_status st = SA_OK;
        if (!sm || rd.reference_length < 0 || rd.n_events < 0 || rd.n_anchors < 0 ||
            (rd.reference_length > 0 && !rd.reference) || (rd.n_events > 0 && !rd.events) ||
            (rd.n_anchors > 0 && !rd.anchors))
            st = SA_E_ARG;
        if (!st && device >= 0 && sm->dev.device != device) st = SA_E_ARG;
        if (!st && sm->emission == SA_EMIT_HDP && !sm->hdp.present) st = SA_E_UNSUPPORTED;
        const int k = sm ? sm->kmer_length : 1;
        // sequence_correctSeqLength (pairwiseAligner.c:456-471)
        const int64_t lX = rd.reference_length == 0 ? 0 : rd.reference_length - (k - 1);
        if (!st && lX < 0) st = SA_E_ARG;
        PathTable pt;
        std::vector<Region> regions;
        if (!st) st = build_paths(sm, rd.reference, lX, rd.degenerate, pt);
        if (!st)
            st = plan_regions(rd.anchors, rd.n_anchors, lX, rd.n_events, p, rd.ragged_left != 0, rd.ragged_right != 0,
                              regions);
        if (st) {
            s->read_status[r] = st;
            continue;
        }
        if (device < 0) device = sm->dev.device;
        // path_checkLegal on k-mer ids: the (k-1)-prefix of id is id / |alphabet|, the (k-1)-suffix
        // id mod |alphabet|^(k-1)
        const int32_t asz = (int32_t) sm->alphabet.size();
        int64_t kpow = 1;
        for (int i = 0; i < k - 1; ++i) kpow *= asz;
        for (Region &rg : regions) {
            PlainRegion pr;
            pr.read = (int32_t) r;
            pr.model = (int32_t) r;
            pr.rg = std::move(rg);
            plan_region(pt, asz, kpow, pr);
            pr.ev_off = s->events.size();
            for (int64_t y = 0; y < pr.rg.lY; ++y) {
                const double *e = rd.events + (pr.rg.y1 + y) * kEventParams;
                s->events.push_back(make_double2(e[0], e[1]));
            }
            const int64_t n = pr.rg.lX + pr.rg.lY;
            cap += 4 * (n + 1) * std::min<int64_t>(pr.max_paths, 4) + 256;
            for (int32_t d = 0; d <= n; ++d) {
                const int64_t x0 = (d + pr.xl[d]) / 2, x1 = (d + pr.xr[d]) / 2;
                s->cells += pr.pfirst[x1 + 1] - pr.pfirst[x0];
            }
            s->regs.push_back(std::move(pr));
        }
        s->read_count[r] = (int64_t) s->regs.size() - s->read_first[r];
    }
    s->device = device < 0 ? 0 : device;
    s->cap = cap;
    // Forward segments (alignment runs): long regions cut at window starts like the batched form's,
    // the automatic cap from twice the set's anti-diagonals per CTA slot (four plain CTAs per SM)
    int32_t policy = -1, warm0 = 1024;
    if (segments) segment_policy(policy, warm0);
    int64_t target = policy;
    if (segments && policy == 0) {
        int64_t diags = 0;
        for (const PlainRegion &pr : s->regs) diags += pr.rg.lX + pr.rg.lY + 1;
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess) {
            cudaGetLastError();
            sms = 0;
        }
        if (sms <= 0) sms = 148;
        target = std::max<int64_t>(segment_min(), 2 * diags / ((int64_t) sms * 4));
    }
    s->task_first.assign(s->regs.size(), 0);
    s->stitch_first.assign(s->regs.size(), 0);
    for (size_t i = 0; i < s->regs.size(); ++i) {
        PlainRegion &pr = s->regs[i];
        pr.cuts.clear();
        pr.warm = 0;
        if (segments && policy >= 0) {
            const int32_t wr = segment_warm(pr.rg, warm0);
            segment_cuts(pr.rg, target, wr, pr.cuts);
            pr.warm = wr;
        }
        s->task_first[i] = s->n_tasks;
        s->stitch_first[i] = s->n_stitch;
        s->n_tasks += 1 + (int64_t) pr.cuts.size();
        s->n_stitch += (int64_t) pr.cuts.size();
    }
    plain_layout(s, nullptr, nullptr);
    if (s->dev_bytes > max_bytes) {
        delete s;
        return SA_E_CAPACITY;
    }
    *out = s;
    return SA_OK;
}

// Device block, staged inputs and their upload (async on `stream`); models must be resident.
sa_status plain_upload(PlainSet *s, cudaStream_t stream) {
    sa_status st = mem_get(MemKind::Device, s->device, s->dev_bytes, s->dev);
    if (!st) st = mem_get(MemKind::Pinned, s->device, s->in_bytes, s->host_in);
    if (!st) st = mem_get(MemKind::Pinned, s->device, s->res_bytes, s->host_res);
    if (st) return st;
    plain_layout(s, static_cast<unsigned char *>(s->host_in.ptr), static_cast<unsigned char *>(s->dev.ptr));
    if (cudaMemcpyAsync(s->dev.ptr, s->host_in.ptr, s->in_bytes, cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return SA_E_CUDA;
    return SA_OK;
}

// One launch: every region one CTA.
sa_status plain_run(PlainSet *s, cudaStream_t stream) {
    auto *dev = static_cast<unsigned char *>(s->dev.ptr);
    if (cudaMemsetAsync(dev + s->res_off, 0, s->res_bytes, stream) != cudaSuccess ||
        cudaMemsetAsync(s->d_P, 0, std::max<size_t>(s->p_bytes, 1), stream) != cudaSuccess)
        return SA_E_CUDA;
    if (s->regs.empty()) return SA_OK;
    SetOut O;
    std::memset(&O, 0, sizeof(O));
    O.out = s->d_out;
    O.tag = s->d_tag;
    O.count = s->d_count;
    O.cap = s->cap;
    O.stitch = s->d_stitch;
    O.stres = s->d_stres;
    O.fail = s->d_fail;
    O.stitch_tol = s->stitch_tol;
    s->n_redone = 0;
    region_kernel<<<(unsigned) s->n_tasks, 128, 0, stream>>>(s->d_models, s->d_tasks, O, nullptr);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? SA_OK : SA_E_CUDA;
}

// Results to the host (synchronises `stream`): per read its pairs in the reference's emission
// order, coordinates shifted back from the regions (alignedPairCoordinateCorrectionFn,
// pairwiseAligner.c:1763-1771), its status and log-likelihood.
sa_status plain_download(PlainSet *s, cudaStream_t stream) {
    if (cudaMemcpyAsync(s->host_res.ptr, static_cast<unsigned char *>(s->dev.ptr) + s->res_off, s->res_bytes,
                        cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return SA_E_CUDA;
    const auto *res = static_cast<const unsigned char *>(s->host_res.ptr);
    const auto *loglik = reinterpret_cast<const double *>(res);
    const auto *rstatus = reinterpret_cast<const int32_t *>(res + s->res_status);
    const auto *stres = reinterpret_cast<const Stitch64Res *>(res + s->res_stres);
    const auto *fail = reinterpret_cast<const int32_t *>(res + s->res_fail);
    // regions whose stitch disagreed run again as whole sweeps (their rings are their first
    // segment's); the pairs of that second launch follow the first launch's in the output
    const size_t nreg = s->regs.size();
    std::vector<char> redone(nreg, 0);
    unsigned long long count0 = *reinterpret_cast<const unsigned long long *>(res + s->res_count);
    {
        std::vector<Region64> redo;
        for (size_t i = 0; i < nreg; ++i)
            if (fail[i]) {
                redone[i] = 1;
                redo.push_back(s->whole[i]);
            }
        if (!redo.empty()) {
            SetOut O;
            std::memset(&O, 0, sizeof(O));
            O.out = s->d_out;
            O.tag = s->d_tag;
            O.count = s->d_count;
            O.cap = s->cap;
            if (cudaMemcpyAsync(s->d_redo, redo.data(), redo.size() * sizeof(Region64), cudaMemcpyHostToDevice,
                                stream) != cudaSuccess)
                return SA_E_CUDA;
            region_kernel<<<(unsigned) redo.size(), 128, 0, stream>>>(s->d_models, s->d_redo, O, nullptr);
            count_launch();
            if (cudaGetLastError() != cudaSuccess ||
                cudaMemcpyAsync(s->host_res.ptr, static_cast<unsigned char *>(s->dev.ptr) + s->res_off, s->res_bytes,
                                cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
                cudaStreamSynchronize(stream) != cudaSuccess)
                return SA_E_CUDA;
            s->n_redone = (int64_t) redo.size();
        }
    }
    const auto count = *reinterpret_cast<const unsigned long long *>(res + s->res_count);
    const size_t npairs = (size_t) std::min<unsigned long long>(count, (unsigned long long) s->cap);
    std::vector<sa_aligned_pair> got(npairs);
    std::vector<int32_t> tag(npairs);
    if (npairs &&
        (cudaMemcpyAsync(got.data(), s->d_out, npairs * sizeof(sa_aligned_pair), cudaMemcpyDeviceToHost, stream) !=
             cudaSuccess ||
         cudaMemcpyAsync(tag.data(), s->d_tag, npairs * sizeof(int32_t), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
         cudaStreamSynchronize(stream) != cudaSuccess))
        return SA_E_CUDA;
    const int64_t n_reads = (int64_t) s->read_status.size();
    std::vector<std::vector<Emitted>> per_read(n_reads);
    for (size_t i = 0; i < npairs; ++i) {
        const int32_t ri = tag[i];
        if (i < count0 && redone[ri]) continue;   // superseded by the whole sweep's pairs
        const PlainRegion &pr = s->regs[ri];
        const sa_aligned_pair &g = got[i];
        Emitted e;
        const int64_t d = g.x + g.y + 2, xmy = g.x - g.y;
        int64_t w = 0;
        while (w < (int64_t) pr.rg.windows.size() && d > pr.rg.windows[w].from) ++w;
        int32_t r = pr.pfirst[g.x + 1];
        while (r + 1 < pr.pfirst[g.x + 2] && pr.pid[r] != g.kmer) ++r;
        e.key_window = ((int64_t) ri << 32) | w;
        e.key_diag = -d;
        e.key_xmy = xmy;
        e.key_path = r;
        e.pair = g;
        e.pair.x += pr.rg.x1;
        e.pair.y += pr.rg.y1;
        per_read[pr.read].push_back(e);
    }
    s->pairs.assign(n_reads, {});
    s->ll.assign(n_reads, 0.0);
    s->status = s->read_status;
    for (int64_t r = 0; r < n_reads; ++r) {
        for (int64_t i = 0; i < s->read_count[r]; ++i) {
            const int64_t ri = s->read_first[r] + i;
            if (rstatus[ri] && !s->status[r]) s->status[r] = rstatus[ri];
            s->ll[r] += loglik[ri];
            // the last segment's total is in its own frame: the stitches' constants bring it back
            if (!redone[ri])
                for (size_t q = 0; q < s->regs[ri].cuts.size(); ++q) s->ll[r] += stres[s->stitch_first[ri] + q].delta;
        }
        if (count > (unsigned long long) s->cap && s->read_count[r] && !s->status[r]) s->status[r] = SA_E_OUTPUT;
        auto &v = per_read[r];
        std::sort(v.begin(), v.end(), [](const Emitted &a, const Emitted &b) {
            if (a.key_window != b.key_window) return a.key_window < b.key_window;
            if (a.key_diag != b.key_diag) return a.key_diag < b.key_diag;
            if (a.key_xmy != b.key_xmy) return a.key_xmy < b.key_xmy;
            return a.key_path < b.key_path;
        });
        s->pairs[r].resize(v.size());
        for (size_t i = 0; i < v.size(); ++i) s->pairs[r][i] = v[i].pair;
    }
    return SA_OK;
}

int plain_device(const PlainSet *s) { return s->device; }
int64_t plain_cells(const PlainSet *s) { return s->cells; }
size_t plain_in_bytes(const PlainSet *s) { return s->in_bytes; }
sa_status plain_read_status(const PlainSet *s, int64_t r) { return (sa_status) s->status[r]; }
const std::vector<sa_aligned_pair> &plain_pairs(const PlainSet *s, int64_t r) { return s->pairs[r]; }
double plain_log_likelihood(const PlainSet *s, int64_t r) { return s->ll[r]; }
void plain_destroy(PlainSet *s) { delete s; }
void plain_set_stitch_tolerance(PlainSet *s, double scale) { s->stitch_tol = scale; }
void plain_segment_info(const PlainSet *s, int64_t *n_tasks, int64_t *n_stitches, int64_t *n_redone) {
    *n_tasks = s->n_tasks;
    *n_stitches = s->n_stitch;
    *n_redone = s->n_redone;
}

}  // namespace sa

using namespace sa;

// Device memory bound of one plain call (the forward and backward rings of a 20 kb read take tens
// of MB; a pathological band of many-path cells is refused rather than allowed to take the GPU).
static constexpr size_t kPlainMaxBytes = (size_t) 32 << 30;
static constexpr size_t kExpectMaxBytes = (size_t) 64 << 30;

extern "C" sa_status sa_getAlignedPairsUsingAnchors(const sa_state_machine *sm_c, const char *reference,
                                                    int64_t reference_length, sa_degenerate degenerate,
                                                    const double *events, int64_t n_events,
                                                    const int64_t *anchors, int64_t n_anchors, const sa_params *p,
                                                    int32_t ragged_left, int32_t ragged_right,
                                                    sa_aligned_pair **pairs_out, int64_t *n_pairs_out,
                                                    double *log_likelihood) {
    if (!sm_c || !p || !pairs_out || !n_pairs_out || reference_length < 0 || n_events < 0 || n_anchors < 0)
        return SA_E_ARG;
    if ((reference_length > 0 && !reference) || (n_events > 0 && !events) || (n_anchors > 0 && !anchors))
        return SA_E_ARG;
    *pairs_out = nullptr;
    *n_pairs_out = 0;
    if (log_likelihood) *log_likelihood = 0.0;
    sa_status st = check_params(*p);
    if (st) return st;
    auto *sm = const_cast<sa_state_machine *>(sm_c);
    sa_read rd;
    std::memset(&rd, 0, sizeof(rd));
    rd.sm = sm;
    rd.reference = reference;
    rd.reference_length = reference_length;
    rd.events = events;
    rd.n_events = n_events;
    rd.anchors = anchors;
    rd.n_anchors = n_anchors;
    rd.scale = sm->scale;
    rd.shift = sm->shift;
    rd.var = sm->var;
    rd.ragged_left = ragged_left;
    rd.ragged_right = ragged_right;
    rd.degenerate = degenerate;
    PlainSet *s = nullptr;
    st = plain_create(&rd, 1, *p, kPlainMaxBytes, &s, true);
    if (st) return st;
    if (s->read_status[0]) {
        st = (sa_status) s->read_status[0];
        plain_destroy(s);
        return st;
    }
    st = ensure_device_model(sm);
    int prev_dev = 0;
    if (!st && cudaGetDevice(&prev_dev) != cudaSuccess) st = SA_E_CUDA;
    if (!st && cudaSetDevice(s->device) != cudaSuccess) st = SA_E_CUDA;
    if (!st) {
        st = plain_upload(s, nullptr);
        if (!st) st = plain_run(s, nullptr);
        if (!st) st = plain_download(s, nullptr);
        if (!st) st = plain_read_status(s, 0);
        cudaSetDevice(prev_dev);
    }
    if (st) {
        plain_destroy(s);
        return st;
    }
    const auto &v = plain_pairs(s, 0);
    auto *outp = (sa_aligned_pair *) std::malloc(std::max<size_t>(1, v.size()) * sizeof(sa_aligned_pair));
    if (!outp) {
        plain_destroy(s);
        return SA_E_NOMEM;
    }
    if (!v.empty()) std::memcpy(outp, v.data(), v.size() * sizeof(sa_aligned_pair));
    *pairs_out = outp;
    *n_pairs_out = (int64_t) v.size();
    if (log_likelihood) *log_likelihood = plain_log_likelihood(s, 0);
    plain_destroy(s);
    return SA_OK;
}

// Expectations of many reads in one launch: CTA i walks read i's regions in order into ex[i]'s
// accumulators (the single-read call is this with one read).  Per read on the device: the
// anti-diagonal scratch and cell masks, the accumulators, and (HDP machines) the assignment lists.
static sa_status expectations_batch(const sa_read *reads, int64_t n, const sa_params &p, sa_expectations *ex,
                                    int32_t *read_status) {
    for (int64_t i = 0; i < n; ++i) {
        read_status[i] = SA_OK;
        const sa_state_machine *sm = reads[i].sm;
        if (!sm || !ex[i].event_expectations || !ex[i].posteriors || !ex[i].observed) {
            read_status[i] = SA_E_ARG;
        } else if (sm->emission == SA_EMIT_HDP) {
            // the HDP machine collects assignments instead (hdpHmm_makeExpectationsHmm)
            if (!sm->hdp.present) read_status[i] = SA_E_UNSUPPORTED;
            else if (ex[i].assignment_capacity > 0 && (!ex[i].assignment_kmers || !ex[i].assignment_events))
                read_status[i] = SA_E_ARG;
        }
    }
    PlainSet *s = nullptr;
    sa_status st = plain_create(reads, n, p, kExpectMaxBytes, &s);
    if (st) return st;
    std::vector<int32_t> width(n, 1);
    for (int64_t i = 0; i < n; ++i) {
        if (!read_status[i]) read_status[i] = s->read_status[i];
        for (int64_t r = s->read_first[i]; r < s->read_first[i] + s->read_count[i]; ++r) {
            if (s->regs[r].max_paths > 1 && !read_status[i]) read_status[i] = SA_E_UNSUPPORTED;   // single-path cells only
            width[i] = std::max(width[i], s->regs[r].stride);
        }
    }
    std::vector<int64_t> run;   // reads that run, in order
    for (int64_t i = 0; i < n; ++i)
        if (!read_status[i] && s->read_count[i] > 0) run.push_back(i);
    if (run.empty()) {   // nothing for the device: no device call at all
        for (int64_t i = 0; i < n; ++i)
            if (!read_status[i]) ex[i].n_assignments = 0;
        plain_destroy(s);
        return SA_OK;
    }
    for (int64_t i : run)
        if (!st) st = ensure_device_model(const_cast<sa_state_machine *>(reads[i].sm));
    int prev_dev = 0;
    if (!st && cudaGetDevice(&prev_dev) != cudaSuccess) st = SA_E_CUDA;
    if (!st && cudaSetDevice(s->device) != cudaSuccess) st = SA_E_CUDA;
    if (st) {
        plain_destroy(s);
        return st;
    }
    // one device block: per running read its buffers, then the ExpectOut array
    struct Off { size_t scratch, mask, acc, ee, po, ob, ak, ae, na; int64_t nk, cap; bool hdp; };
    auto up = [](size_t v) { return (v + 255) & ~(size_t) 255; };
    std::vector<Off> off(run.size());
    size_t total = 0;
    for (size_t j = 0; j < run.size(); ++j) {
        const int64_t i = run[j];
        const sa_state_machine *sm = reads[i].sm;
        Off &o = off[j];
        o.nk = sm->n_kmers;
        o.hdp = sm->emission == SA_EMIT_HDP;
        o.cap = o.hdp ? std::max<int64_t>(ex[i].assignment_capacity, 0) : 0;
        o.scratch = total; total += up(sizeof(double) * kExpectScratch * (size_t) width[i]);
        o.mask = total; total += up(sizeof(int32_t) * (size_t) width[i]);
        o.acc = total; total += up(sizeof(double) * 10);
        o.ee = total; total += up(sizeof(double) * 2 * (size_t) o.nk);
        o.po = total; total += up(sizeof(double) * (size_t) o.nk);
        o.ob = total; total += up((size_t) o.nk);
        o.ak = total; total += up(sizeof(int64_t) * (size_t) std::max<int64_t>(o.cap, 1));
        o.ae = total; total += up(sizeof(int64_t) * (size_t) std::max<int64_t>(o.cap, 1));
        o.na = total; total += up(sizeof(int64_t));
    }
    const size_t o_xs = total;
    total += up(sizeof(ExpectOut) * run.size());
    std::vector<unsigned char> host(total, 0);
    MemBlock blk;
    st = plain_upload(s, nullptr);
    if (!st) st = mem_get(MemKind::Device, s->device, total, blk);
    if (!st) {
        auto *d = static_cast<unsigned char *>(blk.ptr);
        auto *xs = reinterpret_cast<ExpectOut *>(host.data() + o_xs);
        for (size_t j = 0; j < run.size(); ++j) {
            const int64_t i = run[j];
            const Off &o = off[j];
            auto *acc = reinterpret_cast<double *>(host.data() + o.acc);
            acc[0] = ex[i].likelihood;
            for (int k = 0; k < 9; ++k) acc[k + 1] = ex[i].transitions[k];
            std::memcpy(host.data() + o.ee, ex[i].event_expectations, sizeof(double) * 2 * (size_t) o.nk);
            std::memcpy(host.data() + o.po, ex[i].posteriors, sizeof(double) * (size_t) o.nk);
            std::memcpy(host.data() + o.ob, ex[i].observed, (size_t) o.nk);
            ExpectOut &X = xs[j];
            X.on = 1;
            X.first_region = (int32_t) s->read_first[i];
            X.n_regions = (int32_t) s->read_count[i];
            X.hdp = o.hdp ? 1 : 0;
            X.threshold = p.threshold;
            X.scratch = reinterpret_cast<double *>(d + o.scratch);
            X.mask = reinterpret_cast<int32_t *>(d + o.mask);
            X.acc = reinterpret_cast<double *>(d + o.acc);
            X.event_exp = reinterpret_cast<double *>(d + o.ee);
            X.posteriors = reinterpret_cast<double *>(d + o.po);
            X.observed = d + o.ob;
            X.assign_kmer = reinterpret_cast<int64_t *>(d + o.ak);
            X.assign_event = reinterpret_cast<int64_t *>(d + o.ae);
            X.n_assign = reinterpret_cast<int64_t *>(d + o.na);
            X.assign_cap = o.cap;
        }
        SetOut O;
        std::memset(&O, 0, sizeof(O));
        auto *dev = static_cast<unsigned char *>(s->dev.ptr);
        if (cudaMemcpy(d, host.data(), total, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemsetAsync(dev + s->res_off, 0, s->res_bytes, nullptr) != cudaSuccess ||
            cudaMemsetAsync(s->d_P, 0, std::max<size_t>(s->p_bytes, 1), nullptr) != cudaSuccess)
            st = SA_E_CUDA;
        if (!st) {
            region_kernel<<<(unsigned) run.size(), 128>>>(s->d_models, s->d_regions, O,
                                                        reinterpret_cast<const ExpectOut *>(d + o_xs));
            count_launch();
            if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) st = SA_E_CUDA;
        }
        if (!st && cudaMemcpy(host.data(), d, o_xs, cudaMemcpyDeviceToHost) != cudaSuccess) st = SA_E_CUDA;
        if (!st) {
            for (size_t j = 0; j < run.size(); ++j) {
                const int64_t i = run[j];
                const Off &o = off[j];
                const auto *acc = reinterpret_cast<const double *>(host.data() + o.acc);
                ex[i].likelihood = acc[0];
                for (int k = 0; k < 9; ++k) ex[i].transitions[k] = acc[k + 1];
                std::memcpy(ex[i].event_expectations, host.data() + o.ee, sizeof(double) * 2 * (size_t) o.nk);
                std::memcpy(ex[i].posteriors, host.data() + o.po, sizeof(double) * (size_t) o.nk);
                std::memcpy(ex[i].observed, host.data() + o.ob, (size_t) o.nk);
                const int64_t na = *reinterpret_cast<const int64_t *>(host.data() + o.na);
                ex[i].n_assignments = na;
                if (o.hdp) {
                    const int64_t got = std::min(na, o.cap);
                    if (got > 0) {
                        std::memcpy(ex[i].assignment_kmers, host.data() + o.ak, sizeof(int64_t) * (size_t) got);
                        std::memcpy(ex[i].assignment_events, host.data() + o.ae, sizeof(int64_t) * (size_t) got);
                    }
                    if (na > o.cap) read_status[i] = SA_E_OUTPUT;
                }
            }
            for (int64_t i = 0; i < n; ++i)
                if (!read_status[i] && s->read_count[i] == 0) ex[i].n_assignments = 0;
        }
    }
    mem_put(blk);
    cudaSetDevice(prev_dev);
    plain_destroy(s);
    return st;
}

extern "C" sa_status sa_getExpectationsUsingAnchors(const sa_state_machine *sm_c, const char *reference,
                                                    int64_t reference_length, const double *events, int64_t n_events,
                                                    const int64_t *anchors, int64_t n_anchors, const sa_params *p,
                                                    int32_t ragged_left, int32_t ragged_right, sa_expectations *ex) {
    if (!sm_c || !p || !ex || !ex->event_expectations || !ex->posteriors || !ex->observed || reference_length < 0 ||
        n_events < 0 || n_anchors < 0)
        return SA_E_ARG;
    if ((reference_length > 0 && !reference) || (n_events > 0 && !events) || (n_anchors > 0 && !anchors))
        return SA_E_ARG;
    sa_status st = check_params(*p);
    if (st) return st;
    sa_read rd;
    std::memset(&rd, 0, sizeof(rd));
    rd.sm = sm_c;
    rd.reference = reference;
    rd.reference_length = reference_length;
    rd.events = events;
    rd.n_events = n_events;
    rd.anchors = anchors;
    rd.n_anchors = n_anchors;
    rd.scale = sm_c->scale;
    rd.shift = sm_c->shift;
    rd.var = sm_c->var;
    rd.ragged_left = ragged_left;
    rd.ragged_right = ragged_right;
    rd.degenerate = SA_CYTOSINE_METHYLATION3;
    int32_t rs = SA_OK;
    st = expectations_batch(&rd, 1, *p, ex, &rs);
    return st ? st : (sa_status) rs;
}

extern "C" sa_status sa_getExpectationsBatch(const sa_read *reads, int64_t n_reads, const sa_params *p,
                                             sa_expectations *ex, int32_t *read_status) {
    if (n_reads < 0 || !p || (n_reads > 0 && (!reads || !ex || !read_status))) return SA_E_ARG;
    sa_status st = check_params(*p);
    if (st) return st;
    if (n_reads == 0) return SA_OK;
    return expectations_batch(reads, n_reads, *p, ex, read_status);
}
