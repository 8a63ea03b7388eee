// The host steps on either side of the path, as signalMachine runs them for one read: anchor pairs
// from the guide alignment (before), and the ordering, score and posterior files of the aligned
// pairs (after).  Integer and text work, exact with the reference.
#include <algorithm>
#include <cinttypes>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sa_internal.h"

namespace {

using sa::kMaxK;
using sa::kPairProb1;

// The two passes of filterToRemoveOverlap (pairwiseAligner.c:1575-1616) over pairs sorted by (x, y):
// backwards, a pair survives if it is below every later pair in both coordinates; forwards, a pair is
// kept if it is above every earlier pair in both coordinates and its value survived the first pass.
sa_status filter_overlap(const int64_t *in, int64_t n, std::vector<int64_t> &out) {
    // the reference asserts sorted input: x non-decreasing, y non-decreasing for equal x
    for (int64_t i = 1; i < n; ++i) {
        const int64_t px = in[2 * (i - 1)], py = in[2 * (i - 1) + 1], x = in[2 * i], y = in[2 * i + 1];
        if (x < px || (x == px && y < py)) return SA_E_ANCHORS;
    }
    std::vector<char> survive(n, 0);
    int64_t pX = INT64_MAX, pY = INT64_MAX;
    for (int64_t i = n - 1; i >= 0; --i) {
        const int64_t x = in[2 * i], y = in[2 * i + 1];
        if (x < pX && y < pY) survive[i] = 1;
        pX = std::min(pX, x);
        pY = std::min(pY, y);
    }
    // membership is by value (a sorted set of tuples): equal pairs are adjacent in sorted input, so a
    // value survived if any of its run did
    for (int64_t i = 0; i < n;) {
        int64_t j = i;
        char any = 0;
        while (j < n && in[2 * j] == in[2 * i] && in[2 * j + 1] == in[2 * i + 1]) any |= survive[j++];
        for (int64_t k = i; k < j; ++k) survive[k] = any;
        i = j;
    }
    out.clear();
    pX = INT64_MIN;
    pY = INT64_MIN;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t x = in[2 * i], y = in[2 * i + 1];
        if (x > pX && y > pY && survive[i]) {
            out.push_back(x);
            out.push_back(y);
        }
        pX = std::max(pX, x);
        pY = std::max(pY, y);
    }
    return SA_OK;
}

// the k-mer string of id over the sorted alphabet (kmer_id inverted, nanopore_hdp.c:360-393)
void kmer_string(const sa_state_machine *sm, int64_t id, char *buf) {
    const int k = sm->kmer_length;
    const int64_t a = (int64_t) sm->alphabet.size();
    for (int i = k - 1; i >= 0; --i) {
        buf[i] = sm->alphabet[(size_t) (id % a)];
        id /= a;
    }
    buf[k] = 0;
}

// reverse complement as sonLib's stString_reverseComplementString does it: A/C/G/T in either case
// complemented, every other character (N, X, methyl bases) kept
void reverse_complement(const char *in, int k, char *out) {
    for (int i = 0; i < k; ++i) {
        char c = in[k - 1 - i];
        switch (c) {
            case 'A': c = 'T'; break;
            case 'C': c = 'G'; break;
            case 'G': c = 'C'; break;
            case 'T': c = 'A'; break;
            case 'a': c = 't'; break;
            case 'c': c = 'g'; break;
            case 'g': c = 'c'; break;
            case 't': c = 'a'; break;
            default: break;
        }
        out[i] = c;
    }
    out[k] = 0;
}

void append(std::string &s, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void append(std::string &s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    const int n = std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (n < (int) sizeof(buf)) {
        s.append(buf, (size_t) std::max(n, 0));
        return;
    }
    std::vector<char> big((size_t) n + 1);
    va_start(ap, fmt);
    std::vsnprintf(big.data(), big.size(), fmt, ap);
    va_end(ap);
    s.append(big.data(), (size_t) n);
}

sa_status format_alignment(sa_output_format fmt, const sa_state_machine *sm, const sa_output_read *rd,
                           const sa_aligned_pair *pairs, int64_t n, std::string &out) {
    if (!sm || !rd || (n > 0 && !pairs) || !rd->target || rd->target_length < 0 || (rd->n_events > 0 && !rd->events))
        return SA_E_ARG;
    if (fmt == SA_OUTPUT_FULL && (!rd->contig || !rd->read_label)) return SA_E_ARG;
    if (fmt == SA_OUTPUT_VARIANT_CALLER && !rd->read_label) return SA_E_ARG;
    const int k = sm->kmer_length;
    const char *strand_label = rd->strand == 0 ? "t" : "c";
    // (template, forward) and (complement, backward) read the reference as given; the other two
    // through its reverse complement (adjustReferenceCoordinate / makeReferenceKmer /
    // adjustQueryPosition, signalMachine.c:33-66)
    const bool as_given = (rd->strand == 0 && rd->forward) || (rd->strand != 0 && !rd->forward);
    const int64_t ref_length = rd->target_length;
    const int64_t ref_length_kmers = ref_length - k;
    char k_i[kMaxK + 1], ref_kmer[kMaxK + 1], path_kmer[kMaxK + 1];
    for (int64_t i = 0; i < n; ++i) {
        const sa_aligned_pair &pr = pairs[i];
        const int64_t x_i = pr.x;
        const int64_t y = pr.y + rd->event_offset;
        const double p = (double) pr.score / kPairProb1;
        if (pr.kmer < 0 || pr.kmer >= sm->n_kmers) return SA_E_ARG;
        kmer_string(sm, pr.kmer, path_kmer);
        if (fmt == SA_OUTPUT_FULL || fmt == SA_OUTPUT_ASSIGNMENTS) {
            if (y < 0 || y >= rd->n_events) return SA_E_ARG;
        }
        if (fmt != SA_OUTPUT_ASSIGNMENTS) {
            if (x_i < 0 || x_i + k > ref_length) return SA_E_ARG;
            std::memcpy(k_i, rd->target + x_i, (size_t) k);
            k_i[k] = 0;
            if (as_given) std::memcpy(ref_kmer, k_i, (size_t) k + 1);
            else reverse_complement(k_i, k, ref_kmer);
        }
        const int64_t x_adj = as_given ? x_i + rd->reference_offset
                                       : ref_length_kmers - (x_i + (ref_length - rd->reference_offset));
        const double *ev = rd->events ? rd->events + 4 * y : nullptr;
        const double e_mean = sm->match[(size_t) pr.kmer * 5];
        switch (fmt) {
            case SA_OUTPUT_FULL: {
                // writePosteriorProbsFull (signalMachine.c:68-131)
                const double e_noise = sm->match[(size_t) pr.kmer * 5 + 2];
                const double scaled_mean = e_mean * rd->scale + rd->shift;
                const double scaled_noise = e_noise * rd->scale_sd;
                const double descaled = (ev[0] + rd->var * e_mean - rd->scale * e_mean - rd->shift) / rd->var;
                append(out, "%s\t%" PRId64 "\t%s\t%s\t%s\t%" PRId64 "\t%f\t%f\t%f\t%s\t%f\t%f\t%f\t%f\t%f\t%s\n",
                       rd->contig, x_adj, ref_kmer, rd->read_label, strand_label, y, ev[0], ev[1], ev[2], k_i,
                       scaled_mean, scaled_noise, p, descaled, e_mean, path_kmer);
                break;
            }
            case SA_OUTPUT_VARIANT_CALLER: {
                // writePosteriorProbsVC (signalMachine.c:133-200): one line per degenerate ('X')
                // position of the reference k-mer (path_findDegeneratePositions, pairwiseAligner.c:510-524)
                const char *forward_label = rd->forward ? "forward" : "backward";
                for (int q = 0; q < k; ++q) {
                    if (ref_kmer[q] != 'X') continue;
                    const int qpos = as_given ? q : (k - 1) - q;
                    append(out, "%" PRId64 "\t%" PRId64 "\t%c\t%f\t%s\t%s\t%s\n", y, x_adj + q, path_kmer[qpos], p,
                           strand_label, forward_label, rd->read_label);
                }
                break;
            }
            case SA_OUTPUT_ASSIGNMENTS: {
                // writeAssignments (signalMachine.c:202-238)
                const double descaled = (ev[0] + rd->var * e_mean - rd->scale * e_mean - rd->shift) / rd->var;
                append(out, "%s\t%s\t%lf\t%lf\n", path_kmer, strand_label, descaled, p);
                break;
            }
            default:
                return SA_E_ARG;
        }
    }
    return SA_OK;
}

}  // namespace

extern "C" {

sa_status sa_filterToRemoveOverlap(const int64_t *pairs, int64_t n_pairs, int64_t *out, int64_t *n_out) {
    if (n_pairs < 0 || (n_pairs > 0 && (!pairs || !out)) || !n_out) return SA_E_ARG;
    std::vector<int64_t> kept;
    const sa_status st = filter_overlap(pairs, n_pairs, kept);
    if (st) return st;
    if (!kept.empty()) std::memcpy(out, kept.data(), kept.size() * sizeof(int64_t));
    *n_out = (int64_t) kept.size() / 2;
    return SA_OK;
}

sa_status sa_guideAlignmentToRebasedAnchorPairs(sa_guide_alignment *ga, const sa_cigar_op *ops, int64_t n_ops,
                                                int64_t trim, int64_t *out, int64_t capacity, int64_t *n_out) {
    if (!ga || n_ops < 0 || (n_ops > 0 && !ops) || !n_out || capacity < 0 || (capacity > 0 && !out) || trim < 0)
        return SA_E_ARG;
    *n_out = 0;
    // signalUtils_rebasePairwiseAlignmentCoordinates (signalMachineUtils.c:130-140): shift the
    // reference to start at 0, flipping a reverse strand
    const bool flip = ga->strand1 == 0;
    const int64_t shift = ga->strand1 ? ga->start1 : ga->end1;
    ga->start1 -= shift;
    ga->end1 -= shift;
    if (flip) {
        ga->strand1 = 1;
        std::swap(ga->start1, ga->end1);
    }
    // checkPairwiseAlignment: the operations span both sequences' coordinates, on forward strands
    if (ga->strand2 != 1 || ga->start1 > ga->end1 || ga->start2 > ga->end2) return SA_E_ARG;
    int64_t span1 = 0, span2 = 0;
    for (int64_t i = 0; i < n_ops; ++i) {
        if (ops[i].length < 0 || ops[i].op < SA_CIGAR_MATCH || ops[i].op > SA_CIGAR_INDEL_Y) return SA_E_ARG;
        if (ops[i].op != SA_CIGAR_INDEL_Y) span1 += ops[i].length;
        if (ops[i].op != SA_CIGAR_INDEL_X) span2 += ops[i].length;
    }
    if (span1 != ga->end1 - ga->start1 || span2 != ga->end2 - ga->start2) return SA_E_ARG;
    // convertPairwiseForwardStrandAlignmentToAnchorPairs (pairwiseAligner.c:1454-1478)
    std::vector<int64_t> pairs;
    int64_t j = ga->start1, kk = ga->start2;
    for (int64_t i = 0; i < n_ops; ++i) {
        if (ops[i].op == SA_CIGAR_MATCH)
            for (int64_t l = trim; l < ops[i].length - trim; ++l) {
                pairs.push_back(j + l);
                pairs.push_back(kk + l);
            }
        if (ops[i].op != SA_CIGAR_INDEL_Y) j += ops[i].length;
        if (ops[i].op != SA_CIGAR_INDEL_X) kk += ops[i].length;
    }
    // stList_sort by stIntTuple_cmpFn (lexicographic), then filterToRemoveOverlap
    const int64_t np = (int64_t) pairs.size() / 2;
    std::vector<int64_t> idx(np);
    for (int64_t i = 0; i < np; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
        if (pairs[2 * a] != pairs[2 * b]) return pairs[2 * a] < pairs[2 * b];
        return pairs[2 * a + 1] < pairs[2 * b + 1];
    });
    std::vector<int64_t> sorted(2 * np);
    for (int64_t i = 0; i < np; ++i) {
        sorted[2 * i] = pairs[2 * idx[i]];
        sorted[2 * i + 1] = pairs[2 * idx[i] + 1];
    }
    std::vector<int64_t> kept;
    const sa_status st = filter_overlap(sorted.data(), np, kept);
    if (st) return st;
    *n_out = (int64_t) kept.size() / 2;
    if (*n_out > capacity) return SA_E_OUTPUT;
    if (!kept.empty()) std::memcpy(out, kept.data(), kept.size() * sizeof(int64_t));
    return SA_OK;
}

sa_status sa_getRemappedAnchorPairs(const int64_t *anchors, int64_t n_anchors, const int64_t *event_map,
                                    int64_t map_length, int64_t map_offset, int64_t *out, int64_t *n_out) {
    if (n_anchors < 0 || (n_anchors > 0 && (!anchors || !out)) || !n_out || !event_map || map_length <= 0)
        return SA_E_ARG;
    if (map_offset < 0 || map_offset >= map_length) return SA_E_ARG;
    std::vector<int64_t> remapped(2 * (size_t) n_anchors);
    const int64_t base = event_map[map_offset];
    for (int64_t i = 0; i < n_anchors; ++i) {
        const int64_t y = anchors[2 * i + 1];
        if (y < 0 || y >= map_length) return SA_E_ARG;
        remapped[2 * i] = anchors[2 * i];
        remapped[2 * i + 1] = event_map[y] - base;
    }
    std::vector<int64_t> kept;
    const sa_status st = filter_overlap(remapped.data(), n_anchors, kept);
    if (st) return st;
    if (!kept.empty()) std::memcpy(out, kept.data(), kept.size() * sizeof(int64_t));
    *n_out = (int64_t) kept.size() / 2;
    return SA_OK;
}

void sa_sortByXPlusYCoordinate(sa_aligned_pair *pairs, int64_t n_pairs) {
    if (!pairs || n_pairs <= 1) return;
    std::stable_sort(pairs, pairs + n_pairs,
                     [](const sa_aligned_pair &a, const sa_aligned_pair &b) { return a.x + a.y < b.x + b.y; });
}

double sa_scoreByPosteriorProbabilityIgnoringGaps(const sa_aligned_pair *pairs, int64_t n_pairs) {
    // totalScore accumulates the integer scores in a double (signalMachine.c:317-324)
    double total = 0.0;
    for (int64_t i = 0; i < n_pairs; ++i) total += (double) pairs[i].score;
    return 100.0 * total / ((double) n_pairs * sa::kPairProb1);
}

sa_status sa_formatAlignment(sa_output_format fmt, const sa_state_machine *sm, const sa_output_read *rd,
                             const sa_aligned_pair *pairs, int64_t n_pairs, char **text, int64_t *length) {
    if (!text || !length || n_pairs < 0) return SA_E_ARG;
    *text = nullptr;
    *length = 0;
    std::string s;
    const sa_status st = format_alignment(fmt, sm, rd, pairs, n_pairs, s);
    if (st) return st;
    char *buf = static_cast<char *>(std::malloc(s.size() + 1));
    if (!buf) return SA_E_NOMEM;
    std::memcpy(buf, s.data(), s.size());
    buf[s.size()] = 0;
    *text = buf;
    *length = (int64_t) s.size();
    return SA_OK;
}

sa_status sa_outputAlignment(sa_output_format fmt, const char *path, const sa_state_machine *sm,
                             const sa_output_read *rd, const sa_aligned_pair *pairs, int64_t n_pairs) {
    if (!path || n_pairs < 0) return SA_E_ARG;
    std::string s;
    const sa_status st = format_alignment(fmt, sm, rd, pairs, n_pairs, s);
    if (st) return st;
    FILE *f = std::fopen(path, "a");
    if (!f) return SA_E_FILE;
    const size_t w = std::fwrite(s.data(), 1, s.size(), f);
    const int c = std::fclose(f);
    return (w == s.size() && c == 0) ? SA_OK : SA_E_FILE;
}

void sa_free_text(char *text) { std::free(text); }

}  // extern "C"
