// The maximisation step of signalAlign's EM training and its expectations file: the host work that
// follows sa_getExpectationsUsingAnchors (impl/continuousHmm.c, impl/discreteHmm.c).  Exact with the
// reference: the same sums, divisions, square roots and logs in the same order, and its printf
// formats.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "sa_internal.h"

namespace {

constexpr int kStates = 3;   // match, shortGapX (k-mer skip), shortGapY (extra event)

void append(std::string &s, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void append(std::string &s, const char *fmt, ...) {
    char buf[64];
    va_list ap;
    va_start(ap, fmt);
    const int n = std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (n < (int) sizeof buf) {
        s.append(buf, n);
        return;
    }
    std::string big(n + 1, '\0');
    va_start(ap, fmt);
    std::vsnprintf(&big[0], big.size(), fmt, ap);
    va_end(ap);
    s.append(big.data(), n);
}

// hmmContinuous_writeToFile (continuousHmm.c:872-884) through continuousPairHmm_writeToFile
// (:354-406) or hdpHmm_writeToFile (:572-628)
sa_status format_expectations(const sa_state_machine *sm, const sa_expectations *ex, const double *event_model,
                              const double *events, int64_t n_events, std::string &s) {
    if (!sm || !ex || n_events < 0) return SA_E_ARG;
    const bool hdp = sm->type == SA_THREE_STATE_HDP;
    const int64_t n = sm->n_kmers;
    if (!hdp && (!ex->event_expectations || !ex->posteriors || !ex->observed)) return SA_E_ARG;
    if (hdp) {
        if (ex->n_assignments < 0) return SA_E_ARG;
        if (ex->n_assignments > 0 && (!ex->assignment_kmers || !ex->assignment_events || !events)) return SA_E_ARG;
        for (int64_t i = 0; i < ex->n_assignments; ++i) {
            const int64_t kid = ex->assignment_kmers[i], ev = ex->assignment_events[i];
            if (kid < 0 || kid >= n || ev < 0 || ev >= n_events) return SA_E_ARG;
        }
    }
    // hmmContinuous_checkTransitions (:12-22): a NaN transition leaves the file empty
    for (int i = 0; i < kStates * kStates; ++i)
        if (std::isnan(ex->transitions[i])) return SA_OK;
    const double *model = event_model ? event_model : sm->match.data();
    // line 0: stateNumber, alphabetSize, the sorted alphabet, kmerLength
    append(s, "%d\t%d\t%s\t%d\t\n", kStates, (int) sm->alphabet.size(), sm->alphabet.c_str(), sm->kmer_length);
    // line 1: the nine transitions (from * 3 + to), then the likelihood
    for (int i = 0; i < kStates * kStates; ++i) append(s, "%f\t", ex->transitions[i]);
    append(s, "%f\n", ex->likelihood);
    // line 2: the event model, five parameters per k-mer
    for (int64_t i = 0; i < n * 5; ++i) append(s, "%f\t", model[i]);
    s += '\n';
    if (!hdp) {
        for (int64_t i = 0; i < n * 2; ++i) append(s, "%f\t", ex->event_expectations[i]);
        s += '\n';
        for (int64_t i = 0; i < n; ++i) append(s, "%f\t", ex->posteriors[i]);
        s += '\n';
        for (int64_t i = 0; i < n; ++i) append(s, "%d\t", (int) (ex->observed[i] != 0));
        s += '\n';
    } else {
        // the assigned events' (raw) means, then the assigned k-mers
        for (int64_t i = 0; i < ex->n_assignments; ++i) append(s, "%f\t", events[4 * ex->assignment_events[i]]);
        s += '\n';
        for (int64_t i = 0; i < ex->n_assignments; ++i) {
            s += sm->kmer_strings[ex->assignment_kmers[i]];
            s += '\t';
        }
        s += '\n';
    }
    return SA_OK;
}

}  // namespace

extern "C" {

sa_status sa_normalizeExpectations(sa_expectations *ex, int64_t n_kmers, double *event_model) {
    if (!ex || n_kmers < 0) return SA_E_ARG;
    if (event_model && n_kmers > 0 && (!ex->event_expectations || !ex->posteriors || !ex->observed)) return SA_E_ARG;
    // hmmDiscrete_normalizeTransitions (discreteHmm.c:125-137)
    for (int from = 0; from < kStates; ++from) {
        double total = 0.0;
        for (int to = 0; to < kStates; ++to) total += ex->transitions[from * kStates + to];
        for (int to = 0; to < kStates; ++to)
            ex->transitions[from * kStates + to] = ex->transitions[from * kStates + to] / total;
    }
    if (!event_model) return SA_OK;
    // continuousPairHmm_normalize (continuousHmm.c:283-306): u_k = sum(p * e) / sum(p),
    // o_k = sqrt(spread / sum(p)); a zero keeps the previous value
    for (int64_t i = 0; i < n_kmers; ++i) {
        if (!ex->observed[i]) continue;
        const double w = ex->posteriors[i];
        const double u = ex->event_expectations[2 * i] / w;
        const double o = std::sqrt(ex->event_expectations[2 * i + 1] / w);
        double *row = event_model + 5 * i;
        row[0] = u == 0.0 ? row[0] : u;
        row[1] = o == 0.0 ? row[1] : o;
    }
    return SA_OK;
}

sa_status sa_stateMachine_loadExpectations(sa_state_machine *sm, const double transitions[9],
                                           const double *event_model) {
    if (!sm || !transitions) return SA_E_ARG;
    if (event_model && sm->type != SA_THREE_STATE) return SA_E_UNSUPPORTED;
    if (event_model && sm->n_kmers < 2) return SA_E_ARG;   // the gap-Y index i + 5 needs two k-mers
    const double *T = transitions;
    // continuousPairHmm_loadTransitionsIntoStateMachine (continuousHmm.c:321-339); log(0) = -inf is
    // the reference's LOG_ZERO
    sm->t[SA_T_MATCH_CONTINUE] = std::log(T[0]);
    sm->t[SA_T_GAP_OPEN_X] = std::log(T[1]);
    sm->t[SA_T_GAP_OPEN_Y] = std::log(T[2]);
    sm->t[SA_T_MATCH_FROM_GAP_X] = std::log(T[3]);
    sm->t[SA_T_GAP_EXTEND_X] = std::log(T[4]);
    sm->t[SA_T_GAP_SWITCH_TO_Y] = -INFINITY;
    sm->t[SA_T_MATCH_FROM_GAP_Y] = std::log(T[6]);
    sm->t[SA_T_GAP_EXTEND_Y] = std::log(T[8]);
    sm->t[SA_T_GAP_SWITCH_TO_X] = std::log(T[7]);
    if (!event_model) return SA_OK;
    // continuousPairHmm_loadEmissionsIntoStateMachine (:341-352), in its order: the match table takes
    // each k-mer's level mean and sd; the gap-Y table takes the sd x 1.75 at [i * 5 + 1] and the mean
    // at [i + 5], the index the reference writes (so later k-mers' means overwrite rows 1 onwards)
    const int64_t n = sm->n_kmers;
    for (int64_t i = 0; i < n; ++i) {
        const double mean = event_model[5 * i], sd = event_model[5 * i + 1];
        sm->match[5 * i] = mean;
        sm->match[5 * i + 1] = sd;
        sm->gapy[i + 5] = mean;
        sm->gapy[5 * i + 1] = sd * 1.75;
    }
    sm->dev_dirty = true;
    return SA_OK;
}

sa_status sa_formatExpectations(const sa_state_machine *sm, const sa_expectations *ex, const double *event_model,
                                const double *events, int64_t n_events, char **text, int64_t *length) {
    if (!text || !length) return SA_E_ARG;
    *text = nullptr;
    *length = 0;
    std::string s;
    const sa_status st = format_expectations(sm, ex, event_model, events, n_events, s);
    if (st) return st;
    char *buf = static_cast<char *>(std::malloc(s.size() + 1));
    if (!buf) return SA_E_NOMEM;
    std::memcpy(buf, s.data(), s.size());
    buf[s.size()] = 0;
    *text = buf;
    *length = (int64_t) s.size();
    return SA_OK;
}

sa_status sa_writeExpectations(const char *path, const sa_state_machine *sm, const sa_expectations *ex,
                               const double *event_model, const double *events, int64_t n_events) {
    if (!path) return SA_E_ARG;
    std::string s;
    const sa_status st = format_expectations(sm, ex, event_model, events, n_events, s);
    if (st) return st;
    FILE *f = std::fopen(path, "w");   // hmmContinuous_writeToFile opens with "w"
    if (!f) return SA_E_FILE;
    const size_t w = std::fwrite(s.data(), 1, s.size(), f);
    const int c = std::fclose(f);
    return (w == s.size() && c == 0) ? SA_OK : SA_E_FILE;
}

}  // extern "C"
