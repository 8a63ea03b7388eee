// Host side of the engine: state-machine loading (.model / .nhdp), band geometry, split points,
// traceback-window planning, path k-mers and the device copies of the model tables.
//
// The band, split and window logic must reproduce signalAlign bit for bit; each function cites
// the routine it re-implements (paths inside the signalAlign tree).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "sa_internal.h"

namespace sa {

static std::atomic<int64_t> g_launches{0};
void count_launch(int64_t n) { g_launches += n; }

static std::atomic<int64_t> g_allocations{0};
static std::atomic<int64_t> g_allocation_ns{0};

namespace {
template <typename Fn>
cudaError_t counted(Fn &&fn) {
    const auto t0 = std::chrono::steady_clock::now();
    const cudaError_t rc = fn();
    g_allocation_ns += std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count();
    if (rc == cudaSuccess) ++g_allocations;
    return rc;
}
}  // namespace

cudaError_t device_malloc(void **ptr, size_t bytes) {
    return counted([&]() { return cudaMalloc(ptr, bytes); });
}

cudaError_t pinned_malloc(void **ptr, size_t bytes) {
    return counted([&]() { return cudaHostAlloc(ptr, bytes, cudaHostAllocDefault); });
}

// ------------------------------------------------------------------------------------------------
// band geometry
// ------------------------------------------------------------------------------------------------
namespace {
inline int64_t col_x(int64_t xay, int64_t xmy) { return (xay + xmy) / 2; }
inline int64_t row_y(int64_t xay, int64_t xmy) { return (xay - xmy) / 2; }
inline int64_t clamp_to(int64_t z, int64_t hi) { return z < 0 ? 0 : (z > hi ? hi : z); }
}  // namespace

// band_construct / band_setCurrentDiagonal / band_avoidOffByOne / band_boundCoordinate
// (pairwiseAligner.c:97-182).  Between two consecutive anchors (matrix coordinates +1) the band is
// the box spanned by the previous anchor expanded by -expansion/2 in x and +expansion/2 in y and the
// next anchor expanded the other way; each anti-diagonal is that box's intersection, snapped to the
// anti-diagonal's parity.
sa_status band_construct(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY, int64_t expansion,
                         int64_t *xmy_l, int64_t *xmy_r) {
    if (lX < 0 || lY < 0 || expansion < 0 || expansion % 2 != 0) return SA_E_ARG;
    if (n_anchors > 0 && anchors == nullptr) return SA_E_ARG;
    const int64_t last = lX + lY;
    int64_t next_anchor = 0;
    int64_t prev_xay = 0, prev_xmy = 0, next_xay = 0, next_xmy = 0;
    int64_t box_x_lo = 0, box_y_hi = 0, box_x_hi = 0, box_y_lo = 0;
    for (int64_t xay = 0; xay <= last; ++xay) {
        int64_t lo = box_x_lo - box_y_hi, hi = box_x_hi - box_y_lo;
        // band_avoidOffByOne: round up to the anti-diagonal's parity (branch-free: the parity
        // alternates from one anti-diagonal to the next)
        lo += (xay + lo) & 1;
        hi += (xay + hi) & 1;
        int64_t v = col_x(xay, lo);
        if (v < box_x_lo) lo += 2 * (box_x_lo - v);
        v = row_y(xay, lo);
        if (box_y_hi < v) lo += 2 * (v - box_y_hi);
        v = col_x(xay, hi);
        if (box_x_hi < v) hi -= 2 * (v - box_x_hi);
        v = row_y(xay, hi);
        if (v < box_y_lo) hi -= 2 * (box_y_lo - v);
        if (lo > hi) return SA_E_ANCHORS;
        xmy_l[xay] = lo;
        xmy_r[xay] = hi;
        if (xay == next_xay) {
            prev_xay = next_xay;
            prev_xmy = next_xmy;
            int64_t ax = lX, ay = lY;
            if (next_anchor < n_anchors) {
                ax = anchors[2 * next_anchor] + 1;
                ay = anchors[2 * next_anchor + 1] + 1;
                ++next_anchor;
                if (!(ax > col_x(prev_xay, prev_xmy) && ay > row_y(prev_xay, prev_xmy) && ax <= lX && ay <= lY))
                    return SA_E_ANCHORS;
            }
            next_xay = ax + ay;
            next_xmy = ax - ay;
            box_x_lo = clamp_to(col_x(prev_xay, prev_xmy - expansion), lX);
            box_y_hi = clamp_to(row_y(next_xay, next_xmy - expansion), lY);
            box_x_hi = clamp_to(col_x(next_xay, next_xmy + expansion), lX);
            box_y_lo = clamp_to(row_y(prev_xay, prev_xmy + expansion), lY);
        }
    }
    return SA_OK;
}

// getSplitPointsP / getSplitPoints (pairwiseAligner.c:1706-1757)
sa_status split_points(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY, int64_t limit,
                       bool ragged_left, bool ragged_right, std::vector<int64_t> &regions) {
    regions.clear();
    int64_t x1 = 0, y1 = 0, x2 = 0, y2 = 0;
    const int64_t side = (int64_t) std::sqrt((double) limit);
    auto gap = [&](int64_t px, int64_t py, int64_t nx, int64_t ny, bool skip) -> bool {
        int64_t w = nx - px, h = ny - py;
        if (w * h <= limit) return false;
        int64_t hx = w / 2 > side ? side : w / 2;
        int64_t hy = h / 2 > side ? side : h / 2;
        if (!skip) {
            regions.push_back(x1); regions.push_back(y1);
            regions.push_back(px + hx); regions.push_back(py + hy);
        }
        x1 = nx - hx;
        y1 = ny - hy;
        return true;
    };
    for (int64_t i = 0; i < n_anchors; ++i) {
        int64_t ax = anchors[2 * i], ay = anchors[2 * i + 1];
        gap(x2, y2, ax, ay, ragged_left && i == 0);
        if (ax < x2 || ay < y2 || ax >= lX || ay >= lY) return SA_E_ANCHORS;
        x2 = ax + 1;
        y2 = ay + 1;
    }
    if (!gap(x2, y2, lX, lY, ragged_left && n_anchors == 0) || !ragged_right) {
        regions.push_back(x1); regions.push_back(y1);
        regions.push_back(lX); regions.push_back(lY);
    }
    return SA_OK;
}

sa_status check_params(const sa_params &p) {
    // prerequisites of getPosteriorProbsWithBanding (pairwiseAligner.c:1292-1296)
    if (!(p.threshold >= 0.0 && p.threshold <= 1.0)) return SA_E_ARG;
    if (p.traceback_diagonals < 1 || p.diagonal_expansion < 0 || p.diagonal_expansion % 2 != 0) return SA_E_ARG;
    if (p.min_diags_between_traceback < 2 || !(p.traceback_diagonals + 1 < p.min_diags_between_traceback))
        return SA_E_ARG;
    if (p.split_matrix_bigger_than_this < 1) return SA_E_ARG;
    return SA_OK;
}

// Region geometry of getPosteriorProbsWithBandingSplittingAlignmentsByLargeGaps (pairwiseAligner.c:
// 1773-1837) and, per region, the traceback windows of getPosteriorProbsWithBanding (:1319-1350):
// a window closes at the last anti-diagonal, or at the first anti-diagonal at least
// minDiagsBetweenTraceBack past the previous close whose width is at most 2*expansion+1; its
// posteriors stop traceBackDiagonals+1 anti-diagonals short of the close, except at the end.
sa_status plan_regions(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY, const sa_params &p,
                       bool ragged_left, bool ragged_right, std::vector<Region> &regions) {
    sa_status st = check_params(p);
    if (st) return st;
    std::vector<int64_t> splits;
    st = split_points(anchors, n_anchors, lX, lY, p.split_matrix_bigger_than_this, ragged_left, ragged_right,
                      splits);
    if (st) return st;
    const int64_t n_splits = (int64_t) splits.size() / 4;
    regions.clear();
    int64_t j = 0;
    std::vector<int64_t> sub;
    std::vector<int64_t> xl, xr;
    for (int64_t i = 0; i < n_splits; ++i) {
        int64_t x1 = splits[4 * i], y1 = splits[4 * i + 1], x2 = splits[4 * i + 2], y2 = splits[4 * i + 3];
        sub.clear();
        while (j < n_anchors) {
            int64_t ax = anchors[2 * j], ay = anchors[2 * j + 1];
            if (ax + ay >= x2 + y2) break;
            if (!(ax >= x1 && ax < x2 && ay >= y1 && ay < y2)) return SA_E_ANCHORS;
            sub.push_back(ax - x1);
            sub.push_back(ay - y1);
            ++j;
        }
        Region r;
        r.x1 = x1; r.y1 = y1; r.lX = x2 - x1; r.lY = y2 - y1;
        r.ragged_left = (ragged_left || i > 0) ? 1 : 0;
        r.ragged_right = (ragged_right || i < n_splits - 1) ? 1 : 0;
        const int64_t n = r.lX + r.lY;
        if (n == 0) continue;   // trivial region (pairwiseAligner.c:1299-1301)
        if (n >= INT32_MAX / 2) return SA_E_CAPACITY;
        xl.assign(n + 1, 0);
        xr.assign(n + 1, 0);
        st = band_construct(sub.data(), (int64_t) sub.size() / 2, r.lX, r.lY, p.diagonal_expansion, xl.data(),
                            xr.data());
        if (st) return st;
        r.xmy_l.resize(n + 1);
        r.xmy_r.resize(n + 1);
        int64_t cells = 0;
        int32_t maxw = 0;
        for (int64_t d = 0; d <= n; ++d) {
            r.xmy_l[d] = (int32_t) xl[d];
            r.xmy_r[d] = (int32_t) xr[d];
            int32_t w = (int32_t) ((xr[d] - xl[d]) / 2 + 1);
            cells += w;
            maxw = std::max(maxw, w);
        }
        r.cells = cells;
        r.max_width = maxw;
        int64_t traced_back_to = 0;
        for (int64_t d = 1; d <= n; ++d) {
            const bool at_end = d == n;
            const int64_t w = (xr[d] - xl[d]) / 2 + 1;
            const bool tb = d >= traced_back_to + p.min_diags_between_traceback && w <= p.diagonal_expansion * 2 + 1;
            if (at_end || tb) {
                Window win;
                win.T = (int32_t) traced_back_to;
                win.D = (int32_t) d;
                win.from = (int32_t) (d - (at_end ? 0 : p.traceback_diagonals + 1));
                win.at_end = at_end ? 1 : 0;
                r.windows.push_back(win);
                traced_back_to = win.from;
            }
        }
        regions.push_back(std::move(r));
    }
    if (j != n_anchors) return SA_E_ANCHORS;
    return SA_OK;
}

// ------------------------------------------------------------------------------------------------
// path k-mers
// ------------------------------------------------------------------------------------------------
const char *degenerate_options(int32_t degenerate) {
    // sequence_getBaseOptions (pairwiseAligner.c:264-278)
    switch (degenerate) {
        case SA_CYTOSINE_METHYLATION2: return "CE";
        case SA_CYTOSINE_METHYLATION3: return "CEO";
        case SA_ADENOSINE_METHYLATION: return "AI";
        default: return "ACGT";
    }
}

static int64_t kmer_id_of(const char *kmer, int k, const std::string &alpha) {
    int64_t v = 0;
    const int64_t a = (int64_t) alpha.size();
    for (int i = 0; i < k; ++i) {
        size_t j = alpha.find(kmer[i]);
        if (j == std::string::npos) return -1;
        v = v * a + (int64_t) j;
    }
    return v;
}

// hdCell_construct (pairwiseAligner.c:605-650): nbOptions^(#X) paths per column, the first 'X'
// varying slowest (path_permutePattern, :557-569)
sa_status build_paths(const sa_state_machine *sm, const char *reference, int64_t lX, int32_t degenerate,
                      PathTable &pt) {
    const int k = sm->kmer_length;
    const char *opts = degenerate_options(degenerate);
    const int nopt = (int) std::strlen(opts);
    // character -> digit over the sorted alphabet (-1 outside it); 'X' is expanded below
    int8_t code[256];
    std::memset(code, -1, sizeof(code));
    for (size_t i = 0; i < sm->alphabet.size(); ++i) code[(unsigned char) sm->alphabet[i]] = (int8_t) i;
    const int64_t a = (int64_t) sm->alphabet.size();
    pt.lX = lX;
    pt.multi = false;
    pt.first.assign(lX + 2, 0);
    pt.ids.clear();
    pt.ids.reserve(lX + 1);
    pt.ids.push_back(-1);
    pt.first[0] = 0;
    char buf[kMaxK];
    for (int64_t x = 1; x <= lX; ++x) {
        pt.first[x] = (int32_t) pt.ids.size();
        const char *km = reference + (x - 1);
        int pos[kMaxK], nd = 0;
        int64_t id = 0;
        for (int i = 0; i < k; ++i) {
            if (km[i] == 'X') pos[nd++] = i;
            const int8_t c = code[(unsigned char) km[i]];
            id = id * a + c;
            if (c < 0 && km[i] != 'X') return SA_E_ALPHABET;
        }
        if (nd == 0) {   // one path: the k-mer as written
            pt.ids.push_back((int32_t) id);
            continue;
        }
        int64_t np = 1;
        for (int i = 0; i < nd; ++i) np *= nopt;
        if (np > 1) pt.multi = true;
        for (int64_t q = 0; q < np; ++q) {
            std::memcpy(buf, km, k);
            int64_t rem = q;
            for (int i = nd - 1; i >= 0; --i) {
                buf[pos[i]] = opts[rem % nopt];
                rem /= nopt;
            }
            const int64_t pid = kmer_id_of(buf, k, sm->alphabet);
            if (pid < 0) return SA_E_ALPHABET;
            pt.ids.push_back((int32_t) pid);
        }
    }
    pt.first[lX + 1] = (int32_t) pt.ids.size();
    return SA_OK;
}

// ------------------------------------------------------------------------------------------------
// state machine loading
// ------------------------------------------------------------------------------------------------
static std::vector<double> nanopore_default_transitions() {
    // stateMachine3_setTransitionsToNanoporeDefaults (stateMachine.c:1077-1088)
    return {-0.23552123624314988, -0.21880828092192281, -0.013406326748077823, -1.6269694202638481,
            -4.3187242127300092, -1.6269694202638481, -4.3187242127239411, -INFINITY, -INFINITY};
}

static bool sorted_distinct(const std::string &in, std::string &out) {
    out = in;
    std::sort(out.begin(), out.end());
    for (size_t i = 1; i < out.size(); ++i)
        if (out[i] == out[i - 1]) return false;
    return true;
}

static void build_kmer_strings(sa_state_machine *sm) {
    const int k = sm->kmer_length;
    const int64_t a = (int64_t) sm->alphabet.size();
    sm->kmer_strings.assign(sm->n_kmers, std::string());
    for (int64_t id = 0; id < sm->n_kmers; ++id) {
        std::string s(k, '?');
        int64_t v = id;
        for (int i = k - 1; i >= 0; --i) {
            s[i] = sm->alphabet[v % a];
            v /= a;
        }
        sm->kmer_strings[id] = std::move(s);
    }
}

static sa_status new_machine(sa_machine_type type, sa_emission emission, const char *alphabet, int32_t asz,
                             int32_t k, int32_t device, sa_state_machine **out) {
    if (!alphabet || asz <= 0 || k <= 0 || k > kMaxK || (int32_t) std::strlen(alphabet) < asz) return SA_E_ARG;
    if (type != SA_THREE_STATE && type != SA_THREE_STATE_HDP) return SA_E_UNSUPPORTED;
    if ((type == SA_THREE_STATE_HDP) != (emission == SA_EMIT_HDP)) return SA_E_UNSUPPORTED;
    std::string sorted;
    if (!sorted_distinct(std::string(alphabet, asz), sorted)) return SA_E_ARG;
    double n = std::pow((double) asz, (double) k);
    if (n > 1e8) return SA_E_CAPACITY;
    auto *sm = new (std::nothrow) sa_state_machine();
    if (!sm) return SA_E_NOMEM;
    sm->type = type;
    sm->emission = emission;
    sm->alphabet = sorted;
    sm->kmer_length = k;
    sm->n_kmers = (int64_t) n;
    std::vector<double> t = nanopore_default_transitions();
    for (int i = 0; i < SA_N_TRANSITIONS; ++i) sm->t[i] = t[i];
    sm->dev.device = device;
    build_kmer_strings(sm);
    *out = sm;
    return SA_OK;
}

static bool read_line(std::ifstream &in, std::string &line) {
    return (bool) std::getline(in, line);
}

static bool split_doubles(const std::string &line, std::vector<double> &vals) {
    vals.clear();
    const char *s = line.c_str();
    char *end = nullptr;
    while (true) {
        while (*s == ' ' || *s == '\t' || *s == '\r' || *s == '\n') ++s;
        if (!*s) break;
        errno = 0;
        double v = std::strtod(s, &end);
        if (end == s) return false;
        vals.push_back(v);
        s = end;
    }
    return true;
}

static std::vector<std::string> split_tokens(const std::string &line) {
    std::vector<std::string> out;
    std::istringstream ss(line);
    std::string tok;
    while (ss >> tok) out.push_back(tok);
    return out;
}

// stateMachine3_loadFromFile (stateMachine.c:1328-1426) with stateMachine3_loadTransitionsFromFile
// (:1090-1146): line 0 "stateNumber alphabetSize alphabet kmerLength", line 1 nine transition
// probabilities + likelihood, line 2 the k-mer table.  gapY->gapX lands in GAP_SWITCH_TO_Y, so
// GAP_SWITCH_TO_X keeps its default LOG_ZERO.  The gap-Y table's level_sd is scaled by 1.75.
static sa_status load_model_file(const char *path, sa_machine_type type, sa_emission emission, int32_t device,
                                 sa_state_machine **out) {
    std::ifstream in(path);
    if (!in) return SA_E_FILE;
    std::string l0, l1, l2;
    if (!read_line(in, l0) || !read_line(in, l1) || !read_line(in, l2)) return SA_E_FILE;
    auto t0 = split_tokens(l0);
    if (t0.size() != 4) return SA_E_FILE;
    int32_t state_number = std::atoi(t0[0].c_str()), asz = std::atoi(t0[1].c_str()), k = std::atoi(t0[3].c_str());
    if (state_number != 3) return SA_E_UNSUPPORTED;
    if ((int32_t) t0[2].size() != asz) return SA_E_FILE;
    sa_state_machine *sm = nullptr;
    sa_status st = new_machine(type, emission, t0[2].c_str(), asz, k, device, &sm);
    if (st) return st;
    std::vector<double> tr;
    if (!split_doubles(l1, tr) || tr.size() != 10) { delete sm; return SA_E_FILE; }
    sm->t[SA_T_MATCH_CONTINUE] = std::log(tr[0]);
    sm->t[SA_T_GAP_OPEN_X] = std::log(tr[1]);
    sm->t[SA_T_GAP_OPEN_Y] = std::log(tr[2]);
    sm->t[SA_T_MATCH_FROM_GAP_X] = std::log(tr[3]);
    sm->t[SA_T_GAP_EXTEND_X] = std::log(tr[4]);
    sm->t[SA_T_MATCH_FROM_GAP_Y] = std::log(tr[6]);
    sm->t[SA_T_GAP_SWITCH_TO_Y] = std::log(tr[7]);
    sm->t[SA_T_GAP_EXTEND_Y] = std::log(tr[8]);
    std::vector<double> vals;
    if (!split_doubles(l2, vals) || (int64_t) vals.size() != sm->n_kmers * 5) { delete sm; return SA_E_FILE; }
    sm->match = vals;
    sm->gapy = vals;
    for (int64_t i = 1; i < sm->n_kmers * 5; i += 5) sm->gapy[i] *= 1.75;   // EXTRA_EVENT_NOISE_MULTIPLIER
    sm->gapx.assign(sm->n_kmers, kLogPointOne);
    *out = sm;
    return SA_OK;
}

// deserialize_nhdp (nanopore_hdp.c:1071-1098) + deserialize_hdp (hdp.c:3047-3316): the grid, posterior
// predictives and slopes, observed marks (mark_observed_dps, hdp.c:1127-1155) and per k-mer the row
// of the nearest observed ancestor (dir_proc_density, hdp.c:2594-2597).  Factor trees are skipped.
static sa_status load_nhdp(const char *path, sa_state_machine *sm) {
    std::ifstream in(path);
    if (!in) return SA_E_FILE;
    std::string line;
    auto next = [&](std::string &l) { return (bool) std::getline(in, l); };
    if (!next(line)) return SA_E_FILE;
    int64_t asz = std::atoll(line.c_str());
    if (!next(line)) return SA_E_FILE;
    std::string alpha = split_tokens(line).empty() ? std::string() : split_tokens(line)[0];
    if ((int64_t) alpha.size() < asz) return SA_E_FILE;
    alpha = alpha.substr(0, asz);
    if (!next(line)) return SA_E_FILE;
    int64_t k = std::atoll(line.c_str());
    std::string sorted;
    if (!sorted_distinct(alpha, sorted) || sorted != sm->alphabet || k != sm->kmer_length) return SA_E_FILE;
    if (!next(line)) return SA_E_FILE;
    bool splines = std::atoll(line.c_str()) != 0;
    if (!next(line)) return SA_E_FILE;
    bool has_data = std::atoll(line.c_str()) != 0;
    if (!next(line)) return SA_E_FILE;
    bool sample_gamma = std::atoll(line.c_str()) != 0;
    if (!next(line)) return SA_E_FILE;
    int64_t num_dps = std::atoll(line.c_str());
    if (num_dps <= 0) return SA_E_FILE;
    std::vector<int64_t> dp_ids;
    if (has_data) {
        if (!next(line)) return SA_E_FILE;   // data
        if (!next(line)) return SA_E_FILE;
        for (auto &tok : split_tokens(line)) dp_ids.push_back(std::atoll(tok.c_str()));
    }
    if (!next(line)) return SA_E_FILE;   // base params
    if (!next(line)) return SA_E_FILE;   // grid
    std::vector<double> g;
    if (!split_doubles(line, g) || g.size() < 3) return SA_E_FILE;
    double gs = g[0], ge = g[1];
    int64_t gl = (int64_t) g[2];
    if (gl < 2 || !(ge > gs)) return SA_E_FILE;
    if (!next(line)) return SA_E_FILE;   // gamma
    if (sample_gamma)
        for (int i = 0; i < 4; ++i)
            if (!next(line)) return SA_E_FILE;
    std::vector<int64_t> parent(num_dps, -1);
    for (int64_t i = 0; i < num_dps; ++i) {
        if (!next(line)) return SA_E_FILE;
        auto tok = split_tokens(line);
        if (tok.empty()) return SA_E_FILE;
        if (tok[0] != "-") parent[i] = std::atoll(tok[0].c_str());
        if (parent[i] >= num_dps) return SA_E_FILE;
    }
    std::vector<char> observed(num_dps, 0);
    std::vector<std::vector<double>> dens(num_dps), slope(num_dps);
    std::vector<double> vals;
    if (has_data) {
        for (int64_t d : dp_ids) {
            if (d < 0 || d >= num_dps) return SA_E_FILE;
            while (d >= 0 && !observed[d]) {
                observed[d] = 1;
                dens[d].assign(gl, 0.0);
                d = parent[d];
            }
        }
        for (int64_t i = 0; i < num_dps; ++i) {
            if (!next(line)) return SA_E_FILE;
            if (!split_doubles(line, vals)) return SA_E_FILE;
            if (!vals.empty()) {
                if ((int64_t) vals.size() != gl) return SA_E_FILE;
                dens[i] = vals;
            }
        }
    }
    if (splines) {
        for (int64_t i = 0; i < num_dps; ++i) {
            if (!next(line)) return SA_E_FILE;
            if (!split_doubles(line, vals)) return SA_E_FILE;
            if (!vals.empty()) {
                if ((int64_t) vals.size() != gl) return SA_E_FILE;
                slope[i] = vals;
            }
        }
    }
    std::vector<int64_t> row_of(num_dps, -1), rows;
    for (int64_t i = 0; i < num_dps; ++i)
        if (observed[i]) { row_of[i] = (int64_t) rows.size(); rows.push_back(i); }
    std::vector<double> density(rows.size() * gl), slopes(rows.size() * gl, 0.0);
    for (size_t r = 0; r < rows.size(); ++r) {
        std::copy(dens[rows[r]].begin(), dens[rows[r]].end(), density.begin() + r * gl);
        if (!slope[rows[r]].empty()) std::copy(slope[rows[r]].begin(), slope[rows[r]].end(), slopes.begin() + r * gl);
    }
    std::vector<int64_t> kmer_row(sm->n_kmers, -1);
    for (int64_t kid = 0; kid < std::min<int64_t>(sm->n_kmers, num_dps); ++kid) {
        int64_t d = kid;
        while (d >= 0 && !observed[d]) d = parent[d];
        if (d >= 0) kmer_row[kid] = row_of[d];
    }
    sa_status st = sa_stateMachine_setHdp(sm, gs, ge, gl, (int64_t) rows.size(), density.data(), slopes.data(),
                                          kmer_row.data());
    if (st) return st;
    for (int64_t kid = 0; kid < sm->n_kmers; ++kid) sm->hdp.kmer_observed[kid] = kid < num_dps && observed[kid];
    return SA_OK;
}

// stateMachine3_setModelToHdpExpectedValues (stateMachine.c:1163-1192) with dir_proc_expected_val /
// dir_proc_variance (hdp.c:2772-2800)
static void hdp_expected_values(sa_state_machine *sm) {
    const HdpTables &h = sm->hdp;
    for (int64_t kid = 0; kid < sm->n_kmers; ++kid) {
        if (!h.kmer_observed[kid]) continue;
        int64_t row = h.kmer_row[kid];
        if (row < 0) continue;
        const double *distr = h.density.data() + row * h.grid_length;
        double ev = 0.0;
        for (int64_t i = 1; i < h.grid_length; ++i) ev += h.grid[i] * distr[i] * (h.grid[i] - h.grid[i - 1]);
        double var = 0.0;
        for (int64_t i = 1; i < h.grid_length; ++i) {
            double dev = h.grid[i] - ev;
            var += dev * dev * distr[i] * (h.grid[i] - h.grid[i - 1]);
        }
        sm->match[kid * 5] = ev;
        sm->match[kid * 5 + 1] = std::sqrt(var);
    }
    sm->dev_dirty = true;
}

// ------------------------------------------------------------------------------------------------
// device copies of the tables
// ------------------------------------------------------------------------------------------------
void free_device_model(sa_state_machine *sm) {
    DeviceModel &d = sm->dev;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(d.device);
    cudaFree(d.match); cudaFree(d.gapy); cudaFree(d.gapx); cudaFree(d.klog);
    cudaFree(d.hdp_grid); cudaFree(d.hdp_density); cudaFree(d.hdp_slope); cudaFree(d.hdp_kmer_row);
    cudaFree(d.kc32); cudaFree(d.gapx32);
    int dev = d.device;
    d = DeviceModel();
    d.device = dev;
    cudaSetDevice(prev);
}

template <typename T>
static sa_status upload(T **dst, const T *src, size_t n) {
    if (n == 0) return SA_OK;
    if (device_malloc((void **) dst, n * sizeof(T)) != cudaSuccess) return SA_E_NOMEM;
    if (cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return SA_E_CUDA;
    return SA_OK;
}

bool gapy_follows_match(const sa_state_machine *sm) {
    if (sm->emission == SA_EMIT_HDP) return true;   // the HDP density serves both states
    for (int64_t i = 0; i < sm->n_kmers; ++i) {
        const double *m = &sm->match[5 * i], *y = &sm->gapy[5 * i];
        if (!(y[0] == m[0] && y[2] == m[2] && y[4] == m[4])) return false;
    }
    return true;
}

static std::mutex g_model_mutex;

bool model_resident(const sa_state_machine *sm) {
    std::lock_guard<std::mutex> lock(g_model_mutex);
    return !sm->dev_dirty;
}

sa_status ensure_device_model(sa_state_machine *sm) {
    std::lock_guard<std::mutex> lock(g_model_mutex);
    if (!sm->dev_dirty) return SA_OK;
    free_device_model(sm);
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return SA_E_CUDA;
    if (cudaSetDevice(sm->dev.device) != cudaSuccess) return SA_E_CUDA;
    DeviceModel &d = sm->dev;
    sa_status st = SA_OK;
    const int64_t n = sm->n_kmers;
    std::vector<KmerConst32> kc(n);
    std::vector<float> gx(n);
    for (int64_t i = 0; i < n; ++i) {
        const double *m = &sm->match[i * 5], *y = &sm->gapy[i * 5];
        KmerConst32 &c = kc[i];
        const double half_log_lambda = 0.5 * std::log(m[4]);
        c.mu = (float) m[0];
        c.inv_sd_m = (float) (1.0 / m[1]);
        c.inv_sd_y = (float) (1.0 / y[1]);
        c.k_m = (float) (-1.8378770664093453 - std::log(m[1]) + half_log_lambda);
        c.k_y = (float) (-1.8378770664093453 - std::log(y[1]) + half_log_lambda);
        c.inv_nu = (float) (1.0 / m[2]);
        c.half_lambda = (float) (0.5 * m[4]);
        c.gapx = (float) sm->gapx[i];
        gx[i] = (float) sm->gapx[i];
    }
    if (!st) st = upload(&d.match, sm->match.data(), sm->match.size());
    if (!st) st = upload(&d.gapy, sm->gapy.data(), sm->gapy.size());
    if (!st) st = upload(&d.gapx, sm->gapx.data(), sm->gapx.size());
    if (!st) st = upload(&d.kc32, kc.data(), kc.size());
    if (!st) st = upload(&d.gapx32, gx.data(), gx.size());
    if (!st && sm->hdp.present) {
        const HdpTables &h = sm->hdp;
        st = upload(&d.hdp_grid, h.grid.data(), h.grid.size());
        if (!st) st = upload(&d.hdp_density, h.density.data(), h.density.size());
        if (!st) st = upload(&d.hdp_slope, h.slope.data(), h.slope.size());
        if (!st) st = upload(&d.hdp_kmer_row, h.kmer_row.data(), h.kmer_row.size());
    }
    if (!st) st = compute_kmer_logs(sm);
    cudaSetDevice(prev);
    if (st) {
        free_device_model(sm);
        return st;
    }
    sm->dev_dirty = false;
    return SA_OK;
}

}  // namespace sa

using namespace sa;

// ------------------------------------------------------------------------------------------------
// C ABI: state machine
// ------------------------------------------------------------------------------------------------
extern "C" {

sa_status sa_stateMachine_loadFromFile(const char *model_file, sa_machine_type type, sa_emission emission,
                                       const char *nhdp_file, int32_t set_hdp_expected_values, int32_t device,
                                       sa_state_machine **out) {
    if (!model_file || !out) return SA_E_ARG;
    *out = nullptr;
    sa_state_machine *sm = nullptr;
    sa_status st = load_model_file(model_file, type, emission, device, &sm);
    if (st) return st;
    if (type == SA_THREE_STATE_HDP) {
        if (!nhdp_file) { delete sm; return SA_E_ARG; }
        st = load_nhdp(nhdp_file, sm);
        if (st) { delete sm; return st; }
        if (set_hdp_expected_values) hdp_expected_values(sm);
    }
    *out = sm;
    return SA_OK;
}

sa_status sa_stateMachine_fromTables(sa_machine_type type, sa_emission emission, const char *alphabet,
                                     int32_t alphabet_size, int32_t kmer_length,
                                     const double transitions[SA_N_TRANSITIONS], const double *match,
                                     const double *gap_y, const double *gap_x, int32_t device,
                                     sa_state_machine **out) {
    if (!out || !transitions || !match || !gap_y || !gap_x) return SA_E_ARG;
    *out = nullptr;
    sa_state_machine *sm = nullptr;
    sa_status st = new_machine(type, emission, alphabet, alphabet_size, kmer_length, device, &sm);
    if (st) return st;
    for (int i = 0; i < SA_N_TRANSITIONS; ++i) sm->t[i] = transitions[i];
    sm->match.assign(match, match + sm->n_kmers * 5);
    sm->gapy.assign(gap_y, gap_y + sm->n_kmers * 5);
    sm->gapx.assign(gap_x, gap_x + sm->n_kmers);
    *out = sm;
    return SA_OK;
}

sa_status sa_stateMachine_setHdp(sa_state_machine *sm, double grid_start, double grid_stop, int64_t grid_length,
                                 int64_t n_rows, const double *density, const double *slope,
                                 const int64_t *kmer_row) {
    if (!sm || grid_length < 2 || !(grid_stop > grid_start) || n_rows < 0 || !kmer_row) return SA_E_ARG;
    if (n_rows > 0 && (!density || !slope)) return SA_E_ARG;
    HdpTables &h = sm->hdp;
    h.present = true;
    h.grid_start = grid_start;
    h.grid_stop = grid_stop;
    h.grid_length = grid_length;
    h.n_rows = n_rows;
    // linspace (hdp_math_utils.c:497-509)
    h.grid.resize(grid_length);
    const int64_t nn = grid_length - 1;
    const double dx = (grid_stop - grid_start) / ((double) nn);
    for (int64_t i = 0; i < nn; ++i) h.grid[i] = grid_start + i * dx;
    h.grid[nn] = grid_stop;
    h.density.assign(density, density + n_rows * grid_length);
    h.slope.assign(slope, slope + n_rows * grid_length);
    h.kmer_row.assign(kmer_row, kmer_row + sm->n_kmers);
    h.kmer_observed.assign(sm->n_kmers, 0);
    for (int64_t kid = 0; kid < sm->n_kmers; ++kid) {
        if (h.kmer_row[kid] >= n_rows) return SA_E_ARG;
        h.kmer_observed[kid] = h.kmer_row[kid] >= 0;
    }
    sm->dev_dirty = true;
    return SA_OK;
}

sa_status sa_stateMachine_setScaling(sa_state_machine *sm, double scale, double shift, double var) {
    if (!sm) return SA_E_ARG;
    sm->scale = scale;
    sm->shift = shift;
    sm->var = var;
    return SA_OK;
}

sa_status sa_stateMachine_scaleModel(sa_state_machine *sm, double scale, double shift, double var, double scale_sd,
                                     double var_sd) {
    if (!sm) return SA_E_ARG;
    // emissions_signal_scaleModel (stateMachine.c:630-668)
    for (int64_t i = 0; i < sm->n_kmers * 5; i += 5) {
        double *m = &sm->match[i], *y = &sm->gapy[i];
        m[0] = m[0] * scale + shift;
        m[1] = m[1] * var;
        y[0] = y[0] * scale + shift;
        y[1] = y[1] * var;
        m[2] = m[2] * scale_sd;
        m[4] = m[4] * var_sd;
        m[3] = std::sqrt(std::pow(m[2], 3.0) / m[4]);
        y[2] = y[2] * scale_sd;
        y[4] = y[4] * var_sd;
        y[3] = std::sqrt(std::pow(y[2], 3.0) / m[4]);
    }
    sm->dev_dirty = true;
    return SA_OK;
}

sa_status sa_stateMachine_scaleNoise(sa_state_machine *sm, double scale_sd, double var_sd) {
    if (!sm) return SA_E_ARG;
    // emissions_signal_scaleNoise (stateMachine.c:607-628)
    for (int64_t i = 0; i < sm->n_kmers * 5; i += 5) {
        double *m = &sm->match[i], *y = &sm->gapy[i];
        m[2] = m[2] * scale_sd;
        m[4] = m[4] * var_sd;
        m[3] = std::sqrt(std::pow(m[2], 3.0) / m[4]);
        y[2] = y[2] * scale_sd;
        y[4] = y[4] * var_sd;
        y[3] = std::sqrt(std::pow(y[2], 3.0) / m[4]);
    }
    sm->dev_dirty = true;
    return SA_OK;
}

int32_t sa_stateMachine_kmerLength(const sa_state_machine *sm) { return sm ? sm->kmer_length : 0; }

int64_t sa_stateMachine_numberOfKmers(const sa_state_machine *sm) { return sm ? sm->n_kmers : 0; }

const char *sa_stateMachine_kmerString(const sa_state_machine *sm, int64_t kmer_id) {
    if (!sm || kmer_id < 0 || kmer_id >= sm->n_kmers) return nullptr;
    return sm->kmer_strings[kmer_id].c_str();
}

int64_t sa_stateMachine_kmerId(const sa_state_machine *sm, const char *kmer) {
    if (!sm || !kmer || (int64_t) std::strlen(kmer) < sm->kmer_length) return -1;
    return kmer_id_of(kmer, sm->kmer_length, sm->alphabet);
}

sa_status sa_stateMachine_getTables(const sa_state_machine *sm, double *match, double *gap_y, double *gap_x,
                                    double *transitions) {
    if (!sm) return SA_E_ARG;
    if (match) std::copy(sm->match.begin(), sm->match.end(), match);
    if (gap_y) std::copy(sm->gapy.begin(), sm->gapy.end(), gap_y);
    if (gap_x) std::copy(sm->gapx.begin(), sm->gapx.end(), gap_x);
    if (transitions) std::copy(sm->t, sm->t + SA_N_TRANSITIONS, transitions);
    return SA_OK;
}

sa_status sa_stateMachine_getHdpTables(const sa_state_machine *sm, int64_t *grid_length, int64_t *n_rows,
                                       double *grid, double *density, double *slope, int64_t *kmer_row) {
    if (!sm || !grid_length || !n_rows) return SA_E_ARG;
    const HdpTables &h = sm->hdp;
    if (!h.present) return SA_E_UNSUPPORTED;
    *grid_length = h.grid_length;
    *n_rows = h.n_rows;
    if (grid) std::copy(h.grid.begin(), h.grid.end(), grid);
    if (density) std::copy(h.density.begin(), h.density.end(), density);
    if (slope) std::copy(h.slope.begin(), h.slope.end(), slope);
    if (kmer_row) std::copy(h.kmer_row.begin(), h.kmer_row.end(), kmer_row);
    return SA_OK;
}

void sa_stateMachine_destruct(sa_state_machine *sm) {
    if (!sm) return;
    free_device_model(sm);
    delete sm;
}

void sa_params_default(sa_params *p) {
    // pairwiseAlignmentBandingParameters_construct (pairwiseAligner.c:1843-1856)
    if (!p) return;
    p->threshold = 0.01;
    p->min_diags_between_traceback = 1000;
    p->traceback_diagonals = 40;
    p->diagonal_expansion = 20;
    p->constraint_diagonal_trim = 14;
    p->split_matrix_bigger_than_this = (int64_t) 3000 * 3000;
}

sa_status sa_band_construct(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY, int64_t expansion,
                            int64_t *xmy_l, int64_t *xmy_r) {
    if (!xmy_l || !xmy_r || n_anchors < 0) return SA_E_ARG;
    return band_construct(anchors, n_anchors, lX, lY, expansion, xmy_l, xmy_r);
}

sa_status sa_getSplitPoints(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY,
                            int64_t split_matrix_bigger_than_this, int32_t ragged_left, int32_t ragged_right,
                            int64_t *regions, int64_t max_regions, int64_t *n_regions) {
    if (n_anchors < 0 || (n_anchors > 0 && !anchors) || !n_regions || lX < 0 || lY < 0) return SA_E_ARG;
    std::vector<int64_t> r;
    sa_status st = split_points(anchors, n_anchors, lX, lY, split_matrix_bigger_than_this, ragged_left != 0,
                                ragged_right != 0, r);
    if (st) return st;
    *n_regions = (int64_t) r.size() / 4;
    if (*n_regions > max_regions) return SA_E_OUTPUT;
    if (regions) std::copy(r.begin(), r.end(), regions);
    return SA_OK;
}

void sa_free_pairs(sa_aligned_pair *pairs) { std::free(pairs); }

const char *sa_status_string(sa_status s) {
    switch (s) {
        case SA_OK: return "ok";
        case SA_E_ARG: return "bad argument";
        case SA_E_ALPHABET: return "k-mer character outside the model alphabet";
        case SA_E_ANCHORS: return "anchors not strictly increasing or outside the matrix";
        case SA_E_NOMEM: return "out of memory";
        case SA_E_CUDA: return "CUDA error";
        case SA_E_OUTPUT: return "pair output buffer too small";
        case SA_E_UNSUPPORTED: return "unsupported state machine or input";
        case SA_E_FILE: return "model file missing or malformed";
        case SA_E_TIMEOUT: return "device wait timed out";
        case SA_E_DEVICE: return "device consistency check failed";
        case SA_E_CAPACITY: return "request exceeds a fixed capacity";
    }
    return "unknown status";
}

int64_t sa_kernel_launch_count(void) { return g_launches.load(); }

int64_t sa_allocation_count(void) { return g_allocations.load(); }

double sa_allocation_ms(void) { return 1e-6 * (double) g_allocation_ns.load(); }

}  // extern "C"
