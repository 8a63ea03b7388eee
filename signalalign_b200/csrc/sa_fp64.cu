// Plain FP64 form: one region (read, or split sub-region) per kernel launch, one CTA sweeping the
// band anti-diagonal by anti-diagonal in log space with the reference's logAdd, windowed traceback
// and every-10th-anti-diagonal total-probability refresh (getPosteriorProbsWithBanding,
// pairwiseAligner.c:1282-1420).  It is the parity anchor of the engine: results agree with
// signalAlign's CPU code to rounding.  Compiled with -fmad=false.
//
// Device layout of a region (all global memory):
//   xl[d], xr[d]     band of anti-diagonal d (xmy range), d = 0..n
//   coff[d]          index of anti-diagonal d's first cell (prefix sum of widths), n+2 entries
//   kmer[x]          k-mer id of matrix column x (x = 0 is the empty prefix, id -1), lX+1 entries
//   ev[y]            (mean, noise) of event y, lY entries
//   F, B             3 doubles per cell (match, gap-X, gap-Y), forward and backward
//   P                refresh total probabilities, indexed by anti-diagonal
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
    const int32_t *xl, *xr;
    const int64_t *coff;
    const int32_t *kmer;
    const double2 *ev;
    const Window *win;
    double *F, *B, *P;
    double threshold;
    sa_aligned_pair *out;
    unsigned long long *out_count;
    int64_t out_cap;
    int32_t *status;
};

__device__ __forceinline__ double *cell(double *base, const Region64 &R, int32_t d, int32_t xmy) {
    return base + 3 * (R.coff[d] + ((xmy - R.xl[d]) >> 1));
}

__device__ __forceinline__ bool in_band(const Region64 &R, int32_t d, int32_t xmy) {
    return d >= 0 && d <= R.n && xmy >= R.xl[d] && xmy <= R.xr[d];
}

// forward cell by pull: the reference's push order (lower -> gap-X, middle -> match, upper -> gap-Y,
// stateMachine3_cellCalculate, stateMachine.c:1194-1257) with each state accumulated from LOG_ZERO
__device__ void forward_cell(const Model64 &M, const Region64 &R, int32_t d, int32_t xmy) {
    const int32_t x = (d + xmy) >> 1, y = (d - xmy) >> 1;
    const int32_t kid = R.kmer[x];
    double vM = kNegInf, vX = kNegInf, vY = kNegInf;
    if (in_band(R, d - 1, xmy - 1)) {
        const double *l = cell(R.F, R, d - 1, xmy - 1);
        double e = emit_gapx(M, kid);
        vX = log_add(vX, l[S_M] + (e + M.t[T_OX]));
        vX = log_add(vX, l[S_X] + (e + M.t[T_EX]));
        vX = log_add(vX, l[S_Y] + (e + M.t[T_SX]));
    }
    if (d >= 2 && in_band(R, d - 2, xmy)) {
        const double *m = cell(R.F, R, d - 2, xmy);
        double2 ev = R.ev[y - 1];
        double e = emit_event(M, kid, ev.x, ev.y, true);
        vM = log_add(vM, m[S_M] + (e + M.t[T_MC]));
        vM = log_add(vM, m[S_X] + (e + M.t[T_MFGX]));
        vM = log_add(vM, m[S_Y] + (e + M.t[T_MFGY]));
    }
    if (in_band(R, d - 1, xmy + 1)) {
        const double *u = cell(R.F, R, d - 1, xmy + 1);
        double2 ev = R.ev[y - 1];
        double e = emit_event(M, kid, ev.x, ev.y, false);
        vY = log_add(vY, u[S_M] + (e + M.t[T_OY]));
        vY = log_add(vY, u[S_Y] + (e + M.t[T_EY]));
    }
    double *c = cell(R.F, R, d, xmy);
    c[S_M] = vM;
    c[S_X] = vX;
    c[S_Y] = vY;
}

// backward cell by pull.  The reference pushes from later cells into earlier ones
// (doTransitionBackward, pairwiseAligner.c:715-720); a cell on anti-diagonal d receives, in time
// order, the middle contribution of (x+1, y+1) on d+2, then the upper-role contribution of (x, y+1)
// and the lower-role contribution of (x+1, y), both on d+1 (cells there are walked in ascending xmy).
__device__ void backward_cell(const Model64 &M, const Region64 &R, int32_t d, int32_t xmy, int32_t top) {
    const int32_t x = (d + xmy) >> 1, y = (d - xmy) >> 1;
    double vM = kNegInf, vX = kNegInf, vY = kNegInf;
    if (d + 2 <= top && in_band(R, d + 2, xmy)) {
        const double *m = cell(R.B, R, d + 2, xmy);
        double2 ev = R.ev[y];
        double e = emit_event(M, R.kmer[x + 1], ev.x, ev.y, true);
        vM = log_add(vM, m[S_M] + (e + M.t[T_MC]));
        vX = log_add(vX, m[S_M] + (e + M.t[T_MFGX]));
        vY = log_add(vY, m[S_M] + (e + M.t[T_MFGY]));
    }
    if (in_band(R, d + 1, xmy - 1)) {
        const double *u = cell(R.B, R, d + 1, xmy - 1);
        double2 ev = R.ev[y];
        double e = emit_event(M, R.kmer[x], ev.x, ev.y, false);
        vM = log_add(vM, u[S_Y] + (e + M.t[T_OY]));
        vY = log_add(vY, u[S_Y] + (e + M.t[T_EY]));
    }
    if (in_band(R, d + 1, xmy + 1)) {
        const double *l = cell(R.B, R, d + 1, xmy + 1);
        double e = emit_gapx(M, R.kmer[x + 1]);
        vM = log_add(vM, l[S_X] + (e + M.t[T_OX]));
        vX = log_add(vX, l[S_X] + (e + M.t[T_EX]));
        vY = log_add(vY, l[S_X] + (e + M.t[T_SX]));
    }
    double *c = cell(R.B, R, d, xmy);
    c[S_M] = vM;
    c[S_X] = vX;
    c[S_Y] = vY;
}

// diagonalCalculationTotalProbability (pairwiseAligner.c:1182-1200), sequential in the reference's
// order: dot product of F and B on d in ascending xmy, then the matches that jump from d-1 over d
// into d+1, dotted with B[d+1].
__device__ double total_probability(const Model64 &M, const Region64 &R, int32_t d, bool have_next) {
    double total = kNegInf;
    for (int32_t xmy = R.xl[d]; xmy <= R.xr[d]; xmy += 2) {
        const double *f = cell(R.F, R, d, xmy), *b = cell(R.B, R, d, xmy);
        double s = f[S_M] + b[S_M];
        s = log_add(s, f[S_X] + b[S_X]);
        s = log_add(s, f[S_Y] + b[S_Y]);
        total = log_add(total, log_add(kNegInf, s));
    }
    if (d >= 1 && have_next) {
        const int32_t dn = d + 1;
        double through = kNegInf;
        for (int32_t xmy = R.xl[dn]; xmy <= R.xr[dn]; xmy += 2) {
            double m = kNegInf;
            if (in_band(R, d - 1, xmy)) {
                const int32_t x = (dn + xmy) >> 1, y = (dn - xmy) >> 1;
                const double *f = cell(R.F, R, d - 1, xmy);
                double2 ev = R.ev[y - 1];
                double e = emit_event(M, R.kmer[x], ev.x, ev.y, true);
                m = log_add(m, f[S_M] + (e + M.t[T_MC]));
                m = log_add(m, f[S_X] + (e + M.t[T_MFGX]));
                m = log_add(m, f[S_Y] + (e + M.t[T_MFGY]));
            }
            const double *b = cell(R.B, R, dn, xmy);
            double s = m + b[S_M];
            s = log_add(s, kNegInf + b[S_X]);
            s = log_add(s, kNegInf + b[S_Y]);
            through = log_add(through, log_add(kNegInf, s));
        }
        total = log_add(total, through);
    }
    return total;
}

__global__ void __launch_bounds__(128) region_kernel(Model64 M, Region64 R) {
    const int tid = threadIdx.x, nt = blockDim.x;
    // startStateProb / raggedStartStateProb (stateMachine.c:1022-1032) on anti-diagonal 0
    if (tid == 0) {
        double *c = cell(R.F, R, 0, 0);
        c[S_M] = R.ragged_left ? kNegInf : 0.0;
        c[S_X] = R.ragged_left ? 0.0 : kNegInf;
        c[S_Y] = R.ragged_left ? 0.0 : kNegInf;
    }
    __syncthreads();
    int32_t wi = 0;
    Window W = R.win[0];
    for (int32_t d = 1; d <= R.n; ++d) {
        for (int32_t xmy = R.xl[d] + 2 * tid; xmy <= R.xr[d]; xmy += 2 * nt) forward_cell(M, R, d, xmy);
        __syncthreads();
        if (d != W.D) continue;
        // endStateProb / raggedEndStateProb (stateMachine.c:1034-1061) on the traceback anti-diagonal
        const bool ragged_end = W.at_end && R.ragged_right;
        const double e0 = ragged_end ? (M.t[T_OX] + M.t[T_OY]) / 2.0 : M.t[T_MC];
        const double e1 = ragged_end ? M.t[T_EX] : M.t[T_MFGX];
        const double e2 = ragged_end ? M.t[T_EY] : M.t[T_MFGY];
        for (int32_t xmy = R.xl[d] + 2 * tid; xmy <= R.xr[d]; xmy += 2 * nt) {
            double *c = cell(R.B, R, d, xmy);
            c[S_M] = e0;
            c[S_X] = e1;
            c[S_Y] = e2;
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
        // diagonalCalculationPosteriorMatchProbs (pairwiseAligner.c:1202-1253) on (T, from]
        for (int32_t d2 = W.from; d2 > W.T; --d2) {
            const double total = R.P[W.from - 10 * ((W.from - d2) / 10)];
            for (int32_t xmy = R.xl[d2] + 2 * tid; xmy <= R.xr[d2]; xmy += 2 * nt) {
                const int32_t x = (d2 + xmy) >> 1, y = (d2 - xmy) >> 1;
                if (!(x > 0 && y > 0)) continue;
                const double *f = cell(R.F, R, d2, xmy), *b = cell(R.B, R, d2, xmy);
                double p = exp((f[S_M] + b[S_M]) - total);
                if (p >= R.threshold) {
                    if (p > 1.0) p = 1.0;
                    unsigned long long slot = atomicAdd(R.out_count, 1ULL);
                    if ((int64_t) slot < R.out_cap) {
                        sa_aligned_pair o;
                        o.score = (int64_t) floor(p * 10000000.0);
                        o.x = x - 1;
                        o.y = y - 1;
                        o.kmer = R.kmer[x];
                        R.out[slot] = o;
                    } else if (R.status) {
                        atomicExch(R.status, (int32_t) SA_E_OUTPUT);
                    }
                }
            }
        }
        __syncthreads();
        if (W.at_end) break;
        W = R.win[++wi];
    }
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    sa_status alloc(size_t n) {
        if (n == 0) n = 1;
        return cudaMalloc((void **) &p, n * sizeof(T)) == cudaSuccess ? SA_OK : SA_E_NOMEM;
    }
    sa_status put(const T *src, size_t n) {
        sa_status st = alloc(n);
        if (st) return st;
        if (n && cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return SA_E_CUDA;
        return SA_OK;
    }
};

struct Emitted {
    sa_aligned_pair pair;
    int64_t key_window, key_diag, key_xmy;
};

}  // namespace
}  // namespace sa

using namespace sa;

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
    auto *sm = const_cast<sa_state_machine *>(sm_c);
    const int k = sm->kmer_length;
    // sequence_correctSeqLength (pairwiseAligner.c:456-471)
    const int64_t lX = reference_length == 0 ? 0 : reference_length - (k - 1);
    if (lX < 0) return SA_E_ARG;
    const int64_t lY = n_events;
    PathTable pt;
    sa_status st = build_paths(sm, reference, lX, degenerate, pt);
    if (st) return st;
    if (pt.multi) return SA_E_UNSUPPORTED;
    std::vector<Region> regions;
    st = plan_regions(anchors, n_anchors, lX, lY, *p, ragged_left != 0, ragged_right != 0, regions);
    if (st) return st;
    st = ensure_device_model(sm);
    if (st) return st;
    int prev_dev = 0;
    if (cudaGetDevice(&prev_dev) != cudaSuccess) return SA_E_CUDA;
    if (cudaSetDevice(sm->dev.device) != cudaSuccess) return SA_E_CUDA;

    dp64::Model64 M;
    std::memset(&M, 0, sizeof(M));
    M.emission = sm->emission;
    for (int i = 0; i < 9; ++i) M.t[i] = sm->t[i];
    M.match = sm->dev.match;
    M.gapy = sm->dev.gapy;
    M.gapx = sm->dev.gapx;
    M.scale = sm->scale;
    M.shift = sm->shift;
    M.var = sm->var;
    if (sm->emission == SA_EMIT_HDP) {
        if (!sm->hdp.present) { cudaSetDevice(prev_dev); return SA_E_UNSUPPORTED; }
        M.grid_length = sm->hdp.grid_length;
        M.grid = sm->dev.hdp_grid;
        M.density = sm->dev.hdp_density;
        M.slope = sm->dev.hdp_slope;
        M.kmer_row = sm->dev.hdp_kmer_row;
    }

    std::vector<Emitted> all;
    double ll = 0.0;
    for (size_t ri = 0; ri < regions.size() && st == SA_OK; ++ri) {
        const Region &rg = regions[ri];
        const int32_t n = (int32_t) (rg.lX + rg.lY);
        std::vector<int64_t> coff(n + 2, 0);
        for (int32_t d = 0; d <= n; ++d) coff[d + 1] = coff[d] + (rg.xmy_r[d] - rg.xmy_l[d]) / 2 + 1;
        std::vector<int32_t> kmer(rg.lX + 1);
        kmer[0] = -1;
        for (int64_t x = 1; x <= rg.lX; ++x) kmer[x] = pt.ids[pt.first[rg.x1 + x]];
        std::vector<double2> ev(rg.lY);
        for (int64_t y = 0; y < rg.lY; ++y)
            ev[y] = make_double2(events[(rg.y1 + y) * kEventParams], events[(rg.y1 + y) * kEventParams + 1]);
        const int64_t cap = 8 * (int64_t) n + 1024;
        DevBuf<int32_t> d_xl, d_xr, d_kmer, d_status;
        DevBuf<int64_t> d_coff;
        DevBuf<double2> d_ev;
        DevBuf<Window> d_win;
        DevBuf<double> d_F, d_B, d_P;
        DevBuf<sa_aligned_pair> d_out;
        DevBuf<unsigned long long> d_count;
        if (!st) st = d_xl.put(rg.xmy_l.data(), rg.xmy_l.size());
        if (!st) st = d_xr.put(rg.xmy_r.data(), rg.xmy_r.size());
        if (!st) st = d_coff.put(coff.data(), coff.size());
        if (!st) st = d_kmer.put(kmer.data(), kmer.size());
        if (!st) st = d_ev.put(ev.data(), ev.size());
        if (!st) st = d_win.put(rg.windows.data(), rg.windows.size());
        if (!st) st = d_F.alloc(3 * (size_t) coff[n + 1]);
        if (!st) st = d_B.alloc(3 * (size_t) coff[n + 1]);
        if (!st) st = d_P.alloc(n + 1);
        if (!st) st = d_out.alloc(cap);
        if (!st) st = d_count.alloc(1);
        if (!st) st = d_status.alloc(1);
        if (st) break;
        if (cudaMemset(d_count.p, 0, sizeof(unsigned long long)) != cudaSuccess ||
            cudaMemset(d_status.p, 0, sizeof(int32_t)) != cudaSuccess) { st = SA_E_CUDA; break; }
        Region64 R;
        R.lX = (int32_t) rg.lX; R.lY = (int32_t) rg.lY; R.n = n; R.n_windows = (int32_t) rg.windows.size();
        R.ragged_left = rg.ragged_left; R.ragged_right = rg.ragged_right;
        R.xl = d_xl.p; R.xr = d_xr.p; R.coff = d_coff.p; R.kmer = d_kmer.p; R.ev = d_ev.p; R.win = d_win.p;
        R.F = d_F.p; R.B = d_B.p; R.P = d_P.p;
        R.threshold = p->threshold;
        R.out = d_out.p; R.out_count = d_count.p; R.out_cap = cap; R.status = d_status.p;
        region_kernel<<<1, 128>>>(M, R);
        count_launch();
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) { st = SA_E_CUDA; break; }
        unsigned long long cnt = 0;
        int32_t kst = 0;
        double top_p = 0.0;
        if (cudaMemcpy(&cnt, d_count.p, sizeof(cnt), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(&kst, d_status.p, sizeof(kst), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(&top_p, d_P.p + n, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
            st = SA_E_CUDA;
            break;
        }
        if (kst) { st = (sa_status) kst; break; }
        ll += top_p;
        std::vector<sa_aligned_pair> got(cnt);
        if (cnt && cudaMemcpy(got.data(), d_out.p, cnt * sizeof(sa_aligned_pair), cudaMemcpyDeviceToHost) != cudaSuccess) {
            st = SA_E_CUDA;
            break;
        }
        // reference emission order: window by window, anti-diagonals descending, xmy ascending
        for (auto &g : got) {
            Emitted e;
            const int64_t d = g.x + g.y + 2, xmy = g.x - g.y;
            int64_t w = 0;
            while (w < (int64_t) rg.windows.size() && d > rg.windows[w].from) ++w;
            e.key_window = ((int64_t) ri << 32) | w;
            e.key_diag = -d;
            e.key_xmy = xmy;
            e.pair = g;
            e.pair.x += rg.x1;
            e.pair.y += rg.y1;
            all.push_back(e);
        }
    }
    cudaSetDevice(prev_dev);
    if (st) return st;
    std::sort(all.begin(), all.end(), [](const Emitted &a, const Emitted &b) {
        if (a.key_window != b.key_window) return a.key_window < b.key_window;
        if (a.key_diag != b.key_diag) return a.key_diag < b.key_diag;
        return a.key_xmy < b.key_xmy;
    });
    auto *outp = (sa_aligned_pair *) std::malloc(std::max<size_t>(1, all.size()) * sizeof(sa_aligned_pair));
    if (!outp) return SA_E_NOMEM;
    for (size_t i = 0; i < all.size(); ++i) outp[i] = all[i].pair;
    *pairs_out = outp;
    *n_pairs_out = (int64_t) all.size();
    if (log_likelihood) *log_likelihood = ll;
    return SA_OK;
}
