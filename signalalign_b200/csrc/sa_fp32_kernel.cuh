// Batched FP32 kernel: one persistent launch over all regions of a batch.
//
// A CTA is two 128-thread groups working on the same region at once:
//   * the forward group sweeps the band anti-diagonal by anti-diagonal (cells spread over the
//     threads, neighbours through a 3-slot shared-memory ring, one named barrier per
//     anti-diagonal).  For every cell it stores to HBM the forward match value and the two event
//     emissions it used (match, extra event); on the anti-diagonals a total-probability refresh
//     will read, it also stores the two gap-state values;
//   * the backward group follows one traceback window behind (getPosteriorProbsWithBanding,
//     pairwiseAligner.c:1319-1410): once the forward group has passed a window's traceback
//     anti-diagonal it runs that window's backward sweep in its own shared-memory ring, reading the
//     stored emissions instead of recomputing them, with the posterior test fused in, so backward
//     values never leave the SM.
// The hand-off is a window counter in shared memory; the backward group's wait on it is bounded
// (it gives up with SA_E_TIMEOUT), and the forward group never waits on the backward group.
//
// The recursion is bound by instruction issue and latency, so the inner loops are branch-free:
// the rings carry a -inf cell on each side and every slot beyond the anti-diagonal's width holds
// -inf, so an absent neighbour is a clamped index that reads -inf (logAdd and the sums then behave
// exactly like the reference's skipped transitions).  Per-anti-diagonal facts (band start, width,
// window end, refresh, which forward values to store) come packed from the host.  Everything that
// does not depend on the recursion is software-pipelined: band facts three anti-diagonals ahead,
// k-mer ids and events two ahead, k-mer constants one ahead and emissions one anti-diagonal early
// (forward); stored emissions, forward values and bases one anti-diagonal ahead (backward).
//
// Values are log probabilities relative to a per-anti-diagonal FP64 base.  The base of d is the
// base of d-2 plus the largest value stored on d-2 (a lagged renormalisation, so the max reduction
// is off the critical path); the recorded bases are built from the same float shifts the kernel
// applies, so they describe the stored values exactly.
//
// Forward store layout per anti-diagonal d (region-relative float offset 5 * first cell, W = width):
//   [ match | match emission | extra-event emission | gap-X | gap-Y ], W floats each; the last two
//   blocks are written only where a refresh needs them.
#pragma once

namespace sa {
namespace fp32 {

using namespace dp32;

constexpr int kGroup = 128;
constexpr int kGroupWarps = kGroup / 32;
constexpr int kThreads = 2 * kGroup;
constexpr int kMaxCpt = 4;
constexpr int kBarForward = 1;
constexpr int kBarBackward = 2;
constexpr int kStoreStride = 5;
enum { ST_M = 0, ST_EM = 1, ST_EY = 2, ST_X = 3, ST_Y = 4 };

// per-anti-diagonal meta: x = xmy of the first cell, y = width | flags
constexpr int32_t kWidthMask = (1 << 20) - 1;
constexpr int32_t kFlagWindowEnd = 1 << 20;   // a traceback window closes here
constexpr int32_t kFlagStoreGaps = 1 << 21;   // a refresh reads this anti-diagonal's gap states
constexpr int32_t kFlagRefresh = 1 << 22;     // total-probability refresh in its posterior window

enum { T_MC = 0, T_MFGX, T_MFGY, T_OX, T_OY, T_EX, T_EY, T_SX, T_SY };

struct ModelDesc {
    const KmerConst32 *kc;
    Hdp32 hdp;
    int32_t emission;
    int32_t pad;
    float t[9];
    float pad2;
};

struct RegionDesc {
    int32_t n, lX, lY, read;
    int32_t n_windows, model;
    int32_t ragged_left, ragged_right;
    int64_t diag_base;    // first anti-diagonal of this region in the per-anti-diagonal arrays
    int64_t cell_base;    // first cell of this region in the forward store
    int64_t win_base;
    int64_t kmer_base;    // k-mer id of column x >= 1 is kmer[kmer_base + x - 1]
    int64_t event_base;   // event of row y >= 1 is events[event_base + y - 1]
    int64_t out_base, out_cap;
    int64_t x1, y1;
};

struct Args {
    const RegionDesc *regions;
    const int32_t *order;
    int64_t n_regions;
    const ModelDesc *models;
    const ReadScale32 *read_scale;
    const int2 *meta;              // per anti-diagonal {xmy of first cell, width | flags}
    const Window *windows;
    const int32_t *window_off;     // per window: region-relative first cell of its traceback anti-diagonal
    const int32_t *kmer;
    const float *gapx;             // per k-mer position: skip emission of that k-mer
    const Event32 *events;
    float *F;                      // forward store, kStoreStride floats per cell
    double *base;                  // per anti-diagonal FP64 base of the forward store
    float *fshift;                 // per anti-diagonal base(d) - base(d-1)
    sa_aligned_pair *out;
    int64_t *out_count;            // per region
    double *loglik;                // per region: total probability at its last anti-diagonal
    int32_t *status;               // per read
    unsigned int *queue;
    float threshold;
    int32_t wmax;                  // ring width (cells); rings hold wmax + 2 floats per state
    long long spin_limit;          // clock cycles the backward group may wait for a window
};

struct Shared {
    float4 la[16];                 // logAdd cubic pieces by ceil(2 d)
    float fpart[3][kGroupWarps];
    float bpart[3][kGroupWarps];
    int32_t wcnt[2][kMaxCpt][kGroupWarps];
    float fold[2];
    int32_t fwd_done;
    int32_t region;
    int32_t abort;
    int32_t pad;
};

__device__ __forceinline__ void group_bar(int id) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(kGroup) : "memory");
}

// The reference's lookup (pairwiseAligner.c:237-248) picks one of four cubics by d <= 1, <= 2.5,
// <= 4.5; those boundaries are multiples of 1/2, so ceil(2 d) (0..15 below the 7.5 cut) indexes a
// 16-entry table holding, per index, the cubic of its piece with the "- d" of
// logAdd = min + p(d) = max + (p(d) - d) folded into the linear coefficient.
__host__ __device__ inline void log_add_piece(int k, float4 &c) {
    const int seg = k <= 2 ? 0 : (k <= 5 ? 1 : (k <= 9 ? 2 : 3));
    const float a[4] = {-0.009350833524763f, -0.014532321752540f, -0.004605031767994f, -0.000458661602210f};
    const float b[4] = {0.130659527668286f, 0.139942324101744f, 0.063427417320019f, 0.009695946122598f};
    const float cc[4] = {0.498799810682272f, 0.495635523139337f, 0.695956496475118f, 0.930734667215156f};
    const float e[4] = {0.693203116424741f, 0.692140569840976f, 0.514272634594009f, 0.168037164329057f};
    c = make_float4(a[seg], b[seg], cc[seg] - 1.0f, e[seg]);
}

// logAdd in FP32: max(x, y) + h(|x - y|) below the 7.5 cut-off, max(x, y) at or above it (also
// when the smaller argument is -inf: the difference is inf, or NaN if both are -inf)
__device__ __forceinline__ float lae(const float4 *tab, float x, float y) {
    const float mx = fmaxf(x, y), d = fabsf(x - y);
    const int k = min(max(__float2int_ru(2.0f * d), 0), 15);
    const float4 c = tab[k];
    const float h = fmaf(fmaf(fmaf(c.x, d, c.y), d, c.z), d, c.w);
    return d < 7.5f ? mx + h : mx;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sequential logAdd over vals[0..n) in index order, as dpDiagonal_dotProduct folds an
// anti-diagonal one cell at a time (pairwiseAligner.c:1014-1027), run by one warp.
//  * The running result never falls below the running maximum, so a value at least 7.5 below the
//    maximum of the values before it leaves the result unchanged: only the others are folded, in
//    index order (compacted into consecutive lanes first).
//  * Values before the first one within kSeedGap of the overall maximum M enter as one exact
//    log-sum-exp seed: the final result depends on the running result at that point with weight
//    at most exp(-(kSeedGap - 0.7)) < 1e-6, so the reference's approximation error there (< 1e-3)
//    cannot reach the final total.
constexpr float kSeedGap = 15.0f;

__device__ float ordered_fold(const float4 *tab, const float *vals, int n) {
    const int lane = threadIdx.x & 31;
    float mall = kNegInf;
    for (int b = 0; b < n; b += 32) mall = fmaxf(mall, b + lane < n ? vals[b + lane] : kNegInf);
    mall = warp_max(mall);
    if (!(mall > kNegInf)) return kNegInf;
    // first index within kSeedGap of the maximum
    int start = n;
    for (int b = 0; b < n; b += 32) {
        const unsigned m = __ballot_sync(0xffffffffu, b + lane < n && vals[b + lane] >= mall - kSeedGap);
        if (m) { start = b + __ffs(m) - 1; break; }
    }
    float seed = 0.0f, carry = kNegInf;
    for (int b = 0; b < start; b += 32) {
        const float v = b + lane < start ? vals[b + lane] : kNegInf;
        seed += v > kNegInf ? __expf(v - mall) : 0.0f;
        carry = fmaxf(carry, v);
    }
    seed = warp_sum(seed);
    carry = warp_max(carry);
    float r = seed > 0.0f ? mall + __logf(seed) : kNegInf;
    for (int b = start; b < n; b += 32) {
        const float v = b + lane < n ? vals[b + lane] : kNegInf;
        float incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl = fmaxf(incl, t);
        }
        incl = fmaxf(incl, carry);
        float excl = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) excl = carry;
        const unsigned mask = __ballot_sync(0xffffffffu, v > excl - 7.6f);
        const int nc = __popc(mask);
        const unsigned src = lane < nc ? __fns(mask, 0, lane + 1) : 0u;
        const float packed = __shfl_sync(0xffffffffu, v, (int) (src & 31u));
        for (int k = 0; k < nc; ++k) r = lae(tab, r, __shfl_sync(0xffffffffu, packed, k));
        carry = __shfl_sync(0xffffffffu, incl, 31);
    }
    return r;
}

__global__ void prep_events(const double2 *raw, Event32 *out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        const double2 e = raw[i];
        Event32 v;
        v.mean = (float) e.x;
        v.noise = (float) e.y;
        v.c_noise = (float) (-1.5 * log(e.y));
        v.inv_noise = (float) (1.0 / e.y);
        out[i] = v;
    }
}

// ------------------------------------------------------------------------------------------------
// per-region context and loads
// ------------------------------------------------------------------------------------------------
struct Ctx {
    const Args *A;
    RegionDesc R;
    int32_t region_index;
    const ModelDesc *M;
    ReadScale32 rs;
    float t[9];
    bool hdp;
};

__device__ __forceinline__ int32_t load_kid(const Ctx &c, int32_t x) {
    return (x >= 1 && x <= c.R.lX) ? __ldg(c.A->kmer + c.R.kmer_base + x - 1) : -1;
}

__device__ __forceinline__ float load_gapx(const Ctx &c, int32_t x) {
    return (x >= 1 && x <= c.R.lX) ? __ldg(c.A->gapx + c.R.kmer_base + x - 1) : kNegInf;
}

__device__ __forceinline__ Event32 load_event(const Ctx &c, int32_t yi) {
    if (yi >= 0 && yi < c.R.lY) {
        const float4 v = __ldg(reinterpret_cast<const float4 *>(c.A->events + c.R.event_base + yi));
        return Event32{v.x, v.y, v.z, v.w};
    }
    return Event32{0.0f, 1.0f, 0.0f, 1.0f};
}

__device__ __forceinline__ KmerConst32 load_kc(const Ctx &c, int32_t kid) {
    if (kid < 0) return KmerConst32{0, 0, 0, 0, 0, 0, 0, kNegInf};
    const float4 *p = reinterpret_cast<const float4 *>(c.M->kc + kid);
    const float4 a = __ldg(p), b = __ldg(p + 1);
    return KmerConst32{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
}

__device__ __forceinline__ Event32 as_event(float4 v) { return Event32{v.x, v.y, v.z, v.w}; }

// match / extra-event emissions of k-mer kid (constants k) against event ev
__device__ __forceinline__ void emit_event_pair(const Ctx &c, int32_t kid, const KmerConst32 &k, const Event32 &ev,
                                                bool have_event, float &em, float &ey) {
    if (kid < 0 || !have_event) {
        em = ey = kNegInf;
    } else if (c.hdp) {
        em = ey = emit_hdp(c.M->hdp, k, kid, ev, c.rs);
    } else {
        emit_gauss(k, ev, c.rs, em, ey);
    }
}

__device__ __forceinline__ int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return min(max(v, lo), hi); }

// Raw loads: always from a valid address (indices clamped into the region's arrays), never
// followed by a select on the loaded value.  Validity is computed from indices alone and applied
// where the value is consumed, one anti-diagonal later, so the load latency overlaps a whole step.
__device__ __forceinline__ int32_t raw_kid(const Ctx &c, int32_t x) {
    const int64_t at = c.R.lX > 0 ? c.R.kmer_base + clampi(x - 1, 0, c.R.lX - 1) : 0;
    return __ldg(c.A->kmer + at);
}

__device__ __forceinline__ float raw_gapx(const Ctx &c, int32_t x) {
    const int64_t at = c.R.lX > 0 ? c.R.kmer_base + clampi(x - 1, 0, c.R.lX - 1) : 0;
    return __ldg(c.A->gapx + at);
}

__device__ __forceinline__ float4 raw_event(const Ctx &c, int32_t yi) {
    const int64_t at = c.R.lY > 0 ? c.R.event_base + clampi(yi, 0, c.R.lY - 1) : 0;
    return __ldg(reinterpret_cast<const float4 *>(c.A->events + at));
}

__device__ __forceinline__ KmerConst32 raw_kc(const Ctx &c, int32_t kid) {
    const float4 *p = reinterpret_cast<const float4 *>(c.M->kc + max(kid, 0));
    const float4 a = __ldg(p), b = __ldg(p + 1);
    return KmerConst32{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
}

__device__ __forceinline__ int2 raw_meta(const Args &A, int64_t db, int32_t d, int32_t n) {
    return __ldg(A.meta + db + clampi(d, 0, n));
}

struct Meta {
    int32_t L, W, flags;
};

__device__ __forceinline__ Meta decode_meta(int2 m, bool exists) {
    return exists ? Meta{m.x, m.y & kWidthMask, m.y & ~kWidthMask} : Meta{0, 0, 0};
}

__device__ __forceinline__ Meta load_meta(const Args &A, int64_t db, int32_t d, int32_t n) {
    if (d < 0 || d > n) return Meta{0, 0, 0};
    const int2 m = __ldg(A.meta + db + d);
    return Meta{m.x, m.y & kWidthMask, m.y & ~kWidthMask};
}

// ring: 3 slots x 3 states x (wmax + 2) floats; slot pointers point at cell 0 (cell -1 is a pad)
struct Ring {
    float *s[3];   // s[0] = anti-diagonal d (being written), s[1] = d -/+ 1, s[2] = d -/+ 2
    int stride;    // wmax + 2
    __device__ float *st(int k, int state) const { return s[k] + state * stride; }
    __device__ void rotate() {
        float *t = s[2];
        s[2] = s[1];
        s[1] = s[0];
        s[0] = t;
    }
};

__device__ __forceinline__ void ring_init(float *base, int wmax, int tid) {
    const int total = 9 * (wmax + 2);
    for (int i = tid; i < total; i += kGroup) base[i] = kNegInf;
}

// ------------------------------------------------------------------------------------------------
// forward group
// ------------------------------------------------------------------------------------------------
template <int CPT>
__device__ void forward_region(const Ctx &c, Shared *sh, float *fring) {
    const Args &A = *c.A;
    const RegionDesc &R = c.R;
    const float *t = c.t;
    const float4 *tab = sh->la;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wmax = A.wmax;
    const int64_t db = R.diag_base;
    const int32_t n = R.n;
    float *Fd = A.F + kStoreStride * R.cell_base;     // store of the anti-diagonal being computed

    ring_init(fring, wmax, tid);
    group_bar(kBarForward);
    Ring rg;
    rg.stride = wmax + 2;
    // slot of d = 1 is s[0]; s[1] holds d = 0, s[2] holds d = -1 (all -inf)
    rg.s[1] = fring + 1;
    rg.s[2] = fring + 3 * rg.stride + 1;
    rg.s[0] = fring + 6 * rg.stride + 1;

    // anti-diagonal 0: startStateProb / raggedStartStateProb (stateMachine.c:1022-1032)
    const float s0 = R.ragged_left ? kNegInf : 0.0f, s1 = R.ragged_left ? 0.0f : kNegInf;
    if (tid == 0) {
        Fd[ST_M] = s0; Fd[ST_EM] = kNegInf; Fd[ST_EY] = kNegInf; Fd[ST_X] = s1; Fd[ST_Y] = s1;
        rg.st(1, 0)[0] = s0;
        rg.st(1, 1)[0] = s1;
        rg.st(1, 2)[0] = s1;
        A.base[db] = 0.0;
        A.fshift[db] = 0.0f;
    }
    Fd += kStoreStride;   // anti-diagonal 0 has one cell
    Meta m2{0, 0, 0};
    Meta m1 = decode_meta(raw_meta(A, db, 0, n), true), m0 = decode_meta(raw_meta(A, db, 1, n), 1 <= n);
    Meta mn = decode_meta(raw_meta(A, db, 2, n), 2 <= n);
    int2 raw_nn = raw_meta(A, db, 3, n);      // meta of d+2, decoded at the top of each step
    float eX[CPT], eM[CPT], eY[CPT];          // emissions of the current anti-diagonal's cells
    // raw id / event of the next anti-diagonal's cells, with their validity
    int32_t rk1[CPT];
    float4 re1[CPT];
    bool vx1[CPT], vy1[CPT];
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
        const int i = tid + j * kGroup;
        {
            const int32_t xmy = m0.L + 2 * i, x = (1 + xmy) >> 1, y = (1 - xmy) >> 1;
            const bool in = i < m0.W;
            const int32_t kid = in && x >= 1 && x <= R.lX ? raw_kid(c, x) : -1;
            const KmerConst32 kc = raw_kc(c, kid);
            emit_event_pair(c, kid, kc, as_event(raw_event(c, y - 1)), in && y >= 1, eM[j], eY[j]);
            eX[j] = kid < 0 ? kNegInf : (c.hdp ? (float) kLogPointOne : kc.gapx);
        }
        {
            const int32_t xmy = mn.L + 2 * i, x = (2 + xmy) >> 1, y = (2 - xmy) >> 1;
            const bool in = i < mn.W;
            rk1[j] = raw_kid(c, x);
            re1[j] = raw_event(c, y - 1);
            vx1[j] = in && x >= 1 && x <= R.lX;
            vy1[j] = in && y >= 1;
        }
    }
    float lm_prev = tid == 0 ? fmaxf(s0, s1) : kNegInf;   // local max of the previous anti-diagonal
    float delta1 = 0.0f;      // base(d-1) - base(d-2)
    double fbase = 0.0;       // base of d
    int32_t wi = 0;
    group_bar(kBarForward);
    for (int32_t d = 1; d <= n; ++d) {
        // shift of this anti-diagonal: base(d) = base(d-2) + max(d-2)
        float delta0 = 0.0f;
        if (d > 2) {
            const float *fp = sh->fpart[(d - 2) % 3];
            const float mx = fmaxf(fmaxf(fp[0], fp[1]), fmaxf(fp[2], fp[3]));
            delta0 = (mx > kNegInf ? mx : 0.0f) - delta1;
        }
        fbase += (double) delta0;
        const Meta mnn = decode_meta(raw_nn, d + 2 <= n);
        raw_nn = raw_meta(A, db, d + 3, n);
        // stage 1: raw ids and events two anti-diagonals ahead (consumed next step)
        int32_t rk2[CPT];
        float4 re2[CPT];
        bool vx2[CPT], vy2[CPT];
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kGroup;
            const int32_t xmy = mnn.L + 2 * i, x = (d + 2 + xmy) >> 1, y = (d + 2 - xmy) >> 1;
            const bool in = i < mnn.W;
            rk2[j] = raw_kid(c, x);
            re2[j] = raw_event(c, y - 1);
            vx2[j] = in && x >= 1 && x <= R.lX;
            vy2[j] = in && y >= 1;
        }
        // stage 2: k-mer constants one anti-diagonal ahead (ids loaded last step)
        int32_t kid1[CPT];
        KmerConst32 kc1[CPT];
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            kid1[j] = vx1[j] ? rk1[j] : -1;
            kc1[j] = raw_kc(c, kid1[j]);
        }
        // the recursion on anti-diagonal d (stateMachine3_cellCalculate order: lower -> gap-X,
        // middle -> match, upper -> gap-Y, each state accumulated from LOG_ZERO)
        const int32_t W0 = m0.W;
        const float shL = -delta0, shM = -delta1 - delta0;
        const bool store_gaps = (m0.flags & kFlagStoreGaps) != 0;
        float lm = kNegInf;
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kGroup;
            const int32_t xmy = m0.L + 2 * i;
            const int il = clampi((xmy - 1 - m1.L) >> 1, -1, wmax);
            const int iu = clampi((xmy + 1 - m1.L) >> 1, -1, wmax);
            const int im = clampi((xmy - m2.L) >> 1, -1, wmax);
            const float ex = eX[j] + shL, em = eM[j] + shM, ey = eY[j] + shL;
            float vX = rg.st(1, 0)[il] + (ex + t[T_OX]);
            vX = lae(tab, vX, rg.st(1, 1)[il] + (ex + t[T_EX]));
            vX = lae(tab, vX, rg.st(1, 2)[il] + (ex + t[T_SX]));
            float vM = rg.st(2, 0)[im] + (em + t[T_MC]);
            vM = lae(tab, vM, rg.st(2, 1)[im] + (em + t[T_MFGX]));
            vM = lae(tab, vM, rg.st(2, 2)[im] + (em + t[T_MFGY]));
            float vY = rg.st(1, 0)[iu] + (ey + t[T_OY]);
            vY = lae(tab, vY, rg.st(1, 2)[iu] + (ey + t[T_EY]));
            const bool in = i < W0;
            if (!in) vM = vX = vY = kNegInf;
            rg.st(0, 0)[i] = vM;
            rg.st(0, 1)[i] = vX;
            rg.st(0, 2)[i] = vY;
            if (in) {
                Fd[ST_M * W0 + i] = vM;
                Fd[ST_EM * W0 + i] = eM[j];
                Fd[ST_EY * W0 + i] = eY[j];
                if (store_gaps) {
                    Fd[ST_X * W0 + i] = vX;
                    Fd[ST_Y * W0 + i] = vY;
                }
            }
            lm = fmaxf(lm, fmaxf(vM, fmaxf(vX, vY)));
        }
        // lagged reduction of the previous anti-diagonal's maximum
        {
            const float wm = warp_max(lm_prev);
            if (lane == 0) sh->fpart[(d - 1) % 3][warp] = wm;
        }
        // emissions of the next anti-diagonal's cells
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            emit_event_pair(c, kid1[j], kc1[j], as_event(re1[j]), vy1[j], eM[j], eY[j]);
            eX[j] = kid1[j] < 0 ? kNegInf : (c.hdp ? (float) kLogPointOne : kc1[j].gapx);
            rk1[j] = rk2[j]; re1[j] = re2[j]; vx1[j] = vx2[j]; vy1[j] = vy2[j];
        }
        if (tid == 0) {
            A.base[db + d] = fbase;
            A.fshift[db + d] = delta0;
        }
        const bool window_end = (m0.flags & kFlagWindowEnd) != 0;
        if (window_end) __threadfence_block();
        group_bar(kBarForward);
        if (window_end && tid == 0) atomicExch(&sh->fwd_done, ++wi);
        lm_prev = lm;
        delta1 = delta0;
        Fd += kStoreStride * W0;
        rg.rotate();
        m2 = m1; m1 = m0; m0 = mn; mn = mnn;
    }
}

// ------------------------------------------------------------------------------------------------
// backward group: one traceback window at a time, posteriors fused
// ------------------------------------------------------------------------------------------------
template <int CPT>
__device__ __forceinline__ void write_pairs(const Ctx &c, Shared *sh, int32_t pend_d, unsigned pend, const float *pv,
                                            const int32_t *px, const int32_t *py, const int32_t *pk, int64_t &n_out) {
    const Args &A = *c.A;
    const RegionDesc &R = c.R;
    const int tid = threadIdx.x - kGroup, lane = tid & 31, warp = tid >> 5;
    int32_t before = 0;
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
        int32_t mine_before = before;
#pragma unroll
        for (int w = 0; w < kGroupWarps; ++w) {
            const int32_t cw = sh->wcnt[pend_d & 1][j][w];
            if (w < warp) mine_before += cw;
            before += cw;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, (pend >> j) & 1u);
        if ((pend >> j) & 1u) {
            const int64_t slot = n_out + mine_before + __popc(bal & ((1u << lane) - 1u));
            if (slot < R.out_cap) {
                sa_aligned_pair o;
                o.score = (int64_t) floor((double) fminf(pv[j], 1.0f) * 10000000.0);
                o.x = R.x1 + px[j] - 1;
                o.y = R.y1 + py[j] - 1;
                o.kmer = pk[j];
                A.out[R.out_base + slot] = o;
            } else {
                atomicMax(A.status + R.read, (int32_t) SA_E_OUTPUT);
            }
        }
    }
    n_out += before;
}

template <int CPT>
__device__ void backward_region(const Ctx &c, Shared *sh, float *bring, float *chain) {
    const Args &A = *c.A;
    const RegionDesc &R = c.R;
    const float *t = c.t;
    const float4 *tab = sh->la;
    const int tid = threadIdx.x - kGroup, lane = tid & 31, warp = tid >> 5;
    const int wmax = A.wmax;
    const int64_t db = R.diag_base;
    const int32_t n = R.n;
    const float *Freg = A.F + kStoreStride * R.cell_base;
    int64_t n_out = 0;
    double ll = 0.0;
    ring_init(bring, wmax, tid);
    for (int32_t wi = 0; wi < R.n_windows; ++wi) {
        const Window W = A.windows[R.win_base + wi];
        // wait (bounded) for the forward group to pass this window's traceback anti-diagonal
        if (tid == 0) {
            const long long t0 = clock64();
            while (*((volatile int32_t *) &sh->fwd_done) <= wi) {
                __nanosleep(256);
                if (clock64() - t0 > A.spin_limit) {
                    atomicExch(&sh->abort, 1);
                    break;
                }
            }
        }
        group_bar(kBarBackward);
        if (*((volatile int32_t *) &sh->abort)) {
            if (tid == 0) atomicMax(A.status + R.read, (int32_t) SA_E_TIMEOUT);
            return;
        }
        __threadfence_block();
        const int32_t D = W.D, T = W.T, from = W.from;
        // end-state values on D (stateMachine.c:1034-1061)
        const bool ragged_end = W.at_end && R.ragged_right;
        const float e0 = ragged_end ? (t[T_OX] + t[T_OY]) / 2.0f : t[T_MC];
        const float e1 = ragged_end ? t[T_EX] : t[T_MFGX];
        const float e2 = ragged_end ? t[T_EY] : t[T_MFGY];
        float mxD = fmaxf(e0, fmaxf(e1, e2));
        if (!(mxD > kNegInf)) mxD = 0.0f;
        Ring rg;
        rg.stride = wmax + 2;
        rg.s[0] = bring + 1;                      // d = D
        rg.s[1] = bring + 3 * rg.stride + 1;      // d + 1 (none yet: -inf)
        rg.s[2] = bring + 6 * rg.stride + 1;      // d + 2
        // metas of d+2, d+1, d, d-1, d-2 (d = D to start) and store offsets of d+1, d
        Meta mpp{0, 0, 0}, mp{0, 0, 0};
        Meta m0 = decode_meta(raw_meta(A, db, D, n), true);
        Meta mm = decode_meta(raw_meta(A, db, D - 1, n), D - 1 >= 0);
        int2 raw_mmm = raw_meta(A, db, D - 2, n);
        int32_t off0 = __ldg(A.window_off + R.win_base + wi), offp = off0;
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kGroup;
            const bool in = i < m0.W;
            rg.st(0, 0)[i] = in ? e0 : kNegInf;
            rg.st(0, 1)[i] = in ? e1 : kNegInf;
            rg.st(0, 2)[i] = in ? e2 : kNegInf;
            rg.st(1, 0)[i] = kNegInf; rg.st(1, 1)[i] = kNegInf; rg.st(1, 2)[i] = kNegInf;
            rg.st(2, 0)[i] = kNegInf; rg.st(2, 1)[i] = kNegInf; rg.st(2, 2)[i] = kNegInf;
        }
        // operands of the current anti-diagonal's cells, loaded one anti-diagonal ahead
        float eMm[CPT], eYu[CPT], eXl[CPT], fM[CPT];
        // refresh operands: gap states of d, and the match-through inputs of the d+1 cells
        float fX[CPT], fY[CPT], tM[CPT], tX[CPT], tY[CPT], tE[CPT];
        bool tv[CPT];
        double fb = __ldcg(A.base + db + D);
        float fsh = __ldcg(A.fshift + db + D);
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kGroup;
            const int ic = clampi(i, 0, max(m0.W - 1, 0));
            const float *Fd = Freg + kStoreStride * off0;
            eMm[j] = eYu[j] = eXl[j] = kNegInf;
            fM[j] = __ldcg(Fd + ST_M * m0.W + ic);
            fX[j] = __ldcg(Fd + ST_X * m0.W + ic);
            fY[j] = __ldcg(Fd + ST_Y * m0.W + ic);
            tM[j] = tX[j] = tY[j] = tE[j] = kNegInf;
            tv[j] = false;
        }
        float lm_prev = kNegInf;           // local max of B stored on d+1 (lagged reduction)
        float gamma1 = 0.0f;               // base(d+1) - base(d+2)
        double bbase = 0.0;                // base of B on d
        double pref = 0.0;                 // latest refresh total probability (absolute)
        unsigned pend = 0;
        float pv[CPT];
        int32_t px[CPT], py[CPT], pk[CPT];
        int32_t pend_d = -1;
        group_bar(kBarBackward);
        for (int32_t d = D; d > T; --d) {
            const int32_t W0 = m0.W, Wp = mp.W;
            const bool post = d <= from;
            const bool refresh = post && (m0.flags & kFlagRefresh);
            float gamma0 = 0.0f;           // base(d) - base(d+1)
            if (d <= D - 2) {
                float m;
                if (d == D - 2) {
                    m = mxD;
                } else {
                    const float *bp = sh->bpart[(d + 2) % 3];
                    m = fmaxf(fmaxf(bp[0], bp[1]), fmaxf(bp[2], bp[3]));
                    if (!(m > kNegInf)) m = 0.0f;
                }
                gamma0 = m - gamma1;
            }
            bbase += (double) gamma0;
            // prefetch the operands of the d-1 cells: raw loads from clamped indices; a value
            // fetched for an absent neighbour is only ever added to a -inf ring value
            const Meta mmm = decode_meta(raw_mmm, d - 2 >= 0);
            raw_mmm = raw_meta(A, db, d - 3, n);
            const int32_t Wm = mm.W, Wmm = mmm.W;
            const int32_t offm = off0 - Wm, offmm = offm - Wmm;
            const bool live_m = d - 1 > T;
            const bool refresh_m = live_m && d - 1 <= from && (mm.flags & kFlagRefresh);
            float eMm_n[CPT], eYu_n[CPT], eXl_n[CPT], fM_n[CPT], fX_n[CPT], fY_n[CPT];
            float tM_n[CPT], tX_n[CPT], tY_n[CPT], tE_n[CPT];
            bool tv_n[CPT];
            {
                const float *Fd = Freg + kStoreStride * off0;      // d
                const float *Fp = Freg + kStoreStride * offp;      // d+1 (or d at the window top)
                const float *Fm = Freg + kStoreStride * offm;      // d-1
                const float *Fmm = Freg + kStoreStride * (Wmm > 0 ? offmm : offm);   // d-2
                const int32_t Wpl = Wp > 0 ? Wp : W0;              // width of the block Fp points at
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    const int i = tid + j * kGroup;
                    const int32_t xmy = mm.L + 2 * i, x = (d - 1 + xmy) >> 1;
                    eMm_n[j] = __ldcg(Fp + ST_EM * Wpl + clampi((xmy - mp.L) >> 1, 0, max(Wpl - 1, 0)));
                    eYu_n[j] = __ldcg(Fd + ST_EY * W0 + clampi((xmy - 1 - m0.L) >> 1, 0, max(W0 - 1, 0)));
                    eXl_n[j] = raw_gapx(c, x + 1);
                    const int ic = clampi(i, 0, max(Wm - 1, 0));
                    fM_n[j] = __ldcg(Fm + ST_M * Wm + ic);
                    fX_n[j] = __ldcg(Fm + ST_X * Wm + ic);
                    fY_n[j] = __ldcg(Fm + ST_Y * Wm + ic);
                    // match-through inputs for a refresh at d-1: cells of d, F of d-2, emissions of d
                    const int32_t xmy0 = m0.L + 2 * i;
                    const int32_t r = (xmy0 - mmm.L) >> 1;
                    tv_n[j] = refresh_m && i < W0 && Wmm > 0 && xmy0 >= mmm.L && r < Wmm;
                    const int imm = clampi(r, 0, max(Wmm - 1, 0));
                    const int32_t Wml = Wmm > 0 ? Wmm : Wm;
                    tE_n[j] = __ldcg(Fd + ST_EM * W0 + clampi(i, 0, max(W0 - 1, 0)));
                    tM_n[j] = __ldcg(Fmm + ST_M * Wml + imm);
                    tX_n[j] = __ldcg(Fmm + ST_X * Wml + imm);
                    tY_n[j] = __ldcg(Fmm + ST_Y * Wml + imm);
                }
            }
            const double fb_n = __ldcg(A.base + db + max(d - 1, 0));
            const float fsh_n = __ldcg(A.fshift + db + max(d - 1, 0));
            // the recursion on d (D itself holds the end-state values)
            float lm = kNegInf;
            if (d < D) {
                const float shU = -gamma0, shM = -gamma1 - gamma0;
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    const int i = tid + j * kGroup;
                    const int32_t xmy = m0.L + 2 * i;
                    const int ipp = clampi((xmy - mpp.L) >> 1, -1, wmax);
                    const int iu = clampi((xmy - 1 - mp.L) >> 1, -1, wmax);
                    const int il = clampi((xmy + 1 - mp.L) >> 1, -1, wmax);
                    const float bm = rg.st(2, 0)[ipp];
                    const float em = eMm[j] + shM;
                    float vM = bm + (em + t[T_MC]);
                    float vX = bm + (em + t[T_MFGX]);
                    float vY = bm + (em + t[T_MFGY]);
                    const float bu = rg.st(1, 2)[iu];
                    const float ey = eYu[j] + shU;
                    vM = lae(tab, vM, bu + (ey + t[T_OY]));
                    vY = lae(tab, vY, bu + (ey + t[T_EY]));
                    const float bl = rg.st(1, 1)[il];
                    const float ex = eXl[j] + shU;
                    vM = lae(tab, vM, bl + (ex + t[T_OX]));
                    vX = lae(tab, vX, bl + (ex + t[T_EX]));
                    vY = lae(tab, vY, bl + (ex + t[T_SX]));
                    if (i >= W0) vM = vX = vY = kNegInf;
                    rg.st(0, 0)[i] = vM;
                    rg.st(0, 1)[i] = vX;
                    rg.st(0, 2)[i] = vY;
                    lm = fmaxf(lm, fmaxf(vM, fmaxf(vX, vY)));
                }
            }
            {
                const float wm = warp_max(lm_prev);
                if (lane == 0 && d + 1 <= D) sh->bpart[(d + 1) % 3][warp] = wm;
            }
            group_bar(kBarBackward);
            // pairs of the previous anti-diagonal, in the reference's order (ascending xmy)
            if (pend_d >= 0) {
                write_pairs<CPT>(c, sh, pend_d, pend, pv, px, py, pk, n_out);
                pend = 0;
                pend_d = -1;
            }
            if (post) {
                if (refresh) {
                    // diagonalCalculationTotalProbability (pairwiseAligner.c:1182-1200): F.B on d in
                    // ascending cell order, then the matches from d-1 over d into d+1, dotted with B(d+1)
#pragma unroll
                    for (int j = 0; j < CPT; ++j) {
                        const int i = tid + j * kGroup;
                        if (i < W0) {
                            float s = fM[j] + rg.st(0, 0)[i];
                            s = lae(tab, s, fX[j] + rg.st(0, 1)[i]);
                            s = lae(tab, s, fY[j] + rg.st(0, 2)[i]);
                            chain[i] = s;
                        }
                    }
                    const bool have_next = d < D;
                    if (have_next) {
#pragma unroll
                        for (int j = 0; j < CPT; ++j) {
                            const int i = tid + j * kGroup;
                            if (i < Wp) {
                                float mth = kNegInf;
                                if (tv[j]) {
                                    mth = tM[j] + (tE[j] + t[T_MC]);
                                    mth = lae(tab, mth, tX[j] + (tE[j] + t[T_MFGX]));
                                    mth = lae(tab, mth, tY[j] + (tE[j] + t[T_MFGY]));
                                }
                                chain[wmax + i] = mth + rg.st(1, 0)[i];
                            }
                        }
                    }
                    group_bar(kBarBackward);
                    if (warp == 0) {
                        const float f = ordered_fold(tab, chain, W0);
                        if (lane == 0) sh->fold[0] = f;
                    } else if (warp == 1) {
                        const float f = have_next ? ordered_fold(tab, chain + wmax, Wp) : kNegInf;
                        if (lane == 0) sh->fold[1] = f;
                    }
                    group_bar(kBarBackward);
                    // the through-part is relative to base_F(d-1) + base_B(d+1)
                    const float ptil = lae(tab, sh->fold[0], sh->fold[1] - fsh - gamma0);
                    pref = (double) ptil + fb + bbase;
                    if (d == n) ll = pref;
                }
                const float kd = (float) (fb + bbase - pref);
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    const int i = tid + j * kGroup;
                    const int32_t xmy = m0.L + 2 * i, x = (d + xmy) >> 1, y = (d - xmy) >> 1;
                    const float p = __expf(fM[j] + rg.st(0, 0)[i] + kd);
                    const bool hit = i < W0 && x > 0 && y > 0 && p >= A.threshold;
                    pv[j] = p;
                    px[j] = x;
                    py[j] = y;
                    pk[j] = raw_kid(c, x);    // consumed by write_pairs after the next barrier
                    const unsigned bal = __ballot_sync(0xffffffffu, hit);
                    if (hit) pend |= 1u << j;
                    if (lane == 0) sh->wcnt[d & 1][j][warp] = __popc(bal);
                }
                pend_d = d;
            }
#pragma unroll
            for (int j = 0; j < CPT; ++j) {
                eMm[j] = eMm_n[j]; eYu[j] = eYu_n[j]; eXl[j] = eXl_n[j];
                fM[j] = fM_n[j]; fX[j] = fX_n[j]; fY[j] = fY_n[j];
                tM[j] = tM_n[j]; tX[j] = tX_n[j]; tY[j] = tY_n[j]; tE[j] = tE_n[j]; tv[j] = tv_n[j];
            }
            fb = fb_n;
            fsh = fsh_n;
            lm_prev = d == D ? kNegInf : lm;   // D's maximum is known exactly (mxD)
            gamma1 = gamma0;
            offp = off0; off0 = offm;
            rg.rotate();
            mpp = mp; mp = m0; m0 = mm; mm = mmm;
        }
        // flush the last anti-diagonal's pairs
        group_bar(kBarBackward);
        if (pend_d >= 0) write_pairs<CPT>(c, sh, pend_d, pend, pv, px, py, pk, n_out);
        group_bar(kBarBackward);
    }
    if (tid == 0) {
        A.out_count[c.region_index] = n_out;
        A.loglik[c.region_index] = ll;
    }
}

template <int CPT>
__global__ void __launch_bounds__(kThreads) batch_kernel(const __grid_constant__ Args A) {
    extern __shared__ float4 smem_raw[];
    Shared *sh = reinterpret_cast<Shared *>(smem_raw);
    float *fring = reinterpret_cast<float *>(sh + 1);
    float *bring = fring + 9 * (A.wmax + 2);
    float *chain = bring + 9 * (A.wmax + 2);
    if (threadIdx.x < 16) log_add_piece(threadIdx.x, sh->la[threadIdx.x]);
    for (;;) {
        if (threadIdx.x == 0) {
            sh->region = (int32_t) atomicAdd(A.queue, 1u);
            sh->fwd_done = 0;
            sh->abort = 0;
        }
        __syncthreads();
        const int32_t qi = sh->region;
        if (qi >= A.n_regions) break;
        Ctx c;
        c.A = &A;
        c.region_index = A.order[qi];
        c.R = A.regions[c.region_index];
        c.M = A.models + c.R.model;
        c.rs = A.read_scale[c.R.read];
        c.hdp = c.M->emission == SA_EMIT_HDP;
#pragma unroll
        for (int i = 0; i < 9; ++i) c.t[i] = c.M->t[i];
        if (threadIdx.x < kGroup) {
            forward_region<CPT>(c, sh, fring);
        } else {
            backward_region<CPT>(c, sh, bring, chain);
        }
        __syncthreads();
    }
}

}  // namespace fp32
}  // namespace sa
