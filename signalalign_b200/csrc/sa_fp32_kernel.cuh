// Batched FP32 kernel: one persistent launch over all regions of a batch.
//
// A CTA is two 128-thread groups working on the same region at once:
//   * the forward group sweeps the band anti-diagonal by anti-diagonal (cells spread over the
//     threads, neighbours through a 3-slot shared-memory ring, one named barrier per
//     anti-diagonal) and stores every forward cell to HBM;
//   * the backward group follows one traceback window behind (getPosteriorProbsWithBanding,
//     pairwiseAligner.c:1319-1410): once the forward group has passed a window's traceback
//     anti-diagonal it runs that window's backward sweep in its own shared-memory ring with the
//     posterior test fused in, so backward values never leave the SM.
// The hand-off is a window counter in shared memory; the backward group's wait on it is bounded
// (it gives up with SA_E_TIMEOUT), and the forward group never waits on the backward group.
//
// Latency, not arithmetic, bounds one region, so both sweeps software-pipeline everything that does
// not depend on the recursion: band bounds three anti-diagonals ahead, k-mer ids and events two
// ahead, k-mer constants one ahead, emissions computed one anti-diagonal early; the forward store
// is prefetched one anti-diagonal ahead for the posterior.
//
// Values are log probabilities relative to a per-anti-diagonal FP64 base.  The base of d is the
// base of d-2 plus the largest value stored on d-2 (a lagged renormalisation, so the max reduction
// is off the critical path); the recorded bases are built from the same float shifts the kernel
// applies, so they describe the stored values exactly.
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
    const int32_t *xl, *xr;        // per anti-diagonal band
    const int64_t *coff;           // per anti-diagonal first cell (region-relative)
    const Window *windows;
    const int32_t *kmer;
    const Event32 *events;
    float *F;                      // forward store, [M | X | Y] blocks per anti-diagonal
    double *base;                  // per anti-diagonal FP64 base of the forward store
    float *fshift;                 // per anti-diagonal base(d) - base(d-1)
    sa_aligned_pair *out;
    int64_t *out_count;            // per region
    double *loglik;                // per region: total probability at its last anti-diagonal
    int32_t *status;               // per read
    unsigned int *queue;
    float threshold;
    int32_t wmax;
    long long spin_limit;          // clock cycles the backward group may wait for a window
};

struct Shared {
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

// logAdd (pairwiseAligner.c:237-254) in FP32 with the cubic piece chosen by selects (no memory
// access on the recursion's critical path)
__device__ __forceinline__ float lae(float x, float y) {
    const float mx = fmaxf(x, y), mn = fminf(x, y), d = mx - mn;
    const bool p1 = d > 1.0f, p2 = d > 2.5f, p3 = d > 4.5f;
    const float a = p3 ? -0.000458661602210f : (p2 ? -0.004605031767994f : (p1 ? -0.014532321752540f : -0.009350833524763f));
    const float b = p3 ? 0.009695946122598f : (p2 ? 0.063427417320019f : (p1 ? 0.139942324101744f : 0.130659527668286f));
    const float c = p3 ? 0.930734667215156f : (p2 ? 0.695956496475118f : (p1 ? 0.495635523139337f : 0.498799810682272f));
    const float e = p3 ? 0.168037164329057f : (p2 ? 0.514272634594009f : (p1 ? 0.692140569840976f : 0.693203116424741f));
    const float p = fmaf(fmaf(fmaf(a, d, b), d, c), d, e);
    return d < 7.5f ? p + mn : mx;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sequential logAdd over vals[0..n) in index order, exactly as dpDiagonal_dotProduct folds a
// diagonal one cell at a time (pairwiseAligner.c:1014-1027), run by one warp.  The running result
// never falls below the running maximum, so a value at least 7.5 below the maximum of the values
// before it is dropped by logAdd unchanged; only the others are folded, in index order (after being
// compacted into consecutive lanes so their broadcasts do not depend on the running result).
__device__ float ordered_fold(const float *vals, int n) {
    const int lane = threadIdx.x & 31;
    float r = kNegInf, carry = kNegInf;
    for (int b = 0; b < n; b += 32) {
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
        const bool cand = v > excl - 7.6f;
        const unsigned mask = __ballot_sync(0xffffffffu, cand);
        const int nc = __popc(mask);
        // compact: lane k receives the k-th candidate (in index order)
        const unsigned src = lane < nc ? __fns(mask, 0, lane + 1) : 0u;
        const float packed = __shfl_sync(0xffffffffu, v, (int) (src & 31u));
        for (int k = 0; k < nc; ++k) r = lae(r, __shfl_sync(0xffffffffu, packed, k));
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

// match / extra-event / skip emissions of k-mer kid (constants k) against event ev
__device__ __forceinline__ void emit_all(const Ctx &c, int32_t kid, const KmerConst32 &k, const Event32 &ev,
                                         bool have_event, float &em, float &ey, float &ex) {
    if (c.hdp) {
        ex = (float) kLogPointOne;
        em = ey = (kid >= 0 && have_event) ? emit_hdp(c.M->hdp, k, kid, ev, c.rs) : kNegInf;
        return;
    }
    ex = kid >= 0 ? k.gapx : kNegInf;
    if (kid >= 0 && have_event) {
        emit_gauss(k, ev, c.rs, em, ey);
    } else {
        em = ey = kNegInf;
    }
}

__device__ __forceinline__ float *slot_ptr(float *ring, int wmax, int slot, int state) {
    return ring + (slot * 3 + state) * wmax;
}

__device__ __forceinline__ int32_t width_of(int32_t L, int32_t R) { return R >= L ? ((R - L) >> 1) + 1 : 0; }

// ------------------------------------------------------------------------------------------------
// forward group
// ------------------------------------------------------------------------------------------------
template <int CPT>
__device__ void forward_region(const Ctx &c, Shared *sh, float *fring) {
    const Args &A = *c.A;
    const RegionDesc &R = c.R;
    const float *t = c.t;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wmax = A.wmax;
    const int64_t db = R.diag_base;
    const int32_t n = R.n;
    float *Freg = A.F + 3 * R.cell_base;
    auto band_l = [&](int32_t d) -> int32_t { return d <= n ? __ldg(A.xl + db + d) : 0; };
    auto band_r = [&](int32_t d) -> int32_t { return d <= n ? __ldg(A.xr + db + d) : -2; };

    // anti-diagonal 0: startStateProb / raggedStartStateProb (stateMachine.c:1022-1032)
    const float s0 = R.ragged_left ? kNegInf : 0.0f, s1 = R.ragged_left ? 0.0f : kNegInf;
    if (tid == 0) {
        Freg[0] = s0; Freg[1] = s1; Freg[2] = s1;
        slot_ptr(fring, wmax, 0, 0)[0] = s0;
        slot_ptr(fring, wmax, 0, 1)[0] = s1;
        slot_ptr(fring, wmax, 0, 2)[0] = s1;
        A.base[db] = 0.0;
        A.fshift[db] = 0.0f;
    }
    // band bounds: d-2, d-1, d, d+1, d+2
    int32_t L2 = 0, R2 = -2, L1 = band_l(0), R1 = band_r(0);
    int32_t L0 = band_l(1), R0 = band_r(1), Ln = band_l(2), Rn = band_r(2), Lnn = band_l(3), Rnn = band_r(3);
    int64_t off0 = 1;   // anti-diagonal 0 has one cell
    // pipeline registers per owned cell
    float eX[CPT], eM[CPT], eY[CPT];          // emissions of the current anti-diagonal's cells
    int32_t kid1[CPT];                        // k-mer ids of the next anti-diagonal's cells
    Event32 ev1[CPT];
    bool hev1[CPT];
    int32_t kid2[CPT];                        // ... and of the one after
    Event32 ev2[CPT];
    bool hev2[CPT];
    auto cell_xy = [&](int32_t d, int32_t L, int i, int32_t &x, int32_t &y) {
        const int32_t xmy = L + 2 * i;
        x = (d + xmy) >> 1;
        y = (d - xmy) >> 1;
    };
    {
        const int32_t W0 = width_of(L0, R0), Wn = width_of(Ln, Rn);
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kGroup;
            int32_t x = 0, y = 0;
            eX[j] = eM[j] = eY[j] = kNegInf;
            if (i < W0) {
                cell_xy(1, L0, i, x, y);
                const int32_t kid = load_kid(c, x);
                const Event32 ev = load_event(c, y - 1);
                emit_all(c, kid, load_kc(c, kid), ev, y >= 1, eM[j], eY[j], eX[j]);
            }
            kid1[j] = -1; hev1[j] = false; ev1[j] = Event32{0, 1, 0, 1};
            if (i < Wn) {
                cell_xy(2, Ln, i, x, y);
                kid1[j] = load_kid(c, x);
                ev1[j] = load_event(c, y - 1);
                hev1[j] = y >= 1;
            }
        }
    }
    float lm_prev = tid == 0 ? fmaxf(s0, s1) : kNegInf;   // local max of the previous anti-diagonal
    float delta1 = 0.0f;      // base(d-1) - base(d-2)
    float mx2 = 0.0f;         // largest stored value on d-2 (when d-2 >= 0)
    double fbase = 0.0;       // base of d-1, then of d
    int32_t wi = 0;
    int32_t wD = A.windows[R.win_base].D;
    for (int32_t d = 1; d <= n; ++d) {
        // shift of this anti-diagonal: base(d) = base(d-2) + max(d-2)
        float delta0;
        if (d <= 2) {
            delta0 = 0.0f;
        } else {
            float m = sh->fpart[(d - 2) % 3][0];
#pragma unroll
            for (int w = 1; w < kGroupWarps; ++w) m = fmaxf(m, sh->fpart[(d - 2) % 3][w]);
            mx2 = m > kNegInf ? m : 0.0f;
            delta0 = mx2 - delta1;
        }
        fbase += (double) delta0;
        const int32_t L3 = band_l(d + 3), R3 = band_r(d + 3);
        // stage 1: ids and events two anti-diagonals ahead
        const int32_t Wnn = width_of(Lnn, Rnn);
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kGroup;
            kid2[j] = -1; hev2[j] = false; ev2[j] = Event32{0, 1, 0, 1};
            if (i < Wnn) {
                int32_t x, y;
                cell_xy(d + 2, Lnn, i, x, y);
                kid2[j] = load_kid(c, x);
                ev2[j] = load_event(c, y - 1);
                hev2[j] = y >= 1;
            }
        }
        // stage 2: k-mer constants one anti-diagonal ahead
        KmerConst32 kc1[CPT];
#pragma unroll
        for (int j = 0; j < CPT; ++j) kc1[j] = load_kc(c, kid1[j]);
        // the recursion on anti-diagonal d
        const int32_t W0 = width_of(L0, R0);
        const int sl = d % 3, s1l = (d + 2) % 3, s2l = (d + 1) % 3;
        const float shL = -delta0, shM = -delta1 - delta0;
        float *Fd = Freg + 3 * off0;
        float lm = kNegInf;
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kGroup;
            if (i >= W0) break;
            const int32_t xmy = L0 + 2 * i;
            float vM = kNegInf, vX = kNegInf, vY = kNegInf;
            if (xmy - 1 >= L1 && xmy - 1 <= R1) {
                const int il = (xmy - 1 - L1) >> 1;
                const float e = eX[j] + shL;
                vX = slot_ptr(fring, wmax, s1l, 0)[il] + (e + t[T_OX]);
                vX = lae(vX, slot_ptr(fring, wmax, s1l, 1)[il] + (e + t[T_EX]));
                vX = lae(vX, slot_ptr(fring, wmax, s1l, 2)[il] + (e + t[T_SX]));
            }
            if (xmy >= L2 && xmy <= R2) {
                const int im = (xmy - L2) >> 1;
                const float e = eM[j] + shM;
                vM = slot_ptr(fring, wmax, s2l, 0)[im] + (e + t[T_MC]);
                vM = lae(vM, slot_ptr(fring, wmax, s2l, 1)[im] + (e + t[T_MFGX]));
                vM = lae(vM, slot_ptr(fring, wmax, s2l, 2)[im] + (e + t[T_MFGY]));
            }
            if (xmy + 1 >= L1 && xmy + 1 <= R1) {
                const int iu = (xmy + 1 - L1) >> 1;
                const float e = eY[j] + shL;
                vY = slot_ptr(fring, wmax, s1l, 0)[iu] + (e + t[T_OY]);
                vY = lae(vY, slot_ptr(fring, wmax, s1l, 2)[iu] + (e + t[T_EY]));
            }
            slot_ptr(fring, wmax, sl, 0)[i] = vM;
            slot_ptr(fring, wmax, sl, 1)[i] = vX;
            slot_ptr(fring, wmax, sl, 2)[i] = vY;
            Fd[i] = vM;
            Fd[W0 + i] = vX;
            Fd[2 * W0 + i] = vY;
            lm = fmaxf(lm, fmaxf(vM, fmaxf(vX, vY)));
        }
        // lagged reduction of the previous anti-diagonal's maximum
        {
            const float wm = warp_max(lm_prev);
            if (lane == 0) sh->fpart[(d - 1) % 3][warp] = wm;
        }
        // emissions of the next anti-diagonal's cells
        const int32_t Wn = width_of(Ln, Rn);
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kGroup;
            if (i < Wn) {
                emit_all(c, kid1[j], kc1[j], ev1[j], hev1[j], eM[j], eY[j], eX[j]);
            } else {
                eM[j] = eY[j] = eX[j] = kNegInf;
            }
            kid1[j] = kid2[j]; ev1[j] = ev2[j]; hev1[j] = hev2[j];
        }
        if (tid == 0) {
            A.base[db + d] = fbase;
            A.fshift[db + d] = delta0;
        }
        const bool window_end = d == wD;
        if (window_end) __threadfence_block();
        group_bar(kBarForward);
        if (window_end) {
            if (tid == 0) atomicExch(&sh->fwd_done, wi + 1);
            ++wi;
            if (wi < R.n_windows) wD = A.windows[R.win_base + wi].D;
        }
        lm_prev = lm;
        delta1 = delta0;
        off0 += W0;
        L2 = L1; R2 = R1; L1 = L0; R1 = R0; L0 = Ln; R0 = Rn; Ln = Lnn; Rn = Rnn; Lnn = L3; Rnn = R3;
    }
}

// ------------------------------------------------------------------------------------------------
// backward group: one traceback window at a time, posteriors fused
// ------------------------------------------------------------------------------------------------
template <int CPT>
__device__ void backward_region(const Ctx &c, Shared *sh, float *bring, float *chain) {
    const Args &A = *c.A;
    const RegionDesc &R = c.R;
    const float *t = c.t;
    const int tid = threadIdx.x - kGroup, lane = tid & 31, warp = tid >> 5;
    const int wmax = A.wmax;
    const int64_t db = R.diag_base;
    const int32_t n = R.n;
    const float *Freg = A.F + 3 * R.cell_base;
    auto band_l = [&](int32_t d) -> int32_t { return (d >= 0 && d <= n) ? __ldg(A.xl + db + d) : 0; };
    auto band_r = [&](int32_t d) -> int32_t { return (d >= 0 && d <= n) ? __ldg(A.xr + db + d) : -2; };
    int64_t n_out = 0;
    double ll = 0.0;
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
        const int32_t D = W.D;
        // end-state values on D (stateMachine.c:1034-1061)
        const bool ragged_end = W.at_end && R.ragged_right;
        const float e0 = ragged_end ? (t[T_OX] + t[T_OY]) / 2.0f : t[T_MC];
        const float e1 = ragged_end ? t[T_EX] : t[T_MFGX];
        const float e2 = ragged_end ? t[T_EY] : t[T_MFGY];
        float mxD = fmaxf(e0, fmaxf(e1, e2));
        if (!(mxD > kNegInf)) mxD = 0.0f;
        // band bounds: d+2, d+1, d, d-1, d-2 (d = D at the start)
        int32_t Lpp = 0, Rpp = -2, Lp = 0, Rp = -2;
        int32_t L0 = band_l(D), R0 = band_r(D), Lm = band_l(D - 1), Rm = band_r(D - 1), Lmm = band_l(D - 2),
                Rmm = band_r(D - 2);
        int64_t off0 = __ldcg(A.coff + db + D);
        {
            const int32_t W0 = width_of(L0, R0);
            for (int i = tid; i < W0; i += kGroup) {
                slot_ptr(bring, wmax, D % 3, 0)[i] = e0;
                slot_ptr(bring, wmax, D % 3, 1)[i] = e1;
                slot_ptr(bring, wmax, D % 3, 2)[i] = e2;
            }
        }
        // pipeline registers: emissions for the cells of d (eMm: match of k-mer x+1 with event y,
        // eYu: extra event of k-mer x with event y, eXl: skip of k-mer x+1)
        float eMm[CPT], eYu[CPT], eXl[CPT];
        int32_t ka1[CPT], kb1[CPT];
        Event32 ev1[CPT];
        bool hev1[CPT];
        int32_t ka2[CPT], kb2[CPT];
        Event32 ev2[CPT];
        bool hev2[CPT];
        float fM[CPT];   // forward match value (stored) of the cells of d, for the posterior
        auto cell_xy = [&](int32_t d, int32_t L, int i, int32_t &x, int32_t &y) {
            const int32_t xmy = L + 2 * i;
            x = (d + xmy) >> 1;
            y = (d - xmy) >> 1;
        };
        auto backward_emissions = [&](int32_t ka, int32_t kb, const Event32 &ev, bool hev, const KmerConst32 &ca,
                                      const KmerConst32 &cb, float &em, float &ey, float &ex) {
            float a_m, a_y, a_x, b_m, b_y, b_x;
            emit_all(c, kb, cb, ev, hev, b_m, b_y, b_x);
            if (c.hdp) {
                a_y = (ka >= 0 && hev) ? emit_hdp(c.M->hdp, ca, ka, ev, c.rs) : kNegInf;
            } else {
                emit_all(c, ka, ca, ev, hev, a_m, a_y, a_x);
            }
            em = b_m;
            ey = a_y;
            ex = b_x;
        };
        {
            // D has no recursion; the pipeline starts with the ids and events of the D - 1 cells
            const int32_t Wm = width_of(Lm, Rm);
#pragma unroll
            for (int j = 0; j < CPT; ++j) {
                const int i = tid + j * kGroup;
                eMm[j] = eYu[j] = eXl[j] = kNegInf;
                ka1[j] = kb1[j] = -1; hev1[j] = false; ev1[j] = Event32{0, 1, 0, 1};
                if (i < Wm && D - 1 > W.T) {
                    int32_t x, y;
                    cell_xy(D - 1, Lm, i, x, y);
                    ka1[j] = load_kid(c, x);
                    kb1[j] = load_kid(c, x + 1);
                    ev1[j] = load_event(c, y);
                    hev1[j] = y < R.lY;
                }
                fM[j] = kNegInf;
                if (i < width_of(L0, R0) && D <= W.from) fM[j] = __ldcg(Freg + 3 * off0 + i);
            }
        }
        float lm_prev = kNegInf;           // local max of B stored on d+1 (lagged reduction)
        float gamma1 = 0.0f;               // base(d+1) - base(d+2)
        double bbase = 0.0;                // base of B on d
        double pref = 0.0;                 // latest refresh total probability (absolute)
        int32_t k = 0;
        // pending posterior pairs of the previous anti-diagonal (written after the next barrier)
        unsigned pend = 0;
        float pv[CPT];
        int32_t px[CPT], py[CPT], pk[CPT];
        int32_t pend_d = -1;
        group_bar(kBarBackward);
        for (int32_t d = D; d > W.T; --d) {
            const int sl = d % 3, sp = (d + 1) % 3, spp = (d + 2) % 3;
            const int32_t W0 = width_of(L0, R0);
            float gamma0 = 0.0f;           // base(d) - base(d+1)
            if (d <= D - 2) {
                float m;
                if (d == D - 2) {
                    m = mxD;
                } else {
                    m = sh->bpart[(d + 2) % 3][0];
#pragma unroll
                    for (int w = 1; w < kGroupWarps; ++w) m = fmaxf(m, sh->bpart[(d + 2) % 3][w]);
                    if (!(m > kNegInf)) m = 0.0f;
                }
                gamma0 = m - gamma1;
            }
            bbase += (double) gamma0;
            // prefetch: band of d-3, ids/events of d-2 cells (two ahead), constants of d-1 cells
            const int32_t L3 = band_l(d - 3), R3 = band_r(d - 3);
            const int32_t Wmm = width_of(Lmm, Rmm);
#pragma unroll
            for (int j = 0; j < CPT; ++j) {
                const int i = tid + j * kGroup;
                ka2[j] = kb2[j] = -1; hev2[j] = false; ev2[j] = Event32{0, 1, 0, 1};
                if (i < Wmm && d - 2 > W.T) {
                    int32_t x, y;
                    cell_xy(d - 2, Lmm, i, x, y);
                    ka2[j] = load_kid(c, x);
                    kb2[j] = load_kid(c, x + 1);
                    ev2[j] = load_event(c, y);
                    hev2[j] = y < R.lY;
                }
            }
            KmerConst32 ca1[CPT], cb1[CPT];
#pragma unroll
            for (int j = 0; j < CPT; ++j) {
                ca1[j] = load_kc(c, ka1[j]);
                cb1[j] = load_kc(c, kb1[j]);
            }
            const int32_t Wm = width_of(Lm, Rm);
            const int64_t offm = off0 - Wm;
            float fMn[CPT];
#pragma unroll
            for (int j = 0; j < CPT; ++j) {
                const int i = tid + j * kGroup;
                fMn[j] = (i < Wm && d - 1 <= W.from && d - 1 > W.T) ? __ldcg(Freg + 3 * offm + i) : kNegInf;
            }
            const double fb = __ldcg(A.base + db + d);
            // the recursion on d (D itself holds the end-state values)
            float lm = kNegInf;
            if (d < D) {
                const float shU = -gamma0, shM = -gamma1 - gamma0;
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    const int i = tid + j * kGroup;
                    if (i >= W0) break;
                    const int32_t xmy = L0 + 2 * i;
                    float vM = kNegInf, vX = kNegInf, vY = kNegInf;
                    if (d + 2 <= D && xmy >= Lpp && xmy <= Rpp) {
                        const float bm = slot_ptr(bring, wmax, spp, 0)[(xmy - Lpp) >> 1];
                        const float e = eMm[j] + shM;
                        vM = bm + (e + t[T_MC]);
                        vX = bm + (e + t[T_MFGX]);
                        vY = bm + (e + t[T_MFGY]);
                    }
                    if (xmy - 1 >= Lp && xmy - 1 <= Rp) {
                        const float bu = slot_ptr(bring, wmax, sp, 2)[(xmy - 1 - Lp) >> 1];
                        const float e = eYu[j] + shU;
                        vM = lae(vM, bu + (e + t[T_OY]));
                        vY = lae(vY, bu + (e + t[T_EY]));
                    }
                    if (xmy + 1 >= Lp && xmy + 1 <= Rp) {
                        const float bl = slot_ptr(bring, wmax, sp, 1)[(xmy + 1 - Lp) >> 1];
                        const float e = eXl[j] + shU;
                        vM = lae(vM, bl + (e + t[T_OX]));
                        vX = lae(vX, bl + (e + t[T_EX]));
                        vY = lae(vY, bl + (e + t[T_SX]));
                    }
                    slot_ptr(bring, wmax, sl, 0)[i] = vM;
                    slot_ptr(bring, wmax, sl, 1)[i] = vX;
                    slot_ptr(bring, wmax, sl, 2)[i] = vY;
                    lm = fmaxf(lm, fmaxf(vM, fmaxf(vX, vY)));
                }
            }
            {
                const float wm = warp_max(lm_prev);
                if (lane == 0 && d + 1 <= D) sh->bpart[(d + 1) % 3][warp] = wm;
            }
            // emissions of the d-1 cells
#pragma unroll
            for (int j = 0; j < CPT; ++j) {
                const int i = tid + j * kGroup;
                float em = kNegInf, ey = kNegInf, ex = kNegInf;
                if (i < Wm && d - 1 > W.T) backward_emissions(ka1[j], kb1[j], ev1[j], hev1[j], ca1[j], cb1[j], em, ey, ex);
                // the current cells' emissions are no longer needed after the recursion above
                eMm[j] = em; eYu[j] = ey; eXl[j] = ex;
                ka1[j] = ka2[j]; kb1[j] = kb2[j]; ev1[j] = ev2[j]; hev1[j] = hev2[j];
            }
            group_bar(kBarBackward);
            // pairs of the previous anti-diagonal, in the reference's order (ascending xmy)
            if (pend_d >= 0) {
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    int32_t before = 0, tot = 0;
                    for (int jj = 0; jj < j; ++jj)
#pragma unroll
                        for (int w = 0; w < kGroupWarps; ++w) before += sh->wcnt[pend_d & 1][jj][w];
#pragma unroll
                    for (int w = 0; w < kGroupWarps; ++w) {
                        if (w < warp) before += sh->wcnt[pend_d & 1][j][w];
                        tot += sh->wcnt[pend_d & 1][j][w];
                    }
                    (void) tot;
                    const unsigned mine = __ballot_sync(0xffffffffu, (pend >> j) & 1u);
                    if ((pend >> j) & 1u) {
                        const int64_t slot = n_out + before + __popc(mine & ((1u << lane) - 1u));
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
                int32_t all = 0;
#pragma unroll
                for (int j = 0; j < CPT; ++j)
#pragma unroll
                    for (int w = 0; w < kGroupWarps; ++w) all += sh->wcnt[pend_d & 1][j][w];
                n_out += all;
                pend = 0;
                pend_d = -1;
            }
            if (d <= W.from) {
                if (k++ % 10 == 0) {
                    // diagonalCalculationTotalProbability (pairwiseAligner.c:1182-1200): F.B on d in
                    // ascending cell order, then the matches from d-1 over d into d+1, dotted with B(d+1)
                    const int64_t offd = off0;
                    const float *Fd = Freg + 3 * offd;
                    for (int i = tid; i < W0; i += kGroup) {
                        float s = __ldcg(Fd + i) + slot_ptr(bring, wmax, sl, 0)[i];
                        s = lae(s, __ldcg(Fd + W0 + i) + slot_ptr(bring, wmax, sl, 1)[i]);
                        s = lae(s, __ldcg(Fd + 2 * W0 + i) + slot_ptr(bring, wmax, sl, 2)[i]);
                        chain[i] = s;
                    }
                    const bool have_next = d < D;
                    const int32_t Wp = width_of(Lp, Rp);
                    float mshift = 0.0f;
                    if (have_next) {
                        const float fsh = __ldcg(A.fshift + db + d);
                        mshift = -fsh - gamma0;
                        const float *Fm = Freg + 3 * (off0 - Wm);
                        for (int i = tid; i < Wp; i += kGroup) {
                            const int32_t xmy = Lp + 2 * i;
                            float m = kNegInf;
                            if (xmy >= Lm && xmy <= Rm) {
                                int32_t x, y;
                                cell_xy(d + 1, Lp, i, x, y);
                                const int32_t kid = load_kid(c, x);
                                float em, ey, ex;
                                emit_all(c, kid, load_kc(c, kid), load_event(c, y - 1), y >= 1, em, ey, ex);
                                const int im = (xmy - Lm) >> 1;
                                m = __ldcg(Fm + im) + (em + t[T_MC]);
                                m = lae(m, __ldcg(Fm + Wm + im) + (em + t[T_MFGX]));
                                m = lae(m, __ldcg(Fm + 2 * Wm + im) + (em + t[T_MFGY]));
                            }
                            chain[wmax + i] = m + slot_ptr(bring, wmax, sp, 0)[i];
                        }
                    }
                    group_bar(kBarBackward);
                    if (warp == 0) {
                        const float f = ordered_fold(chain, W0);
                        if (lane == 0) sh->fold[0] = f;
                    } else if (warp == 1) {
                        const float f = have_next ? ordered_fold(chain + wmax, Wp) : kNegInf;
                        if (lane == 0) sh->fold[1] = f;
                    }
                    group_bar(kBarBackward);
                    const float ptil = lae(sh->fold[0], sh->fold[1] + mshift);
                    pref = (double) ptil + fb + bbase;
                    if (d == n) ll = pref;
                }
                const float kd = (float) (fb + bbase - pref);
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    const int i = tid + j * kGroup;
                    bool hit = false;
                    if (i < W0) {
                        int32_t x, y;
                        cell_xy(d, L0, i, x, y);
                        if (x > 0 && y > 0) {
                            const float p = __expf(fM[j] + slot_ptr(bring, wmax, sl, 0)[i] + kd);
                            if (p >= A.threshold) {
                                hit = true;
                                pv[j] = p;
                                px[j] = x;
                                py[j] = y;
                                pk[j] = load_kid(c, x);
                            }
                        }
                    }
                    const unsigned bal = __ballot_sync(0xffffffffu, hit);
                    if (hit) pend |= 1u << j;
                    if (lane == 0) sh->wcnt[d & 1][j][warp] = __popc(bal);
                }
                pend_d = d;
            }
#pragma unroll
            for (int j = 0; j < CPT; ++j) fM[j] = fMn[j];
            lm_prev = lm;
            if (d == D) lm_prev = kNegInf;   // D's maximum is known exactly (mxD)
            gamma1 = gamma0;
            off0 = offm;
            Lpp = Lp; Rpp = Rp; Lp = L0; Rp = R0; L0 = Lm; R0 = Rm; Lm = Lmm; Rm = Rmm; Lmm = L3; Rmm = R3;
        }
        // flush the last anti-diagonal's pairs
        group_bar(kBarBackward);
        if (pend_d >= 0) {
#pragma unroll
            for (int j = 0; j < CPT; ++j) {
                int32_t before = 0;
                for (int jj = 0; jj < j; ++jj)
#pragma unroll
                    for (int w = 0; w < kGroupWarps; ++w) before += sh->wcnt[pend_d & 1][jj][w];
#pragma unroll
                for (int w = 0; w < kGroupWarps; ++w)
                    if (w < warp) before += sh->wcnt[pend_d & 1][j][w];
                const unsigned mine = __ballot_sync(0xffffffffu, (pend >> j) & 1u);
                if ((pend >> j) & 1u) {
                    const int64_t slot = n_out + before + __popc(mine & ((1u << lane) - 1u));
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
            int32_t all = 0;
#pragma unroll
            for (int j = 0; j < CPT; ++j)
#pragma unroll
                for (int w = 0; w < kGroupWarps; ++w) all += sh->wcnt[pend_d & 1][j][w];
            n_out += all;
        }
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
    float *bring = fring + 9 * A.wmax;
    float *chain = bring + 9 * A.wmax;
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
