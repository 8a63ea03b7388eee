// Batched FP32 form, warp kernels: every task is run by one warp.
//
//   * forward task: one region's forward sweep, anti-diagonal by anti-diagonal;
//   * window task: one traceback window's backward sweep with the posterior test and the
//     total-probability refreshes fused in (getPosteriorProbsWithBanding, pairwiseAligner.c:
//     1282-1420).
//
// Cells live in registers.  A warp covers 128 consecutive columns ("slots") of the matrix: lane l
// holds the four slots 4l .. 4l+3 of the window base Xb (absolute column x = Xb + slot), chosen per
// anti-diagonal by the host so that the bands of d-1, d and d+1 lie in [Xb + 1, Xb + 126] (Xb a
// multiple of 4, changed rarely).  Indexed by column, the recursion's neighbours sit at fixed
// slots: cell (x, y) on d takes its lower neighbour (x-1, y) and its upper neighbour (x, y-1) from
// d-1 at slots x-1 and x, and its middle neighbour (x-1, y-1) from d-2 at slot x-1; the backward
// sweep takes its successors from slots x+1 and x.  So a step moves one value per state across a
// lane boundary (a shuffle) and nothing else moves; when Xb changes, whole lanes shift.
//
// Emissions: Gaussian machines compute them in place from per-slot k-mer constants (loaded when Xb
// changes) and per-cell events (one new event per lane per step, the others rotate through four
// registers); HDP machines read them from emission rows written beforehand by emission_rows_kernel
// (the spline density in FP64; its tails underflow FP32).
//
// Forward values go to a per-region ring of ring_rows anti-diagonals (3 planes of 128 floats:
// match, and the gap states on anti-diagonals a refresh reads), not a whole-matrix store.  Before
// it overwrites a row, the forward sweep waits (bounded) until every window reading that row is
// done.  Windows are published to a ready queue as the sweep passes their traceback anti-diagonal;
// warps claim them from the queue once no forward sweep is left for them to claim.  A fixed share of
// the warps never takes a forward sweep, so the queue is served even when a batch has more regions
// than the grid has warps, and every wait of a forward sweep ends.
//
// Every wait is bounded (spin_limit clock cycles); a wait that runs out sets the batch's error flag,
// every other waiter and every forward sweep leaves, and the launch ends normally.
#pragma once

namespace sa {
namespace wk {

using namespace dp32;
using fp32::kFlagRefresh;
using fp32::kFlagStoreGaps;
using fp32::kFlagWindowEnd;
using fp32::kWidthMask;
using fp32::lae;

constexpr int kCpl = 4;                  // slots per lane
constexpr int kSlots = 32 * kCpl;        // slots per warp
constexpr int kWarps = 4;                // warps per CTA
constexpr int kRowFloats = 3 * kSlots;   // ring row: match, gap-X, gap-Y planes

enum { T_MC = 0, T_MFGX, T_MFGY, T_OX, T_OY, T_EX, T_EY, T_SX, T_SY };

struct WRegion {
    int32_t n, lX, lY, read;
    int32_t n_windows, model;
    int32_t ragged_left, ragged_right;
    int64_t diag_base;      // first anti-diagonal of the region in the per-anti-diagonal arrays
    int64_t win_base;       // first window of the region
    int64_t kmer_base;      // k-mer id of column x >= 1 is kmer[kmer_base + x - 1]
    int64_t event_base;     // event of row y >= 1 is events[event_base + y - 1]
    int64_t x1, y1;         // offset of the region in read coordinates
    int64_t ring_base;      // float offset of the region's forward ring
    int64_t e_base;         // float offset of its emission rows (stored emissions), else -1
    int32_t ring_rows;      // power of two
    int32_t stored;         // emissions from emission rows (HDP machine)
};

struct WModel {
    const float4 *kc;       // per k-mer two float4: {mu, -1/(2 sd^2), -1/(2 sd_y^2), k_m},
                            // {k_y, 1/noise mean, -lambda/2, gap-X log probability}
    fp32::Hdp64 hdp64;
    int32_t emission;
    int32_t has_sx;         // SWITCH_TO_X is finite (a .model file leaves it LOG_ZERO)
    float t[9];
    float pad;
};

struct WArgs {
    const WRegion *regions;
    const int32_t *order;           // forward claims: regions by band area, largest first
    int64_t n_regions;
    const WModel *models;
    const ReadScale32 *read_scale;
    const fp32::ReadScale64 *read_scale64;
    const double2 *events_raw;      // per event FP64 (mean, noise)
    float4 *events;                 // per event {mean / var, noise, -1.5 log noise, 1 / noise}
    const int4 *meta;               // per anti-diagonal {xmy of first cell, width | flags, Xb, row offset}
    const Window *windows;
    const fp32::WindowTask *wtask;
    int64_t n_windows;
    int32_t *wflag;                 // per window: 2 once its backward sweep is done
    const int32_t *kmer;
    float *F;                       // forward rings
    float *E;                       // emission rows (stored-emission regions)
    double *base;                   // per anti-diagonal FP64 base of the forward values
    float *fshift;                  // per anti-diagonal base(d) - base(d-1)
    int32_t *ready;                 // ready queue of windows (-1: not yet published)
    sa_aligned_pair *out;           // per-window output segments
    int64_t *wcount;                // per window: pairs written (may exceed its capacity)
    double *loglik;                 // per region: total probability at its last anti-diagonal
    int32_t *status;                // per read
    fp32::Control *ctl;
    float threshold;
    int32_t pad;
    long long spin_limit;           // clock cycles a warp may wait
    // emission rows (stored-emission regions)
    const fp32::Chunk *echunks;     // runs of anti-diagonals of such regions
    int64_t n_echunks;
};

constexpr float kNInf = kNegInf;

// ------------------------------------------------------------------------------------------------
// lane helpers
// ------------------------------------------------------------------------------------------------
// value of slot 4l + j - 1 for v holding slots 4l .. 4l + 3 (slot -1 of lane 0: -inf)
__device__ __forceinline__ float from_left(const float (&v)[kCpl], int j, int lane) {
    if (j > 0) return v[j - 1];
    const float t = __shfl_up_sync(0xffffffffu, v[kCpl - 1], 1);
    return lane > 0 ? t : kNInf;
}

// value of slot 4l + j + 1 (slot 128 of lane 31: -inf)
__device__ __forceinline__ float from_right(const float (&v)[kCpl], int j, int lane) {
    if (j < kCpl - 1) return v[j + 1];
    const float t = __shfl_down_sync(0xffffffffu, v[0], 1);
    return lane < 31 ? t : kNInf;
}

// whole-lane move for a change of window base: new lane l takes old lane l + k (-inf past the ends)
__device__ __forceinline__ void shift_lanes(float (&v)[kCpl], int k, int lane) {
    const int src = lane + k;
    const bool ok = src >= 0 && src < 32;
#pragma unroll
    for (int j = 0; j < kCpl; ++j) {
        const float t = __shfl_sync(0xffffffffu, v[j], src & 31);
        v[j] = ok ? t : kNInf;
    }
}

__device__ __forceinline__ float lane_max(const float (&a)[kCpl], const float (&b)[kCpl], const float (&c)[kCpl]) {
    float m = fmaxf(fmaxf(a[0], b[0]), c[0]);
#pragma unroll
    for (int j = 1; j < kCpl; ++j) m = fmaxf(m, fmaxf(fmaxf(a[j], b[j]), c[j]));
    return m;
}

__device__ __forceinline__ float4 ld4(const float *p) { return __ldcg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void st4(float *p, const float (&v)[kCpl]) {
    __stcg(reinterpret_cast<float4 *>(p), make_float4(v[0], v[1], v[2], v[3]));
}
__device__ __forceinline__ void unpack(const float4 &q, float (&v)[kCpl]) {
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}

struct MetaW {
    int32_t L, W, flags, xb, eoff;
};

__device__ __forceinline__ MetaW decode(int4 m) {
    return MetaW{m.x, m.y & kWidthMask, m.y & ~kWidthMask, m.z, m.w};
}

// ------------------------------------------------------------------------------------------------
// emissions of a lane's four cells
// ------------------------------------------------------------------------------------------------
// Per-slot constants of the Gaussian emissions (the k-mer of column x, the read's scaling folded
// into the level mean); a column without a k-mer (x < 1 or x > lX) has -inf log constants, so both
// of its emissions and its skip emission are -inf (the reference's NULL k-mer, stateMachine.c:498-545).
struct SlotK {
    float mu, cm, cy, km, ky, inu, nhl, gx;
};

struct Emit {
    SlotK k[kCpl];
    float4 ev[kCpl];        // the cells' events in four rotating registers
    float4 pre[2];          // the next new event, loaded one step ahead
    int32_t kid[kCpl];      // k-mer id per slot (pair output)
};

__device__ __forceinline__ void load_slot_consts(const WArgs &A, const WRegion &R, const WModel &M,
                                                 const ReadScale32 &rs, int32_t xb, int lane, Emit &e,
                                                 bool gauss) {
#pragma unroll
    for (int j = 0; j < kCpl; ++j) {
        const int32_t x = xb + 4 * lane + j;
        const bool ok = x >= 1 && x <= R.lX;
        const int32_t kid = ok ? __ldg(A.kmer + R.kmer_base + x - 1) : 0;
        e.kid[j] = kid;
        if (gauss) {
            const float4 a = __ldg(M.kc + 2 * (int64_t) kid), b = __ldg(M.kc + 2 * (int64_t) kid + 1);
            SlotK &s = e.k[j];
            s.mu = fmaf(rs.scale, a.x, rs.shift) * rs.inv_var;
            s.cm = a.y;
            s.cy = a.z;
            s.km = ok ? a.w : kNInf;
            s.ky = ok ? b.x : kNInf;
            s.inu = b.y;
            s.nhl = b.z;
            s.gx = ok ? b.w : kNInf;
        }
    }
}

__device__ __forceinline__ float4 load_event(const WArgs &A, const WRegion &R, int32_t y) {
    const int32_t yc = min(max(y - 1, 0), max(R.lY - 1, 0));
    return __ldg(A.events + R.event_base + yc);
}

// emissions of match and extra event (stateMachine.c:498-545 with :226-247, :285-289): the
// descaled residual r = (mean - scale mu - shift) / var, log N(r; 0, sd) + log IG(noise; nu, lambda)
__device__ __forceinline__ void gauss2(const SlotK &s, const float4 &v, float &em, float &ey) {
    const float r = v.x - s.mu;
    const float r2 = r * r;
    const float b = fmaf(v.y, s.inu, -1.0f);
    const float common = fmaf(s.nhl, (b * v.w) * b, v.z);
    em = fmaf(r2, s.cm, s.km + common);
    ey = fmaf(r2, s.cy, s.ky + common);
}

// the four cells' emissions on one anti-diagonal (match, extra event, skip); cell j's event is in
// register (R0 + DIR * j) mod 4
template <bool kStored, int R0, int DIR>
__device__ __forceinline__ void cell_emissions(const Emit &e, const float4 &erow, float gx_stored,
                                               float (&eM)[kCpl], float (&eY)[kCpl], float (&eX)[kCpl]) {
    if (kStored) {
        unpack(erow, eM);
#pragma unroll
        for (int j = 0; j < kCpl; ++j) {
            eY[j] = eM[j];
            eX[j] = gx_stored;
        }
    } else {
#pragma unroll
        for (int j = 0; j < kCpl; ++j) {
            gauss2(e.k[j], e.ev[(R0 + DIR * j) & 3], eM[j], eY[j]);
            eX[j] = e.k[j].gx;
        }
    }
}

// emission row of anti-diagonal d for this lane's four slots (stored emissions)
__device__ __forceinline__ float4 load_erow(const WArgs &A, const WRegion &R, int32_t d, const MetaW &m, int lane) {
    const int32_t xL = (d + m.L) >> 1, xR = xL + m.W - 1;
    const int32_t xa = xL & ~3, len = ((xR - xa + 1) + 3) & ~3;
    const int32_t x0 = m.xb + 4 * lane;
    if (m.W > 0 && x0 >= xa && x0 < xa + len)
        return __ldg(reinterpret_cast<const float4 *>(A.E + R.e_base + m.eoff + (x0 - xa)));
    return make_float4(kNInf, kNInf, kNInf, kNInf);
}

// -inf mask of the band: 0 for slots inside [xL, xR], -inf outside
__device__ __forceinline__ void band_mask(int32_t d, const MetaW &m, int lane, float (&mk)[kCpl]) {
    const int32_t xL = (d + m.L) >> 1;
    const int32_t lo = xL - m.xb - 4 * lane;
#pragma unroll
    for (int j = 0; j < kCpl; ++j) mk[j] = (unsigned) (j - lo) < (unsigned) m.W ? 0.0f : kNInf;
}

// ------------------------------------------------------------------------------------------------
// bounded waits
// ------------------------------------------------------------------------------------------------
// one lane: until `flag` reaches `want`; false if the wait gave up (error flag set)
__device__ __forceinline__ bool wait_flag(const WArgs &A, const int32_t *flag, int32_t want) {
    const long long t0 = clock64();
    for (;;) {
        if (*((volatile const int32_t *) flag) >= want) {
            __threadfence();
            return true;
        }
        if (*((volatile int32_t *) &A.ctl->error)) return false;
        if (clock64() - t0 > A.spin_limit) {
            atomicExch(&A.ctl->error, 1);
            return false;
        }
        __nanosleep(256);
    }
}

// one lane: until ready-queue slot `slot` is published; -1 if the wait gave up
__device__ __forceinline__ int32_t wait_ready(const WArgs &A, int64_t slot) {
    const long long t0 = clock64();
    for (;;) {
        const int32_t v = *((volatile int32_t *) (A.ready + slot));
        if (v >= 0) {
            __threadfence();
            return v;
        }
        if (*((volatile int32_t *) &A.ctl->error)) return -1;
        if (clock64() - t0 > A.spin_limit) {
            atomicExch(&A.ctl->error, 1);
            return -1;
        }
        __nanosleep(512);
    }
}

// ------------------------------------------------------------------------------------------------
// forward sweep of one region
// ------------------------------------------------------------------------------------------------
template <bool kStored>
struct Forward {
    const WArgs &A;
    WRegion R;
    const WModel *M;
    const float4 *tab;
    ReadScale32 rs;
    float t[9];
    bool has_sx;
    float gx_stored;
    int lane;
    int32_t n, rmask;
    int64_t db;
    float *ring;
    // rows d-1 and d-2 by parity of the anti-diagonal, and the slot-0 element of the slot-shifted
    // copy of each (its value of slot -1; the other elements alias the row itself)
    float S[2][3][kCpl];
    float U0[2][3];
    int32_t xb;
    Emit e;
    float4 erow[4];         // stored emissions of d .. d+3 by d mod 4
    int4 mq[4];             // raw metas of d .. d+3 by d mod 4
    MetaW m0;               // meta of d
    float wm[2];            // warp maxima of the last two rows (by parity)
    float delta1;           // delta(d-1)
    double base0;           // base(d-1)
    double qbase;           // lane q keeps base and shift of the last anti-diagonal d with d mod 32 == q
    float qshift;
    int32_t wi;             // next window of the region to publish
    int32_t lo;             // lowest window not known to be done
    int32_t t_lo;           // its first forward row
    bool failed;

    __device__ __forceinline__ Forward(const WArgs &a, const float4 *tb) : A(a), tab(tb) {}

    __device__ __forceinline__ int4 raw_meta(int32_t d) const { return __ldg(A.meta + db + min(max(d, 0), n)); }

    // the window base moves to new_xb at anti-diagonal d (phase P: d = 4k + P + 1): rows d-1 and
    // d-2 shift by whole lanes, the slot constants and the events of d are reloaded
    template <int P>
    __device__ __forceinline__ void rebase(int32_t d, int32_t new_xb) {
        constexpr int c = (P + 1) & 1;
        const int k = (new_xb - xb) >> 2;
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int s = 0; s < 3; ++s) shift_lanes(S[q][s], k, lane);
        // slot-0 elements of the shifted row d-2 (the middle neighbours of d)
#pragma unroll
        for (int s = 0; s < 3; ++s) U0[c][s] = from_left(S[c][s], 0, lane);
        xb = new_xb;
        load_slot_consts(A, R, *M, rs, xb, lane, e, !kStored);
        if (!kStored) {
#pragma unroll
            for (int j = 0; j < kCpl; ++j) e.ev[(P + 1 - j) & 3] = load_event(A, R, d - xb - 4 * lane - j);
            e.pre[P & 1] = load_event(A, R, d + 1 - xb - 4 * lane);
        } else {
            // emission rows of d .. d+2 were loaded for the old base (mq still holds d .. d+3)
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (d + q <= n) {
                    MetaW mm = decode(mq[(P + 1 + q) & 3]);
                    mm.xb = xb;
                    erow[(P + 1 + q) & 3] = load_erow(A, R, d + q, mm, lane);
                }
            }
        }
    }

    // before row d goes into the ring: every window that reads the row it replaces is done.  Those
    // windows were published (the ring holds more than a window's span), and the warps that serve
    // the ready queue take them in publication order, so the wait ends; it is bounded anyway.
    __device__ __forceinline__ bool make_room(int32_t d) {
        const int32_t w = d - R.ring_rows;
        while (lo < R.n_windows && t_lo <= w) {
            bool ok = true;
            if (lane == 0) ok = wait_flag(A, A.wflag + R.win_base + lo, 2);
            if (!__shfl_sync(0xffffffffu, (int) ok, 0)) return false;
            ++lo;
            if (lo < R.n_windows) t_lo = __ldg(&A.windows[R.win_base + lo].T);
        }
        return true;
    }

    template <int P>
    __device__ __forceinline__ void step(int32_t d) {
        constexpr int c = (P + 1) & 1;    // parity of d (d = 4k + P + 1)
        constexpr int p = c ^ 1;          // parity of d-1
        constexpr int r0 = (P + 1) & 3;   // d mod 4
        // band facts: meta of d (requested four steps ago); request d+4 after a possible rebase
        m0 = decode(mq[r0]);
        if (m0.xb != xb) rebase<P>(d, m0.xb);
        mq[r0] = raw_meta(d + 4);
        if (kStored && d + 3 <= n) erow[(r0 + 3) & 3] = load_erow(A, R, d + 3, decode(mq[(r0 + 3) & 3]), lane);
        // renormalisation: base(d) = base(d-2) + max(d-2), so delta(d) = max(d-2) - delta(d-1)
        const float mx2 = wm[c];
        const float delta0 = (mx2 > kNInf ? mx2 : 0.0f) - delta1;
        const float shL = -delta0, shM = -delta0 - delta1;
        // emissions of d and the band mask
        float eM[kCpl], eY[kCpl], eX[kCpl], mk[kCpl];
        cell_emissions<kStored, r0, -1>(e, erow[r0], gx_stored, eM, eY, eX);
        band_mask(d, m0, lane, mk);
        // the recursion (stateMachine3_cellCalculate, stateMachine.c:1194-1257, in its order:
        // lower -> gap-X, middle -> match, upper -> gap-Y, each state accumulated from LOG_ZERO).
        // lower and upper come from d-1 (slots q-1, q), middle from d-2 (slot q-1).
        float nM[kCpl], nX[kCpl], nY[kCpl];
        float u0[3];
#pragma unroll
        for (int s = 0; s < 3; ++s) u0[s] = from_left(S[p][s], 0, lane);
#pragma unroll
        for (int j = 0; j < kCpl; ++j) {
            const float lM = j ? S[p][0][j - 1] : u0[0];
            const float lX = j ? S[p][1][j - 1] : u0[1];
            const float lY = j ? S[p][2][j - 1] : u0[2];
            const float mM = j ? S[c][0][j - 1] : U0[c][0];
            const float mX = j ? S[c][1][j - 1] : U0[c][1];
            const float mY = j ? S[c][2][j - 1] : U0[c][2];
            const float uM = S[p][0][j], uY = S[p][2][j];
            // logAdd depends only on the difference of its arguments, so the cell's emission (and
            // the shift to this anti-diagonal's base, and the band mask) is added once after each
            // state's fold
            float vX = lae(tab, lM + t[T_OX], lX + t[T_EX]);
            if (has_sx) vX = lae(tab, vX, lY + t[T_SX]);
            vX = vX + (eX[j] + (shL + mk[j]));
            float vM = lae(tab, mM + t[T_MC], mX + t[T_MFGX]);
            vM = lae(tab, vM, mY + t[T_MFGY]) + (eM[j] + (shM + mk[j]));
            const float vY = lae(tab, uM + t[T_OY], uY + t[T_EY]) + (eY[j] + (shL + mk[j]));
            nM[j] = vM;
            nX[j] = vX;
            nY[j] = vY;
        }
        // row d replaces row d-2: keep the slot-shifted copy of d-1 for d+1's middle neighbours
#pragma unroll
        for (int s = 0; s < 3; ++s) U0[p][s] = u0[s];
#pragma unroll
        for (int j = 0; j < kCpl; ++j) {
            S[c][0][j] = nM[j];
            S[c][1][j] = nX[j];
            S[c][2][j] = nY[j];
        }
        // the event of cell 0 of d+1 (the others rotate), and the one of d+2 requested
        if (!kStored) {
            e.ev[(r0 + 1) & 3] = e.pre[P & 1];
            e.pre[(P + 1) & 1] = load_event(A, R, d + 2 - xb - 4 * lane);
        }
        // forward ring
        if (d >= R.ring_rows && !make_room(d)) {
            failed = true;
            return;
        }
        float *row = ring + (int64_t) (d & rmask) * kRowFloats + 4 * lane;
        st4(row, nM);
        if (m0.flags & kFlagStoreGaps) {
            st4(row + kSlots, nX);
            st4(row + 2 * kSlots, nY);
        }
        // warp maximum of d for base(d+2)
        wm[c] = fp32::warp_max1(lane_max(nM, nX, nY));
        // base and shift of d: lane d mod 32 keeps them; written 32 at a time and before a window
        // is published (its backward sweep reads them)
        base0 += (double) delta0;
        delta1 = delta0;
        const int q = d & 31;
        if (lane == q) {
            qbase = base0;
            qshift = delta0;
        }
        const bool window_end = (m0.flags & kFlagWindowEnd) != 0;
        if ((q == 31 || window_end || d == n) && lane <= q) {
            A.base[db + (d - q) + lane] = qbase;
            A.fshift[db + (d - q) + lane] = qshift;
        }
        if (window_end) {
            __threadfence();
            __syncwarp();
            if (lane == 0) {
                const unsigned slot = atomicAdd(&A.ctl->pub, 1u);
                atomicExch(A.ready + slot, (int32_t) (R.win_base + wi));
            }
            ++wi;
        }
    }

    __device__ __forceinline__ void run(int32_t region) {
        lane = threadIdx.x & 31;
        R = A.regions[region];
        M = A.models + R.model;
        rs = A.read_scale[R.read];
#pragma unroll
        for (int i = 0; i < 9; ++i) t[i] = M->t[i];
        has_sx = M->has_sx != 0;
        gx_stored = (float) kLogPointOne;
        n = R.n;
        db = R.diag_base;
        rmask = R.ring_rows - 1;
        ring = A.F + R.ring_base;
        failed = false;
        wi = 0;
        lo = 0;
        t_lo = R.n_windows > 0 ? __ldg(&A.windows[R.win_base].T) : 0;
        // anti-diagonal 0: the start states (startStateProb / raggedStartStateProb,
        // stateMachine.c:1022-1032) in the slot of x = 0
        m0 = decode(raw_meta(0));
        xb = m0.xb;
        const float s0 = R.ragged_left ? kNInf : 0.0f, s1 = R.ragged_left ? 0.0f : kNInf;
        const int q0 = -xb;   // slot of x = 0
#pragma unroll
        for (int j = 0; j < kCpl; ++j) {
            const bool here = 4 * lane + j == q0;
            S[0][0][j] = here ? s0 : kNInf;
            S[0][1][j] = here ? s1 : kNInf;
            S[0][2][j] = here ? s1 : kNInf;
            S[1][0][j] = S[1][1][j] = S[1][2][j] = kNInf;   // row -1
        }
        // slot-shifted copies: row -1 (the middle of d = 1) is all -inf
        U0[0][0] = U0[0][1] = U0[0][2] = kNInf;
        U0[1][0] = U0[1][1] = U0[1][2] = kNInf;
        {
            float *row = ring + 4 * lane;
            st4(row, S[0][0]);
            st4(row + kSlots, S[0][1]);
            st4(row + 2 * kSlots, S[0][2]);
        }
        if (lane == 0) {
            A.base[db] = 0.0;
            A.fshift[db] = 0.0f;
        }
        load_slot_consts(A, R, *M, rs, xb, lane, e, !kStored);
        if (!kStored) {
            // d = 1: cell j's event in register (1 - j) mod 4; the new event of d = 2 in pre[0]
#pragma unroll
            for (int j = 0; j < kCpl; ++j) e.ev[(1 - j) & 3] = load_event(A, R, 1 - xb - 4 * lane - j);
            e.pre[0] = load_event(A, R, 2 - xb - 4 * lane);
            e.pre[1] = e.pre[0];
        } else {
#pragma unroll
            for (int q = 1; q <= 3; ++q)
                if (q <= n) erow[q & 3] = load_erow(A, R, q, decode(raw_meta(q)), lane);
        }
#pragma unroll
        for (int q = 1; q <= 4; ++q) mq[q & 3] = raw_meta(q);
        // maxima of row 0 (for delta(2) = max(0)) and row -1 (taken as 0: delta(1) = 0)
        wm[0] = fp32::warp_max1(lane_max(S[0][0], S[0][1], S[0][2]));
        wm[1] = 0.0f;
        delta1 = 0.0f;                   // delta(0)
        base0 = 0.0;
        qbase = 0.0;
        qshift = 0.0f;
        // d = 1, 2, 3, 4, ... : phase P = (d - 1) mod 4
        for (int32_t d = 1; d <= n; d += 4) {
            step<0>(d);
            if (failed || d + 1 > n) break;
            step<1>(d + 1);
            if (failed || d + 2 > n) break;
            step<2>(d + 2);
            if (failed || d + 3 > n) break;
            step<3>(d + 3);
            if (failed) break;
        }
    }
};

// ------------------------------------------------------------------------------------------------
// backward sweep of one traceback window, posteriors and refreshes fused
// ------------------------------------------------------------------------------------------------
template <bool kStored>
struct Backward {
    const WArgs &A;
    WRegion R;
    const WModel *M;
    const float4 *tab;
    float *chain;           // this warp's 2 x kSlots floats: refresh terms of d and of d+1
    ReadScale32 rs;
    float t[9];
    bool has_sx;
    float gx_stored;
    int lane;
    int32_t n, rmask, D, T, from;
    int64_t db;
    const float *ring;
    // successors: P = B + own emission of rows d+1 and d+2 by parity of D - row; B_M and e_M of d+1
    float PM[2][kCpl], PX[2][kCpl], PY[2][kCpl];
    float BM1[kCpl], EM1[kCpl];
    int32_t xb;
    Emit e;
    float4 erow[4];         // stored emissions of d .. d-3 by (D - d) mod 4
    int4 mq[4];             // raw metas of d .. d-3 by (D - d) mod 4
    MetaW mp, m0;           // metas of d+1 and d
    float4 fq[2];           // forward match values of d (prefetched one step ahead) by (D - d) mod 2
    double fbq[2];
    float fsq[2];
    float mx[2];            // warp maxima of B on the last two rows (by parity)
    float gamma1, mxD;
    float e0, e1, e2;
    double bbase, pref, ll;
    int64_t n_out;
    fp32::WindowTask wt;

    __device__ __forceinline__ Backward(const WArgs &a, const float4 *tb, float *ch) : A(a), tab(tb), chain(ch) {}

    __device__ __forceinline__ int4 raw_meta(int32_t d) const { return __ldg(A.meta + db + min(max(d, 0), n)); }

    template <int Q>
    __device__ __forceinline__ void prefetch_f(int32_t d) {
        if (d <= T) return;
        fq[Q] = ld4(ring + (int64_t) (d & rmask) * kRowFloats + 4 * lane);
        fbq[Q] = __ldcg(A.base + db + d);
        fsq[Q] = __ldcg(A.fshift + db + d);
    }

    // the window base moves to new_xb at anti-diagonal d (phase P: d = D - 4k - P)
    template <int P>
    __device__ __forceinline__ void rebase(int32_t d, int32_t new_xb) {
        const int k = (new_xb - xb) >> 2;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            shift_lanes(PM[q], k, lane);
            shift_lanes(PX[q], k, lane);
            shift_lanes(PY[q], k, lane);
        }
        shift_lanes(BM1, k, lane);
        shift_lanes(EM1, k, lane);
        xb = new_xb;
        load_slot_consts(A, R, *M, rs, xb, lane, e, !kStored);
        if (!kStored) {
            // cell j of d uses event register (P + j) mod 4; the next new event (cell 3 of d-1)
#pragma unroll
            for (int j = 0; j < kCpl; ++j) e.ev[(P + j) & 3] = load_event(A, R, d - xb - 4 * lane - j);
            e.pre[(P + 1) & 1] = load_event(A, R, d - 1 - xb - 4 * lane - 3);
        } else {
            // emission rows of d .. d-2 were loaded for the old base (mq still holds d .. d-3)
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (d - q > T) {
                    MetaW mm = decode(mq[(P + q) & 3]);
                    mm.xb = xb;
                    erow[(P + q) & 3] = load_erow(A, R, d - q, mm, lane);
                }
            }
        }
        // the forward row of d (prefetched) was stored by the forward sweep with d's own base: no move
    }

    // forward row dd (match, gap-X, gap-Y planes), in the current slot mapping
    __device__ __forceinline__ void load_frow(int32_t dd, float (&fm)[kCpl], float (&fx)[kCpl], float (&fy)[kCpl]) {
        const float *row = ring + (int64_t) (dd & rmask) * kRowFloats + 4 * lane;
        unpack(ld4(row), fm);
        unpack(ld4(row + kSlots), fx);
        unpack(ld4(row + 2 * kSlots), fy);
        const int32_t rxb = decode(raw_meta(dd)).xb;
        if (rxb != xb) {
            const int k = (xb - rxb) >> 2;
            shift_lanes(fm, k, lane);
            shift_lanes(fx, k, lane);
            shift_lanes(fy, k, lane);
        }
    }

    template <int P>
    __device__ __forceinline__ void step(int32_t d) {
        constexpr int c = P & 1;          // parity of D - d (d = D - 4k - P)
        constexpr int p = c ^ 1;          // parity of D - (d+1) (d+2 has parity c)
        const bool first = d == D;
        mp = m0;
        m0 = decode(mq[P]);
        if (m0.xb != xb) rebase<P>(d, m0.xb);
        mq[P] = raw_meta(d - 4);
        if (kStored && d - 3 > T) erow[(P + 3) & 3] = load_erow(A, R, d - 3, decode(mq[(P + 3) & 3]), lane);
        // backward base: base(d) = base(d+2) + max(d+2), gamma0 = base(d) - base(d+1)
        float gamma0 = 0.0f;
        if (d <= D - 2) {
            float m = d == D - 2 ? mxD : mx[c];
            if (!(m > kNInf)) m = 0.0f;
            gamma0 = m - gamma1;
        }
        bbase += (double) gamma0;
        const float shU = -gamma0, shM = -gamma1 - gamma0;
        float mk[kCpl];
        band_mask(d, m0, lane, mk);
        float bM[kCpl], bX[kCpl], bY[kCpl];
        if (first) {
#pragma unroll
            for (int j = 0; j < kCpl; ++j) {
                bM[j] = e0 + mk[j];
                bX[j] = e1 + mk[j];
                bY[j] = e2 + mk[j];
            }
        } else {
            // successors: match (x+1, y+1) on d+2 at slot q+1, upper (x, y+1) on d+1 at slot q,
            // lower (x+1, y) on d+1 at slot q+1; each already holds its own emission
#pragma unroll
            for (int j = 0; j < kCpl; ++j) {
                const float me = from_right(PM[c], j, lane) + shM;
                const float ue = PY[p][j] + shU;
                const float le = from_right(PX[p], j, lane) + shU;
                float vM = me + t[T_MC];
                float vX = me + t[T_MFGX];
                float vY = me + t[T_MFGY];
                vM = lae(tab, vM, ue + t[T_OY]);
                vY = lae(tab, vY, ue + t[T_EY]);
                vM = lae(tab, vM, le + t[T_OX]);
                vX = lae(tab, vX, le + t[T_EX]);
                if (has_sx) vY = lae(tab, vY, le + t[T_SX]);
                bM[j] = vM + mk[j];
                bX[j] = vX + mk[j];
                bY[j] = vY + mk[j];
            }
        }
        // this row's warp maximum for the base of d-2 (D's maximum is known exactly)
        const float lmx = fp32::warp_max1(lane_max(bM, bX, bY));
        // emissions of d (for the successor sums of d-1 and d-2)
        float eM[kCpl], eY[kCpl], eX[kCpl];
        cell_emissions<kStored, P, 1>(e, erow[P], gx_stored, eM, eY, eX);
        const double fb = fbq[c];
        const float fsh = fsq[c];
        float fM[kCpl];
        unpack(fq[c], fM);
        prefetch_f<p>(d - 1);
        if (d <= from) {
            if (m0.flags & kFlagRefresh) refresh(d, first, bM, bX, bY, fM, fb, fsh, gamma0);
            posteriors(d, bM, fM, fb);
        }
        // sums for the predecessors, and the row's facts for d-1's refresh
#pragma unroll
        for (int j = 0; j < kCpl; ++j) {
            PM[c][j] = bM[j] + eM[j];
            PX[c][j] = bX[j] + eX[j];
            PY[c][j] = bY[j] + eY[j];
            BM1[j] = bM[j];
            EM1[j] = eM[j];
        }
        if (!kStored) {
            // cell 3 of d-1 takes the register cell 0 of d used; the one of d-2 is requested
            e.ev[P & 3] = e.pre[(P + 1) & 1];
            e.pre[P & 1] = load_event(A, R, d - 2 - xb - 4 * lane - 3);
        }
        mx[c] = first ? kNInf : lmx;   // D's own maximum is mxD
        gamma1 = gamma0;
    }

    // diagonalCalculationTotalProbability (pairwiseAligner.c:1182-1200): F.B on d in ascending cell
    // order, then the matches from d-1 over d into d+1 dotted with B(d+1), folded in the reference's
    // sequential order
    __device__ __forceinline__ void refresh(int32_t d, bool first, const float (&bM)[kCpl], const float (&bX)[kCpl],
                                            const float (&bY)[kCpl], const float (&fM)[kCpl], double fb, float fsh,
                                            float gamma0) {
        float fm[kCpl], fx[kCpl], fy[kCpl];
        load_frow(d, fm, fx, fy);
        float c0[kCpl], c1[kCpl];
#pragma unroll
        for (int j = 0; j < kCpl; ++j) {
            float v = fM[j] + bM[j];
            v = lae(tab, v, fx[j] + bX[j]);
            c0[j] = lae(tab, v, fy[j] + bY[j]);
        }
        const int32_t xL = (d + m0.L) >> 1;
        int32_t n1 = 0, xL1 = xL;
        if (!first) {
            // cells of d+1 through their match predecessors on d-1 (slot q-1)
            float gm[kCpl], gx[kCpl], gy[kCpl];
            if (d - 1 >= 0) {
                load_frow(d - 1, gm, gx, gy);
            } else {
#pragma unroll
                for (int j = 0; j < kCpl; ++j) gm[j] = gx[j] = gy[j] = kNInf;
            }
            float mk1[kCpl];
            band_mask(d + 1, MetaW{mp.L, mp.W, 0, xb, 0}, lane, mk1);
#pragma unroll
            for (int j = 0; j < kCpl; ++j) {
                const float tm = from_left(gm, j, lane), tx = from_left(gx, j, lane), ty = from_left(gy, j, lane);
                const float te = EM1[j];
                float mth = tm + (te + t[T_MC]);
                mth = lae(tab, mth, tx + (te + t[T_MFGX]));
                mth = lae(tab, mth, ty + (te + t[T_MFGY]));
                c1[j] = (mth + BM1[j]) + mk1[j];
            }
            n1 = mp.W;
            xL1 = (d + 1 + mp.L) >> 1;
        }
        float *ca = chain, *cb = chain + kSlots;
        reinterpret_cast<float4 *>(ca)[lane] = make_float4(c0[0], c0[1], c0[2], c0[3]);
        if (!first) reinterpret_cast<float4 *>(cb)[lane] = make_float4(c1[0], c1[1], c1[2], c1[3]);
        __syncwarp();
        const float2 ff = fp32::ordered_fold2(tab, ca + (xL - xb), m0.W, cb + (xL1 - xb), n1);
        // the through-part is relative to base_F(d-1) + base_B(d+1)
        const float ptil = lae(tab, ff.x, ff.y - fsh - gamma0);
        pref = (double) ptil + fb + bbase;
        if (d == n) ll = pref;
        __syncwarp();
    }

    // posterior match probabilities of d (diagonalCalculationPosteriorMatchProbs,
    // pairwiseAligner.c:1202-1253), emitted in ascending cell order
    __device__ __forceinline__ void posteriors(int32_t d, const float (&bM)[kCpl], const float (&fM)[kCpl], double fb) {
        const float kd = (float) (fb + bbase - pref);
        float pv[kCpl];
        unsigned hits = 0;
        const int32_t xL = (d + m0.L) >> 1;
        const int32_t lo = xL - xb - 4 * lane;
#pragma unroll
        for (int j = 0; j < kCpl; ++j) {
            const int32_t x = xb + 4 * lane + j, y = d - x;
            pv[j] = __expf(fM[j] + bM[j] + kd);
            const bool hit = (unsigned) (j - lo) < (unsigned) m0.W && x > 0 && y > 0 && pv[j] >= A.threshold;
            hits |= (unsigned) hit << j;
        }
        const unsigned below = (1u << lane) - 1u;
        int32_t before = 0, total = 0;
#pragma unroll
        for (int j = 0; j < kCpl; ++j) {
            const unsigned b = __ballot_sync(0xffffffffu, (hits >> j) & 1u);
            before += __popc(b & below);
            total += __popc(b);
        }
        if (hits) {
            int32_t k = 0;
#pragma unroll
            for (int j = 0; j < kCpl; ++j) {
                if (!((hits >> j) & 1u)) continue;
                const int64_t slot = n_out + before + k;
                ++k;
                if (slot < wt.out_cap) {
                    const int32_t x = xb + 4 * lane + j, y = d - x;
                    sa_aligned_pair o;
                    o.score = (int64_t) floor((double) fminf(pv[j], 1.0f) * 10000000.0);
                    o.x = R.x1 + x - 1;
                    o.y = R.y1 + y - 1;
                    o.kmer = e.kid[j];
                    A.out[wt.out_base + slot] = o;
                } else {
                    atomicMax(A.status + R.read, (int32_t) SA_E_OUTPUT);
                }
            }
        }
        n_out += total;
    }

    __device__ __forceinline__ void run(int64_t gw) {
        lane = threadIdx.x & 31;
        wt = A.wtask[gw];
        R = A.regions[wt.region];
        M = A.models + R.model;
        rs = A.read_scale[R.read];
#pragma unroll
        for (int i = 0; i < 9; ++i) t[i] = M->t[i];
        has_sx = M->has_sx != 0;
        gx_stored = (float) kLogPointOne;
        n = R.n;
        db = R.diag_base;
        rmask = R.ring_rows - 1;
        ring = A.F + R.ring_base;
        const Window Wn = A.windows[gw];
        D = Wn.D;
        T = Wn.T;
        from = Wn.from;
        // end-state values on D (stateMachine.c:1034-1061)
        const bool ragged_end = Wn.at_end && R.ragged_right;
        e0 = ragged_end ? (t[T_OX] + t[T_OY]) / 2.0f : t[T_MC];
        e1 = ragged_end ? t[T_EX] : t[T_MFGX];
        e2 = ragged_end ? t[T_EY] : t[T_MFGY];
        mxD = fmaxf(e0, fmaxf(e1, e2));
        if (!(mxD > kNInf)) mxD = 0.0f;
        m0 = decode(raw_meta(D + 1));   // becomes mp of D (unused there)
        xb = decode(raw_meta(D)).xb;
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int j = 0; j < kCpl; ++j) PM[q][j] = PX[q][j] = PY[q][j] = kNInf;
#pragma unroll
        for (int j = 0; j < kCpl; ++j) BM1[j] = EM1[j] = kNInf;
        load_slot_consts(A, R, *M, rs, xb, lane, e, !kStored);
#pragma unroll
        for (int q = 0; q < 4; ++q) mq[q] = raw_meta(D - q);
        if (!kStored) {
            // phase 0 at D: cell j's event in register j; cell 3 of D-1 in pre[1]
#pragma unroll
            for (int j = 0; j < kCpl; ++j) e.ev[j] = load_event(A, R, D - xb - 4 * lane - j);
            e.pre[1] = load_event(A, R, D - 1 - xb - 4 * lane - 3);
            e.pre[0] = e.pre[1];
        } else {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (D - q > T) {
                    MetaW mm = decode(mq[q]);
                    mm.xb = xb;
                    erow[q] = load_erow(A, R, D - q, mm, lane);
                }
            }
        }
        prefetch_f<0>(D);
        mx[0] = mx[1] = kNInf;
        gamma1 = 0.0f;
        bbase = pref = ll = 0.0;
        n_out = 0;
        for (int32_t d = D; d > T; d -= 4) {
            step<0>(d);
            if (d - 1 <= T) break;
            step<1>(d - 1);
            if (d - 2 <= T) break;
            step<2>(d - 2);
            if (d - 3 <= T) break;
            step<3>(d - 3);
        }
        if (lane == 0) {
            A.wcount[gw] = n_out;
            if (Wn.at_end) A.loglik[wt.region] = ll;
        }
        __syncwarp();
    }
};

template <bool kStored>
__device__ __noinline__ void window_task(const WArgs &A, int64_t gw, const float4 *tab, float *chain) {
    Backward<kStored> b(A, tab, chain);
    b.run(gw);
}

template <bool kStored>
__device__ __noinline__ void forward_task(const WArgs &A, int32_t region, const float4 *tab) {
    Forward<kStored> f(A, tab);
    f.run(region);
}

// window gw claimed by this warp: run it and mark it done (after all its reads of the ring)
__device__ __noinline__ void run_window(const WArgs &A, int64_t gw, const float4 *tab, float *chain) {
    const int32_t region = A.wtask[gw].region;
    if (A.regions[region].stored) window_task<true>(A, gw, tab, chain);
    else window_task<false>(A, gw, tab, chain);
    __syncwarp();
    __threadfence();
    if ((threadIdx.x & 31) == 0) atomicExch(A.wflag + gw, 2);
    __syncwarp();
}

// ------------------------------------------------------------------------------------------------
// the persistent worker: forward sweeps first (largest band first), then windows
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(32 * kWarps) warp_worker(const __grid_constant__ WArgs A) {
    __shared__ float4 tab[16];
    __shared__ __align__(16) float chain[kWarps][2 * kSlots];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < 16) fp32::log_add_piece(threadIdx.x, tab[threadIdx.x]);
    __syncthreads();
    float *ch = chain[warp];
    // the last eighth of the grid's warps serve only the ready queue
    const int64_t gwarp = (int64_t) blockIdx.x * kWarps + warp, nwarps = (int64_t) gridDim.x * kWarps;
    const int64_t reserve = nwarps / 8 > 1 ? nwarps / 8 : 1;
    const bool may_forward = gwarp < nwarps - reserve || nwarps == 1;
    while (may_forward) {
        int32_t id = -1;
        if (lane == 0) {
            const unsigned claim = atomicAdd(&A.ctl->claim, 1u);
            id = claim < (unsigned) A.n_regions ? A.order[claim] : -1;
        }
        id = __shfl_sync(0xffffffffu, id, 0);
        if (id < 0) break;
        if (*((volatile int32_t *) &A.ctl->error)) continue;   // claim the rest, run nothing
        if (A.regions[id].stored) forward_task<true>(A, id, tab);
        else forward_task<false>(A, id, tab);
    }
    for (;;) {
        int32_t id = -1;
        if (lane == 0) {
            const unsigned claim = atomicAdd(&A.ctl->wclaim, 1u);
            if ((int64_t) claim < A.n_windows) id = wait_ready(A, claim);
        }
        id = __shfl_sync(0xffffffffu, id, 0);
        if (id < 0) break;
        run_window(A, id, tab, ch);
    }
}

// ------------------------------------------------------------------------------------------------
// per-event FP32 records: {mean / var, noise, -1.5 log noise, 1 / noise}, per region with its read's
// variance (Gaussian regions)
// ------------------------------------------------------------------------------------------------
__global__ void prep_events_w(const __grid_constant__ WArgs A) {
    for (int64_t r = blockIdx.x; r < A.n_regions; r += gridDim.x) {
        const WRegion R = A.regions[r];
        if (R.stored) continue;
        const float inv_var = A.read_scale[R.read].inv_var;
        for (int32_t y = threadIdx.x; y < R.lY; y += blockDim.x) {
            const double2 v = A.events_raw[R.event_base + y];
            float4 o;
            o.x = (float) v.x * inv_var;
            o.y = (float) v.y;
            o.z = (float) (-1.5 * log(v.y));
            o.w = (float) (1.0 / v.y);
            A.events[R.event_base + y] = o;
        }
    }
}

// ------------------------------------------------------------------------------------------------
// emission rows of stored-emission (HDP) regions: per anti-diagonal the slots [xa, xa + len) with
// xa the band's first column rounded down to a multiple of 4; -inf outside the band, at x = 0 and
// at y = 0 (the reference's NULL k-mer / event)
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) emission_rows_kernel(const __grid_constant__ WArgs A) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t) gridDim.x * (blockDim.x >> 5);
    for (int64_t ch = blockIdx.x * (int64_t) (blockDim.x >> 5) + (threadIdx.x >> 5); ch < A.n_echunks; ch += warps) {
        const fp32::Chunk C = A.echunks[ch];
        const WRegion R = A.regions[C.region];
        const WModel &M = A.models[R.model];
        const fp32::ReadScale64 rs = A.read_scale64[R.read];
        for (int k = 0; k < C.nd; ++k) {
            const int32_t d = C.d0 + k;
            const MetaW m = decode(__ldg(A.meta + R.diag_base + d));
            const int32_t xL = (d + m.L) >> 1, xR = xL + m.W - 1;
            const int32_t xa = xL & ~3, len = ((xR - xa + 1) + 3) & ~3;
            float *row = A.E + R.e_base + m.eoff;
            for (int32_t i = lane; i < len; i += 32) {
                const int32_t x = xa + i, y = d - x;
                float v = kNInf;
                if (x >= xL && x <= xR && x >= 1 && y >= 1 && x <= R.lX && y <= R.lY) {
                    const int32_t kid = __ldg(A.kmer + R.kmer_base + x - 1);
                    v = fp32::emit_hdp64(M.hdp64, kid, __ldg(A.events_raw + R.event_base + y - 1).x, rs);
                }
                row[i] = v;
            }
        }
    }
}

}  // namespace wk
}  // namespace sa
