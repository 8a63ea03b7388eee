// Batched FP32 kernels: all regions of a batch in three launches.
//
//   1. emission_kernel: the match and extra-event emissions of every band cell, written to the
//      emission store.  Fully parallel (a warp per run of 32 anti-diagonals); it takes the
//      Gaussian / HDP density work off the sequential sweeps.
//   2. worker_kernel: persistent CTAs of 128 threads pull tasks from one device counter.  The first
//      claims are forward segments (longest first); every later claim is a slot of a ready queue of
//      traceback windows.  A forward segment sweeps a run of a region's anti-diagonals (the whole
//      region, or a piece of a long one; see Segment) anti-diagonal by anti-diagonal (cells spread
//      over the threads, neighbours through a 3-slot shared-memory ring, one barrier per
//      anti-diagonal), stores the forward match values (and, on the anti-diagonals a
//      total-probability refresh reads, the gap states) to HBM, and publishes each traceback window
//      of getPosteriorProbsWithBanding (pairwiseAligner.c:1319-1333) to the ready queue as soon as it
//      has passed the last anti-diagonal whose forward values the window reads.  A window task runs
//      that window's backward sweep in its own ring with the posterior test and the reference's
//      total-probability refreshes fused in, and writes its pairs to the window's output segment.
//      Windows of one region are independent given the forward store, so the backward work of a
//      long read spreads over many CTAs while its forward sweep is still running.
//   3. gather_pairs: per read, the windows' segments concatenated in order (regions, then windows:
//      the reference's emission order) into one packed buffer.
//
// A window slot is claimed only after every forward segment has been claimed, and forward segments
// never wait (a stitch is checked by whichever of its two segments finishes second), so every wait
// on the ready queue ends once the forward sweeps progress; the wait is bounded anyway
// (SA_E_TIMEOUT).
//
// The recursion is bound by instruction issue and latency, so the inner loops are branch-free: the
// rings carry a -inf cell on each side and every slot beyond the anti-diagonal's width holds -inf,
// so an absent neighbour is a clamped index that reads -inf (logAdd and the sums then behave
// exactly like the reference's skipped transitions).  Per-anti-diagonal facts (band start, width,
// window end, refresh, which forward values to store) come packed from the host.  Loads that do not
// depend on the recursion are issued two anti-diagonals ahead from clamped (always valid) addresses
// and masked where they are consumed.
//
// Values are log probabilities relative to a per-anti-diagonal FP64 base.  The forward base of d is
// the base of d-3 plus the largest value computed on d-3, the backward base of d the base of d+2
// plus the largest value on d+2 (lagged renormalisations, so the max reductions are off the
// critical path); the recorded bases are built from the same float shifts the kernel applies, so
// they describe the stored values exactly.
//
// Stores, per anti-diagonal d with first cell c (region relative) and width W:
//   emission store at 2c: [ match emission | extra-event emission ], W floats each;
//   forward store at 3c:  [ match | gap-X | gap-Y ], W floats each; the gap states only where a
//   refresh reads them.
#pragma once

namespace sa {
namespace fp32 {

using namespace dp32;

constexpr int kThreads = 128;                  // one CTA = one worker
constexpr int kWarps = kThreads / 32;
constexpr int kMaxCpt = 4;                     // cells per thread: bands up to 512 cells wide
constexpr int kChunkDiags = 32;                // anti-diagonals per emission-kernel chunk
enum { ST_M = 0, ST_X = 1, ST_Y = 2 };         // forward store blocks
enum { SE_M = 0, SE_Y = 1 };                   // emission store blocks

// per-anti-diagonal meta: x = xmy of the first cell, y = width | flags
constexpr int32_t kWidthMask = (1 << 20) - 1;
constexpr int32_t kFlagWindowEnd = 1 << 20;   // a traceback window closes here
constexpr int32_t kFlagStoreGaps = 1 << 21;   // a refresh reads this anti-diagonal's gap states
constexpr int32_t kFlagRefresh = 1 << 22;     // total-probability refresh in its posterior window

enum { T_MC = 0, T_MFGX, T_MFGY, T_OX, T_OY, T_EX, T_EY, T_SX, T_SY };

// FP64 HDP tables of a model (the emission kernel evaluates HDP densities in FP64: they reach far
// below the FP32 range in the tails, and the spline's terms cancel there)
struct Hdp64 {
    const double *match;      // n_kmers x 5 (level mean in column 0)
    const double *grid;       // grid_length knots
    const double *density;    // rows x grid_length
    const double *slope;      // rows x grid_length
    const int64_t *kmer_row;  // n_kmers
    int64_t grid_length;
};

struct ModelDesc {
    const KmerConst32 *kc;
    Hdp64 hdp64;
    int32_t emission;
    int32_t gapx_uniform;   // every k-mer's skip emission is gapx_value (log 0.1 in .model machines)
    float t[9];
    float gapx_value;
};

// per-read FP64 descaling parameters (HDP emissions)
struct ReadScale64 {
    double scale, shift, var, pad;
};

struct RegionDesc {
    int32_t n, lX, lY, read;
    int32_t n_windows, model;
    int32_t ragged_left, ragged_right;
    int64_t diag_base;    // first anti-diagonal of this region in the per-anti-diagonal arrays
    int64_t cell_base;    // first cell of this region in the stores
    int64_t win_base;     // first window of this region in the per-window arrays
    int64_t kmer_base;    // k-mer id of column x >= 1 is kmer[kmer_base + x - 1]
    int64_t event_base;   // event of row y >= 1 is events[event_base + y - 1]
    int64_t x1, y1;
};

// one traceback window as a task
struct WindowTask {
    int32_t region;
    int32_t first_cell;   // region-relative first cell of its traceback anti-diagonal D
    int32_t out_cap;      // pair slots of its output segment
    int32_t side;         // T starts a forward segment: the stitch whose copy of T it reads, else -1
    int64_t out_base;     // first pair slot of its output segment
};

// One forward segment: a run of a region's anti-diagonals swept by one CTA.  A region's forward
// sweep is cut at traceback-window starts into segments that run at the same time on different
// CTAs.  Every segment after the first starts `warm` anti-diagonals before its first owned one
// from a flat vector (every band cell 0 in every state).  The recursion commutes with adding a
// constant to every value (logAdd(x + c, y + c) = logAdd(x, y) + c, pairwiseAligner.c:234-254), and
// the influence of the start vector dies out: within a few hundred anti-diagonals the segment's
// values are the true ones minus one constant, and the stitch where two segments meet checks that
// on both anti-diagonals the recursion carries over (b-1 and b).  Posteriors are unaffected by the
// constant: a window's total probability comes from its own forward values, so it cancels.
struct Segment {
    int32_t region;
    int32_t d_begin;      // owned anti-diagonals: (d_begin, d_end]; the first segment also owns 0
    int32_t d_end;
    int32_t warm;         // anti-diagonals swept before d_begin (0 for a region's first segment)
    int32_t wi0;          // region-relative index of the first window it publishes
    int32_t stitch_in;    // stitch at d_begin (-1: first segment)
    int32_t stitch_out;   // stitch at d_end (-1: last segment)
    int32_t pad;
    int64_t cell0;        // region-relative first cell of the first anti-diagonal it computes
};

// where two segments meet, at anti-diagonal b: values of b-1 and b from both sides
struct StitchDesc {
    int32_t region, read;
    int32_t w0, w1;       // widths of b-1 and b
    int64_t voff;         // first float of [later segment: b-1, b | earlier segment: b-1, b], M|X|Y each
};

// result of a stitch (cleared before every run)
struct StitchRes {
    double sbase[2];      // FP64 bases of b-1, b in the later segment's sweep
    double tbase[2];      // and in the earlier segment's
    double delta;         // earlier-segment value - later-segment value (the constant)
    float spread;         // largest deviation from the constant, over the cells (diagnostic)
    int32_t arrive;       // sides that have written their values
    int32_t result;       // 0 pending, 1 agreed, 2 disagreed
    int32_t pad;
};
constexpr int kStitchAgreed = 1, kStitchDisagreed = 2;

// a run of up to kChunkDiags anti-diagonals of one region (emission kernel)
struct Chunk {
    int32_t region;
    int32_t d0;
    int32_t nd;
    int32_t pad;
    int64_t cell;         // batch-absolute first cell of anti-diagonal d0
};

// device counters, cleared before every launch
struct Control {
    unsigned int claim;   // next forward-sweep claim
    unsigned int wclaim;  // next ready-queue slot claim
    unsigned int pub;     // next ready-queue slot to publish into
    int32_t error;        // a bounded wait gave up
    unsigned long long packed;   // pairs in the packed output
};

// per-warp window area (floats) when windows run one per warp: ring, refresh chain (2 rows) and
// the staged operands of the next refresh (6 rows)
constexpr int kWarpWindowCpt = 4;
constexpr int kWarpWindowWidth = 32 * kWarpWindowCpt;
constexpr int kWarpWindowFloats = 9 * (kWarpWindowWidth + 2) + 8 * kWarpWindowWidth;

// dynamic shared memory of the worker after the Shared header, in floats
__host__ __device__ constexpr int worker_area_floats(int cpt) {
    return cpt == 1 ? kWarps * kWarpWindowFloats : 9 * (cpt * kThreads + 2) + 2 * cpt * kThreads;
}

struct Args {
    const RegionDesc *regions;
    int64_t n_regions;
    const Segment *segs;
    const int32_t *order;           // forward claims: segments by length, longest first
    int64_t n_segs;
    const StitchDesc *stitch;
    StitchRes *stitch_res;
    float *stitch_vals;
    int32_t *seg_fail;              // per read: a stitch disagreed (the read is re-run unsegmented)
    float stitch_tol;               // scale of the stitch tolerance (negative: every stitch disagrees)
    int32_t use_side;               // windows at segment starts read the stitch copy of T
    const ModelDesc *models;
    const ReadScale32 *read_scale;
    const ReadScale64 *read_scale64;
    const double2 *events_raw;      // per event FP64 (mean, noise)
    const int2 *meta;               // per anti-diagonal {xmy of first cell, width | flags}
    const Window *windows;
    const WindowTask *wtask;
    int64_t n_windows;
    const Chunk *chunks;
    int64_t n_chunks;
    const int32_t *kmer;
    const float *gapx;              // per k-mer position: skip emission of that k-mer
    const Event32 *events;
    float *E;                       // emission store, 2 floats per cell
    float *F;                       // forward store, 3 floats per cell
    double *base;                   // per anti-diagonal FP64 base of the forward store
    float *fshift;                  // per anti-diagonal base(d) - base(d-1)
    int32_t *ready;                 // ready queue of windows (-1: not yet published)
    sa_aligned_pair *out;           // per-window output segments
    int64_t *wcount;                // per window: pairs written (may exceed its capacity)
    double *loglik;                 // per region: total probability at its last anti-diagonal
    int32_t *status;                // per read
    Control *ctl;
    float threshold;
    int32_t wmax;                   // ring width (cells); rings hold wmax + 2 floats per state
    int32_t warp_windows;           // bands up to 128 cells: a window per warp (else per CTA)
    long long spin_limit;           // clock cycles a worker may wait for a window
    // gather
    int64_t n_reads;
    const int64_t *read_win;        // per read: first window, window count, first region, region
                                    // count, first stitch, stitch count, units (windows + stitches), 0
    sa_aligned_pair *packed;
    int64_t *read_base;             // per read: first pair in the packed output
    int64_t *read_count;
    // per-read completion (null: the gather launch packs every read after the worker)
    int32_t *read_wdone;            // per read: windows finished
    ReadDone *done_host;            // per read: record in mapped host memory
    int32_t done_seq;               // this run's number, written to a record's `done`
};

struct Shared {
    float4 la[16];                  // logAdd cubic pieces by ceil(2 d)
    float part[3][kWarps];          // per-warp maxima of the last anti-diagonals
    int32_t wcnt[2][kMaxCpt][kWarps];
    float fold[2];
    int32_t task_id;
    int32_t done_read;
    long long red[kWarps + 1];
    double cmp[3][kWarps];          // stitch check: per-warp largest value, its difference, spread
};

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
// when the smaller argument is -inf: the difference is inf, or NaN if both are -inf).
// The table index ceil(2 d) comes from one add rounded toward +inf: 2 d + 2^23 lands on the
// integer 2^23 + ceil(2 d) for 0 <= 2 d <= 15, whose low four bits are the index; beyond the
// cut-off (or for inf / NaN) the low bits are some index in 0..15 whose value is discarded.
__device__ __forceinline__ float lae(const float4 *tab, float x, float y) {
    const float mx = fmaxf(x, y), d = fabsf(x - y);
    const int k = __float_as_int(__fmaf_ru(d, 2.0f, 8388608.0f)) & 15;
    const float4 c = tab[k];
    const float h = fmaf(fmaf(fmaf(c.x, d, c.y), d, c.z), d, c.w);
    return d < 7.5f ? mx + h : mx;
}

// warp-wide maximum in one instruction
__device__ __forceinline__ float warp_max1(float v) {
    float r;
    asm volatile("redux.sync.max.f32 %0, %1, 0xffffffff;" : "=f"(r) : "f"(v));
    return r;
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
//  * Values before the first one within kSeedGap of the overall maximum M enter as one exact
//    log-sum-exp seed: the final result depends on the running result at that point with weight
//    at most exp(-(kSeedGap - 0.7)) < 1e-6, so the reference's approximation error there (< 1e-3)
//    cannot reach the final total.
//  * From there on the running result r never falls below the running maximum, which is at least
//    M - kSeedGap, and logAdd(r, v) is exactly r once r - v >= 7.5.  So a value at or below
//    M - kSeedGap - 7.6 leaves the result unchanged: only the values above that bound are folded,
//    in index order (compacted into consecutive lanes first).  Folding a few that would also have
//    left r unchanged costs a step but changes nothing, so no running maximum is needed to pick them.
constexpr float kSeedGap = 15.0f;
constexpr float kFoldGap = kSeedGap + 7.6f;

// lane-compacted values of vals[q .. q+32) above `lo` with index >= start, and their count
__device__ __forceinline__ int fold_candidates(const float *vals, int q, int start, int n, float lo, float &packed) {
    const int lane = threadIdx.x & 31;
    const float v = q + lane < n ? vals[q + lane] : kNegInf;
    const unsigned mask = __ballot_sync(0xffffffffu, q + lane >= start && v > lo);
    const int nc = __popc(mask);
    if (nc == 0) return 0;
    const unsigned src = lane < nc ? __fns(mask, 0, lane + 1) : 0u;
    packed = __shfl_sync(0xffffffffu, v, (int) (src & 31u));
    return nc;
}

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
    float seed = 0.0f;
    for (int b = 0; b < start; b += 32) {
        const float v = b + lane < start ? vals[b + lane] : kNegInf;
        seed += v > kNegInf ? __expf(v - mall) : 0.0f;
    }
    seed = warp_sum(seed);
    float r = seed > 0.0f ? mall + __logf(seed) : kNegInf;
    for (int b = start & ~31; b < n; b += 32) {
        float packed = kNegInf;
        const int nc = fold_candidates(vals, b, start, n, mall - kFoldGap, packed);
        for (int k = 0; k < nc; ++k) r = lae(tab, r, __shfl_sync(0xffffffffu, packed, k));
    }
    return r;
}

// Two independent ordered folds (ordered_fold on a[0..na) and on b[0..nb)) run by one warp with
// their sequential logAdd chains interleaved.
__device__ __forceinline__ float2 ordered_fold2(const float4 *tab, const float *a, int na, const float *b, int nb) {
    const int lane = threadIdx.x & 31;
    float ma = kNegInf, mb = kNegInf;
    for (int q = 0; q < max(na, nb); q += 32) {
        ma = fmaxf(ma, q + lane < na ? a[q + lane] : kNegInf);
        mb = fmaxf(mb, q + lane < nb ? b[q + lane] : kNegInf);
    }
    ma = warp_max(ma);
    mb = warp_max(mb);
    // first index within kSeedGap of each maximum
    int sa = na, sb = nb;
    for (int q = 0; q < na; q += 32) {
        const unsigned m = __ballot_sync(0xffffffffu, q + lane < na && a[q + lane] >= ma - kSeedGap);
        if (m) { sa = q + __ffs(m) - 1; break; }
    }
    for (int q = 0; q < nb; q += 32) {
        const unsigned m = __ballot_sync(0xffffffffu, q + lane < nb && b[q + lane] >= mb - kSeedGap);
        if (m) { sb = q + __ffs(m) - 1; break; }
    }
    float seed_a = 0.0f, seed_b = 0.0f;
    for (int q = 0; q < max(sa, sb); q += 32) {
        const float va = q + lane < sa ? a[q + lane] : kNegInf;
        const float vb = q + lane < sb ? b[q + lane] : kNegInf;
        seed_a += va > kNegInf ? __expf(va - ma) : 0.0f;
        seed_b += vb > kNegInf ? __expf(vb - mb) : 0.0f;
    }
    seed_a = warp_sum(seed_a);
    seed_b = warp_sum(seed_b);
    float ra = ma > kNegInf && seed_a > 0.0f ? ma + __logf(seed_a) : kNegInf;
    float rb = mb > kNegInf && seed_b > 0.0f ? mb + __logf(seed_b) : kNegInf;
    const int ea = ma > kNegInf ? na : 0, eb = mb > kNegInf ? nb : 0;
    // chunk by chunk: candidates compacted, then both sequential chains side by side
    for (int ca = sa & ~31, cb = sb & ~31; ca < ea || cb < eb; ca += 32, cb += 32) {
        float pa = kNegInf, pb = kNegInf;
        const int nca = ca < ea ? fold_candidates(a, ca, sa, ea, ma - kFoldGap, pa) : 0;
        const int ncb = cb < eb ? fold_candidates(b, cb, sb, eb, mb - kFoldGap, pb) : 0;
        for (int k = 0; k < max(nca, ncb); ++k) {
            const float xa = __shfl_sync(0xffffffffu, pa, k), xb = __shfl_sync(0xffffffffu, pb, k);
            if (k < nca) ra = lae(tab, ra, xa);
            if (k < ncb) rb = lae(tab, rb, xb);
        }
    }
    return make_float2(ra, rb);
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
    bool gx_uniform;   // the skip emission is gx for every column: no per-column load
    float gx;
};

__device__ __forceinline__ void ctx_init(Ctx &c, const Args &A, int32_t region) {
    c.A = &A;
    c.region_index = region;
    c.R = A.regions[region];
    c.M = A.models + c.R.model;
    c.rs = A.read_scale[c.R.read];
    c.hdp = c.M->emission == SA_EMIT_HDP;
    c.gx_uniform = c.M->gapx_uniform != 0;
    c.gx = c.M->gapx_value;
#pragma unroll
    for (int i = 0; i < 9; ++i) c.t[i] = c.M->t[i];
}

__device__ __forceinline__ int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return min(max(v, lo), hi); }

// Raw loads: always from a valid address (indices clamped into the region's arrays); validity is
// computed from indices alone and applied where the value is consumed.
__device__ __forceinline__ float raw_gapx(const Ctx &c, int32_t x) {
    if (c.gx_uniform) return c.gx;
    const int64_t at = c.R.lX > 0 ? c.R.kmer_base + clampi(x - 1, 0, c.R.lX - 1) : 0;
    return __ldg(c.A->gapx + at);
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

__device__ __forceinline__ void ring_init(float *base, int wmax) {
    const int total = 9 * (wmax + 2);
    for (int i = threadIdx.x; i < total; i += kThreads) base[i] = kNegInf;
}

// ------------------------------------------------------------------------------------------------
// emission kernel: match / extra-event emissions of every band cell
// ------------------------------------------------------------------------------------------------
// match / extra-event emissions of every band cell (the emission calls of stateMachine3_cellCalculate,
// stateMachine.c:1194-1257, and of its HDP form, :1259-1325); -inf without a k-mer (x = 0) or
// without an event (y = 0)
// Per warp, one chunk of anti-diagonals at a time.  The chunk's cells cover a small range of
// columns and rows (the band drifts by under one cell per anti-diagonal), so the k-mer constants of
// its columns and the events of its rows are gathered once into the warp's shared memory and every
// cell reads them from there; a chunk whose ranges exceed kEmitSpan reads global memory per cell.
constexpr int kEmitWarps = 4;
constexpr int kEmitSpan = 192;
constexpr int kEmitCols = 4;   // column slots per lane of the column-stationary Gaussian path
// The k-mer constants are staged as two float4 halves in separate arrays: lanes reading consecutive
// columns then load 16-byte strides, which shared memory serves without bank conflicts (32-byte
// records would put two lanes on every bank group).
struct EmitStage {
    float4 kca[kEmitSpan], kcb[kEmitSpan];
    float4 ev[kEmitSpan];
    double mean[kEmitSpan];     // FP64 event means (HDP)
    int32_t kid[kEmitSpan];
};

// getHdpKmerDensity (stateMachine.c:468-495): log((1/var) * max(0, spline(descaled mean))) with the
// spline of grid_spline_interp (hdp_math_utils.c:471-495), in FP64 as the reference computes it
__device__ __forceinline__ float emit_hdp64(const Hdp64 &h, int32_t kid, double mean, const ReadScale64 &rs) {
    const int64_t row = h.kmer_row[kid];
    if (row < 0) return kNegInf;
    const double mu = h.match[(int64_t) kid * 5];
    const double u = (mean + rs.var * mu - rs.scale * mu - rs.shift) / rs.var;
    const double *x = h.grid, *y = h.density + row * h.grid_length, *sl = h.slope + row * h.grid_length;
    const int64_t len = h.grid_length;
    double d;
    if (u <= x[0]) {
        d = y[0] - sl[0] * (x[0] - u);
    } else if (u >= x[len - 1]) {
        d = y[len - 1] + sl[len - 1] * (u - x[len - 1]);
    } else {
        const double dx = x[1] - x[0];
        int64_t il = (int64_t) ((u - x[0]) / dx);
        il = il > len - 2 ? len - 2 : (il < 0 ? 0 : il);
        const double dy = y[il + 1] - y[il];
        const double a = sl[il] * dx - dy, b = dy - sl[il + 1] * dx;
        const double tl = (u - x[il]) / dx, tr = 1.0 - tl;
        d = tr * y[il] + tl * y[il + 1] + tl * tr * (a * tr + b * tl);
    }
    return d > 0.0 ? (float) log((1.0 / rs.var) * d) : kNegInf;
}

__device__ __forceinline__ void emit_cell(const Ctx &c, const KmerConst32 &k, int32_t kid, const float4 &v,
                                          double mean64, bool ok, float &em, float &ey) {
    em = ey = kNegInf;
    if (!ok) return;
    if (c.hdp) {
        em = ey = emit_hdp64(c.M->hdp64, kid, mean64, c.A->read_scale64[c.R.read]);
    } else {
        const Event32 e{v.x, v.y, v.z, v.w};
        emit_gauss(k, e, c.rs, em, ey);
    }
}

__global__ void __launch_bounds__(32 * kEmitWarps) emission_kernel(const __grid_constant__ Args A) {
    __shared__ EmitStage stage[kEmitWarps];
    const int lane = threadIdx.x & 31;
    EmitStage &st = stage[threadIdx.x >> 5];
    const int64_t warps = (int64_t) gridDim.x * (blockDim.x >> 5);
    for (int64_t ch = blockIdx.x * (int64_t) (blockDim.x >> 5) + (threadIdx.x >> 5); ch < A.n_chunks; ch += warps) {
        const Chunk C = A.chunks[ch];
        Ctx c;
        ctx_init(c, A, C.region);
        const int2 mt = lane < C.nd ? __ldg(A.meta + c.R.diag_base + C.d0 + lane) : make_int2(0, 0);
        const int32_t w = mt.y & kWidthMask;
        int32_t off = w;   // inclusive prefix of the widths, then exclusive
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t t = __shfl_up_sync(0xffffffffu, off, o);
            if (lane >= o) off += t;
        }
        off -= w;
        // column and row ranges of the chunk's cells, over all its anti-diagonals
        int32_t xlo, xhi, ylo, yhi;
        {
            const int32_t dk = C.d0 + lane, Lk = mt.x, Rk = mt.x + 2 * (w - 1);
            const bool in = lane < C.nd;
            xlo = __reduce_min_sync(0xffffffffu, in ? (dk + Lk) >> 1 : INT32_MAX);
            xhi = __reduce_max_sync(0xffffffffu, in ? (dk + Rk) >> 1 : INT32_MIN);
            ylo = __reduce_min_sync(0xffffffffu, in ? (dk - Rk) >> 1 : INT32_MAX);
            yhi = __reduce_max_sync(0xffffffffu, in ? (dk - Lk) >> 1 : INT32_MIN);
        }
        const bool staged = xhi - xlo < kEmitSpan && yhi - ylo < kEmitSpan;
        const bool by_column = staged && !c.hdp && xhi - xlo < 32 * kEmitCols;
        if (by_column) {
            // Gaussian emissions, column-stationary: lane l owns columns xlo + l + 32 q and keeps their
            // k-mer constants in registers for the whole chunk, so a cell reads only its event from
            // shared memory (16 B instead of 52 B with the constants staged too); on each
            // anti-diagonal the lanes' columns are consecutive cells, so the stores coalesce
            constexpr int kCols = kEmitCols;
            const int nq = (xhi - xlo + 32) / 32;
            KmerConst32 kk[kCols];
            bool col_ok[kCols];
#pragma unroll
            for (int q = 0; q < kCols; ++q) {
                const int32_t x = xlo + lane + 32 * q;
                col_ok[q] = q < nq && x <= xhi && x >= 1 && x <= c.R.lX;
                const int32_t kid = col_ok[q] ? __ldg(A.kmer + c.R.kmer_base + x - 1) : 0;
                const float4 *kp = reinterpret_cast<const float4 *>(c.M->kc + kid);
                const float4 ka = q < nq ? __ldg(kp) : make_float4(0.f, 0.f, 0.f, 0.f);
                const float4 kb = q < nq ? __ldg(kp + 1) : make_float4(0.f, 0.f, 0.f, 0.f);
                kk[q] = KmerConst32{ka.x, ka.y, ka.z, ka.w, kb.x, kb.y, kb.z, kb.w};
            }
            for (int q = lane; q <= yhi - ylo; q += 32) {
                const int32_t yc = clampi(ylo + q - 1, 0, max(c.R.lY - 1, 0));
                st.ev[q] = __ldg(reinterpret_cast<const float4 *>(A.events + c.R.event_base + yc));
            }
            __syncwarp();
            for (int k = 0; k < C.nd; ++k) {
                const int32_t d = C.d0 + k;
                const int32_t L = __shfl_sync(0xffffffffu, mt.x, k);
                const int32_t W = __shfl_sync(0xffffffffu, w, k);
                float *Ed = A.E + 2 * (C.cell + __shfl_sync(0xffffffffu, off, k));
                const int32_t xfirst = (d + L) >> 1;   // column of the anti-diagonal's cell 0
#pragma unroll
                for (int q = 0; q < kCols; ++q) {
                    if (q >= nq) break;
                    const int32_t x = xlo + lane + 32 * q, i = x - xfirst, y = d - x;
                    if (i < 0 || i >= W) continue;
                    float em = kNegInf, ey = kNegInf;
                    if (col_ok[q] && y >= 1 && y <= c.R.lY) {
                        const float4 v = st.ev[y - ylo];
                        emit_gauss(kk[q], Event32{v.x, v.y, v.z, v.w}, c.rs, em, ey);
                    }
                    Ed[SE_M * W + i] = em;
                    Ed[SE_Y * W + i] = ey;
                }
            }
        } else if (staged) {
            for (int q = lane; q <= xhi - xlo; q += 32) {
                const int32_t x = xlo + q;
                const bool ok = x >= 1 && x <= c.R.lX;
                const int32_t kid = ok ? __ldg(A.kmer + c.R.kmer_base + x - 1) : 0;
                const float4 *kp = reinterpret_cast<const float4 *>(c.M->kc + kid);
                const float4 ka = __ldg(kp), kb = __ldg(kp + 1);
                st.kca[q] = ka;
                st.kcb[q] = kb;
                st.kid[q] = kid;
            }
            for (int q = lane; q <= yhi - ylo; q += 32) {
                const int32_t y = ylo + q;
                const int32_t yc = clampi(y - 1, 0, max(c.R.lY - 1, 0));
                st.ev[q] = __ldg(reinterpret_cast<const float4 *>(A.events + c.R.event_base + yc));
                if (c.hdp) st.mean[q] = __ldg(A.events_raw + c.R.event_base + yc).x;
            }
            __syncwarp();
        }
        // every other chunk (HDP emissions, or a chunk spanning more than 128 columns or the stage's
        // rows): a lane per cell of each anti-diagonal
        for (int k = 0; k < (by_column ? 0 : C.nd); ++k) {
            const int32_t d = C.d0 + k;
            const int32_t L = __shfl_sync(0xffffffffu, mt.x, k);
            const int32_t W = __shfl_sync(0xffffffffu, w, k);
            float *Ed = A.E + 2 * (C.cell + __shfl_sync(0xffffffffu, off, k));
            for (int i = lane; i < W; i += 32) {
                const int32_t xmy = L + 2 * i, x = (d + xmy) >> 1, y = (d - xmy) >> 1;
                const bool ok = x >= 1 && x <= c.R.lX && y >= 1 && y <= c.R.lY;
                float em, ey;
                if (staged) {
                    const float4 ka = st.kca[x - xlo], kb = st.kcb[x - xlo];
                    const KmerConst32 kk{ka.x, ka.y, ka.z, ka.w, kb.x, kb.y, kb.z, kb.w};
                    emit_cell(c, kk, st.kid[x - xlo], st.ev[y - ylo], c.hdp ? st.mean[y - ylo] : 0.0, ok,
                              em, ey);
                } else {
                    const int32_t kid = ok ? __ldg(A.kmer + c.R.kmer_base + x - 1) : 0;
                    const float4 *kp = reinterpret_cast<const float4 *>(c.M->kc + kid);
                    const float4 ka = __ldg(kp), kb = __ldg(kp + 1);
                    const KmerConst32 kk{ka.x, ka.y, ka.z, ka.w, kb.x, kb.y, kb.z, kb.w};
                    const int32_t yc = clampi(y - 1, 0, max(c.R.lY - 1, 0));
                    const float4 v = __ldg(reinterpret_cast<const float4 *>(A.events + c.R.event_base + yc));
                    emit_cell(c, kk, kid, v, c.hdp ? __ldg(A.events_raw + c.R.event_base + yc).x : 0.0, ok, em, ey);
                }
                Ed[SE_M * W + i] = em;
                Ed[SE_Y * W + i] = ey;
            }
        }
        __syncwarp();   // the stage is rewritten by the warp's next chunk
    }
}

// ------------------------------------------------------------------------------------------------
// forward sweep of one region
// ------------------------------------------------------------------------------------------------
// The sweep is unrolled by three anti-diagonals: ring slots, shared maxima and the look-ahead
// registers are indexed by d mod 3 at compile time, so nothing rotates and every look-ahead load
// has three anti-diagonals to land.
// kSX: the machine's SWITCH_TO_X transition is finite.  A .model file leaves it at LOG_ZERO
// (stateMachine3_loadTransitionsFromFile stores gap-Y -> gap-X in SWITCH_TO_Y, stateMachine.c:1139),
// and logAdd(v, LOG_ZERO) is v exactly, so without it the gap-X state of the forward sweep and the
// gap-Y state of the backward sweep take one logAdd less (the same values, bit for bit).
template <int NT>
__device__ void read_unit_done(const Args &A, int32_t r, int tid, Shared *sh);

// Checks stitch si once both segments have written their values of b-1 and b (whole CTA).  With
// a_i the earlier segment's FP64 value of a cell and s_i the later one's, the stitch agrees when
// both have the same -inf cells and every a_i - s_i lies within 2e-5 + 1e-6 (a_max - a_i) of the
// difference at the largest a_i (FP32 rounding of each sweep's values is a few ulp of their
// magnitude below the anti-diagonal's maximum).  The difference at the largest value becomes the
// stitch's constant; a disagreement marks the read for an unsegmented re-run.
__device__ __forceinline__ void stitch_check(const Args &A, Shared *sh, int32_t si) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const StitchDesc sd = A.stitch[si];
    StitchRes &res = A.stitch_res[si];
    const double sb0 = __ldcg(&res.sbase[0]), sb1 = __ldcg(&res.sbase[1]);
    const double tb0 = __ldcg(&res.tbase[0]), tb1 = __ldcg(&res.tbase[1]);
    const int32_t nv = 3 * (sd.w0 + sd.w1);
    const float *spec = A.stitch_vals + sd.voff, *tru = spec + nv;
    // the largest earlier-segment value and the difference there
    double amax = -INFINITY, dref = 0.0;
    for (int q = tid; q < nv; q += kThreads) {
        const bool j = q >= 3 * sd.w0;
        const float tv = __ldcg(tru + q), sv = __ldcg(spec + q);
        if (tv > kNegInf && sv > kNegInf) {
            const double a = (double) tv + (j ? tb1 : tb0);
            if (a > amax) {
                amax = a;
                dref = a - ((double) sv + (j ? sb1 : sb0));
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double a2 = __shfl_xor_sync(0xffffffffu, amax, o), d2 = __shfl_xor_sync(0xffffffffu, dref, o);
        if (a2 > amax || (a2 == amax && d2 < dref)) {
            amax = a2;
            dref = d2;
        }
    }
    if (lane == 0) {
        sh->cmp[0][warp] = amax;
        sh->cmp[1][warp] = dref;
    }
    __syncthreads();
    amax = sh->cmp[0][0];
    dref = sh->cmp[1][0];
    for (int w = 1; w < kWarps; ++w) {
        const double a2 = sh->cmp[0][w], d2 = sh->cmp[1][w];
        if (a2 > amax || (a2 == amax && d2 < dref)) {
            amax = a2;
            dref = d2;
        }
    }
    // every cell against it
    const double scale = (double) A.stitch_tol;
    bool ok = scale >= 0.0;
    double spread = 0.0;
    for (int q = tid; q < nv; q += kThreads) {
        const bool j = q >= 3 * sd.w0;
        const float tv = __ldcg(tru + q), sv = __ldcg(spec + q);
        const bool ft = tv > kNegInf, fs = sv > kNegInf;
        if (ft != fs) {
            ok = false;
        } else if (ft) {
            const double a = (double) tv + (j ? tb1 : tb0);
            const double dev = fabs((a - ((double) sv + (j ? sb1 : sb0))) - dref);
            spread = fmax(spread, dev);
            if (!(dev <= scale * (2e-5 + 1e-6 * (amax - a)))) ok = false;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) spread = fmax(spread, __shfl_xor_sync(0xffffffffu, spread, o));
    __syncthreads();   // cmp[0..1] read by every thread
    if (lane == 0) sh->cmp[2][warp] = spread;
    ok = __syncthreads_and(ok);
    if (tid == 0) {
        for (int w = 1; w < kWarps; ++w) spread = fmax(spread, sh->cmp[2][w]);
        res.delta = dref;
        res.spread = (float) spread;
        res.result = ok ? kStitchAgreed : kStitchDisagreed;
        if (!ok) atomicExch(A.seg_fail + sd.read, 1);
        __threadfence();
    }
    __syncthreads();
    read_unit_done<kThreads>(A, sd.read, tid, sh);
}

// One side of stitch si has written its values (whole CTA, after its sweep): the side that arrives
// second checks the stitch.
__device__ __forceinline__ void stitch_arrive(const Args &A, Shared *sh, int32_t si) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        sh->done_read = atomicAdd(&A.stitch_res[si].arrive, 1);
        __threadfence();
    }
    __syncthreads();
    const bool second = sh->done_read == 1;
    __syncthreads();
    if (second) stitch_check(A, sh, si);
}

template <int CPT, bool kSX>
struct ForwardSweep {
    const Ctx &c;
    const Args &A;
    const RegionDesc &R;
    const Segment &S;
    Shared *sh;
    float *ring;                  // 3 slots x 3 states x (wmax + 2); slot of d is (d - s) mod 3
    const float4 *tab;
    int tid, lane, warp, wmax, stride;
    int64_t db;
    int32_t n;
    int32_t dbeg, dend;           // owned anti-diagonals (dbeg, dend] (0 is owned by a first segment)
    float *Fd;                    // forward store of the anti-diagonal being computed
    const float *Ereg;
    // band facts: metas of d-2, d-1, d (m2, m1, m0); by phase, decoded metas of d+1 .. d+3 and
    // raw metas of d+3 .. d+5 (loaded three steps before they are decoded)
    Meta m2, m1, m0;
    Meta near[3];
    int2 raw[3];
    int32_t eoff3;                // first cell of d+3
    // look-ahead emissions by phase: match, extra event, skip (and whether the column exists)
    float pM[3][CPT], pY[3][CPT], pX[3][CPT];
    bool pV[3][CPT];
    float lm_prev;
    float delta0, delta1;         // delta(d) = base(d) - base(d-1), delta(d-1)
    double base0;                 // base(d)
    double qbase;                 // lane q of warp 0: base and shift of the last anti-diagonal d
    float qshift;                 // with d mod 32 == q
    int32_t wi;

    __device__ __forceinline__ ForwardSweep(const Ctx &cc, const Segment &sg, Shared *s, float *r)
        : c(cc), A(*cc.A), R(cc.R), S(sg), sh(s), ring(r) {}

    __device__ __forceinline__ float *slot(int k, int state) const { return ring + (k * 3 + state) * stride + 1; }

    // issue the look-ahead loads of anti-diagonal dd (meta m, first cell off) into phase P
    template <int P>
    __device__ __forceinline__ void prefetch(int32_t dd, const Meta &m, int32_t off) {
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kThreads;
            const int32_t xmy = m.L + 2 * i, x = (dd + xmy) >> 1;
            const int ic = clampi(i, 0, max(m.W - 1, 0));
            pM[P][j] = __ldg(Ereg + 2 * off + SE_M * m.W + ic);
            pY[P][j] = __ldg(Ereg + 2 * off + SE_Y * m.W + ic);
            pX[P][j] = raw_gapx(c, x);
            pV[P][j] = x >= 1;
        }
    }

    template <int P>
    __device__ __forceinline__ void step(int32_t d) {
        constexpr int S0 = P, S1 = (P + 2) % 3, S2 = (P + 1) % 3;   // slots of d, d-1, d-2
        const float *t = c.t;
        // the recursion's operands first: ring reads right after the barrier, ahead of any
        // shared-memory store of this step that would have to be ordered before them
        const int32_t W0 = m0.W;
        const int32_t dl = (m0.L - 1 - m1.L) >> 1, du = (m0.L + 1 - m1.L) >> 1, dm = (m0.L - m2.L) >> 1;
        float lM[CPT], lX[CPT], lY[CPT], mM[CPT], mX[CPT], mY[CPT], uM[CPT], uY[CPT];
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kThreads;
            const int il = clampi(i + dl, -1, wmax);
            const int iu = clampi(i + du, -1, wmax);
            const int im = clampi(i + dm, -1, wmax);
            lM[j] = slot(S1, 0)[il];
            lX[j] = slot(S1, 1)[il];
            lY[j] = slot(S1, 2)[il];
            mM[j] = slot(S2, 0)[im];
            mX[j] = slot(S2, 1)[im];
            mY[j] = slot(S2, 2)[im];
            uM[j] = slot(S1, 0)[iu];
            uY[j] = slot(S1, 2)[iu];
        }
        // emissions of d (landed three steps ago)
        float eM[CPT], eY[CPT], eX[CPT];
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            eM[j] = pM[P][j];
            eY[j] = pY[P][j];
            eX[j] = pV[P][j] ? pX[P][j] : kNegInf;
        }
        // shift of d+1 from the maximum of d-2 (complete since the last barrier):
        // base(d+1) - base(d) = max(d-2) - delta(d) - delta(d-1)
        float delta_next = 0.0f;
        if (d >= 2) {
            const float *fp = sh->part[S2];
            const float mx = fmaxf(fmaxf(fp[0], fp[1]), fmaxf(fp[2], fp[3]));
            delta_next = ((mx > kNegInf ? mx : 0.0f) - delta0) - delta1;
        }
        // band facts: d+3 decoded (loaded three steps ago), d+6 requested; loads of d+3
        const Meta m3 = decode_meta(raw[P], d + 3 <= n);
        near[P] = m3;
        raw[P] = raw_meta(A, db, d + 6, n);
        prefetch<P>(d + 3, m3, eoff3);
        eoff3 += m3.W;
        // the recursion on d (stateMachine3_cellCalculate order: lower -> gap-X, middle -> match,
        // upper -> gap-Y, each state accumulated from LOG_ZERO)
        const float shL = -delta0, shM = -delta1 - delta0;
        const bool own = d > dbeg;   // warm-up anti-diagonals of a later segment store nothing
        const bool store_gaps = (m0.flags & kFlagStoreGaps) != 0;
        float lm = kNegInf;
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kThreads;
            // logAdd depends only on the difference of its arguments, so the cell's emission (and
            // the shift to this anti-diagonal's base) is added once after each state's fold
            float vX = lae(tab, lM[j] + t[T_OX], lX[j] + t[T_EX]);
            if (kSX) vX = lae(tab, vX, lY[j] + t[T_SX]);
            vX = vX + (eX[j] + shL);
            float vM = lae(tab, mM[j] + t[T_MC], mX[j] + t[T_MFGX]);
            vM = lae(tab, vM, mY[j] + t[T_MFGY]) + (eM[j] + shM);
            float vY = lae(tab, uM[j] + t[T_OY], uY[j] + t[T_EY]) + (eY[j] + shL);
            const bool in = i < W0;
            if (!in) vM = vX = vY = kNegInf;
            slot(S0, 0)[i] = vM;
            slot(S0, 1)[i] = vX;
            slot(S0, 2)[i] = vY;
            if (in && own) {
                Fd[ST_M * W0 + i] = vM;
                if (store_gaps) {
                    Fd[ST_X * W0 + i] = vX;
                    Fd[ST_Y * W0 + i] = vY;
                }
            }
            lm = fmaxf(lm, fmaxf(vM, fmaxf(vX, vY)));
        }
        // maximum of d-1 (one instruction per warp), published for the shift of d+2
        {
            const float wm = warp_max1(lm_prev);
            if (lane == 0) sh->part[S1][warp] = wm;
        }
        // base and shift of d: lane d mod 32 of warp 0 keeps them, and the warp writes them out 32
        // at a time and before a window is published (its backward sweep reads them); only the
        // segment's own anti-diagonals
        const bool window_end = own && (m0.flags & kFlagWindowEnd) != 0;
        if (warp == 0) {
            const int q = d & 31;
            if (lane == q) {
                qbase = base0;
                qshift = delta0;
            }
            if ((q == 31 || window_end || d == dend) && lane <= q && d - q + lane > dbeg) {
                A.base[db + (d - q) + lane] = qbase;
                A.fshift[db + (d - q) + lane] = qshift;
            }
        }
        if (window_end) __threadfence();   // this anti-diagonal and all before it, device-wide
        __syncthreads();
        if (window_end && tid == 0) {
            const unsigned q = atomicAdd(&A.ctl->pub, 1u);
            if ((int64_t) q < A.n_windows) atomicExch(A.ready + q, (int32_t) (R.win_base + wi));
            ++wi;
        }
        lm_prev = lm;
        delta1 = delta0;
        delta0 = delta_next;
        base0 += (double) delta_next;   // only warp 0 stores it
        Fd += 3 * W0;
        m2 = m1;
        m1 = m0;
        m0 = near[(P + 1) % 3];   // meta of d+1, decoded two steps ago
    }

    // After the step of anti-diagonal b (the ring holds b-2, b-1, b): the values of b-1 and b go to
    // stitch si with their FP64 bases, as its later side (this segment starts at b) or its earlier
    // side (this segment ends at b).  base0 and delta0 / delta1 already describe b+1.
    __device__ void stitch_capture(int32_t si, bool later, int32_t b, int32_t s) {
        const StitchDesc sd = A.stitch[si];
        float *v = A.stitch_vals + sd.voff + (later ? 0 : 3 * (sd.w0 + sd.w1));
        const double base_b = base0 - (double) delta0, base_b1 = base_b - (double) delta1;
#pragma unroll
        for (int part = 0; part < 2; ++part) {
            const int k = ((b - 1 + part - s) % 3 + 3) % 3;   // ring slot of anti-diagonal x: (x - s) mod 3
            const int32_t W = part ? sd.w1 : sd.w0;
            float *o = v + (part ? 3 * sd.w0 : 0);
            for (int i = tid; i < W; i += kThreads) {
                o[i] = slot(k, 0)[i];
                o[W + i] = slot(k, 1)[i];
                o[2 * W + i] = slot(k, 2)[i];
            }
        }
        if (tid == 0) {
            double *bs = later ? A.stitch_res[si].sbase : A.stitch_res[si].tbase;
            bs[0] = base_b1;
            bs[1] = base_b;
        }
    }

    // The sweep starts at anti-diagonal s = d_begin - warm (1 for a region's first segment); the
    // phase of anti-diagonal d (its ring slot and look-ahead registers) is (d - s) mod 3.  A later
    // segment's warm is 2 mod 3 (the planner picks it so): d_begin is the last step of a group of
    // three, so the stepping loop can stop there, with d_begin - 1 and d_begin in the ring.
    __device__ void run() {
        tab = sh->la;
        tid = threadIdx.x;
        lane = tid & 31;
        warp = tid >> 5;
        wmax = A.wmax;
        stride = wmax + 2;
        db = R.diag_base;
        n = R.n;
        dbeg = S.d_begin;
        dend = S.d_end;
        const int32_t s = dbeg - S.warm + (dbeg == 0 ? 1 : 0);
        Fd = A.F + 3 * (R.cell_base + S.cell0);
        Ereg = A.E + 2 * R.cell_base;
        ring_init(ring, wmax);
        __syncthreads();
        if (dbeg == 0) {
            // anti-diagonal 0 (slot 2): startStateProb / raggedStartStateProb (stateMachine.c:1022-1032)
            const float s0 = R.ragged_left ? kNegInf : 0.0f, s1 = R.ragged_left ? 0.0f : kNegInf;
            if (tid == 0) {
                float *F0 = A.F + 3 * R.cell_base;   // anti-diagonal 0 has one cell
                F0[ST_M] = s0; F0[ST_X] = s1; F0[ST_Y] = s1;
                slot(2, 0)[0] = s0;
                slot(2, 1)[0] = s1;
                slot(2, 2)[0] = s1;
                A.base[db] = 0.0;
                A.fshift[db] = 0.0f;
            }
            m2 = Meta{0, 0, 0};
            m1 = decode_meta(raw_meta(A, db, 0, n), true);
            lm_prev = tid == 0 ? fmaxf(s0, s1) : kNegInf;
        } else {
            // a later segment: every band cell of s-2 (slot 1) and s-1 (slot 2) starts at 0
            m2 = decode_meta(raw_meta(A, db, s - 2, n), true);
            m1 = decode_meta(raw_meta(A, db, s - 1, n), true);
            for (int i = tid; i < wmax; i += kThreads) {
#pragma unroll
                for (int st = 0; st < 3; ++st) {
                    if (i < m2.W) slot(1, st)[i] = 0.0f;
                    if (i < m1.W) slot(2, st)[i] = 0.0f;
                }
            }
            if (tid < kWarps) sh->part[1][tid] = 0.0f;   // maximum of s-2
            lm_prev = 0.0f;                               // maximum of s-1
        }
        // look-ahead: metas of s, s+1, s+2 decoded, s+3 .. s+5 raw; emissions of s .. s+2 requested
        int32_t off = (int32_t) S.cell0;
        m0 = decode_meta(raw_meta(A, db, s, n), s <= n);
        const Meta ma = decode_meta(raw_meta(A, db, s + 1, n), s + 1 <= n);
        const Meta mb = decode_meta(raw_meta(A, db, s + 2, n), s + 2 <= n);
        prefetch<0>(s, m0, off);
        off += m0.W;
        prefetch<1>(s + 1, ma, off);
        off += ma.W;
        prefetch<2>(s + 2, mb, off);
        off += mb.W;
        eoff3 = off;   // first cell of s + 3
        near[0] = Meta{0, 0, 0};
        near[1] = ma;
        near[2] = mb;
        raw[0] = raw_meta(A, db, s + 3, n);
        raw[1] = raw_meta(A, db, s + 4, n);
        raw[2] = raw_meta(A, db, s + 5, n);
        // Renormalisation: base(d + 1) = base(d - 2) + max(d - 2), known one step ahead, so neither
        // the reduction nor the shared-memory read of the warps' maxima sits on the recursion's
        // path.  delta(d) = base(d) - base(d-1) is a float and base(d) = base(d-1) + delta(d).
        delta0 = delta1 = 0.0f;
        base0 = 0.0;
        qbase = 0.0;   // anti-diagonal 0 (lane 0 of the first block): base 0, shift 0
        qshift = 0.0f;
        wi = S.wi0;
        __syncthreads();
        // the stepping loop stops once at d_begin when the segment starts at a stitch
        int32_t d = s, stop = S.stitch_in >= 0 ? dbeg : dend;
        for (;;) {
            for (; d <= stop; d += 3) {
                step<0>(d);
                if (d + 1 > stop) break;
                step<1>(d + 1);
                if (d + 2 > stop) break;
                step<2>(d + 2);
            }
            if (stop == dend) break;
            stitch_capture(S.stitch_in, true, dbeg, s);   // whole groups ran: d == d_begin + 1
            stop = dend;
        }
        if (S.stitch_out >= 0) stitch_capture(S.stitch_out, false, dend, s);
        if (S.stitch_in >= 0) stitch_arrive(A, sh, S.stitch_in);
        if (S.stitch_out >= 0) stitch_arrive(A, sh, S.stitch_out);
    }
};

template <int CPT>
__device__ void forward_task(const Ctx &c, const Segment &sg, Shared *sh, float *ring) {
    if (c.t[T_SX] > kNegInf) {
        ForwardSweep<CPT, true> f(c, sg, sh, ring);
        f.run();
    } else {
        ForwardSweep<CPT, false> f(c, sg, sh, ring);
        f.run();
    }
}

// ------------------------------------------------------------------------------------------------
// backward sweep of one traceback window, posteriors fused
// ------------------------------------------------------------------------------------------------
template <int CPT>
__device__ __forceinline__ void write_pairs(const Ctx &c, Shared *sh, const WindowTask &wt, int32_t pend_d,
                                            unsigned pend, const float *pv, const int32_t *px, const int32_t *py,
                                            const int32_t *pk, int64_t &n_out) {
    const Args &A = *c.A;
    const RegionDesc &R = c.R;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int32_t before = 0;
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
        int32_t mine_before = before;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const int32_t cw = sh->wcnt[pend_d & 1][j][w];
            if (w < warp) mine_before += cw;
            before += cw;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, (pend >> j) & 1u);
        if ((pend >> j) & 1u) {
            const int64_t slot = n_out + mine_before + __popc(bal & ((1u << lane) - 1u));
            if (slot < wt.out_cap) {
                sa_aligned_pair o;
                o.score = (int64_t) floor((double) fminf(pv[j], 1.0f) * 10000000.0);
                o.x = R.x1 + px[j] - 1;
                o.y = R.y1 + py[j] - 1;
                o.kmer = pk[j];
                A.out[wt.out_base + slot] = o;
            } else {
                atomicMax(A.status + R.read, (int32_t) SA_E_OUTPUT);
            }
        }
    }
    n_out += before;
}

template <int CPT, bool kSX>
__device__ void window_task(const Ctx &c, Shared *sh, float *ring, float *chain, int64_t gw) {
    const Args &A = *c.A;
    const RegionDesc &R = c.R;
    const float *t = c.t;
    const float4 *tab = sh->la;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wmax = A.wmax;
    const int64_t db = R.diag_base;
    const int32_t n = R.n;
    const float *Freg = A.F + 3 * R.cell_base;
    const float *Ereg = A.E + 2 * R.cell_base;
    const Window W = A.windows[gw];
    const WindowTask wt = A.wtask[gw];
    // a window whose T starts a forward segment reads that segment's own copy of T, kept by the
    // stitch: the store holds the earlier segment's, whose values differ by the stitch's constant
    const float *Tside = A.use_side && wt.side >= 0 ? A.stitch_vals + A.stitch[wt.side].voff + 3 * A.stitch[wt.side].w0
                                                    : nullptr;
    int64_t n_out = 0;
    double ll = 0.0;
    ring_init(ring, wmax);
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
    rg.s[0] = ring + 1;                      // d = D
    rg.s[1] = ring + 3 * rg.stride + 1;      // d + 1 (none yet: -inf)
    rg.s[2] = ring + 6 * rg.stride + 1;      // d + 2
    // metas of d+2, d+1, d, d-1 (d = D to start), raw meta of d-2, first cells of d+1, d
    Meta mpp{0, 0, 0}, mp{0, 0, 0};
    Meta m0 = decode_meta(raw_meta(A, db, D, n), true);
    Meta mm = decode_meta(raw_meta(A, db, D - 1, n), D - 1 >= 0);
    int2 raw_mmm = raw_meta(A, db, D - 2, n);
    int32_t off0 = wt.first_cell, offp = off0;
    __syncthreads();   // ring cleared
#pragma unroll
    for (int j = 0; j < CPT; ++j) {
        const int i = tid + j * kThreads;
        const bool in = i < m0.W;
        rg.st(0, 0)[i] = in ? e0 : kNegInf;
        rg.st(0, 1)[i] = in ? e1 : kNegInf;
        rg.st(0, 2)[i] = in ? e2 : kNegInf;
    }
    // operands of the current anti-diagonal's cells, loaded one anti-diagonal ahead
    float eMm[CPT], eYu[CPT], eXl[CPT], fM[CPT];
    // refresh operands: gap states of d, and the match-through inputs of the d+1 cells
    float fX[CPT], fY[CPT], tM[CPT], tX[CPT], tY[CPT], tE[CPT];
    bool tv[CPT];
    double fb = __ldcg(A.base + db + D);
    float fsh = __ldcg(A.fshift + db + D);
    {
        const bool refreshD = D <= from && (m0.flags & kFlagRefresh);
        const float *Fd = Freg + 3 * off0;
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
            const int i = tid + j * kThreads;
            const int ic = clampi(i, 0, max(m0.W - 1, 0));
            eMm[j] = eYu[j] = eXl[j] = kNegInf;
            fM[j] = __ldcg(Fd + ST_M * m0.W + ic);
            fX[j] = refreshD ? __ldcg(Fd + ST_X * m0.W + ic) : kNegInf;
            fY[j] = refreshD ? __ldcg(Fd + ST_Y * m0.W + ic) : kNegInf;
            tM[j] = tX[j] = tY[j] = tE[j] = kNegInf;
            tv[j] = false;
        }
    }
    float lm_prev = kNegInf;           // local max of B stored on d+1 (lagged reduction)
    float gamma1 = 0.0f;               // base(d+1) - base(d+2)
    double bbase = 0.0;                // base of B on d
    double pref = 0.0;                 // latest refresh total probability (absolute)
    unsigned pend = 0;
    float pv[CPT];
    int32_t px[CPT], py[CPT], pk[CPT];
    int32_t pend_d = -1;
    __syncthreads();
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
                const float *bp = sh->part[(d + 2) % 3];
                m = fmaxf(fmaxf(bp[0], bp[1]), fmaxf(bp[2], bp[3]));
                if (!(m > kNegInf)) m = 0.0f;
            }
            gamma0 = m - gamma1;
        }
        bbase += (double) gamma0;
        // prefetch the operands of the d-1 cells: raw loads from clamped indices; a value fetched
        // for an absent neighbour is only ever added to a -inf ring value
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
            const float *Ed = Ereg + 2 * off0;                  // emissions of d
            const float *Ep = Ereg + 2 * offp;                  // of d+1 (or d at the window top)
            const float *Fm = Freg + 3 * offm;                  // forward values of d-1
            const int32_t Wpl = Wp > 0 ? Wp : W0;               // width of the block Ep points at
#pragma unroll
            for (int j = 0; j < CPT; ++j) {
                const int i = tid + j * kThreads;
                const int32_t xmy = mm.L + 2 * i, x = (d - 1 + xmy) >> 1;
                eMm_n[j] = __ldg(Ep + SE_M * Wpl + clampi((xmy - mp.L) >> 1, 0, max(Wpl - 1, 0)));
                eYu_n[j] = __ldg(Ed + SE_Y * W0 + clampi((xmy - 1 - m0.L) >> 1, 0, max(W0 - 1, 0)));
                eXl_n[j] = raw_gapx(c, x + 1);
                fM_n[j] = __ldcg(Fm + ST_M * Wm + clampi(i, 0, max(Wm - 1, 0)));
                tv_n[j] = false;
                fX_n[j] = fY_n[j] = tM_n[j] = tX_n[j] = tY_n[j] = tE_n[j] = kNegInf;
            }
            if (refresh_m) {
                // gap states of d-1; match-through inputs of a refresh at d-1: match emissions of
                // the d cells and forward values of d-2
                const float *Fmm = Tside && d - 2 == T ? Tside : Freg + 3 * (Wmm > 0 ? offmm : offm);
                const int32_t Wml = Wmm > 0 ? Wmm : Wm;
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    const int i = tid + j * kThreads;
                    const int ic = clampi(i, 0, max(Wm - 1, 0));
                    fX_n[j] = __ldcg(Fm + ST_X * Wm + ic);
                    fY_n[j] = __ldcg(Fm + ST_Y * Wm + ic);
                    const int32_t xmy0 = m0.L + 2 * i;
                    const int32_t r = (xmy0 - mmm.L) >> 1;
                    tv_n[j] = i < W0 && Wmm > 0 && xmy0 >= mmm.L && r < Wmm;
                    const int imm = clampi(r, 0, max(Wmm - 1, 0));
                    tE_n[j] = __ldg(Ed + SE_M * W0 + clampi(i, 0, max(W0 - 1, 0)));
                    tM_n[j] = __ldcg(Fmm + ST_M * Wml + imm);
                    tX_n[j] = __ldcg(Fmm + ST_X * Wml + imm);
                    tY_n[j] = __ldcg(Fmm + ST_Y * Wml + imm);
                }
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
                const int i = tid + j * kThreads;
                const int32_t xmy = m0.L + 2 * i;
                const int ipp = clampi((xmy - mpp.L) >> 1, -1, wmax);
                const int iu = clampi((xmy - 1 - mp.L) >> 1, -1, wmax);
                const int il = clampi((xmy + 1 - mp.L) >> 1, -1, wmax);
                // each successor's backward value plus its emission, shared by the transitions into it
                const float bme = rg.st(2, 0)[ipp] + (eMm[j] + shM);
                float vM = bme + t[T_MC];
                float vX = bme + t[T_MFGX];
                float vY = bme + t[T_MFGY];
                const float bue = rg.st(1, 2)[iu] + (eYu[j] + shU);
                vM = lae(tab, vM, bue + t[T_OY]);
                vY = lae(tab, vY, bue + t[T_EY]);
                const float ble = rg.st(1, 1)[il] + (eXl[j] + shU);
                vM = lae(tab, vM, ble + t[T_OX]);
                vX = lae(tab, vX, ble + t[T_EX]);
                if (kSX) vY = lae(tab, vY, ble + t[T_SX]);
                if (i >= W0) vM = vX = vY = kNegInf;
                rg.st(0, 0)[i] = vM;
                rg.st(0, 1)[i] = vX;
                rg.st(0, 2)[i] = vY;
                lm = fmaxf(lm, fmaxf(vM, fmaxf(vX, vY)));
            }
        }
        {
            const float wm = warp_max(lm_prev);
            if (lane == 0 && d + 1 <= D) sh->part[(d + 1) % 3][warp] = wm;
        }
        __syncthreads();
        // pairs of the previous anti-diagonal, in the reference's order (ascending xmy)
        if (pend_d >= 0) {
            write_pairs<CPT>(c, sh, wt, pend_d, pend, pv, px, py, pk, n_out);
            pend = 0;
            pend_d = -1;
        }
        if (post) {
            if (refresh) {
                // diagonalCalculationTotalProbability (pairwiseAligner.c:1182-1200): F.B on d in
                // ascending cell order, then the matches from d-1 over d into d+1, dotted with B(d+1)
#pragma unroll
                for (int j = 0; j < CPT; ++j) {
                    const int i = tid + j * kThreads;
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
                        const int i = tid + j * kThreads;
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
                __syncthreads();
                if (warp == 0) {
                    const float f = ordered_fold(tab, chain, W0);
                    if (lane == 0) sh->fold[0] = f;
                } else if (warp == 1) {
                    const float f = have_next ? ordered_fold(tab, chain + wmax, Wp) : kNegInf;
                    if (lane == 0) sh->fold[1] = f;
                }
                __syncthreads();
                // the through-part is relative to base_F(d-1) + base_B(d+1)
                const float ptil = lae(tab, sh->fold[0], sh->fold[1] - fsh - gamma0);
                pref = (double) ptil + fb + bbase;
                if (d == n) ll = pref;
            }
            const float kd = (float) (fb + bbase - pref);
#pragma unroll
            for (int j = 0; j < CPT; ++j) {
                const int i = tid + j * kThreads;
                const int32_t xmy = m0.L + 2 * i, x = (d + xmy) >> 1, y = (d - xmy) >> 1;
                const float p = __expf(fM[j] + rg.st(0, 0)[i] + kd);
                const bool hit = i < W0 && x > 0 && y > 0 && p >= A.threshold;
                pv[j] = p;
                px[j] = x;
                py[j] = y;
                pk[j] = __ldg(A.kmer + R.kmer_base + clampi(x - 1, 0, max(R.lX - 1, 0)));
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
    __syncthreads();
    if (pend_d >= 0) write_pairs<CPT>(c, sh, wt, pend_d, pend, pv, px, py, pk, n_out);
    if (tid == 0) {
        A.wcount[gw] = n_out;
        if (W.at_end) A.loglik[c.region_index] = ll;
    }
}

// ------------------------------------------------------------------------------------------------
// backward sweep of one traceback window by one warp (bands up to 32 * WCPT cells wide)
// ------------------------------------------------------------------------------------------------
// The same recursion, posterior and refreshes as window_task, with the anti-diagonal's cells spread
// over one warp (cell i on lane i mod 32): warp-synchronous exchange through the ring, maxima by one
// warp reduction, pairs numbered by ballots, no block barrier.  Look-ahead loads go to registers
// indexed by the parity of the step, so they land without register moves; the operands of a
// refresh (one anti-diagonal in ten) are loaded when it happens.
template <int WCPT, bool kSX>
struct WarpWindow {
    const Ctx &c;
    const Args &A;
    const RegionDesc &R;
    const float4 *tab;
    float *ring;                  // 3 slots x 3 states x (wmax + 2)
    float *chain;                 // 2 x wmax: refresh terms, then 6 x wmax: staged refresh operands
    int lane, wmax, stride;
    int64_t db;
    int32_t n, D, T, from;
    const float *Freg, *Ereg;
    const float *Tside;           // the forward segment's own copy of T (see window_task), or null
    float *s0, *s1, *s2;          // ring slots of d, d+1, d+2
    Meta mpp, mp, m0, mm;         // band facts of d+2, d+1, d, d-1
    int2 raw_mmm;                 // raw band facts of d-2
    int32_t off0, offp;           // first cells of d and d+1
    // look-ahead operands of a step's cells, by step parity: match emission of the match
    // successor, extra-event emission of the upper successor, skip emission of the lower
    // successor, forward match value; and the forward base and shift
    float qM[2][WCPT], qY[2][WCPT], qX[2][WCPT], qF[2][WCPT];
    double qB[2];
    float qS[2];
    float mxD, mx_last, lm_prev, gamma1;
    float e0, e1, e2;             // end states on D
    double bbase, pref, ll;
    int64_t n_out;

    __device__ __forceinline__ WarpWindow(const Ctx &cc, float *r, float *ch, const float4 *tb)
        : c(cc), A(*cc.A), R(cc.R), tab(tb), ring(r), chain(ch) {}

    // operands of the cells of anti-diagonal dd (meta m, first cell off) into parity Q; m1 / off1
    // describe dd+1 (upper successors), m2 / off2 dd+2 (match successors)
    template <int Q>
    __device__ __forceinline__ void prefetch(int32_t dd, const Meta &m, int32_t off, const Meta &m1, int32_t off1,
                                             const Meta &m2, int32_t off2) {
        const float *E2 = Ereg + 2 * off2, *E1 = Ereg + 2 * off1, *Fm = Freg + 3 * off;
#pragma unroll
        for (int j = 0; j < WCPT; ++j) {
            const int i = lane + 32 * j;
            const int32_t xmy = m.L + 2 * i, x = (dd + xmy) >> 1;
            qM[Q][j] = __ldg(E2 + SE_M * m2.W + clampi((xmy - m2.L) >> 1, 0, max(m2.W - 1, 0)));
            qY[Q][j] = __ldg(E1 + SE_Y * m1.W + clampi((xmy - 1 - m1.L) >> 1, 0, max(m1.W - 1, 0)));
            qX[Q][j] = raw_gapx(c, x + 1);
            qF[Q][j] = __ldcg(Fm + ST_M * m.W + clampi(i, 0, max(m.W - 1, 0)));
        }
        qB[Q] = __ldcg(A.base + db + max(dd, 0));
        qS[Q] = __ldcg(A.fshift + db + max(dd, 0));
    }

    // Operands of a refresh at anti-diagonal dd (meta m, first cell off): its gap states, and for
    // the cells of dd+1 (m1, off1) the forward values of dd-1 (m_1, off_1) on their match
    // predecessors and their match emissions.  At the end of the step before the refresh,
    // load_refresh loads them (forward values through L2: other CTAs wrote them during this
    // launch) and store_refresh puts them in this warp's staging rows.
    struct RefreshOps {
        float x[WCPT], y[WCPT], m[WCPT], tx[WCPT], ty[WCPT], e[WCPT];
    };

    __device__ __forceinline__ void load_refresh(RefreshOps &o, const Meta &m, int32_t off, const Meta &m1, int32_t off1,
                                                 const Meta &m_1, int32_t off_1, int32_t d_1) const {
        const float *Fd = Freg + 3 * off, *E1 = Ereg + 2 * off1;
        const float *Fm = Tside && d_1 == T ? Tside : Freg + 3 * off_1;
#pragma unroll
        for (int j = 0; j < WCPT; ++j) {
            const int i = lane + 32 * j;
            const int ic = clampi(i, 0, max(m.W - 1, 0));
            o.x[j] = __ldcg(Fd + ST_X * m.W + ic);
            o.y[j] = __ldcg(Fd + ST_Y * m.W + ic);
            const int32_t r = clampi((m1.L + 2 * i - m_1.L) >> 1, 0, max(m_1.W - 1, 0));
            o.m[j] = __ldcg(Fm + ST_M * m_1.W + r);
            o.tx[j] = __ldcg(Fm + ST_X * m_1.W + r);
            o.ty[j] = __ldcg(Fm + ST_Y * m_1.W + r);
            o.e[j] = __ldg(E1 + SE_M * m1.W + clampi(i, 0, max(m1.W - 1, 0)));
        }
    }

    __device__ __forceinline__ void store_refresh(const RefreshOps &o) const {
        float *stg = chain + 2 * wmax;
#pragma unroll
        for (int j = 0; j < WCPT; ++j) {
            const int i = lane + 32 * j;
            stg[i] = o.x[j];
            stg[wmax + i] = o.y[j];
            stg[2 * wmax + i] = o.m[j];
            stg[3 * wmax + i] = o.tx[j];
            stg[4 * wmax + i] = o.ty[j];
            stg[5 * wmax + i] = o.e[j];
        }
    }

    // anti-diagonal d; K = (D - d) & 1 is the parity of its operands
    template <int K>
    __device__ __forceinline__ void step(int32_t d, const WindowTask &wt) {
        const float *t = c.t;
        const int32_t W0 = m0.W, Wp = mp.W;
        // maximum of B on d+1 for the shift of d-1 (d+1 = D holds the end states: known exactly)
        const float mx_new = warp_max1(lm_prev);
        float gamma0 = 0.0f;           // base(d) - base(d+1) = max(d+2) - gamma1
        if (d <= D - 2) {
            float m = d == D - 2 ? mxD : mx_last;
            if (!(m > kNegInf)) m = 0.0f;
            gamma0 = m - gamma1;
        }
        bbase += (double) gamma0;
        // operands of the d-1 cells
        const Meta mmm = decode_meta(raw_mmm, d - 2 >= 0);
        raw_mmm = raw_meta(A, db, d - 3, n);
        const int32_t offm = off0 - mm.W;
        prefetch<1 - K>(d - 1, mm, offm, m0, off0, mp, offp);
        const bool refresh_next = d - 1 > T && d - 1 <= from && (mm.flags & kFlagRefresh) != 0;
        // the recursion on d (D itself holds the end-state values); B of the cells kept in registers
        float lm = kNegInf;
        float bM[WCPT], bX[WCPT], bY[WCPT];
        if (d == D) {
#pragma unroll
            for (int j = 0; j < WCPT; ++j) {
                const bool in = lane + 32 * j < W0;
                bM[j] = in ? e0 : kNegInf;
                bX[j] = in ? e1 : kNegInf;
                bY[j] = in ? e2 : kNegInf;
            }
        } else {
            const float shU = -gamma0, shM = -gamma1 - gamma0;
            // all ring reads first, then the arithmetic, then the ring writes: the cells' chains are
            // independent, and no shared-memory store sits between them to order them
            float bme[WCPT], bue[WCPT], ble[WCPT];
#pragma unroll
            for (int j = 0; j < WCPT; ++j) {
                const int i = lane + 32 * j;
                const int32_t xmy = m0.L + 2 * i;
                const int ipp = clampi((xmy - mpp.L) >> 1, -1, wmax);
                const int iu = clampi((xmy - 1 - mp.L) >> 1, -1, wmax);
                const int il = clampi((xmy + 1 - mp.L) >> 1, -1, wmax);
                bme[j] = s2[ipp];
                bue[j] = s1[2 * stride + iu];
                ble[j] = s1[stride + il];
            }
#pragma unroll
            for (int j = 0; j < WCPT; ++j) {
                // each successor's backward value plus its emission, shared by the transitions into it
                const float me = bme[j] + (qM[K][j] + shM);
                float vM = me + t[T_MC];
                float vX = me + t[T_MFGX];
                float vY = me + t[T_MFGY];
                const float ue = bue[j] + (qY[K][j] + shU);
                vM = lae(tab, vM, ue + t[T_OY]);
                vY = lae(tab, vY, ue + t[T_EY]);
                const float le = ble[j] + (qX[K][j] + shU);
                vM = lae(tab, vM, le + t[T_OX]);
                vX = lae(tab, vX, le + t[T_EX]);
                if (kSX) vY = lae(tab, vY, le + t[T_SX]);
                const bool in = lane + 32 * j < W0;
                bM[j] = in ? vM : kNegInf;
                bX[j] = in ? vX : kNegInf;
                bY[j] = in ? vY : kNegInf;
                lm = fmaxf(lm, fmaxf(bM[j], fmaxf(bX[j], bY[j])));
            }
#pragma unroll
            for (int j = 0; j < WCPT; ++j) {
                const int i = lane + 32 * j;
                s0[i] = bM[j];
                s0[stride + i] = bX[j];
                s0[2 * stride + i] = bY[j];
            }
        }
        __syncwarp();
        const double fb = qB[K];
        const float fsh = qS[K];
        if (d <= from) {
            if ((m0.flags & kFlagRefresh) != 0) {
                // diagonalCalculationTotalProbability (pairwiseAligner.c:1182-1200): F.B on d in
                // ascending cell order, then the matches from d-1 over d into d+1, dotted with B(d+1)
                const float *stg = chain + 2 * wmax;
                const bool have_next = d < D;
                const int32_t Wm = mm.W;
                float sx[WCPT], sy[WCPT], tm[WCPT], tx[WCPT], ty[WCPT], te[WCPT], b1[WCPT];
#pragma unroll
                for (int j = 0; j < WCPT; ++j) {
                    const int i = lane + 32 * j;
                    sx[j] = stg[i];
                    sy[j] = stg[wmax + i];
                    tm[j] = stg[2 * wmax + i];
                    tx[j] = stg[3 * wmax + i];
                    ty[j] = stg[4 * wmax + i];
                    te[j] = stg[5 * wmax + i];
                    b1[j] = s1[i];
                }
                float c0[WCPT], c1[WCPT];
#pragma unroll
                for (int j = 0; j < WCPT; ++j) {
                    const int i = lane + 32 * j;
                    float v = qF[K][j] + bM[j];
                    v = lae(tab, v, sx[j] + bX[j]);
                    c0[j] = lae(tab, v, sy[j] + bY[j]);
                    const int32_t xmy1 = mp.L + 2 * i;
                    const int32_t r = (xmy1 - mm.L) >> 1;
                    float mth = kNegInf;
                    if (Wm > 0 && xmy1 >= mm.L && r < Wm) {
                        const float e = te[j];
                        mth = tm[j] + (e + t[T_MC]);
                        mth = lae(tab, mth, tx[j] + (e + t[T_MFGX]));
                        mth = lae(tab, mth, ty[j] + (e + t[T_MFGY]));
                    }
                    c1[j] = mth + b1[j];
                }
#pragma unroll
                for (int j = 0; j < WCPT; ++j) {
                    const int i = lane + 32 * j;
                    if (i < W0) chain[i] = c0[j];
                    if (have_next && i < Wp) chain[wmax + i] = c1[j];
                }
                __syncwarp();
                const float2 ff = ordered_fold2(tab, chain, W0, chain + wmax, have_next ? Wp : 0);
                const float f0 = ff.x, f1 = ff.y;
                // the through-part is relative to base_F(d-1) + base_B(d+1)
                const float ptil = lae(tab, f0, f1 - fsh - gamma0);
                pref = (double) ptil + fb + bbase;
                if (d == n) ll = pref;
                __syncwarp();
            }
            // posteriors of d, emitted in ascending cell order (the reference's order)
            const float kd = (float) (fb + bbase - pref);
            int64_t before = n_out;
#pragma unroll
            for (int j = 0; j < WCPT; ++j) {
                const int i = lane + 32 * j;
                const int32_t xmy = m0.L + 2 * i, x = (d + xmy) >> 1, y = (d - xmy) >> 1;
                const float p = __expf(qF[K][j] + bM[j] + kd);
                const bool hit = i < W0 && x > 0 && y > 0 && p >= A.threshold;
                const unsigned bal = __ballot_sync(0xffffffffu, hit);
                if (hit) {
                    const int64_t q = before + __popc(bal & ((1u << lane) - 1u));
                    if (q < wt.out_cap) {
                        sa_aligned_pair o;
                        o.score = (int64_t) floor((double) fminf(p, 1.0f) * 10000000.0);
                        o.x = R.x1 + x - 1;
                        o.y = R.y1 + y - 1;
                        o.kmer = __ldg(A.kmer + R.kmer_base + x - 1);   // 1 <= x <= lX for a pair
                        A.out[wt.out_base + q] = o;
                    } else {
                        atomicMax(A.status + R.read, (int32_t) SA_E_OUTPUT);
                    }
                }
                before += __popc(bal);
            }
            n_out = before;
        }
        if (refresh_next) {
            // loaded here rather than a step early: held across the step, the 6 x WCPT operands
            // pushed the 3-CTAs-per-SM build into spilling (312 B per thread; 16 B this way), and
            // the latency is paid one step in ten
            RefreshOps rops;
            load_refresh(rops, mm, offm, m0, off0, mmm, offm - mmm.W, d - 2);
            __syncwarp();   // this step's refresh (if any) has read the staging rows
            store_refresh(rops);
        }
        mx_last = mx_new;
        lm_prev = d == D ? kNegInf : lm;   // D's maximum is known exactly (mxD)
        gamma1 = gamma0;
        offp = off0;
        off0 = offm;
        float *fr = s2;
        s2 = s1;
        s1 = s0;
        s0 = fr;
        mpp = mp; mp = m0; m0 = mm; mm = mmm;
    }

    __device__ void run(int64_t gw) {
        lane = threadIdx.x & 31;
        wmax = 32 * WCPT;
        stride = wmax + 2;
        db = R.diag_base;
        n = R.n;
        Freg = A.F + 3 * R.cell_base;
        Ereg = A.E + 2 * R.cell_base;
        const Window Wn = A.windows[gw];
        const WindowTask wt = A.wtask[gw];
        D = Wn.D;
        T = Wn.T;
        from = Wn.from;
        Tside = A.use_side && wt.side >= 0 ? A.stitch_vals + A.stitch[wt.side].voff + 3 * A.stitch[wt.side].w0 : nullptr;
        for (int i = lane; i < 9 * stride; i += 32) ring[i] = kNegInf;
        s0 = ring + 1;
        s1 = ring + 3 * stride + 1;
        s2 = ring + 6 * stride + 1;
        // end-state values on D (stateMachine.c:1034-1061)
        const float *t = c.t;
        const bool ragged_end = Wn.at_end && R.ragged_right;
        e0 = ragged_end ? (t[T_OX] + t[T_OY]) / 2.0f : t[T_MC];
        e1 = ragged_end ? t[T_EX] : t[T_MFGX];
        e2 = ragged_end ? t[T_EY] : t[T_MFGY];
        mxD = fmaxf(e0, fmaxf(e1, e2));
        if (!(mxD > kNegInf)) mxD = 0.0f;
        mpp = mp = Meta{0, 0, 0};
        m0 = decode_meta(raw_meta(A, db, D, n), true);
        mm = decode_meta(raw_meta(A, db, D - 1, n), D - 1 >= 0);
        raw_mmm = raw_meta(A, db, D - 2, n);
        off0 = offp = wt.first_cell;
        __syncwarp();
#pragma unroll
        for (int j = 0; j < WCPT; ++j) {
            const int i = lane + 32 * j;
            if (i < m0.W) {
                s0[i] = e0;
                s0[stride + i] = e1;
                s0[2 * stride + i] = e2;
            }
        }
        prefetch<0>(D, m0, off0, mp, offp, mpp, offp);
        if (D <= from && (m0.flags & kFlagRefresh) != 0) {
            RefreshOps o;
            load_refresh(o, m0, off0, mp, offp, mm, off0 - mm.W, D - 1);
            store_refresh(o);
        }
        mx_last = kNegInf;
        lm_prev = kNegInf;
        gamma1 = 0.0f;
        bbase = pref = ll = 0.0;
        n_out = 0;
        __syncwarp();
        for (int32_t d = D; d > T; d -= 2) {
            step<0>(d, wt);
            if (d - 1 <= T) break;
            step<1>(d - 1, wt);
        }
        if (lane == 0) {
            A.wcount[gw] = n_out;
            if (Wn.at_end) A.loglik[c.region_index] = ll;
        }
        __syncwarp();
    }
};

// ------------------------------------------------------------------------------------------------
// the persistent worker
// ------------------------------------------------------------------------------------------------
// Bounded wait (one thread) until a forward sweep publishes into ready-queue slot `slot`; -1 if
// the wait gave up (SA_E_TIMEOUT for the batch) or another worker already did.
__device__ __forceinline__ int32_t wait_ready(const Args &A, int64_t slot) {
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
// per-read gather and completion
// ------------------------------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ void group_sync() {
    if (NT == 32) __syncwarp();
    else __syncthreads();
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One read's windows' pairs concatenated in window order (regions, then windows: the reference's
// emission order) into a range of the packed output claimed from the packed counter; sets the
// read's range.  Run by a group of NT threads (one warp, or a whole CTA of NT threads with `red`
// holding NT / 32 + 1 shared slots); every thread returns the range.  Window counts and pairs were
// written by other CTAs, so they are read through L2.
template <int NT>
__device__ void gather_read(const Args &A, int64_t r, int tid, long long *red, long long &base, long long &tot) {
    const int64_t w0 = A.read_win[8 * r], nw = A.read_win[8 * r + 1];
    long long mine = 0;
    for (int64_t k = tid; k < nw; k += NT)
        mine += min(__ldcg(A.wcount + w0 + k), (int64_t) A.wtask[w0 + k].out_cap);
    mine = warp_sum_ll(mine);
    if (NT == 32) {
        tot = mine;
        base = tid == 0 && tot > 0 ? (long long) atomicAdd(&A.ctl->packed, (unsigned long long) tot) : 0;
        base = __shfl_sync(0xffffffffu, base, 0);
    } else {
        if ((tid & 31) == 0) red[tid >> 5] = mine;
        __syncthreads();
        tot = 0;
        for (int w = 0; w < NT / 32; ++w) tot += red[w];
        if (tid == 0) red[NT / 32] = tot > 0 ? (long long) atomicAdd(&A.ctl->packed, (unsigned long long) tot) : 0;
        __syncthreads();
        base = red[NT / 32];
    }
    // 32 windows at a time: lane j of every warp holds window k0 + j's count and an inclusive scan
    // of the counts, so the group copies window after window without a barrier between them
    const int j = tid & 31;
    long long run = 0;
    for (int64_t k0 = 0; k0 < nw; k0 += 32) {
        long long cnt = 0, ob = 0;
        if (k0 + j < nw) {
            cnt = min(__ldcg(A.wcount + w0 + k0 + j), (int64_t) A.wtask[w0 + k0 + j].out_cap);
            ob = A.wtask[w0 + k0 + j].out_base;
        }
        long long inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long v = __shfl_up_sync(0xffffffffu, inc, o);
            if (j >= o) inc += v;
        }
        const int m = (int) min((int64_t) 32, nw - k0);
        for (int jj = 0; jj < m; ++jj) {
            const long long c = __shfl_sync(0xffffffffu, cnt, jj);
            const long long at = run + __shfl_sync(0xffffffffu, inc, jj) - c;
            const int4 *src = reinterpret_cast<const int4 *>(A.out + __shfl_sync(0xffffffffu, ob, jj));
            int4 *dst = reinterpret_cast<int4 *>(A.packed + base + at);
            for (long long q = tid; q < 2 * c; q += NT) dst[q] = __ldcg(src + q);
        }
        run += __shfl_sync(0xffffffffu, inc, 31);
    }
    group_sync<NT>();
    if (tid == 0) {
        A.read_base[r] = base;
        A.read_count[r] = tot;
    }
}

// After a group of NT threads (tid 0..NT-1) finished a unit of read r (a traceback window, or the
// check of a stitch between two forward segments), with batches that publish reads as they finish:
// the unit is counted against its read, and the group that finishes the read's last unit gathers
// the read and writes its record to mapped host memory, `done` last after a system-scope fence (the
// host then copies the pairs while the kernel runs on).  A read with a disagreeing stitch gets no
// record: the host re-runs it unsegmented and its result comes from the download.
template <int NT>
__device__ void read_unit_done(const Args &A, int32_t r, int tid, Shared *sh) {
    if (!A.done_host) return;
    __threadfence();   // this thread's pairs, count and total before the count below
    group_sync<NT>();
    int32_t last = -1;
    if (tid == 0) {
        if (atomicAdd(A.read_wdone + r, 1) + 1 == (int32_t) A.read_win[8 * r + 6]) last = r;
        __threadfence();
        if (last >= 0 && __ldcg(A.seg_fail + r)) last = -1;
    }
    if (NT == 32) {
        last = __shfl_sync(0xffffffffu, last, 0);
    } else {
        if (tid == 0) sh->done_read = last;
        __syncthreads();
        last = sh->done_read;
        __syncthreads();
    }
    if (last < 0) return;
    __threadfence();   // the read's other windows, counted before the last increment
    long long base, tot;
    gather_read<NT>(A, last, tid, sh->red, base, tot);
    __threadfence_system();   // this thread's packed pairs before the record
    group_sync<NT>();
    if (tid == 0) {
        const int64_t g0 = A.read_win[8 * last + 2], ng = A.read_win[8 * last + 3];
        const int64_t s0 = A.read_win[8 * last + 4], ns = A.read_win[8 * last + 5];
        double ll = 0.0;
        for (int64_t g = 0; g < ng; ++g) ll += __ldcg(A.loglik + g0 + g);
        // each region's last window is in its last segment's frame: add the stitches' constants
        for (int64_t q = 0; q < ns; ++q) ll += __ldcg(&A.stitch_res[s0 + q].delta);
        ReadDone *rec = A.done_host + last;
        rec->first_pair = base;
        rec->n_pairs = tot;
        rec->log_likelihood = ll;
        rec->status = __ldcg(A.status + last);
        __threadfence_system();
        *((volatile int32_t *) &rec->done) = A.done_seq;
    }
    group_sync<NT>();
}

// CPT: cells per thread of the forward sweep (128 threads per region).  The first claims are
// forward sweeps, one per CTA; once none is left, windows are claimed: one per warp for bands up to
// kWarpWindowWidth cells wide, one per CTA for wider bands.  MINB: CTAs per SM the registers are
// budgeted for (2: 255 registers per thread; 3: 168, with some spilling, for batches bound by their
// total work rather than by one forward chain).
template <int CPT, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) worker_kernel(const __grid_constant__ Args A) {
    extern __shared__ float4 smem_raw[];
    Shared *sh = reinterpret_cast<Shared *>(smem_raw);
    float *area = reinterpret_cast<float *>(sh + 1);
    const int tid = threadIdx.x;
    if (tid < 16) log_add_piece(tid, sh->la[tid]);
    // forward segments
    for (;;) {
        if (tid == 0) {
            const unsigned claim = atomicAdd(&A.ctl->claim, 1u);
            sh->task_id = claim < (unsigned) A.n_segs ? A.order[claim] : -1;
        }
        __syncthreads();
        const int32_t id = sh->task_id;
        if (id < 0) break;
        const Segment sg = A.segs[id];
        Ctx c;
        ctx_init(c, A, sg.region);
        forward_task<CPT>(c, sg, sh, area);
        __syncthreads();
    }
    // traceback windows, in publication order: one per warp for bands up to 128 cells (when the
    // launch configuration asks for it), else one per CTA
    if (CPT == 1 && A.warp_windows) {
        const int lane = tid & 31, warp = tid >> 5;
        float *wring = area + warp * kWarpWindowFloats;
        float *wchain = wring + 9 * (kWarpWindowWidth + 2);
        for (;;) {
            int32_t id = -1;
            if (lane == 0) {
                const unsigned claim = atomicAdd(&A.ctl->wclaim, 1u);
                if ((int64_t) claim < A.n_windows) id = wait_ready(A, claim);
            }
            id = __shfl_sync(0xffffffffu, id, 0);
            if (id < 0) break;
            Ctx c;
            ctx_init(c, A, A.wtask[id].region);
            if (c.t[T_SX] > kNegInf) {
                WarpWindow<kWarpWindowCpt, true> w(c, wring, wchain, sh->la);
                w.run(id);
            } else {
                WarpWindow<kWarpWindowCpt, false> w(c, wring, wchain, sh->la);
                w.run(id);
            }
            read_unit_done<32>(A, c.R.read, lane, sh);
        }
    } else {
        float *ring = area, *chain = area + 9 * (A.wmax + 2);
        for (;;) {
            if (tid == 0) {
                const unsigned claim = atomicAdd(&A.ctl->wclaim, 1u);
                sh->task_id = (int64_t) claim < A.n_windows ? wait_ready(A, claim) : -1;
            }
            __syncthreads();
            const int32_t id = sh->task_id;
            if (id < 0) break;
            Ctx c;
            ctx_init(c, A, A.wtask[id].region);
            if (c.t[T_SX] > kNegInf) window_task<CPT, true>(c, sh, ring, chain, id);
            else window_task<CPT, false>(c, sh, ring, chain, id);
            __syncthreads();
            read_unit_done<kThreads>(A, c.R.read, tid, sh);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// gather: per read, its windows' pairs in order into the packed output
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) gather_pairs(const __grid_constant__ Args A) {
    __shared__ long long red[256 / 32 + 1];
    long long base, tot;
    for (int64_t r = blockIdx.x; r < A.n_reads; r += gridDim.x) {
        gather_read<256>(A, r, threadIdx.x, red, base, tot);
        __syncthreads();
    }
}

}  // namespace fp32
}  // namespace sa
