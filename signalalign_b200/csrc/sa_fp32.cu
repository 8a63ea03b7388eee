// Batched FP32 form: host side.  Plans a batch (band geometry, traceback windows, k-mer ids,
// emission chunks, output segments), owns its device buffers, and runs the three kernels of
// sa_fp32_kernel.cuh: emissions of every band cell, the persistent worker (forward sweeps and
// traceback-window backward sweeps pulled from a device queue), and the per-read gather of pairs.
//
// Every buffer of a batch is placed by one function (layout): the inputs first, staged on the host
// in exactly the device layout so that one copy uploads them; then the small results block, which
// one copy downloads; then the device-only stores.  The device block and the pinned host blocks
// come from reusable pools (sa_memory.cpp); the no-allocation entry lays the same set out in its
// static array and stages on the heap.  Host planning runs on all host threads.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "sa_dp32.cuh"
#include "sa_internal.h"

namespace sa {
namespace fp32 {

using namespace dp32;

}  // namespace fp32
}  // namespace sa

#include "sa_fp32_kernel.cuh"

namespace sa {
namespace fp32 {

// FP32 issue-rate probe for the roofline denominator: 8 independent FMA chains per thread.
__global__ void __launch_bounds__(256) fma_probe(float *sink, int iters, float seed) {
    float a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = seed + threadIdx.x * 1e-7f + i;
    const float m = 0.999999f, c = 1e-7f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = fmaf(a[i], m, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == 12345.678f) sink[0] = s;
}

// Slack after the emission and forward stores: the kernels' clamped look-ahead loads past a
// region's last anti-diagonal stay inside the allocation.
constexpr size_t kStoreSlack = 1024;

// device memory bound of a batch's plain-form reads
constexpr size_t kPlainBatchMaxBytes = (size_t) 64 << 30;

}  // namespace fp32
}  // namespace sa

// ------------------------------------------------------------------------------------------------
// host side of the batch
// ------------------------------------------------------------------------------------------------
using namespace sa;
using namespace sa::fp32;

// a typed view into a host block
template <typename T>
struct Span {
    T *p = nullptr;
    size_t n = 0;
    T *data() const { return p; }
    size_t size() const { return n; }
    T &operator[](size_t i) const { return p[i]; }
};

// ------------------------------------------------------------------------------------------------
// launch configurations of the batched kernels, per device name and band-width class
// ------------------------------------------------------------------------------------------------
namespace {

std::mutex g_launch_mutex;
std::map<std::pair<std::string, int>, sa_launch_config> g_launch;   // (device name, width class)

// the choices measured on B200: two worker CTAs per SM, at most three CTAs per region (a forward CTA
// and about two CTAs of window warps, so small batches on other streams run beside it), a window
// per warp for bands up to 128 cells, 16 emission CTAs per SM
sa_launch_config default_launch() { return sa_launch_config{2, 3, 1, 16}; }

bool valid_launch(const sa_launch_config &c) {
    return c.ctas_per_sm >= 1 && c.ctas_per_sm <= 32 && c.grid_per_region >= 1 && c.grid_per_region <= 64 &&
           (c.warp_windows == 0 || c.warp_windows == 1) && c.emission_ctas_per_sm >= 1 &&
           c.emission_ctas_per_sm <= 64;
}

bool valid_width_class(int w) { return w == 1 || w == 2 || w == 4; }

std::string device_name(int device) {
    static std::mutex m;
    static std::map<int, std::string> names;
    std::lock_guard<std::mutex> lock(m);
    auto it = names.find(device);
    if (it != names.end()) return it->second;
    cudaDeviceProp prop;
    std::string name;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) name = prop.name;
    else cudaGetLastError();
    if (!name.empty()) names[device] = name;
    return name;
}

sa_launch_config launch_for(int device, int width_class) {
    const std::string name = device_name(device);
    std::lock_guard<std::mutex> lock(g_launch_mutex);
    auto it = g_launch.find({name, width_class});
    return it != g_launch.end() ? it->second : default_launch();
}

}  // namespace

struct sa_batch {
    int device = 0;
    int64_t n_reads = 0;
    bool host_pinned = true;      // staging and results in pinned pool blocks (else heap)
    bool owns_device = true;      // device block from the pool (else memory of the caller)
    std::vector<sa_state_machine *> models;
    std::vector<int32_t> read_status;       // host planning status per read
    std::vector<int64_t> read_first_region, read_n_regions;
    int64_t n_regions = 0, n_diags = 0, n_windows = 0, n_chunks = 0, n_kmers = 0, n_events = 0;
    int64_t n_segs = 0, n_stitch = 0, stitch_floats = 0;
    int64_t cells = 0, out_total = 0;
    int32_t max_width = 0;
    float threshold = 0.01f;
    // inputs, staged on the host with the device layout (one copy uploads them all)
    Span<RegionDesc> regions;
    Span<Segment> segs;
    Span<int32_t> order;
    Span<StitchDesc> stitch;
    Span<ModelDesc> mdesc;
    Span<ReadScale32> read_scale;
    Span<ReadScale64> read_scale64;
    Span<int2> meta;
    Span<Window> windows;
    Span<WindowTask> wtask;
    Span<Chunk> chunks;
    Span<int32_t> kmer;
    Span<float> gapx;
    Span<double2> events;
    Span<int64_t> read_win;                 // per read: first window, window count, first region, region
                                            // count, first stitch, stitch count, units, 0
    // results, mirrored from one contiguous device range (one copy downloads them all)
    Span<int64_t> read_base, read_count;
    Span<double> loglik;
    Span<int32_t> dev_status;
    Span<int32_t> read_wdone;
    Span<int32_t> seg_fail;
    Span<StitchRes> stitch_res;
    Span<Control> ctl;
    size_t in_bytes = 0, res_off = 0, res_bytes = 0, dev_bytes = 0;
    // device pointers
    RegionDesc *d_regions = nullptr;
    Segment *d_segs = nullptr;
    int32_t *d_order = nullptr;
    StitchDesc *d_stitch = nullptr;
    StitchRes *d_stitch_res = nullptr;
    float *d_stitch_vals = nullptr;
    int32_t *d_seg_fail = nullptr;
    Segment *d_redo_segs = nullptr;         // reads re-run unsegmented after a disagreeing stitch
    int32_t *d_redo_order = nullptr;
    ModelDesc *d_models = nullptr;
    ReadScale32 *d_read_scale = nullptr;
    ReadScale64 *d_read_scale64 = nullptr;
    int2 *d_meta = nullptr;
    Window *d_windows = nullptr;
    WindowTask *d_wtask = nullptr;
    Chunk *d_chunks = nullptr;
    int32_t *d_kmer = nullptr;
    float *d_gapx = nullptr;
    double2 *d_events_raw = nullptr;
    int64_t *d_read_win = nullptr;
    int64_t *d_read_base = nullptr, *d_read_count = nullptr;
    double *d_loglik = nullptr;
    int32_t *d_status = nullptr;
    int32_t *d_read_wdone = nullptr;
    Control *d_ctl = nullptr;
    Event32 *d_events = nullptr;
    float *d_E = nullptr, *d_F = nullptr, *d_fshift = nullptr;
    double *d_base = nullptr;
    int32_t *d_ready = nullptr;
    sa_aligned_pair *d_out = nullptr, *d_packed = nullptr;
    int64_t *d_wcount = nullptr;
    // memory
    MemBlock host_in, host_res, host_pairs, dev;
    MemBlock host_done;                     // per-read completion records (mapped pinned memory)
    ReadDone *d_done = nullptr;             // their device address
    int32_t run_seq = 0;                    // runs with per-read completion (a record's `done`)
    unsigned char *dev_base = nullptr;
    std::vector<double> read_ll;
    bool downloaded = false;
    long long wait_limit = 20000000000LL;   // clock cycles a worker may wait for a window (~10 s)
    float stitch_tol = 1.0f;                // scale of the stitch tolerance (negative: all disagree)
    std::vector<char> redone;               // per read: re-run unsegmented after a disagreement
    int64_t n_redone = 0;
    bool has_cfg = false;                   // the tuner's candidate instead of the device's table
    sa_launch_config cfg{};
    int width_class = 1;
    // device timing of the last run's kernels (batches that own their device memory only)
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool timed = false;
    // reads whose references have degenerate positions (multi-path cells), or whose machine's gap-Y
    // table does not follow its match table, run in the plain FP64 form
    std::vector<int64_t> plain_of;          // per read: its index in `plain`, or -1
    std::vector<sa_read> plain_reads;
    PlainSet *plain = nullptr;

    ~sa_batch() {
        if (plain) plain_destroy(plain);
        for (cudaEvent_t &e : ev)
            if (e) cudaEventDestroy(e);
        mem_put(host_in);
        mem_put(host_res);
        mem_put(host_pairs);
        mem_put(host_done);
        if (owns_device) mem_put(dev);
    }
};

namespace {

// Lays out the batch's buffers, 256-byte aligned, in three groups: inputs (staged on the host in
// the same layout), results (mirrored to the host), work buffers (device only).  With non-null bases
// the host spans and device pointers are set.  Returns the device bytes; sets in/res offsets.
size_t layout(sa_batch *b, unsigned char *host_in, unsigned char *host_res, unsigned char *dev) {
    size_t at = 0;
    auto place = [&](auto &span, auto *&dptr, size_t n, unsigned char *host, size_t host_origin) {
        using T = std::remove_reference_t<decltype(*dptr)>;
        at = (at + 255) & ~(size_t) 255;
        if (host) {
            span.p = reinterpret_cast<T *>(host + (at - host_origin));
            span.n = n;
        }
        if (dev) dptr = reinterpret_cast<T *>(dev + at);
        at += std::max<size_t>(n, 1) * sizeof(T);
    };
    auto work = [&](auto *&dptr, size_t n) {
        using T = std::remove_reference_t<decltype(*dptr)>;
        at = (at + 255) & ~(size_t) 255;
        if (dev) dptr = reinterpret_cast<T *>(dev + at);
        at += std::max<size_t>(n, 1) * sizeof(T);
    };
    const size_t nr = (size_t) b->n_regions, nd = (size_t) b->n_diags, nw = (size_t) b->n_windows;
    const size_t nreads = (size_t) b->n_reads, cells = (size_t) b->cells;
    place(b->regions, b->d_regions, nr, host_in, 0);
    place(b->segs, b->d_segs, (size_t) b->n_segs, host_in, 0);
    place(b->order, b->d_order, (size_t) b->n_segs, host_in, 0);
    place(b->stitch, b->d_stitch, (size_t) b->n_stitch, host_in, 0);
    place(b->mdesc, b->d_models, b->models.size(), host_in, 0);
    place(b->read_scale, b->d_read_scale, nreads, host_in, 0);
    place(b->read_scale64, b->d_read_scale64, nreads, host_in, 0);
    place(b->meta, b->d_meta, nd, host_in, 0);
    place(b->windows, b->d_windows, nw, host_in, 0);
    place(b->wtask, b->d_wtask, nw, host_in, 0);
    place(b->chunks, b->d_chunks, (size_t) b->n_chunks, host_in, 0);
    place(b->kmer, b->d_kmer, (size_t) b->n_kmers, host_in, 0);
    place(b->gapx, b->d_gapx, (size_t) b->n_kmers, host_in, 0);
    place(b->events, b->d_events_raw, (size_t) b->n_events, host_in, 0);
    place(b->read_win, b->d_read_win, 8 * nreads, host_in, 0);
    b->in_bytes = (at + 255) & ~(size_t) 255;
    at = b->in_bytes;
    b->res_off = at;
    place(b->read_base, b->d_read_base, nreads, host_res, b->res_off);
    place(b->read_count, b->d_read_count, nreads, host_res, b->res_off);
    place(b->loglik, b->d_loglik, nr, host_res, b->res_off);
    place(b->dev_status, b->d_status, nreads, host_res, b->res_off);
    place(b->read_wdone, b->d_read_wdone, nreads, host_res, b->res_off);
    place(b->seg_fail, b->d_seg_fail, nreads, host_res, b->res_off);
    place(b->stitch_res, b->d_stitch_res, (size_t) b->n_stitch, host_res, b->res_off);
    place(b->ctl, b->d_ctl, 1, host_res, b->res_off);
    b->res_bytes = ((at + 255) & ~(size_t) 255) - b->res_off;
    work(b->d_events, (size_t) b->n_events);
    work(b->d_E, 2 * cells + kStoreSlack);
    work(b->d_F, 3 * cells + kStoreSlack);
    work(b->d_base, nd);
    work(b->d_fshift, nd);
    work(b->d_ready, nw);
    work(b->d_out, (size_t) b->out_total);
    work(b->d_wcount, nw);
    work(b->d_packed, (size_t) b->out_total);
    work(b->d_stitch_vals, (size_t) b->stitch_floats);
    work(b->d_redo_segs, nr);
    work(b->d_redo_order, nr);
    b->dev_bytes = (at + 255) & ~(size_t) 255;
    return b->dev_bytes;
}

// Runs fn(i) for i in [0, n) on up to `threads` host threads (the calling thread included).
template <typename Fn>
void parallel_for(int64_t n, int threads, Fn &&fn) {
    threads = (int) std::max<int64_t>(1, std::min<int64_t>(threads, n));
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (int64_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) fn(i);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
}

int planning_threads() {
    if (const char *e = std::getenv("SA_PLAN_THREADS")) {
        const int v = std::atoi(e);
        if (v > 0) return v;
    }
    return (int) std::max(1u, std::thread::hardware_concurrency());
}

// Forward segments.  A region's forward sweep is cut at traceback-window starts into segments that
// run at the same time; every later segment first sweeps `warm` anti-diagonals from a flat start.
// Policy: segment_diags < 0 keeps every region whole, > 0 caps a segment's sweep (warm-up included)
// at that many anti-diagonals, 0 picks the cap from the batch: twice the forward anti-diagonals per
// worker CTA, at least kSegMin.  A batch's worker time is about the larger of its longest forward
// chain and its total work (forward and traceback-window work per anti-diagonal together cost about
// twice a worker CTA's forward step, measured on B200), so only chains longer than the total work
// are cut: a large batch keeps nearly every region whole (no warm-up overhead), a small one (a
// serving micro-batch) splits its long reads for latency.
std::atomic<int32_t> g_seg_target{0};
std::atomic<int32_t> g_seg_warm{1024};
constexpr int64_t kSegMin = 4096;

// Warm-up of a region's later segments: the start's influence dies out over a few band widths
// (measured on the oracle's FP64 sweep: within 4.2 widths at diagonal expansion 50, 5.9 at 200), so
// ten widths of the region's widest anti-diagonal, and at least the policy's warm-up.
int32_t region_warm(const Region &rg, int32_t warm) { return std::max<int32_t>(warm, 10 * rg.max_width); }

// Window indices (>= 1) whose T starts a new segment of region rg: k pieces of about equal sweep
// time (L + warm each; the first piece owns L + warm anti-diagonals and needs no warm-up, and L is
// at least warm), each cut at the first window start at or after its ideal place, none leaving less
// than L / 2 behind.
void plan_cuts(const Region &rg, int64_t target, int32_t warm, std::vector<int32_t> &cuts) {
    cuts.clear();
    const int64_t n = rg.lX + rg.lY;
    if (target <= (int64_t) warm + 64 || n <= target) return;
    // pieces: sweeps of at most `target`, and none owning fewer anti-diagonals than its warm-up
    const int64_t k = std::min((n - warm + (target - warm) - 1) / (target - warm), (n - warm) / warm);
    if (k < 2) return;
    const double L = (double) (n - warm) / (double) k;
    size_t j = 1;
    for (int64_t i = 1; i < k; ++i) {
        const double want = (double) warm + (double) i * L;
        while (j < rg.windows.size() && (double) rg.windows[j].T < want) ++j;
        if (j >= rg.windows.size() || (double) (n - rg.windows[j].T) < L / 2) break;
        cuts.push_back((int32_t) j);
        ++j;
    }
}

// one read's plan before packing
struct ReadPlan {
    sa_status status = SA_OK;
    bool plain = false;         // degenerate positions, or a machine whose gap-Y table has its own
                                // level mean or noise: aligned by the plain FP64 form
    int32_t model = -1;
    int64_t lX = 0;
    std::vector<int32_t> kid;   // k-mer id per column 1..lX
    std::vector<Region> regs;
    std::vector<std::vector<int32_t>> cuts;   // per region: windows that start a forward segment
    int64_t diags = 0, cells = 0, windows = 0, chunks = 0, out = 0;
    int64_t segs = 0, stitches = 0, stitch_floats = 0;
    int32_t max_width = 0;
    // packing offsets
    int64_t region_base = 0, diag_base = 0, cell_base = 0, win_base = 0, chunk_base = 0, kmer_base = 0,
            event_base = 0, out_base = 0, seg_base = 0, stitch_base = 0, stitch_voff = 0;
};

int32_t band_width(const Region &rg, int64_t d) { return (rg.xmy_r[d] - rg.xmy_l[d]) / 2 + 1; }

// Host planning of a batch (no device work): per read its regions and their windows (in parallel
// over reads), then the packed inputs, written straight into a host staging block (pinned when
// `pinned`): per region its descriptor, per-anti-diagonal meta and emission chunks, per window its
// task and output segment, per read its k-mer ids, skip emissions and events; and the LPT order.
// Returns SA_E_CAPACITY for a band wider than the kernel's widest ring.
sa_status plan_batch(const sa_read *reads, int64_t n_reads, const sa_params *p, bool pinned, sa_batch *b) {
    b->n_reads = n_reads;
    b->host_pinned = pinned;
    b->threshold = (float) p->threshold;
    b->read_status.assign(n_reads, SA_OK);
    b->read_first_region.assign(n_reads, 0);
    b->read_n_regions.assign(n_reads, 0);
    std::vector<ReadScale32> scale(n_reads);
    std::vector<ReadScale64> scale64(n_reads);
    std::vector<ReadPlan> plan(n_reads);
    // arguments, devices and models (serial: models are shared)
    int device = -1;
    for (int64_t r = 0; r < n_reads; ++r) {
        const sa_read &rd = reads[r];
        ReadPlan &rp = plan[r];
        auto *sm = const_cast<sa_state_machine *>(rd.sm);
        std::memset(&scale[r], 0, sizeof(ReadScale32));
        scale64[r] = ReadScale64{1.0, 0.0, 1.0, 0.0};
        if (!sm || rd.reference_length < 0 || rd.n_events < 0 || rd.n_anchors < 0 ||
            (rd.reference_length > 0 && !rd.reference) || (rd.n_events > 0 && !rd.events) ||
            (rd.n_anchors > 0 && !rd.anchors) || !(rd.var != 0.0)) {
            rp.status = SA_E_ARG;
            continue;
        }
        if (device < 0) device = sm->dev.device;
        if (sm->dev.device != device) { rp.status = SA_E_ARG; continue; }
        if (sm->emission == SA_EMIT_HDP && !sm->hdp.present) { rp.status = SA_E_UNSUPPORTED; continue; }
        const int k = sm->kmer_length;
        rp.lX = rd.reference_length == 0 ? 0 : rd.reference_length - (k - 1);
        if (rp.lX < 0) { rp.status = SA_E_ARG; continue; }
        for (size_t i = 0; i < b->models.size(); ++i)
            if (b->models[i] == sm) rp.model = (int32_t) i;
        if (rp.model < 0) { rp.model = (int32_t) b->models.size(); b->models.push_back(sm); }
        const double var = sm->emission == SA_EMIT_PLAIN ? 1.0 : rd.var;
        ReadScale32 &rs = scale[r];
        rs.scale = sm->emission == SA_EMIT_PLAIN ? 1.0f : (float) rd.scale;
        rs.shift = sm->emission == SA_EMIT_PLAIN ? 0.0f : (float) rd.shift;
        rs.inv_var = (float) (1.0 / var);
        rs.log_inv_var = (float) std::log(1.0 / var);
        scale64[r] = ReadScale64{sm->emission == SA_EMIT_PLAIN ? 1.0 : rd.scale, sm->emission == SA_EMIT_PLAIN ? 0.0 : rd.shift,
                                 var, 0.0};
    }
    std::vector<char> fp32_tables(b->models.size());
    for (size_t i = 0; i < b->models.size(); ++i) fp32_tables[i] = gapy_follows_match(b->models[i]);
    // a thread per few reads: starting a thread costs about as much as planning a short read, so
    // micro-batches of a few reads (a serving loop's) plan on the calling thread alone
    const int threads = (int) std::min<int64_t>(planning_threads(), std::max<int64_t>(1, n_reads / 4));
    // k-mer ids, regions and windows of each read
    parallel_for(n_reads, threads, [&](int64_t r) {
        ReadPlan &rp = plan[r];
        if (rp.status) return;
        const sa_read &rd = reads[r];
        PathTable pt;
        sa_status st = build_paths(rd.sm, rd.reference, rp.lX, rd.degenerate, pt);
        if (!st && (pt.multi || !fp32_tables[rp.model])) {
            rp.plain = true;
            return;
        }
        if (!st)
            st = plan_regions(rd.anchors, rd.n_anchors, rp.lX, rd.n_events, *p, rd.ragged_left != 0,
                              rd.ragged_right != 0, rp.regs);
        if (st) {
            rp.status = st;
            rp.regs.clear();
            return;
        }
        rp.kid.resize(rp.lX);
        for (int64_t x = 1; x <= rp.lX; ++x) rp.kid[x - 1] = pt.ids[pt.first[x]];
        for (const Region &rg : rp.regs) {
            const int64_t n = rg.lX + rg.lY;
            rp.diags += n + 1;
            rp.cells += rg.cells;
            rp.windows += (int64_t) rg.windows.size();
            rp.chunks += (n + kChunkDiags) / kChunkDiags;
            for (const Window &w : rg.windows) rp.out += 4 * (int64_t) (w.from - w.T) + 64;
            rp.max_width = std::max(rp.max_width, rg.max_width);
        }
    });
    // forward segments: the cap from the policy and the batch's forward anti-diagonals per worker CTA
    {
        int64_t fwd_diags = 0;
        int32_t mw = 0;
        for (int64_t r = 0; r < n_reads; ++r) {
            fwd_diags += plan[r].diags;
            mw = std::max(mw, plan[r].max_width);
        }
        const int32_t policy = g_seg_target.load(), warm = g_seg_warm.load();
        int64_t target = policy;
        if (policy == 0) {
            const int cpt = std::max(1, (mw + kThreads - 1) / kThreads);
            const int wc = cpt <= 1 ? 1 : (cpt <= 2 ? 2 : 4);
            int sms = 0;
            if (device < 0 || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
                cudaGetLastError();
                sms = 0;
            }
            if (sms <= 0) sms = 148;
            const int64_t slots = (int64_t) sms * std::max(1, launch_for(std::max(device, 0), wc).ctas_per_sm);
            target = std::max<int64_t>(kSegMin, 2 * fwd_diags / slots);
        }
        for (int64_t r = 0; r < n_reads; ++r) {
            ReadPlan &rp = plan[r];
            rp.cuts.assign(rp.regs.size(), {});
            for (size_t gi = 0; gi < rp.regs.size(); ++gi) {
                const Region &rg = rp.regs[gi];
                if (policy >= 0) plan_cuts(rg, target, region_warm(rg, warm), rp.cuts[gi]);
                rp.segs += 1 + (int64_t) rp.cuts[gi].size();
                rp.stitches += (int64_t) rp.cuts[gi].size();
                for (int32_t j : rp.cuts[gi]) {
                    const int32_t bd = rg.windows[j].T;
                    rp.stitch_floats += 6 * (int64_t) (band_width(rg, bd - 1) + band_width(rg, bd));
                }
            }
        }
    }
    // packing offsets
    int64_t nreg = 0, ndiag = 0, ncell = 0, nwin = 0, nchunk = 0, nkmer = 0, nevent = 0, nout = 0;
    int64_t nseg = 0, nstitch = 0, nsfloat = 0;
    for (int64_t r = 0; r < n_reads; ++r) {
        ReadPlan &rp = plan[r];
        b->read_status[r] = rp.status;
        rp.region_base = nreg; rp.diag_base = ndiag; rp.cell_base = ncell; rp.win_base = nwin;
        rp.chunk_base = nchunk; rp.kmer_base = nkmer; rp.event_base = nevent; rp.out_base = nout;
        rp.seg_base = nseg; rp.stitch_base = nstitch; rp.stitch_voff = nsfloat;
        b->read_first_region[r] = nreg;
        b->read_n_regions[r] = (int64_t) rp.regs.size();
        nreg += (int64_t) rp.regs.size(); ndiag += rp.diags; ncell += rp.cells; nwin += rp.windows;
        nchunk += rp.chunks; nout += rp.out;
        nseg += rp.segs; nstitch += rp.stitches; nsfloat += rp.stitch_floats;
        if (!rp.status && !rp.plain) {
            nkmer += rp.lX;
            nevent += reads[r].n_events;
        }
        b->max_width = std::max(b->max_width, rp.max_width);
    }
    b->plain_of.assign(n_reads, -1);
    for (int64_t r = 0; r < n_reads; ++r)
        if (plan[r].plain && !plan[r].status) {
            b->plain_of[r] = (int64_t) b->plain_reads.size();
            b->plain_reads.push_back(reads[r]);
        }
    if (b->max_width > kMaxCpt * kThreads) return SA_E_CAPACITY;
    b->device = device < 0 ? 0 : device;
    b->n_regions = nreg; b->n_diags = ndiag; b->n_windows = nwin; b->n_chunks = nchunk;
    b->n_segs = nseg; b->n_stitch = nstitch; b->stitch_floats = nsfloat;
    b->n_kmers = nkmer; b->n_events = nevent;
    b->cells = ncell;
    b->out_total = nout;
    layout(b, nullptr, nullptr, nullptr);
    sa_status st = mem_get(pinned ? MemKind::Pinned : MemKind::Heap, b->device, b->in_bytes, b->host_in);
    if (st) return st;
    layout(b, static_cast<unsigned char *>(b->host_in.ptr), nullptr, nullptr);
    for (int64_t r = 0; r < n_reads; ++r) {
        b->read_scale[r] = scale[r];
        b->read_scale64[r] = scale64[r];
        b->read_win[8 * r] = plan[r].win_base;
        b->read_win[8 * r + 1] = plan[r].windows;
        b->read_win[8 * r + 2] = plan[r].region_base;
        b->read_win[8 * r + 3] = (int64_t) plan[r].regs.size();
        b->read_win[8 * r + 4] = plan[r].stitch_base;
        b->read_win[8 * r + 5] = plan[r].stitches;
        b->read_win[8 * r + 6] = plan[r].windows + plan[r].stitches;
        b->read_win[8 * r + 7] = 0;
    }
    // the packed inputs, read by read
    parallel_for(n_reads, threads, [&](int64_t r) {
        const ReadPlan &rp = plan[r];
        if (rp.status || rp.plain) return;
        const sa_read &rd = reads[r];
        const sa_state_machine *sm = rd.sm;
        for (int64_t x = 0; x < rp.lX; ++x) {
            const int32_t kid = rp.kid[x];
            b->kmer[rp.kmer_base + x] = kid;
            b->gapx[rp.kmer_base + x] = sm->emission == SA_EMIT_HDP ? (float) kLogPointOne : (float) sm->gapx[kid];
        }
        for (int64_t y = 0; y < rd.n_events; ++y)
            b->events[rp.event_base + y] = make_double2(rd.events[y * kEventParams], rd.events[y * kEventParams + 1]);
        int64_t dbase = rp.diag_base, cbase = rp.cell_base, wbase = rp.win_base, chbase = rp.chunk_base,
                obase = rp.out_base, sgbase = rp.seg_base, stbase = rp.stitch_base, vbase = rp.stitch_voff;
        const int32_t warm = g_seg_warm.load();
        std::vector<int32_t> flags;
        std::vector<int64_t> off;
        for (size_t gi = 0; gi < rp.regs.size(); ++gi) {
            const Region &rg = rp.regs[gi];
            const int32_t region = (int32_t) (rp.region_base + (int64_t) gi);
            RegionDesc d;
            std::memset(&d, 0, sizeof(d));
            d.n = (int32_t) (rg.lX + rg.lY);
            d.lX = (int32_t) rg.lX;
            d.lY = (int32_t) rg.lY;
            d.read = (int32_t) r;
            d.n_windows = (int32_t) rg.windows.size();
            d.model = rp.model;
            d.ragged_left = rg.ragged_left;
            d.ragged_right = rg.ragged_right;
            d.diag_base = dbase;
            d.cell_base = cbase;
            d.win_base = wbase;
            d.kmer_base = rp.kmer_base + rg.x1;
            d.event_base = rp.event_base + rg.y1;
            d.x1 = rg.x1;
            d.y1 = rg.y1;
            // per anti-diagonal meta: band start, width, window end / refresh / stored gap states
            flags.assign(d.n + 2, 0);
            // a window is published once the forward sweep has passed the last anti-diagonal it
            // reads (`from`), not its traceback anti-diagonal D: its backward sweep from D reads
            // emissions only above `from`
            for (const Window &w : rg.windows) {
                flags[w.from] |= kFlagWindowEnd;
                for (int32_t q = w.from; q > w.T; q -= 10) flags[q] |= kFlagRefresh;
            }
            off.resize(d.n + 1);
            int64_t acc = 0;
            for (int32_t dd = 0; dd <= d.n; ++dd) {
                const int32_t w = (rg.xmy_r[dd] - rg.xmy_l[dd]) / 2 + 1;
                int32_t f = flags[dd];
                if ((flags[dd] | flags[dd + 1]) & kFlagRefresh) f |= kFlagStoreGaps;
                b->meta[dbase + dd] = make_int2(rg.xmy_l[dd], w | f);
                off[dd] = acc;
                acc += w;
            }
            for (int32_t d0 = 0; d0 <= d.n; d0 += kChunkDiags) {
                Chunk &ch = b->chunks[chbase++];
                ch.region = region;
                ch.d0 = d0;
                ch.nd = std::min(kChunkDiags, d.n + 1 - d0);
                ch.pad = 0;
                ch.cell = cbase + off[d0];
            }
            for (size_t wi = 0; wi < rg.windows.size(); ++wi) {
                const Window &w = rg.windows[wi];
                WindowTask &t = b->wtask[wbase + (int64_t) wi];
                t.region = region;
                t.first_cell = (int32_t) off[w.D];
                t.out_cap = 4 * (w.from - w.T) + 64;
                t.side = -1;
                t.out_base = obase;
                obase += t.out_cap;
                b->windows[wbase + (int64_t) wi] = w;
            }
            // forward segments and the stitches between them
            const std::vector<int32_t> &cuts = rp.cuts[gi];
            for (size_t q = 0; q <= cuts.size(); ++q) {
                Segment sg;
                std::memset(&sg, 0, sizeof(sg));
                sg.region = region;
                sg.d_begin = q == 0 ? 0 : rg.windows[cuts[q - 1]].T;
                sg.d_end = q == cuts.size() ? d.n : rg.windows[cuts[q]].T;
                sg.stitch_in = q == 0 ? -1 : (int32_t) (stbase + (int64_t) q - 1);
                sg.stitch_out = q == cuts.size() ? -1 : (int32_t) (stbase + (int64_t) q);
                if (q == 0) {
                    sg.warm = 0;
                    sg.wi0 = 0;
                    sg.cell0 = 1;   // anti-diagonal 0 has one cell
                } else {
                    // warm = 2 mod 3: d_begin closes a group of three steps of the sweep
                    const int32_t wr = region_warm(rg, warm);
                    sg.warm = wr + ((2 - wr) % 3 + 3) % 3;
                    sg.wi0 = cuts[q - 1];
                    sg.cell0 = off[sg.d_begin - sg.warm];
                }
                b->segs[sgbase + (int64_t) q] = sg;
            }
            for (size_t q = 0; q < cuts.size(); ++q) {
                const int32_t bd = rg.windows[cuts[q]].T;
                StitchDesc &sd = b->stitch[stbase + (int64_t) q];
                sd.region = region;
                sd.read = (int32_t) r;
                sd.w0 = band_width(rg, bd - 1);
                sd.w1 = band_width(rg, bd);
                sd.voff = vbase;
                vbase += 6 * (int64_t) (sd.w0 + sd.w1);
                b->wtask[wbase + cuts[q]].side = (int32_t) (stbase + (int64_t) q);
            }
            sgbase += 1 + (int64_t) cuts.size();
            stbase += (int64_t) cuts.size();
            b->regions[region] = d;
            dbase += d.n + 1;
            cbase += acc;
            wbase += (int64_t) rg.windows.size();
        }
    });
    // longest sweep first (LPT order of the forward claims)
    std::vector<int32_t> order(nseg);
    std::iota(order.begin(), order.end(), 0);
    std::vector<int64_t> len(nseg);
    for (int64_t i = 0; i < nseg; ++i) len[i] = (int64_t) b->segs[i].d_end - b->segs[i].d_begin + b->segs[i].warm;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t c) { return len[a] > len[c]; });
    std::copy(order.begin(), order.end(), b->order.data());
    b->redone.assign(n_reads, 0);
    b->n_redone = 0;
    return SA_OK;
}

// kernel arguments of a batch's run (launch-dependent fields set by the caller)
Args batch_args(const sa_batch *b) {
    Args a;
    std::memset(&a, 0, sizeof(a));
    a.regions = b->d_regions;
    a.n_regions = b->n_regions;
    a.segs = b->d_segs;
    a.order = b->d_order;
    a.n_segs = b->n_segs;
    a.stitch = b->d_stitch;
    a.stitch_res = b->d_stitch_res;
    a.stitch_vals = b->d_stitch_vals;
    a.seg_fail = b->d_seg_fail;
    a.stitch_tol = b->stitch_tol;
    a.use_side = 1;
    a.models = b->d_models;
    a.read_scale = b->d_read_scale;
    a.read_scale64 = b->d_read_scale64;
    a.events_raw = b->d_events_raw;
    a.meta = b->d_meta;
    a.windows = b->d_windows;
    a.wtask = b->d_wtask;
    a.n_windows = b->n_windows;
    a.chunks = b->d_chunks;
    a.n_chunks = b->n_chunks;
    a.kmer = b->d_kmer;
    a.gapx = b->d_gapx;
    a.events = b->d_events;
    a.E = b->d_E;
    a.F = b->d_F;
    a.base = b->d_base;
    a.fshift = b->d_fshift;
    a.ready = b->d_ready;
    a.out = b->d_out;
    a.wcount = b->d_wcount;
    a.loglik = b->d_loglik;
    a.status = b->d_status;
    a.ctl = b->d_ctl;
    a.threshold = b->threshold;
    a.n_reads = b->n_reads;
    a.read_win = b->d_read_win;
    a.packed = b->d_packed;
    a.read_base = b->d_read_base;
    a.read_count = b->d_read_count;
    a.read_wdone = b->d_read_wdone;
    a.done_host = b->d_done;
    a.done_seq = b->run_seq;
    const int cpt = std::max(1, (b->max_width + kThreads - 1) / kThreads);
    a.wmax = (cpt <= 1 ? 1 : (cpt <= 2 ? 2 : 4)) * kThreads;
    a.warp_windows = 1;
    a.spin_limit = b->wait_limit;
    return a;
}

// the persistent worker over a.n_segs forward segments and a.n_windows windows
void launch_worker(const sa_batch *b, const Args &a, const sa_launch_config &cfg, int sms, cudaStream_t s) {
    const int cls = a.wmax / kThreads;
    const size_t smem = sizeof(Shared) + sizeof(float) * (size_t) worker_area_floats(cls);
    auto launch = [&](auto kern) {
        int per_sm = 0;
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
        per_sm = std::max(1, std::min(per_sm, cfg.ctas_per_sm));
        const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((int64_t) sms * per_sm,
                                                                    (int64_t) cfg.grid_per_region * a.n_segs));
        kern<<<(unsigned) grid, kThreads, smem, s>>>(a);
    };
    if (cls == 1 && cfg.ctas_per_sm >= 3) launch(worker_kernel<1, 3>);
    else if (cls == 1) launch(worker_kernel<1, 2>);
    else if (cls == 2) launch(worker_kernel<2, 1>);
    else launch(worker_kernel<4, 1>);
}

// Reads whose stitch disagreed run again with every region as one segment (after the batch's
// results were downloaded): their windows are re-run and every read re-gathered.  The stitch
// tolerance makes this rare; the redo keeps the result exact whatever the input.
sa_status redo_disagreed(sa_batch *b, cudaStream_t s) {
    std::vector<Segment> segs;
    int64_t nwin = 0;
    for (int64_t r = 0; r < b->n_reads; ++r) {
        if (!b->seg_fail[r] || b->redone[r]) continue;
        b->redone[r] = 1;
        ++b->n_redone;
        for (int64_t g = b->read_first_region[r]; g < b->read_first_region[r] + b->read_n_regions[r]; ++g) {
            Segment sg;
            std::memset(&sg, 0, sizeof(sg));
            sg.region = (int32_t) g;
            sg.d_end = b->regions[g].n;
            sg.stitch_in = sg.stitch_out = -1;
            sg.cell0 = 1;
            segs.push_back(sg);
            nwin += b->regions[g].n_windows;
        }
    }
    if (segs.empty()) return SA_OK;
    std::vector<int32_t> order(segs.size());
    std::iota(order.begin(), order.end(), 0);
    const size_t nw = (size_t) std::max<int64_t>(1, nwin);
    if (cudaMemcpyAsync(b->d_redo_segs, segs.data(), sizeof(Segment) * segs.size(), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(b->d_redo_order, order.data(), sizeof(int32_t) * order.size(), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemsetAsync(b->d_ctl, 0, sizeof(Control), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_ready, 0xff, sizeof(int32_t) * nw, s) != cudaSuccess)
        return SA_E_CUDA;
    Args a = batch_args(b);
    a.segs = b->d_redo_segs;
    a.order = b->d_redo_order;
    a.n_segs = (int64_t) segs.size();
    a.n_windows = nwin;
    a.use_side = 0;          // T of every window comes from the unsegmented sweep's store
    a.done_host = nullptr;   // every read is gathered below
    const sa_launch_config cfg = b->has_cfg ? b->cfg : launch_for(b->device, a.wmax / kThreads);
    a.warp_windows = cfg.warp_windows;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    sms = std::max(1, sms);
    launch_worker(b, a, cfg, sms, s);
    gather_pairs<<<(unsigned) std::max<int64_t>(1, std::min<int64_t>(b->n_reads, sms * 4)), 256, 0, s>>>(a);
    count_launch(2);
    // the pages the host reads in the pageable copies above stay alive until the stream drains
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return SA_E_CUDA;
    return SA_OK;
}

}  // namespace

extern "C" {

sa_status sa_batch_create(const sa_read *reads, int64_t n_reads, const sa_params *p, sa_batch **out) {
    if (!reads || n_reads < 0 || !p || !out) return SA_E_ARG;
    *out = nullptr;
    sa_status st = check_params(*p);
    if (st) return st;
    auto *b = new (std::nothrow) sa_batch();
    if (!b) return SA_E_NOMEM;
    st = plan_batch(reads, n_reads, p, true, b);
    if (!st) {
        int prev = 0;
        cudaGetDevice(&prev);
        if (cudaSetDevice(b->device) != cudaSuccess) st = SA_E_CUDA;
        for (auto *sm : b->models)
            if (!st) st = ensure_device_model(sm);
        cudaSetDevice(prev);
    }
    if (!st && !b->plain_reads.empty()) {
        st = plain_create(b->plain_reads.data(), (int64_t) b->plain_reads.size(), *p, kPlainBatchMaxBytes, &b->plain,
                          true);
        if (!st && plain_device(b->plain) != b->device) st = SA_E_ARG;
    }
    if (!st) st = mem_get(MemKind::Device, b->device, b->dev_bytes, b->dev);
    if (!st) st = mem_get(MemKind::Pinned, b->device, b->res_bytes, b->host_res);
    if (st) {
        delete b;
        return st;
    }
    b->dev_base = static_cast<unsigned char *>(b->dev.ptr);
    layout(b, static_cast<unsigned char *>(b->host_in.ptr), static_cast<unsigned char *>(b->host_res.ptr), b->dev_base);
    *out = b;
    return SA_OK;
}

sa_status sa_batch_upload(sa_batch *b, void *stream) {
    if (!b) return SA_E_ARG;
    cudaStream_t s = (cudaStream_t) stream;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(b->device) != cudaSuccess) return SA_E_CUDA;
    for (size_t i = 0; i < b->models.size(); ++i) {
        const sa_state_machine *sm = b->models[i];
        ModelDesc &m = b->mdesc[i];
        std::memset(&m, 0, sizeof(m));
        m.kc = sm->dev.kc32;
        m.emission = sm->emission;
        // a skip emission the same for every k-mer (log 0.1 for HDP machines and .model files)
        // is passed as a value instead of loaded per column
        if (sm->emission == SA_EMIT_HDP) {
            m.gapx_uniform = 1;
            m.gapx_value = (float) kLogPointOne;
        } else {
            bool uni = !sm->gapx.empty();
            for (size_t q = 1; q < sm->gapx.size() && uni; ++q) uni = (float) sm->gapx[q] == (float) sm->gapx[0];
            m.gapx_uniform = uni ? 1 : 0;
            m.gapx_value = uni ? (float) sm->gapx[0] : 0.0f;
        }
        for (int j = 0; j < 9; ++j) m.t[j] = (float) sm->t[j];
        if (sm->emission == SA_EMIT_HDP) {
            const HdpTables &h = sm->hdp;
            m.hdp64.match = sm->dev.match;
            m.hdp64.grid = sm->dev.hdp_grid;
            m.hdp64.density = sm->dev.hdp_density;
            m.hdp64.slope = sm->dev.hdp_slope;
            m.hdp64.kmer_row = sm->dev.hdp_kmer_row;
            m.hdp64.grid_length = h.grid_length;
        }
    }
    sa_status st = SA_OK;
    // every input in one copy: the staging block has the device layout
    if (cudaMemcpyAsync(b->dev_base, b->host_in.ptr, b->in_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        st = SA_E_CUDA;
    if (!st && b->n_events > 0) {
        const int64_t n = b->n_events;
        prep_events<<<(unsigned) std::min<int64_t>((n + 255) / 256, 4096), 256, 0, s>>>(b->d_events_raw, b->d_events, n);
        count_launch();
        if (cudaGetLastError() != cudaSuccess) st = SA_E_CUDA;
    }
    if (!st && b->plain) st = plain_upload(b->plain, s);
    cudaSetDevice(prev);
    b->downloaded = false;
    return st;
}

sa_status sa_batch_run(sa_batch *b, void *stream) {
    if (!b) return SA_E_ARG;
    cudaStream_t s = (cudaStream_t) stream;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(b->device) != cudaSuccess) return SA_E_CUDA;
    const size_t nr = (size_t) b->n_regions, nw = (size_t) b->n_windows;
    sa_status st = SA_OK;
    // every run gets a new number (from 1), also one that launches nothing: a record counts for the
    // run whose number it holds
    if (b->d_done) ++b->run_seq;
    // re-runs after a disagreeing stitch belong to one run's download
    std::fill(b->redone.begin(), b->redone.end(), 0);
    b->n_redone = 0;
    // what the kernels expect cleared: the results block (counters, per-read status and pair
    // ranges, log-likelihoods), the window pair counts, and the ready queue (-1 = empty)
    if (cudaMemsetAsync(b->dev_base + b->res_off, 0, b->res_bytes, s) != cudaSuccess ||
        cudaMemsetAsync(b->d_wcount, 0, sizeof(int64_t) * std::max<size_t>(1, nw), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_ready, 0xff, sizeof(int32_t) * std::max<size_t>(1, nw), s) != cudaSuccess)
        st = SA_E_CUDA;
    if (!st && nr > 0) {
        Args a = batch_args(b);
        const int cpt = std::max(1, (b->max_width + kThreads - 1) / kThreads);
        const int cpt_pow2 = cpt <= 1 ? 1 : (cpt <= 2 ? 2 : 4);
        b->width_class = cpt_pow2;
        const sa_launch_config cfg = b->has_cfg ? b->cfg : launch_for(b->device, cpt_pow2);
        a.warp_windows = cfg.warp_windows;
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
        sms = std::max(1, sms);
        b->timed = false;
        if (b->owns_device && !b->ev[0])
            for (cudaEvent_t &e : b->ev) cudaEventCreate(&e);
        const bool timing = b->owns_device && b->ev[3];
        if (timing) cudaEventRecord(b->ev[0], s);
        emission_kernel<<<(unsigned) std::max<int64_t>(1, std::min<int64_t>((int64_t) sms * cfg.emission_ctas_per_sm,
                                                                            (a.n_chunks + kEmitWarps - 1) / kEmitWarps)),
                          32 * kEmitWarps, 0, s>>>(a);
        if (timing) cudaEventRecord(b->ev[1], s);
        launch_worker(b, a, cfg, sms, s);
        if (timing) cudaEventRecord(b->ev[2], s);
        // with per-read completion the worker has gathered every read it finished
        if (!b->d_done)
            gather_pairs<<<(unsigned) std::max<int64_t>(1, std::min<int64_t>(b->n_reads, sms * 4)), 256, 0, s>>>(a);
        if (timing) {
            cudaEventRecord(b->ev[3], s);
            b->timed = true;
        }
        count_launch(b->d_done ? 2 : 3);
        if (cudaGetLastError() != cudaSuccess) st = SA_E_CUDA;
    }
    if (!st && b->plain) st = plain_run(b->plain, s);
    cudaSetDevice(prev);
    b->downloaded = false;
    return st;
}
sa_status sa_batch_download(sa_batch *b, void *stream) {
    if (!b) return SA_E_ARG;
    cudaStream_t s = (cudaStream_t) stream;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(b->device) != cudaSuccess) return SA_E_CUDA;
    const MemKind host_kind = b->host_pinned ? MemKind::Pinned : MemKind::Heap;
    sa_status st = SA_OK;
    if (!b->host_res.ptr) {
        st = mem_get(host_kind, b->device, b->res_bytes, b->host_res);
        if (!st) layout(b, nullptr, static_cast<unsigned char *>(b->host_res.ptr), nullptr);
    }
    // the results block in one copy, then the packed pairs in one copy
    if (!st && cudaMemcpyAsync(b->host_res.ptr, b->dev_base + b->res_off, b->res_bytes, cudaMemcpyDeviceToHost, s) !=
                   cudaSuccess)
        st = SA_E_CUDA;
    if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = SA_E_CUDA;
    // reads whose stitch disagreed: re-run unsegmented, then the results block again
    bool redo = false;
    for (int64_t r = 0; r < b->n_reads && !st && b->n_stitch > 0; ++r) redo = redo || (b->seg_fail[r] && !b->redone[r]);
    if (redo && !st) {
        st = redo_disagreed(b, s);
        if (!st && cudaMemcpyAsync(b->host_res.ptr, b->dev_base + b->res_off, b->res_bytes, cudaMemcpyDeviceToHost,
                                   s) != cudaSuccess)
            st = SA_E_CUDA;
        if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = SA_E_CUDA;
    }
    const size_t npairs = st ? 0 : (size_t) b->ctl[0].packed;
    const size_t pair_bytes = std::max<size_t>(npairs, 1) * sizeof(sa_aligned_pair);
    if (!st && b->host_pairs.bytes < pair_bytes) {
        mem_put(b->host_pairs);
        st = mem_get(host_kind, b->device, pair_bytes, b->host_pairs);
    }
    if (!st && npairs > 0 &&
        cudaMemcpyAsync(b->host_pairs.ptr, b->d_packed, npairs * sizeof(sa_aligned_pair), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess)
        st = SA_E_CUDA;
    if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = SA_E_CUDA;
    if (!st && b->plain) st = plain_download(b->plain, s);
    b->read_ll.assign(b->n_reads, 0.0);
    for (int64_t r = 0; r < b->n_reads && !st; ++r) {
        if (b->plain_of[r] >= 0) {
            // the no-allocation entry makes no plain set: its reads report SA_E_UNSUPPORTED
            if (b->plain) b->read_ll[r] = plain_log_likelihood(b->plain, b->plain_of[r]);
            continue;
        }
        for (int64_t i = 0; i < b->read_n_regions[r]; ++i) b->read_ll[r] += b->loglik[b->read_first_region[r] + i];
        // each region's total is in its last segment's frame: the stitches' constants bring it back
        if (!b->redone[r])
            for (int64_t q = 0; q < b->read_win[8 * r + 5]; ++q) b->read_ll[r] += b->stitch_res[b->read_win[8 * r + 4] + q].delta;
    }
    cudaSetDevice(prev);
    b->downloaded = st == SA_OK;
    return st;
}

sa_status sa_align_batch(const sa_read *reads, int64_t n_reads, const sa_params *p, void *stream, sa_batch **out) {
    sa_status st = sa_batch_create(reads, n_reads, p, out);
    if (st) return st;
    st = sa_batch_upload(*out, stream);
    if (!st) st = sa_batch_run(*out, stream);
    if (!st) st = sa_batch_download(*out, stream);
    return st;
}

sa_status sa_batch_read_status(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads) return SA_E_ARG;
    if (b->read_status[read]) return (sa_status) b->read_status[read];
    if (!b->plain_of.empty() && b->plain_of[read] >= 0 && !b->plain) return SA_E_UNSUPPORTED;
    if (!b->downloaded) return SA_E_ARG;
    if (!b->plain_of.empty() && b->plain_of[read] >= 0) return plain_read_status(b->plain, b->plain_of[read]);
    if (b->ctl[0].error) return SA_E_TIMEOUT;
    return (sa_status) b->dev_status[read];
}

int64_t sa_batch_pair_count(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads || !b->downloaded) return -1;
    if (b->read_status[read]) return 0;
    if (b->plain_of[read] >= 0) return b->plain ? (int64_t) plain_pairs(b->plain, b->plain_of[read]).size() : 0;
    return b->read_count[read];
}

const sa_aligned_pair *sa_batch_pairs(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads || !b->downloaded) return nullptr;
    if (!b->read_status[read] && b->plain_of[read] >= 0 && b->plain) {
        const auto &v = plain_pairs(b->plain, b->plain_of[read]);
        if (!v.empty()) return v.data();
    }
    return static_cast<const sa_aligned_pair *>(b->host_pairs.ptr) + (b->read_status[read] ? 0 : b->read_base[read]);
}

double sa_batch_log_likelihood(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads || !b->downloaded) return 0.0;
    return b->read_ll[read];
}

int64_t sa_batch_cells(const sa_batch *b) { return b ? b->cells + (b->plain ? plain_cells(b->plain) : 0) : 0; }

sa_status sa_batch_kernel_ms(const sa_batch *b, double *emission_ms, double *worker_ms, double *gather_ms) {
    if (!b || !emission_ms || !worker_ms || !gather_ms) return SA_E_ARG;
    if (!b->timed) return SA_E_ARG;
    float t[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k)
        if (cudaEventSynchronize(b->ev[k + 1]) != cudaSuccess || cudaEventElapsedTime(&t[k], b->ev[k], b->ev[k + 1]) != cudaSuccess)
            return SA_E_CUDA;
    *emission_ms = t[0];
    *worker_ms = t[1];
    *gather_ms = t[2];
    return SA_OK;
}

sa_status sa_batch_transfer_bytes(const sa_batch *b, int64_t *h2d_bytes, int64_t *d2h_bytes) {
    if (!b || !h2d_bytes || !d2h_bytes) return SA_E_ARG;
    *h2d_bytes = (int64_t) b->in_bytes;
    *d2h_bytes = (int64_t) b->res_bytes + (b->downloaded ? (int64_t) (b->ctl[0].packed * sizeof(sa_aligned_pair)) : 0);
    return SA_OK;
}

sa_status sa_measure_fp32_peak(int32_t device, double *tflops) {
    if (!tflops) return SA_E_ARG;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return SA_E_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    float *sink = nullptr;
    if (device_malloc(reinterpret_cast<void **>(&sink), sizeof(float)) != cudaSuccess) { cudaSetDevice(prev); return SA_E_NOMEM; }
    const int blocks = sms * 8, threads = 256, iters = 1 << 16;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        fma_probe<<<blocks, threads>>>(sink, iters, 1.0f + rep);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best = std::min(best, ms);
    }
    count_launch(4);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    const sa_status st = cudaGetLastError() == cudaSuccess ? SA_OK : SA_E_CUDA;
    cudaSetDevice(prev);
    *tflops = 2.0 * 8.0 * (double) iters * blocks * threads / (best * 1e-3) / 1e12;
    return st;
}

int64_t sa_batch_regions(const sa_batch *b) { return b ? (int64_t) b->regions.size() : 0; }

sa_status sa_batch_set_wait_limit(sa_batch *b, int64_t cycles) {
    if (!b || cycles < 1) return SA_E_ARG;
    b->wait_limit = (long long) cycles;
    return SA_OK;
}

sa_status sa_setSegmentPolicy(int32_t segment_diags, int32_t warmup_diags) {
    if (warmup_diags < 64 || (segment_diags > 0 && segment_diags <= warmup_diags + 64)) return SA_E_ARG;
    g_seg_target.store(segment_diags < 0 ? -1 : segment_diags);
    g_seg_warm.store(warmup_diags);
    return SA_OK;
}

sa_status sa_planForwardSegments(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY,
                                 const sa_params *p, int32_t segment_diags, int32_t warmup_diags, int64_t *out,
                                 int64_t capacity, int64_t *n_segments) {
    if ((n_anchors > 0 && !anchors) || lX < 0 || lY < 0 || !p || !n_segments || capacity < 0 ||
        (capacity > 0 && !out) || warmup_diags < 64 || segment_diags == 0)
        return SA_E_ARG;
    std::vector<Region> regs;
    sa_status st = plan_regions(anchors, n_anchors, lX, lY, *p, true, true, regs);
    if (st) return st;
    int64_t k = 0;
    std::vector<int32_t> cuts;
    for (size_t g = 0; g < regs.size(); ++g) {
        const Region &rg = regs[g];
        const int32_t wr = region_warm(rg, warmup_diags);
        cuts.clear();
        if (segment_diags > 0) plan_cuts(rg, segment_diags, wr, cuts);
        for (size_t q = 0; q <= cuts.size(); ++q, ++k) {
            if (k >= capacity) continue;
            const int64_t b = q == 0 ? 0 : rg.windows[cuts[q - 1]].T;
            int64_t *o = out + 6 * k;
            o[0] = (int64_t) g;
            o[1] = b;
            o[2] = q == cuts.size() ? rg.lX + rg.lY : rg.windows[cuts[q]].T;
            o[3] = q == 0 ? 0 : wr + ((2 - wr) % 3 + 3) % 3;
            o[4] = q == 0 ? 0 : cuts[q - 1];
            o[5] = rg.max_width;
        }
    }
    *n_segments = k;
    return k > capacity ? SA_E_OUTPUT : SA_OK;
}

sa_status sa_getSegmentPolicy(int32_t *segment_diags, int32_t *warmup_diags) {
    if (!segment_diags || !warmup_diags) return SA_E_ARG;
    *segment_diags = g_seg_target.load();
    *warmup_diags = g_seg_warm.load();
    return SA_OK;
}

sa_status sa_batch_segment_info(const sa_batch *b, int64_t *n_segments, int64_t *n_stitches, int64_t *n_redone,
                                double *max_spread) {
    if (!b || !n_segments || !n_stitches || !n_redone || !max_spread) return SA_E_ARG;
    *n_segments = b->n_segs;
    *n_stitches = b->n_stitch;
    *n_redone = b->downloaded ? b->n_redone : 0;
    if (b->plain) {   // the batch's reads in the plain FP64 form (regions re-run whole)
        int64_t t = 0, st = 0, rd = 0;
        plain_segment_info(b->plain, &t, &st, &rd);
        *n_segments += t;
        *n_stitches += st;
        if (b->downloaded) *n_redone += rd;
    }
    double m = 0.0;
    if (b->downloaded)
        for (int64_t q = 0; q < b->n_stitch; ++q)
            if (b->stitch_res[q].result == kStitchAgreed) m = std::max(m, (double) b->stitch_res[q].spread);
    *max_spread = m;
    return SA_OK;
}

sa_status sa_batch_set_stitch_tolerance(sa_batch *b, double scale) {
    if (!b || !(scale == scale)) return SA_E_ARG;
    b->stitch_tol = (float) scale;
    if (b->plain) plain_set_stitch_tolerance(b->plain, scale);
    return SA_OK;
}

sa_status sa_getLaunchConfig(int32_t device, int32_t width_class, sa_launch_config *cfg) {
    if (!cfg || device < 0 || !valid_width_class(width_class)) return SA_E_ARG;
    *cfg = launch_for(device, width_class);
    return SA_OK;
}

sa_status sa_setLaunchConfig(int32_t device, int32_t width_class, const sa_launch_config *cfg) {
    if (!cfg || device < 0 || !valid_width_class(width_class) || !valid_launch(*cfg)) return SA_E_ARG;
    const std::string name = device_name(device);
    if (name.empty()) return SA_E_CUDA;
    std::lock_guard<std::mutex> lock(g_launch_mutex);
    g_launch[{name, width_class}] = *cfg;
    return SA_OK;
}

sa_status sa_loadLaunchConfigs(const char *path) {
    if (!path) return SA_E_ARG;
    std::ifstream in(path);
    if (!in) return SA_E_FILE;
    std::string line;
    std::vector<std::pair<std::pair<std::string, int>, sa_launch_config>> rows;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::vector<std::string> f;
        std::stringstream ss(line);
        std::string tok;
        while (std::getline(ss, tok, '\t')) f.push_back(tok);
        if (f.size() != 6) return SA_E_FILE;
        sa_launch_config c;
        int wc = 0;
        try {
            wc = std::stoi(f[1]);
            c.ctas_per_sm = std::stoi(f[2]);
            c.grid_per_region = std::stoi(f[3]);
            c.warp_windows = std::stoi(f[4]);
            c.emission_ctas_per_sm = std::stoi(f[5]);
        } catch (...) {
            return SA_E_FILE;
        }
        if (!valid_width_class(wc) || !valid_launch(c)) return SA_E_FILE;
        rows.push_back({{f[0], wc}, c});
    }
    std::lock_guard<std::mutex> lock(g_launch_mutex);
    for (const auto &r : rows) g_launch[r.first] = r.second;
    return SA_OK;
}

sa_status sa_tuneLaunchConfig(sa_batch *b, void *stream, int32_t repeats, sa_launch_config *best, double *best_ms,
                              int32_t *n_tried) {
    if (!b || !best || !best_ms || !n_tried || repeats < 1 || !b->owns_device) return SA_E_ARG;
    const int cpt = std::max(1, (b->max_width + kThreads - 1) / kThreads);
    const int wc = cpt <= 1 ? 1 : (cpt <= 2 ? 2 : 4);
    std::vector<sa_launch_config> cand;
    for (int cps : {1, 2, 3})
        for (int gpr : {2, 3, 4, 6})
            for (int ww : {1, 0})
                for (int ecs : {8, 16, 32}) {
                    if (wc != 1 && (ww == 0 || cps >= 2)) continue;   // wider bands: CTA windows, one CTA per SM
                    cand.push_back(sa_launch_config{cps, gpr, ww, ecs});
                }
    double best_t = 1e300;
    sa_launch_config best_c = default_launch();
    int tried = 0;
    for (const sa_launch_config &c : cand) {
        b->has_cfg = true;
        b->cfg = c;
        double total = 0.0;
        for (int r = 0; r <= repeats; ++r) {
            sa_status st = sa_batch_run(b, stream);
            double em = 0, wk = 0, ga = 0;
            if (!st) st = sa_batch_kernel_ms(b, &em, &wk, &ga);
            if (st) {
                b->has_cfg = false;
                return st;
            }
            if (r > 0) total += em + wk + ga;   // the first run is untimed
        }
        ++tried;
        const double t = total / repeats;
        if (t < best_t) {
            best_t = t;
            best_c = c;
        }
    }
    b->has_cfg = false;
    *best = best_c;
    *best_ms = best_t;
    *n_tried = tried;
    return sa_setLaunchConfig(b->device, wc, &best_c);
}

void sa_batch_destroy(sa_batch *b) { delete b; }

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// batches whose device buffers live in caller-provided device memory (sa_noalloc.cu)
// ------------------------------------------------------------------------------------------------
namespace sa {

sa_status batch_plan_host(const sa_read *reads, int64_t n_reads, const sa_params *p, sa_batch **out) {
    if (!reads || n_reads < 0 || !p || !out) return SA_E_ARG;
    *out = nullptr;
    sa_status st = check_params(*p);
    if (st) return st;
    auto *b = new (std::nothrow) sa_batch();
    if (!b) return SA_E_NOMEM;
    st = plan_batch(reads, n_reads, p, false, b);
    if (st) {
        delete b;
        return st;
    }
    *out = b;
    return SA_OK;
}

int batch_device(const sa_batch *b) { return b->device; }

void segment_policy(int32_t &target, int32_t &warm) {
    target = g_seg_target.load();
    warm = g_seg_warm.load();
}
int64_t segment_min() { return kSegMin; }
int32_t segment_warm(const Region &rg, int32_t warm) { return region_warm(rg, warm); }
void segment_cuts(const Region &rg, int64_t target, int32_t warm, std::vector<int32_t> &cuts) {
    plan_cuts(rg, target, warm, cuts);
}


bool batch_models_resident(const sa_batch *b) {
    // only the machines of reads the FP32 kernels run: reads routed to the plain form report
    // SA_E_UNSUPPORTED on this path and never touch their machine's device tables
    std::vector<char> used(b->models.size(), 0);
    for (int64_t r = 0; r < b->n_regions; ++r) used[(size_t) b->regions[r].model] = 1;
    for (size_t i = 0; i < b->models.size(); ++i)
        if (used[i] && !model_resident(b->models[i])) return false;
    return true;
}

size_t batch_bind_scratch(sa_batch *b, unsigned char *base) {
    b->owns_device = false;
    b->dev_base = base;
    return layout(b, nullptr, nullptr, base);
}

void batch_release_host(sa_batch *b) { delete b; }

sa_status batch_publish_reads(sa_batch *b) {
    if (!b || !b->owns_device) return SA_E_ARG;
    if (b->d_done) return SA_OK;
    const size_t bytes = sizeof(ReadDone) * (size_t) std::max<int64_t>(1, b->n_reads);
    sa_status st = mem_get(MemKind::Pinned, b->device, bytes, b->host_done);
    if (st) return st;
    // pinned memory is mapped into every device's address space (unified addressing)
    void *dptr = nullptr;
    if (cudaHostGetDevicePointer(&dptr, b->host_done.ptr, 0) != cudaSuccess) {
        cudaGetLastError();
        mem_put(b->host_done);
        return SA_E_CUDA;
    }
    std::memset(b->host_done.ptr, 0, bytes);
    b->d_done = static_cast<ReadDone *>(dptr);
    return SA_OK;
}

const ReadDone *batch_read_records(const sa_batch *b) {
    return b && b->d_done ? static_cast<const ReadDone *>(b->host_done.ptr) : nullptr;
}

int32_t batch_run_seq(const sa_batch *b) { return b ? b->run_seq : 0; }

sa_status batch_fetch_read(const sa_batch *b, const ReadDone &rec, sa_aligned_pair *dst, cudaStream_t stream) {
    if (!b || rec.n_pairs < 0 || rec.first_pair < 0 || rec.first_pair + rec.n_pairs > b->out_total) return SA_E_ARG;
    if (rec.n_pairs == 0) return SA_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(b->device) != cudaSuccess) return SA_E_CUDA;
    const bool ok = cudaMemcpyAsync(dst, b->d_packed + rec.first_pair, sizeof(sa_aligned_pair) * (size_t) rec.n_pairs,
                                    cudaMemcpyDeviceToHost, stream) == cudaSuccess &&
                    cudaStreamSynchronize(stream) == cudaSuccess;
    cudaSetDevice(prev);
    return ok ? SA_OK : SA_E_CUDA;
}

bool batch_run_events(const sa_batch *b, cudaEvent_t *start, cudaEvent_t *end) {
    if (!b || !b->timed) return false;
    *start = b->ev[0];
    *end = b->ev[2];
    return true;
}

}  // namespace sa
