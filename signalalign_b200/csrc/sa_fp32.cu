// Batched FP32 form: host side.  Plans a batch (band geometry, traceback windows, k-mer ids,
// emission chunks, output segments), owns its device buffers, and runs the three kernels of
// sa_fp32_kernel.cuh: emissions of every band cell, the persistent worker (forward sweeps and
// traceback-window backward sweeps pulled from a device queue), and the per-read gather of pairs.
//
// Every device buffer of a batch is listed once (for_each_buffer), so the allocating path
// (sa_batch_create) and the path that carves them from caller-provided memory
// (batch_bind_scratch) lay out the same set.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
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

}  // namespace fp32
}  // namespace sa

// ------------------------------------------------------------------------------------------------
// host side of the batch
// ------------------------------------------------------------------------------------------------
using namespace sa;
using namespace sa::fp32;

struct sa_batch {
    int device = 0;
    int64_t n_reads = 0;
    std::vector<sa_state_machine *> models;
    std::vector<RegionDesc> regions;
    std::vector<int32_t> order;
    std::vector<int32_t> read_status;       // host planning status per read
    std::vector<int64_t> read_first_region, read_n_regions;
    std::vector<int64_t> read_win;          // per read: first window, window count
    std::vector<ReadScale32> read_scale;
    std::vector<int2> meta;
    std::vector<Window> windows;
    std::vector<WindowTask> wtask;
    std::vector<Chunk> chunks;
    std::vector<int32_t> kmer;
    std::vector<float> gapx;
    std::vector<double2> events;
    int64_t cells = 0, out_total = 0;
    int32_t max_width = 0;
    float threshold = 0.01f;
    // device
    RegionDesc *d_regions = nullptr;
    int32_t *d_order = nullptr;
    ModelDesc *d_models = nullptr;
    ReadScale32 *d_read_scale = nullptr;
    int2 *d_meta = nullptr;
    Window *d_windows = nullptr;
    WindowTask *d_wtask = nullptr;
    Chunk *d_chunks = nullptr;
    int32_t *d_kmer = nullptr;
    float *d_gapx = nullptr;
    double2 *d_events_raw = nullptr;
    Event32 *d_events = nullptr;
    float *d_E = nullptr, *d_F = nullptr, *d_fshift = nullptr;
    double *d_base = nullptr, *d_loglik = nullptr;
    int32_t *d_ready = nullptr, *d_status = nullptr;
    sa_aligned_pair *d_out = nullptr, *d_packed = nullptr;
    int64_t *d_wcount = nullptr, *d_read_win = nullptr, *d_read_base = nullptr, *d_read_count = nullptr;
    Control *d_ctl = nullptr;
    // results
    std::vector<int64_t> read_base, read_count;
    std::vector<double> loglik;
    std::vector<int32_t> dev_status;
    Control ctl{};
    std::vector<std::vector<sa_aligned_pair>> read_pairs;
    std::vector<double> read_ll;
    bool downloaded = false;
};

namespace {

// Calls fn(pointer, element count) for every device buffer of the batch.
template <typename Fn>
void for_each_buffer(sa_batch *b, Fn &&fn) {
    const size_t nr = b->regions.size(), nd = b->meta.size(), nw = b->windows.size(), nreads = (size_t) b->n_reads;
    const size_t cells = (size_t) b->cells;
    fn(b->d_regions, nr);
    fn(b->d_order, b->order.size());
    fn(b->d_models, b->models.size());
    fn(b->d_read_scale, b->read_scale.size());
    fn(b->d_meta, nd);
    fn(b->d_windows, nw);
    fn(b->d_wtask, nw);
    fn(b->d_chunks, b->chunks.size());
    fn(b->d_kmer, b->kmer.size());
    fn(b->d_gapx, b->gapx.size());
    fn(b->d_events_raw, b->events.size());
    fn(b->d_events, b->events.size());
    fn(b->d_E, 2 * cells + kStoreSlack);
    fn(b->d_F, 3 * cells + kStoreSlack);
    fn(b->d_base, nd);
    fn(b->d_fshift, nd);
    fn(b->d_ready, nw);
    fn(b->d_out, (size_t) b->out_total);
    fn(b->d_wcount, nw);
    fn(b->d_loglik, nr);
    fn(b->d_status, nreads);
    fn(b->d_ctl, (size_t) 1);
    fn(b->d_read_win, 2 * nreads);
    fn(b->d_packed, (size_t) b->out_total);
    fn(b->d_read_base, nreads);
    fn(b->d_read_count, nreads);
}

template <typename T>
sa_status h2d(T *dst, const std::vector<T> &src, cudaStream_t s) {
    if (src.empty()) return SA_OK;
    return cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s) == cudaSuccess
               ? SA_OK : SA_E_CUDA;
}

template <typename T>
sa_status d2h(std::vector<T> &dst, const T *src, size_t n, cudaStream_t s) {
    dst.resize(n);
    if (n == 0) return SA_OK;
    return cudaMemcpyAsync(dst.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, s) == cudaSuccess ? SA_OK
                                                                                                     : SA_E_CUDA;
}

void free_batch_device(sa_batch *b) {
    for_each_buffer(b, [](auto *&p, size_t) {
        cudaFree(p);
        p = nullptr;
    });
}

// Host planning of a batch (no device work): per read k-mer ids, events and regions, per region its
// windows, per-anti-diagonal meta and emission chunks, per window its task and output segment, the
// LPT order.  Returns SA_E_CAPACITY for a band wider than the kernel's widest ring.
sa_status plan_batch(const sa_read *reads, int64_t n_reads, const sa_params *p, sa_batch *b) {
    sa_status st = SA_OK;
    b->n_reads = n_reads;
    b->threshold = (float) p->threshold;
    b->read_status.assign(n_reads, SA_OK);
    b->read_first_region.assign(n_reads, 0);
    b->read_n_regions.assign(n_reads, 0);
    b->read_win.assign(2 * n_reads, 0);
    b->read_scale.resize(n_reads);
    std::vector<Region> regs;
    PathTable pt;
    int device = -1;
    for (int64_t r = 0; r < n_reads; ++r) {
        const sa_read &rd = reads[r];
        auto *sm = const_cast<sa_state_machine *>(rd.sm);
        b->read_first_region[r] = (int64_t) b->regions.size();
        b->read_win[2 * r] = (int64_t) b->windows.size();
        if (!sm || rd.reference_length < 0 || rd.n_events < 0 || rd.n_anchors < 0 ||
            (rd.reference_length > 0 && !rd.reference) || (rd.n_events > 0 && !rd.events) ||
            (rd.n_anchors > 0 && !rd.anchors) || !(rd.var != 0.0)) {
            b->read_status[r] = SA_E_ARG;
            continue;
        }
        if (device < 0) device = sm->dev.device;
        if (sm->dev.device != device) { b->read_status[r] = SA_E_ARG; continue; }
        if (sm->emission == SA_EMIT_HDP && !sm->hdp.present) { b->read_status[r] = SA_E_UNSUPPORTED; continue; }
        const int k = sm->kmer_length;
        const int64_t lX = rd.reference_length == 0 ? 0 : rd.reference_length - (k - 1);
        if (lX < 0) { b->read_status[r] = SA_E_ARG; continue; }
        st = build_paths(sm, rd.reference, lX, rd.degenerate, pt);
        if (st) { b->read_status[r] = st; continue; }
        if (pt.multi) { b->read_status[r] = SA_E_UNSUPPORTED; continue; }
        st = plan_regions(rd.anchors, rd.n_anchors, lX, rd.n_events, *p, rd.ragged_left != 0, rd.ragged_right != 0,
                          regs);
        if (st) { b->read_status[r] = st; continue; }
        int32_t model = -1;
        for (size_t i = 0; i < b->models.size(); ++i)
            if (b->models[i] == sm) model = (int32_t) i;
        if (model < 0) { model = (int32_t) b->models.size(); b->models.push_back(sm); }
        const double var = sm->emission == SA_EMIT_PLAIN ? 1.0 : rd.var;
        ReadScale32 &rs = b->read_scale[r];
        rs.scale = sm->emission == SA_EMIT_PLAIN ? 1.0f : (float) rd.scale;
        rs.shift = sm->emission == SA_EMIT_PLAIN ? 0.0f : (float) rd.shift;
        rs.inv_var = (float) (1.0 / var);
        rs.log_inv_var = (float) std::log(1.0 / var);
        const int64_t kmer_base = (int64_t) b->kmer.size();
        for (int64_t x = 1; x <= lX; ++x) {
            const int32_t kid = pt.ids[pt.first[x]];
            b->kmer.push_back(kid);
            b->gapx.push_back(sm->emission == SA_EMIT_HDP ? (float) kLogPointOne : (float) sm->gapx[kid]);
        }
        const int64_t event_base = (int64_t) b->events.size();
        for (int64_t y = 0; y < rd.n_events; ++y)
            b->events.push_back(make_double2(rd.events[y * kEventParams], rd.events[y * kEventParams + 1]));
        for (const Region &rg : regs) {
            const int32_t region = (int32_t) b->regions.size();
            RegionDesc d;
            std::memset(&d, 0, sizeof(d));
            d.n = (int32_t) (rg.lX + rg.lY);
            d.lX = (int32_t) rg.lX;
            d.lY = (int32_t) rg.lY;
            d.read = (int32_t) r;
            d.n_windows = (int32_t) rg.windows.size();
            d.model = model;
            d.ragged_left = rg.ragged_left;
            d.ragged_right = rg.ragged_right;
            d.diag_base = (int64_t) b->meta.size();
            d.cell_base = b->cells;
            d.win_base = (int64_t) b->windows.size();
            d.kmer_base = kmer_base + rg.x1;
            d.event_base = event_base + rg.y1;
            d.x1 = rg.x1;
            d.y1 = rg.y1;
            // per anti-diagonal meta: band start, width, window end / refresh / stored gap states
            std::vector<int32_t> flags(d.n + 2, 0);
            for (const Window &w : rg.windows) {
                flags[w.D] |= kFlagWindowEnd;
                for (int32_t q = w.from; q > w.T; q -= 10) flags[q] |= kFlagRefresh;
            }
            std::vector<int64_t> off(d.n + 1, 0);
            int64_t acc = 0;
            for (int32_t dd = 0; dd <= d.n; ++dd) {
                const int32_t w = (rg.xmy_r[dd] - rg.xmy_l[dd]) / 2 + 1;
                int32_t f = flags[dd];
                if ((flags[dd] | flags[dd + 1]) & kFlagRefresh) f |= kFlagStoreGaps;
                b->meta.push_back(make_int2(rg.xmy_l[dd], w | f));
                off[dd] = acc;
                acc += w;
            }
            for (int32_t d0 = 0; d0 <= d.n; d0 += kChunkDiags) {
                Chunk ch;
                ch.region = region;
                ch.d0 = d0;
                ch.nd = std::min(kChunkDiags, d.n + 1 - d0);
                ch.pad = 0;
                ch.cell = d.cell_base + off[d0];
                b->chunks.push_back(ch);
            }
            for (const Window &w : rg.windows) {
                WindowTask t;
                t.region = region;
                t.first_cell = (int32_t) off[w.D];
                t.out_cap = 4 * (w.from - w.T) + 64;
                t.pad = 0;
                t.out_base = b->out_total;
                b->out_total += t.out_cap;
                b->wtask.push_back(t);
            }
            b->cells += acc;
            b->max_width = std::max(b->max_width, rg.max_width);
            b->windows.insert(b->windows.end(), rg.windows.begin(), rg.windows.end());
            b->regions.push_back(d);
        }
        b->read_n_regions[r] = (int64_t) b->regions.size() - b->read_first_region[r];
        b->read_win[2 * r + 1] = (int64_t) b->windows.size() - b->read_win[2 * r];
    }
    if (b->max_width > kMaxCpt * kThreads) return SA_E_CAPACITY;
    b->device = device < 0 ? 0 : device;
    // largest band area first (LPT order of the forward claims)
    b->order.resize(b->regions.size());
    std::iota(b->order.begin(), b->order.end(), 0);
    std::vector<int64_t> area(b->regions.size());
    for (size_t i = 0; i < b->regions.size(); ++i) {
        const RegionDesc &d = b->regions[i];
        area[i] = (i + 1 < b->regions.size() ? b->regions[i + 1].cell_base : b->cells) - d.cell_base;
    }
    std::stable_sort(b->order.begin(), b->order.end(), [&](int32_t a, int32_t c) { return area[a] > area[c]; });
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
    st = plan_batch(reads, n_reads, p, b);
    if (st) {
        delete b;
        return st;
    }
    // device buffers
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(b->device) != cudaSuccess) { delete b; return SA_E_CUDA; }
    for (auto *sm : b->models) {
        st = ensure_device_model(sm);
        if (st) { cudaSetDevice(prev); delete b; return st; }
    }
    for_each_buffer(b, [&](auto *&ptr, size_t n) {
        using T = std::remove_reference_t<decltype(*ptr)>;
        if (!st && cudaMalloc((void **) &ptr, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) st = SA_E_NOMEM;
    });
    cudaSetDevice(prev);
    if (st) {
        free_batch_device(b);
        delete b;
        return st;
    }
    *out = b;
    return SA_OK;
}

sa_status sa_batch_upload(sa_batch *b, void *stream) {
    if (!b) return SA_E_ARG;
    cudaStream_t s = (cudaStream_t) stream;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(b->device) != cudaSuccess) return SA_E_CUDA;
    std::vector<ModelDesc> md(b->models.size());
    for (size_t i = 0; i < b->models.size(); ++i) {
        const sa_state_machine *sm = b->models[i];
        ModelDesc &m = md[i];
        std::memset(&m, 0, sizeof(m));
        m.kc = sm->dev.kc32;
        m.emission = sm->emission;
        for (int j = 0; j < 9; ++j) m.t[j] = (float) sm->t[j];
        if (sm->emission == SA_EMIT_HDP) {
            const HdpTables &h = sm->hdp;
            m.hdp.knots = sm->dev.hdp_knots32;
            m.hdp.kmer_row = sm->dev.hdp_row32;
            m.hdp.x0 = (float) h.grid[0];
            m.hdp.dx = (float) (h.grid[1] - h.grid[0]);
            m.hdp.inv_dx = (float) (1.0 / (h.grid[1] - h.grid[0]));
            m.hdp.x_last = (float) h.grid[h.grid_length - 1];
            m.hdp.grid_length = (int32_t) h.grid_length;
        }
    }
    sa_status st = SA_OK;
    if (!st) st = h2d(b->d_regions, b->regions, s);
    if (!st) st = h2d(b->d_order, b->order, s);
    if (!st) st = h2d(b->d_models, md, s);
    if (!st) st = h2d(b->d_read_scale, b->read_scale, s);
    if (!st) st = h2d(b->d_meta, b->meta, s);
    if (!st) st = h2d(b->d_windows, b->windows, s);
    if (!st) st = h2d(b->d_wtask, b->wtask, s);
    if (!st) st = h2d(b->d_chunks, b->chunks, s);
    if (!st) st = h2d(b->d_kmer, b->kmer, s);
    if (!st) st = h2d(b->d_gapx, b->gapx, s);
    if (!st) st = h2d(b->d_events_raw, b->events, s);
    if (!st) st = h2d(b->d_read_win, b->read_win, s);
    if (!st && !b->events.empty()) {
        const int64_t n = (int64_t) b->events.size();
        prep_events<<<(unsigned) std::min<int64_t>((n + 255) / 256, 4096), 256, 0, s>>>(b->d_events_raw, b->d_events, n);
        count_launch();
        if (cudaGetLastError() != cudaSuccess) st = SA_E_CUDA;
    }
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
    const size_t nr = b->regions.size(), nw = b->windows.size();
    sa_status st = SA_OK;
    // what the kernels expect cleared: counters, per-read status, window counts, log-likelihoods,
    // and the ready queue (-1 = empty)
    if (cudaMemsetAsync(b->d_ctl, 0, sizeof(Control), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_status, 0, sizeof(int32_t) * std::max<int64_t>(1, b->n_reads), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_wcount, 0, sizeof(int64_t) * std::max<size_t>(1, nw), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_loglik, 0, sizeof(double) * std::max<size_t>(1, nr), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_ready, 0xff, sizeof(int32_t) * std::max<size_t>(1, nw), s) != cudaSuccess)
        st = SA_E_CUDA;
    if (!st && nr > 0) {
        Args a;
        std::memset(&a, 0, sizeof(a));
        a.regions = b->d_regions;
        a.order = b->d_order;
        a.n_regions = (int64_t) nr;
        a.models = b->d_models;
        a.read_scale = b->d_read_scale;
        a.meta = b->d_meta;
        a.windows = b->d_windows;
        a.wtask = b->d_wtask;
        a.n_windows = (int64_t) nw;
        a.chunks = b->d_chunks;
        a.n_chunks = (int64_t) b->chunks.size();
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
        const int cpt = std::max(1, (b->max_width + kThreads - 1) / kThreads);
        const int cpt_pow2 = cpt <= 1 ? 1 : (cpt <= 2 ? 2 : 4);
        a.wmax = cpt_pow2 * kThreads;
        a.spin_limit = 20000000000LL;   // ~10 s at 2 GHz: far beyond any forward sweep
        const size_t smem = sizeof(Shared) + sizeof(float) * (size_t) (9 * (a.wmax + 2) + 2 * a.wmax);
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
        sms = std::max(1, sms);
        emission_kernel<<<(unsigned) std::max<int64_t>(1, std::min<int64_t>(sms * 8, (a.n_chunks + 7) / 8)), 256, 0,
                          s>>>(a);
        auto launch = [&](auto kern) {
            if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
            const int64_t grid = (int64_t) sms * std::max(1, per_sm);
            kern<<<(unsigned) grid, kThreads, smem, s>>>(a);
        };
        if (cpt_pow2 == 1) launch(worker_kernel<1>);
        else if (cpt_pow2 == 2) launch(worker_kernel<2>);
        else launch(worker_kernel<4>);
        gather_pairs<<<(unsigned) std::max<int64_t>(1, std::min<int64_t>(b->n_reads, sms * 4)), 256, 0, s>>>(a);
        count_launch(3);
        if (cudaGetLastError() != cudaSuccess) st = SA_E_CUDA;
    }
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
    const size_t nr = b->regions.size(), nreads = (size_t) b->n_reads;
    sa_status st = SA_OK;
    b->ctl = Control{};
    if (!st) st = d2h(b->read_base, b->d_read_base, nr ? nreads : 0, s);
    if (!st) st = d2h(b->read_count, b->d_read_count, nr ? nreads : 0, s);
    if (!st) st = d2h(b->loglik, b->d_loglik, nr, s);
    if (!st) st = d2h(b->dev_status, b->d_status, nreads, s);
    if (!st && nr && cudaMemcpyAsync(&b->ctl, b->d_ctl, sizeof(Control), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        st = SA_E_CUDA;
    if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = SA_E_CUDA;
    if (!nr) {
        b->read_base.assign(nreads, 0);
        b->read_count.assign(nreads, 0);
    }
    // the packed pairs in one copy, then split per read on the host
    std::vector<sa_aligned_pair> packed;
    if (!st) st = d2h(packed, b->d_packed, (size_t) b->ctl.packed, s);
    if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = SA_E_CUDA;
    b->read_pairs.assign(nreads, {});
    b->read_ll.assign(nreads, 0.0);
    for (size_t r = 0; r < nreads && !st; ++r) {
        const int64_t base = b->read_base[r], cnt = b->read_count[r];
        if (cnt > 0 && base >= 0 && base + cnt <= (int64_t) packed.size())
            b->read_pairs[r].assign(packed.begin() + base, packed.begin() + base + cnt);
        for (int64_t i = 0; i < b->read_n_regions[r]; ++i) b->read_ll[r] += b->loglik[b->read_first_region[r] + i];
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
    if (!b->downloaded) return SA_E_ARG;
    if (b->ctl.error) return SA_E_TIMEOUT;
    return (sa_status) b->dev_status[read];
}

int64_t sa_batch_pair_count(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads || !b->downloaded) return -1;
    return (int64_t) b->read_pairs[read].size();
}

const sa_aligned_pair *sa_batch_pairs(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads || !b->downloaded) return nullptr;
    return b->read_pairs[read].data();
}

double sa_batch_log_likelihood(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads || !b->downloaded) return 0.0;
    return b->read_ll[read];
}

int64_t sa_batch_cells(const sa_batch *b) { return b ? b->cells : 0; }

sa_status sa_batch_transfer_bytes(const sa_batch *b, int64_t *h2d_bytes, int64_t *d2h_bytes) {
    if (!b || !h2d_bytes || !d2h_bytes) return SA_E_ARG;
    auto bytes = [](const auto &v) { return (int64_t) (v.size() * sizeof(v[0])); };
    *h2d_bytes = bytes(b->regions) + bytes(b->order) + (int64_t) (b->models.size() * sizeof(ModelDesc)) +
                 bytes(b->read_scale) + bytes(b->meta) + bytes(b->windows) + bytes(b->wtask) + bytes(b->chunks) +
                 bytes(b->kmer) + bytes(b->gapx) + bytes(b->events) + bytes(b->read_win);
    int64_t pairs = 0;
    for (const auto &rp : b->read_pairs) pairs += (int64_t) rp.size();
    *d2h_bytes = bytes(b->read_base) + bytes(b->read_count) + bytes(b->loglik) + bytes(b->dev_status) +
                 (int64_t) sizeof(Control) + pairs * (int64_t) sizeof(sa_aligned_pair);
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
    if (cudaMalloc(&sink, sizeof(float)) != cudaSuccess) { cudaSetDevice(prev); return SA_E_NOMEM; }
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

void sa_batch_destroy(sa_batch *b) {
    if (!b) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    free_batch_device(b);
    cudaSetDevice(prev);
    delete b;
}

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
    st = plan_batch(reads, n_reads, p, b);
    if (st) {
        delete b;
        return st;
    }
    *out = b;
    return SA_OK;
}

int batch_device(const sa_batch *b) { return b->device; }

bool batch_models_resident(const sa_batch *b) {
    for (const sa_state_machine *sm : b->models)
        if (sm->dev_dirty) return false;
    return true;
}

size_t batch_bind_scratch(sa_batch *b, unsigned char *base) {
    size_t at = 0;
    for_each_buffer(b, [&](auto *&ptr, size_t n) {
        using T = std::remove_reference_t<decltype(*ptr)>;
        at = (at + 255) & ~(size_t) 255;
        if (base) ptr = reinterpret_cast<T *>(base + at);
        at += std::max<size_t>(n, 1) * sizeof(T);
    });
    return (at + 255) & ~(size_t) 255;
}

void batch_release_host(sa_batch *b) { delete b; }

}  // namespace sa
