// Batched FP32 form: all regions of all reads in one persistent launch.
//
// Work distribution: regions are sorted by band area (largest first) on the host; persistent CTAs
// of 128 threads pull the next region from a device counter.  A CTA sweeps its region's band one
// anti-diagonal at a time (cells of an anti-diagonal spread over the threads, neighbours exchanged
// through a 3-slot shared-memory ring, one barrier per anti-diagonal).  Forward values go to HBM
// (3 floats per cell, SoA per anti-diagonal) together with each anti-diagonal's FP64 base.  At each
// traceback point of getPosteriorProbsWithBanding (pairwiseAligner.c:1319-1333) the CTA runs the
// window's backward sweep in shared memory with the posterior test fused into it, so backward
// values never leave the SM.  Total probabilities are refreshed on the reference's schedule
// (every 10th posterior anti-diagonal, :1370-1380) and accumulated in the reference's sequential
// cell order, which the 7.5 cut-off of logAdd makes order dependent.
//
// Values are log probabilities relative to a per-anti-diagonal base: the base of anti-diagonal d is
// the base of d-1 plus the largest value stored on d-1 (FP64, carried by every thread), so stored
// FP32 values stay near zero.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
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
    std::vector<ReadScale32> read_scale;
    std::vector<int2> meta;
    std::vector<int32_t> window_off;
    std::vector<Window> windows;
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
    int32_t *d_window_off = nullptr, *d_kmer = nullptr, *d_status = nullptr;
    float *d_gapx = nullptr;
    int64_t *d_out_count = nullptr;
    Window *d_windows = nullptr;
    double2 *d_events_raw = nullptr;
    Event32 *d_events = nullptr;
    float *d_F = nullptr, *d_fshift = nullptr;
    double *d_base = nullptr, *d_loglik = nullptr;
    sa_aligned_pair *d_out = nullptr;
    unsigned int *d_queue = nullptr;
    // results
    std::vector<int64_t> out_count;
    std::vector<double> loglik;
    std::vector<int32_t> dev_status;
    std::vector<sa_aligned_pair> out;
    std::vector<std::vector<sa_aligned_pair>> read_pairs;
    std::vector<double> read_ll;
    bool downloaded = false;
};

namespace {

template <typename T>
sa_status dalloc(T **p, size_t n) {
    if (n == 0) n = 1;
    return cudaMalloc((void **) p, n * sizeof(T)) == cudaSuccess ? SA_OK : SA_E_NOMEM;
}

template <typename T>
sa_status h2d(T *dst, const std::vector<T> &src, cudaStream_t s) {
    if (src.empty()) return SA_OK;
    return cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s) == cudaSuccess
               ? SA_OK : SA_E_CUDA;
}

void free_batch_device(sa_batch *b) {
    cudaFree(b->d_regions); cudaFree(b->d_order); cudaFree(b->d_models); cudaFree(b->d_read_scale);
    cudaFree(b->d_meta); cudaFree(b->d_window_off); cudaFree(b->d_kmer); cudaFree(b->d_gapx); cudaFree(b->d_status);
    cudaFree(b->d_out_count); cudaFree(b->d_windows); cudaFree(b->d_events_raw); cudaFree(b->d_events);
    cudaFree(b->d_F); cudaFree(b->d_fshift); cudaFree(b->d_base); cudaFree(b->d_loglik); cudaFree(b->d_out);
    cudaFree(b->d_queue);
}

// Host planning of a batch (no device work): per read k-mer ids, events and regions, per region its
// windows and per-anti-diagonal meta, the LPT order.  Returns SA_E_CAPACITY for a band wider than
// the kernel's widest ring.
sa_status plan_batch(const sa_read *reads, int64_t n_reads, const sa_params *p, sa_batch *b) {
    sa_status st = SA_OK;
    b->n_reads = n_reads;
    b->threshold = (float) p->threshold;
    b->read_status.assign(n_reads, SA_OK);
    b->read_first_region.assign(n_reads, 0);
    b->read_n_regions.assign(n_reads, 0);
    b->read_scale.resize(n_reads);
    std::vector<Region> regs;
    PathTable pt;
    int device = -1;
    for (int64_t r = 0; r < n_reads; ++r) {
        const sa_read &rd = reads[r];
        auto *sm = const_cast<sa_state_machine *>(rd.sm);
        b->read_first_region[r] = (int64_t) b->regions.size();
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
            d.out_cap = 4 * (int64_t) d.n + 256;
            d.out_base = b->out_total;
            b->out_total += d.out_cap;
            // per anti-diagonal meta: band start, width, window end / refresh / stored gap states
            std::vector<int32_t> flags(d.n + 2, 0);
            for (const Window &w : rg.windows) {
                flags[w.D] |= kFlagWindowEnd;
                for (int32_t r = w.from; r > w.T; r -= 10) flags[r] |= kFlagRefresh;
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
            for (const Window &w : rg.windows) b->window_off.push_back((int32_t) off[w.D]);
            b->cells += acc;
            b->max_width = std::max(b->max_width, rg.max_width);
            b->windows.insert(b->windows.end(), rg.windows.begin(), rg.windows.end());
            b->regions.push_back(d);
        }
        b->read_n_regions[r] = (int64_t) b->regions.size() - b->read_first_region[r];
    }
    if (b->max_width > kMaxCpt * kGroup) return SA_E_CAPACITY;
    b->device = device < 0 ? 0 : device;
    // largest band area first (LPT order for the persistent CTAs)
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
    const size_t nd = b->meta.size();
    st = SA_OK;
    if (!st) st = dalloc(&b->d_regions, b->regions.size());
    if (!st) st = dalloc(&b->d_order, b->order.size());
    if (!st) st = dalloc(&b->d_models, b->models.size());
    if (!st) st = dalloc(&b->d_read_scale, b->read_scale.size());
    if (!st) st = dalloc(&b->d_meta, nd);
    if (!st) st = dalloc(&b->d_window_off, b->window_off.size());
    if (!st) st = dalloc(&b->d_windows, b->windows.size());
    if (!st) st = dalloc(&b->d_kmer, b->kmer.size());
    if (!st) st = dalloc(&b->d_gapx, b->gapx.size());
    if (!st) st = dalloc(&b->d_events_raw, b->events.size());
    if (!st) st = dalloc(&b->d_events, b->events.size());
    if (!st) st = dalloc(&b->d_F, (size_t) kStoreStride * (size_t) b->cells);
    if (!st) st = dalloc(&b->d_base, nd);
    if (!st) st = dalloc(&b->d_fshift, nd);
    if (!st) st = dalloc(&b->d_out, (size_t) b->out_total);
    if (!st) st = dalloc(&b->d_out_count, b->regions.size());
    if (!st) st = dalloc(&b->d_loglik, b->regions.size());
    if (!st) st = dalloc(&b->d_status, (size_t) n_reads);
    if (!st) st = dalloc(&b->d_queue, 1);
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
    if (!st) st = h2d(b->d_window_off, b->window_off, s);
    if (!st) st = h2d(b->d_windows, b->windows, s);
    if (!st) st = h2d(b->d_kmer, b->kmer, s);
    if (!st) st = h2d(b->d_gapx, b->gapx, s);
    if (!st) st = h2d(b->d_events_raw, b->events, s);
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
    sa_status st = SA_OK;
    if (cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned int), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_status, 0, sizeof(int32_t) * std::max<int64_t>(1, b->n_reads), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_out_count, 0, sizeof(int64_t) * std::max<size_t>(1, b->regions.size()), s) != cudaSuccess)
        st = SA_E_CUDA;
    if (!st && !b->regions.empty()) {
        Args a;
        std::memset(&a, 0, sizeof(a));
        a.regions = b->d_regions;
        a.order = b->d_order;
        a.n_regions = (int64_t) b->regions.size();
        a.models = b->d_models;
        a.read_scale = b->d_read_scale;
        a.meta = b->d_meta;
        a.window_off = b->d_window_off;
        a.windows = b->d_windows;
        a.kmer = b->d_kmer;
        a.gapx = b->d_gapx;
        a.events = b->d_events;
        a.F = b->d_F;
        a.base = b->d_base;
        a.fshift = b->d_fshift;
        a.out = b->d_out;
        a.out_count = b->d_out_count;
        a.loglik = b->d_loglik;
        a.status = b->d_status;
        a.queue = b->d_queue;
        a.threshold = b->threshold;
        const int cpt = std::max(1, (b->max_width + kGroup - 1) / kGroup);
        const int cpt_pow2 = cpt <= 1 ? 1 : (cpt <= 2 ? 2 : 4);
        a.wmax = cpt_pow2 * kGroup;
        a.spin_limit = 20000000000LL;   // ~10 s at 2 GHz: far beyond any window's forward time
        const size_t smem = sizeof(Shared) + sizeof(float) * (size_t) (18 * (a.wmax + 2) + 2 * a.wmax);
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
        auto launch = [&](auto kern) {
            if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
            int64_t grid = (int64_t) std::max(1, sms) * std::max(1, per_sm);
            grid = std::min<int64_t>(grid, (int64_t) b->regions.size());
            kern<<<(unsigned) grid, kThreads, smem, s>>>(a);
        };
        if (cpt_pow2 == 1) launch(batch_kernel<1>);
        else if (cpt_pow2 == 2) launch(batch_kernel<2>);
        else launch(batch_kernel<4>);
        count_launch();
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
    const size_t nr = b->regions.size();
    b->out_count.assign(nr, 0);
    b->loglik.assign(nr, 0.0);
    b->dev_status.assign(b->n_reads, 0);
    sa_status st = SA_OK;
    if (nr) {
        if (cudaMemcpyAsync(b->out_count.data(), b->d_out_count, nr * sizeof(int64_t), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaMemcpyAsync(b->loglik.data(), b->d_loglik, nr * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
            st = SA_E_CUDA;
    }
    if (!st && b->n_reads &&
        cudaMemcpyAsync(b->dev_status.data(), b->d_status, b->n_reads * sizeof(int32_t), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess)
        st = SA_E_CUDA;
    if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = SA_E_CUDA;
    // pairs: one copy per region segment in use
    b->read_pairs.assign(b->n_reads, {});
    b->read_ll.assign(b->n_reads, 0.0);
    for (int64_t r = 0; r < b->n_reads && !st; ++r) {
        int64_t total = 0;
        for (int64_t i = 0; i < b->read_n_regions[r]; ++i) {
            const int64_t ri = b->read_first_region[r] + i;
            total += std::min(b->out_count[ri], b->regions[ri].out_cap);
        }
        b->read_pairs[r].resize(total);
        int64_t at = 0;
        for (int64_t i = 0; i < b->read_n_regions[r]; ++i) {
            const int64_t ri = b->read_first_region[r] + i;
            const int64_t cnt = std::min(b->out_count[ri], b->regions[ri].out_cap);
            if (cnt > 0 && cudaMemcpyAsync(b->read_pairs[r].data() + at, b->d_out + b->regions[ri].out_base,
                                           cnt * sizeof(sa_aligned_pair), cudaMemcpyDeviceToHost, s) != cudaSuccess) {
                st = SA_E_CUDA;
                break;
            }
            at += cnt;
            b->read_ll[r] += b->loglik[ri];
        }
    }
    if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = SA_E_CUDA;
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

sa_status sa_batch_transfer_bytes(const sa_batch *b, int64_t *h2d, int64_t *d2h) {
    if (!b || !h2d || !d2h) return SA_E_ARG;
    auto bytes = [](const auto &v) { return (int64_t) (v.size() * sizeof(v[0])); };
    *h2d = bytes(b->regions) + bytes(b->order) + (int64_t) (b->models.size() * sizeof(ModelDesc)) +
           bytes(b->read_scale) + bytes(b->meta) + bytes(b->window_off) + bytes(b->windows) + bytes(b->kmer) + bytes(b->gapx) +
           bytes(b->events);
    int64_t pairs = 0;
    for (const auto &rp : b->read_pairs) pairs += (int64_t) rp.size();
    *d2h = (int64_t) (b->regions.size() * (sizeof(int64_t) + sizeof(double))) + b->n_reads * (int64_t) sizeof(int32_t) +
           pairs * (int64_t) sizeof(sa_aligned_pair);
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
    auto carve = [&](auto **ptr, size_t n) {
        using T = std::remove_reference_t<decltype(**ptr)>;
        at = (at + 255) & ~(size_t) 255;
        if (base) *ptr = reinterpret_cast<T *>(base + at);
        at += std::max<size_t>(n, 1) * sizeof(T);
    };
    const size_t nd = b->meta.size(), nr = b->regions.size();
    carve(&b->d_regions, nr);
    carve(&b->d_order, b->order.size());
    carve(&b->d_models, b->models.size());
    carve(&b->d_read_scale, b->read_scale.size());
    carve(&b->d_meta, nd);
    carve(&b->d_window_off, b->window_off.size());
    carve(&b->d_windows, b->windows.size());
    carve(&b->d_kmer, b->kmer.size());
    carve(&b->d_gapx, b->gapx.size());
    carve(&b->d_events_raw, b->events.size());
    carve(&b->d_events, b->events.size());
    carve(&b->d_F, (size_t) kStoreStride * (size_t) b->cells);
    carve(&b->d_base, nd);
    carve(&b->d_fshift, nd);
    carve(&b->d_out, (size_t) b->out_total);
    carve(&b->d_out_count, nr);
    carve(&b->d_loglik, nr);
    carve(&b->d_status, (size_t) b->n_reads);
    carve(&b->d_queue, 1);
    return (at + 255) & ~(size_t) 255;
}

void batch_release_host(sa_batch *b) { delete b; }

}  // namespace sa
