// Per-read scale / shift / drift / variance estimation, the step before the path
// (signalUtils_estimateNanoporeParams, impl/signalMachineUtils.c:186-223): the read's 1D event <->
// k-mer assignments (nanopore_getOneDAssignmentsFromRead, impl/nanopore.c:503-533) feed two weighted
// least-squares fits (nanopore_compute_mean_scale_params with drift and variance, :650-781;
// nanopore_compute_noise_scale_params, :783-848).  The assignments are extracted on the host; the
// fits run on the GPU, one CTA per read: FP64 sums reduced over the CTA, the normal equations solved
// by Gaussian elimination as the reference does (nanopore_lineq_solve, :586-648), then a second
// reduction for the dispersions.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sa_internal.h"

namespace sa {
namespace {

constexpr int kParamThreads = 256;

struct Assignment {
    double mean, sd, dt;   // event mean, event noise, event delta time (events[4 i + 3])
    int64_t kmer;
};

struct ParamTask {
    int64_t first, count;        // assignments of the read
    const double *model;         // the read's match table: 5 doubles per k-mer (mean, sd, noise mean, noise sd, lambda)
};

// nanopore_lineq_solve: Gauss-Jordan elimination without pivoting on these symmetric positive
// systems (the reference swaps rows only for a pivot below machine epsilon, which a weighted normal
// matrix of distinct levels never has; a singular system returns false here instead of exiting)
template <int N>
__device__ bool lineq_solve(double (&a)[N][N], double (&x)[N]) {
    for (int i = 0; i < N; ++i) {
        if (!(fabs(a[i][i]) >= 1.11022302462515654042E-16)) return false;
        const double f = 1.0 / a[i][i];
        x[i] *= f;
        for (int j = 0; j < N; ++j) a[i][j] *= f;
        for (int s = i + 1; s < N; ++s) {
            const double g = a[s][i];
            x[s] -= g * x[i];
            for (int j = 0; j < N; ++j) a[s][j] -= g * a[i][j];
        }
    }
    for (int i = N - 1; i >= 0; --i)
        for (int s = i - 1; s >= 0; --s) {
            const double g = a[s][i];
            x[s] -= g * x[i];
            for (int j = 0; j < N; ++j) a[s][j] -= g * a[i][j];
        }
    return true;
}

// sum of v over the CTA (every thread gets it)
template <int K>
__device__ void block_sum(double (&v)[K], double (*scratch)[K]) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0)
        for (int k = 0; k < K; ++k) scratch[warp][k] = v[k];
    __syncthreads();
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int w = 0; w < kParamThreads / 32; ++w) s += scratch[w][k];
        v[k] = s;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kParamThreads) estimate_params_kernel(const ParamTask *tasks, const Assignment *as,
                                                                        sa_read_params *out, int32_t *status) {
    __shared__ double scratch[kParamThreads / 32][14];
    const ParamTask t = tasks[blockIdx.x];
    const Assignment *a = as + t.first;
    const double *model = t.model;
    // normal equations: level mean (shift, scale, drift) and noise (shift_sd, scale_sd), weighted by
    // the inverse variance of the k-mer's level and noise distributions
    double s[14] = {0};
    for (int64_t i = threadIdx.x; i < t.count; i += kParamThreads) {
        const Assignment e = a[i];
        const double lm = model[e.kmer * 5], lsd = model[e.kmer * 5 + 1];
        const double nm = model[e.kmer * 5 + 2], nsd = model[e.kmer * 5 + 3];
        const double iv = 1.0 / (lsd * lsd), sm = lm * iv, st = e.dt * iv;
        s[0] += iv; s[1] += sm; s[2] += st; s[3] += sm * lm; s[4] += sm * e.dt; s[5] += st * e.dt;
        s[6] += iv * e.mean; s[7] += sm * e.mean; s[8] += st * e.mean;
        const double inv = 1.0 / (nsd * nsd), snm = nm * inv;
        s[9] += inv; s[10] += snm; s[11] += snm * nm;
        s[12] += inv * e.sd; s[13] += snm * e.sd;
    }
    block_sum<14>(s, scratch);
    double m[3][3] = {{s[0], s[1], s[2]}, {s[1], s[3], s[4]}, {s[2], s[4], s[5]}};
    double beta[3] = {s[6], s[7], s[8]};
    double q[2][2] = {{s[9], s[10]}, {s[10], s[11]}};
    double gamma[2] = {s[12], s[13]};
    const bool ok = t.count > 0 && lineq_solve<3>(m, beta) && lineq_solve<2>(q, gamma);
    // dispersions of the residuals, weighted by the level (noise) variance
    double r[2] = {0.0, 0.0};
    if (ok)
        for (int64_t i = threadIdx.x; i < t.count; i += kParamThreads) {
            const Assignment e = a[i];
            const double lm = model[e.kmer * 5], lsd = model[e.kmer * 5 + 1];
            const double nm = model[e.kmer * 5 + 2], nsd = model[e.kmer * 5 + 3];
            const double res = e.mean - (beta[0] + beta[1] * lm + beta[2] * e.dt);
            r[0] += (res * res) / (lsd * lsd);
            const double rn = e.sd - (gamma[0] + gamma[1] * nm);
            r[1] += (rn * rn) / (nsd * nsd);
        }
    block_sum<2>(r, reinterpret_cast<double(*)[2]>(&scratch[0][0]));
    if (threadIdx.x == 0) {
        if (!ok) {
            status[blockIdx.x] = SA_E_ARG;
            return;
        }
        sa_read_params p = out[blockIdx.x];
        p.shift = beta[0];
        p.scale = beta[1];
        p.drift = beta[2];
        p.var = sqrt(r[0] / (double) t.count);
        p.shift_sd = gamma[0];
        p.scale_sd = gamma[1];
        p.var_sd = sqrt(r[1] / (double) t.count);
        out[blockIdx.x] = p;
        status[blockIdx.x] = SA_OK;
    }
}

// nanopore_getOneDAssignmentsFromRead: for each k-mer of the strand's read, its event, kept only for
// the first position an event maps to (later ones fill skipped k-mers)
sa_status one_d_assignments(const sa_param_read &rd, std::vector<Assignment> &out) {
    const sa_state_machine *sm = rd.sm;
    const int k = sm->kmer_length;
    const int64_t rows = rd.read_length - (k - 1);
    int64_t prev = -1;
    for (int64_t i = 0; i < rows; ++i) {
        const int64_t ev = rd.event_map[i];
        if (ev < 0 || ev >= rd.n_events) return SA_E_ARG;
        int64_t id = 0;
        for (int j = 0; j < k; ++j) {
            const size_t pos = sm->alphabet.find(rd.read[i + j]);
            if (pos == std::string::npos) return SA_E_ALPHABET;
            id = id * (int64_t) sm->alphabet.size() + (int64_t) pos;
        }
        if (ev > prev) {
            const double *e = rd.events + 4 * ev;
            out.push_back(Assignment{e[0], e[1], e[3], id});
            prev = ev;
        }
    }
    return SA_OK;
}

}  // namespace
}  // namespace sa

using namespace sa;

extern "C" {

sa_status sa_oneDAssignmentsFromRead(const sa_param_read *read, int64_t *kmer_ids, double *event_params,
                                     int64_t capacity, int64_t *n_out) {
    if (!read || !read->sm || !n_out || read->read_length < 0 || read->n_events < 0 ||
        (read->read_length > 0 && (!read->read || !read->event_map)) || (read->n_events > 0 && !read->events))
        return SA_E_ARG;
    std::vector<Assignment> v;
    const sa_status st = one_d_assignments(*read, v);
    if (st) return st;
    *n_out = (int64_t) v.size();
    if ((int64_t) v.size() > capacity) return SA_E_OUTPUT;
    for (size_t i = 0; i < v.size(); ++i) {
        if (kmer_ids) kmer_ids[i] = v[i].kmer;
        if (event_params) {
            event_params[3 * i] = v[i].mean;
            event_params[3 * i + 1] = v[i].sd;
            event_params[3 * i + 2] = v[i].dt;
        }
    }
    return SA_OK;
}

sa_status sa_estimateNanoporeParams(const sa_param_read *reads, int64_t n_reads, sa_read_params *params,
                                    int32_t *read_status, void *stream) {
    if (n_reads < 0 || (n_reads > 0 && (!reads || !params || !read_status))) return SA_E_ARG;
    if (n_reads == 0) return SA_OK;
    // assignments of every read, packed
    std::vector<Assignment> all;
    std::vector<ParamTask> tasks(n_reads);
    int device = -1;
    for (int64_t r = 0; r < n_reads; ++r) {
        const sa_param_read &rd = reads[r];
        if (!rd.sm || rd.read_length < 0 || rd.n_events < 0 || (rd.read_length > 0 && (!rd.read || !rd.event_map)) ||
            (rd.n_events > 0 && !rd.events))
            return SA_E_ARG;
        if (device < 0) device = rd.sm->dev.device;
        if (rd.sm->dev.device != device) return SA_E_ARG;
        tasks[r].first = (int64_t) all.size();
        const sa_status st = one_d_assignments(rd, all);
        if (st) return st;
        tasks[r].count = (int64_t) all.size() - tasks[r].first;
        read_status[r] = tasks[r].count > 0 ? SA_OK : SA_E_ARG;   // the reference aborts with no assignments
    }
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return SA_E_CUDA;
    sa_status st = SA_OK;
    for (int64_t r = 0; r < n_reads && !st; ++r) {
        st = ensure_device_model(const_cast<sa_state_machine *>(reads[r].sm));
        tasks[r].model = reads[r].sm->dev.match;
    }
    // one device block and one pinned block: tasks, assignments, parameters, statuses
    const size_t tb = sizeof(ParamTask) * (size_t) n_reads, ab = sizeof(Assignment) * std::max<size_t>(all.size(), 1);
    const size_t pb = sizeof(sa_read_params) * (size_t) n_reads, sb = sizeof(int32_t) * (size_t) n_reads;
    auto up = [](size_t v) { return (v + 255) & ~(size_t) 255; };
    const size_t o_a = up(tb), o_p = o_a + up(ab), o_s = o_p + up(pb), total = o_s + up(sb);
    MemBlock dev, host;
    if (!st) st = mem_get(MemKind::Device, device, total, dev);
    if (!st) st = mem_get(MemKind::Pinned, device, total, host);
    if (!st) {
        auto *h = static_cast<unsigned char *>(host.ptr);
        std::memcpy(h, tasks.data(), tb);
        if (!all.empty()) std::memcpy(h + o_a, all.data(), sizeof(Assignment) * all.size());
        std::memcpy(h + o_p, params, pb);
        cudaStream_t s = (cudaStream_t) stream;
        auto *d = static_cast<unsigned char *>(dev.ptr);
        if (cudaMemcpyAsync(d, h, o_s, cudaMemcpyHostToDevice, s) != cudaSuccess) st = SA_E_CUDA;
        if (!st) {
            estimate_params_kernel<<<(unsigned) n_reads, kParamThreads, 0, s>>>(
                reinterpret_cast<const ParamTask *>(d), reinterpret_cast<const Assignment *>(d + o_a),
                reinterpret_cast<sa_read_params *>(d + o_p), reinterpret_cast<int32_t *>(d + o_s));
            count_launch();
            if (cudaGetLastError() != cudaSuccess) st = SA_E_CUDA;
        }
        if (!st && (cudaMemcpyAsync(h + o_p, d + o_p, total - o_p, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                    cudaStreamSynchronize(s) != cudaSuccess))
            st = SA_E_CUDA;
        if (!st) {
            std::memcpy(params, h + o_p, pb);
            const auto *ks = reinterpret_cast<const int32_t *>(h + o_s);
            for (int64_t r = 0; r < n_reads; ++r)
                if (!read_status[r]) read_status[r] = ks[r];
        }
    }
    mem_put(dev);
    mem_put(host);
    cudaSetDevice(prev);
    return st;
}

sa_status sa_adjustEventsForDrift(double *events, int64_t n_events, double drift) {
    if (n_events < 0 || (n_events > 0 && !events)) return SA_E_ARG;
    // nanopore_adjustEventsForDriftP (nanopore.c:535-540): mean -= delta time x drift
    for (int64_t i = 0; i < n_events; ++i) events[4 * i] = events[4 * i] - events[4 * i + 3] * drift;
    return SA_OK;
}

}  // extern "C"
