// sa_align_batch_noalloc: the batched FP32 alignment with its device buffers carved from one static
// device array instead of cudaMalloc.
//
// Who needs it: a host process embedded in a framework that keeps nearly all of the GPU's memory in
// its own pool cannot count on cudaMalloc succeeding (and making room would mean asking the
// framework to shrink its pool), and a latency-bound serving loop cannot afford cudaMalloc /
// cudaFree, which may synchronise the device and stall the other streams.  Both can still run
// alignments through this entry point: the array below is reserved when the library's device code
// is loaded on a device, and each call only reuses it.
//
// Sharing: one array per device for the whole process, so calls on a device must not overlap.  A
// per-device mutex held for the whole (synchronous) call serialises callers on different host
// threads.
#include <cstring>
#include <mutex>

#include "sa_internal.h"

namespace {

// The scratch array: inputs, forward store, base arrays, counters and pair output of one batch.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SA_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;

std::mutex g_device_mutex[kMaxDevices];
unsigned char *g_scratch_addr[kMaxDevices] = {};   // looked up once per device, under its mutex

// Address of the array on the current device (which must be `device`); the first call per device
// does the lookup.
sa_status scratch_address(int device, unsigned char **out) {
    if (!g_scratch_addr[device]) {
        void *ptr = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (rc != cudaSuccess || !ptr) return SA_E_CUDA;
        g_scratch_addr[device] = static_cast<unsigned char *>(ptr);
    }
    *out = g_scratch_addr[device];
    return SA_OK;
}

}  // namespace

extern "C" sa_status sa_align_batch_noalloc(const sa_read *reads, int64_t n_reads, const sa_params *p, void *stream,
                                            sa_aligned_pair *pairs, int64_t pair_capacity, int64_t *pair_offsets,
                                            int32_t *read_status, double *log_likelihood, int64_t *scratch_bytes) {
    if (!pair_offsets || !read_status || pair_capacity < 0 || (pair_capacity > 0 && !pairs)) return SA_E_ARG;
    sa_batch *b = nullptr;
    sa_status st = sa::batch_plan_host(reads, n_reads, p, &b);
    if (st) return st;
    // host-only checks first: size, then the models' device tables
    const size_t need = sa::batch_bind_scratch(b, nullptr);
    if (scratch_bytes) *scratch_bytes = (int64_t) need;
    const int device = sa::batch_device(b);
    if (need > (size_t) SA_NOALLOC_SCRATCH_BYTES) st = SA_E_CAPACITY;
    else if (!sa::batch_models_resident(b)) st = SA_E_ARG;
    else if (device < 0 || device >= kMaxDevices) st = SA_E_ARG;
    if (st) {
        sa::batch_release_host(b);
        return st;
    }
    {
        std::lock_guard<std::mutex> lock(g_device_mutex[device]);
        int prev = 0;
        unsigned char *base = nullptr;
        if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) st = SA_E_CUDA;
        if (!st) st = scratch_address(device, &base);
        if (!st) {
            sa::batch_bind_scratch(b, base);
            st = sa_batch_upload(b, stream);
            if (!st) st = sa_batch_run(b, stream);
            if (!st) st = sa_batch_download(b, stream);
            // a failed step may leave copies or kernels queued that still write the array: let the
            // stream drain before the lock lets the next caller in
            if (st) cudaStreamSynchronize((cudaStream_t) stream);
        }
        cudaSetDevice(prev);
    }
    if (!st) {
        int64_t at = 0;
        pair_offsets[0] = 0;
        for (int64_t r = 0; r < n_reads; ++r) {
            read_status[r] = (int32_t) sa_batch_read_status(b, r);
            const int64_t n = read_status[r] == SA_OK ? sa_batch_pair_count(b, r) : 0;
            at += n > 0 ? n : 0;
            pair_offsets[r + 1] = at;
            if (log_likelihood) log_likelihood[r] = sa_batch_log_likelihood(b, r);
        }
        if (at > pair_capacity) {
            st = SA_E_OUTPUT;
        } else {
            for (int64_t r = 0; r < n_reads; ++r) {
                const int64_t n = pair_offsets[r + 1] - pair_offsets[r];
                if (n > 0) std::memcpy(pairs + pair_offsets[r], sa_batch_pairs(b, r), (size_t) n * sizeof(sa_aligned_pair));
            }
        }
    }
    sa::batch_release_host(b);
    return st;
}
