// Device and pinned-host blocks kept for reuse across batches.
//
// A batch needs one device block (inputs, stores, outputs) and two pinned host blocks (staged
// inputs, results).  cudaMalloc / cudaHostAlloc of hundreds of megabytes cost milliseconds and can
// synchronise the device, so released blocks go to a free list and the next batch of a similar size
// takes one from there.  Blocks come in power-of-two sizes (2 MiB and up), so batches whose sizes
// vary (a serving loop's micro-batches) settle on a few size classes and stop allocating: a request
// takes the smallest free block that is at least as large, otherwise a new block of the request's
// class: an allocation (pinning host pages, mapping device memory) takes milliseconds, which a
// serving loop cannot hide, while a larger block costs only idle memory.  If an allocation fails,
// the free blocks of that kind are released and the allocation is tried once more.
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "sa_internal.h"

namespace sa {
namespace {

constexpr size_t kRound = size_t(2) << 20;

std::mutex g_pool_mutex;
std::vector<MemBlock> g_free;   // blocks not in use

void release_free(MemKind kind, int device) {
    // g_pool_mutex held by the caller
    std::vector<MemBlock> keep;
    for (MemBlock &b : g_free) {
        if (b.kind == kind && (kind != MemKind::Device || b.device == device)) {
            if (kind == MemKind::Device) {
                int prev = 0;
                cudaGetDevice(&prev);
                cudaSetDevice(b.device);
                cudaFree(b.ptr);
                cudaSetDevice(prev);
            } else {
                cudaFreeHost(b.ptr);
            }
        } else {
            keep.push_back(b);
        }
    }
    g_free.swap(keep);
}

bool allocate(MemKind kind, int device, size_t bytes, void **ptr) {
    if (kind == MemKind::Device) {
        int prev = 0;
        cudaGetDevice(&prev);
        bool ok = cudaSetDevice(device) == cudaSuccess && device_malloc(ptr, bytes) == cudaSuccess;
        cudaSetDevice(prev);
        if (!ok) cudaGetLastError();
        return ok;
    }
    const bool ok = pinned_malloc(ptr, bytes) == cudaSuccess;
    if (!ok) cudaGetLastError();
    return ok;
}

}  // namespace

sa_status mem_get(MemKind kind, int device, size_t bytes, MemBlock &out) {
    out = MemBlock{};
    if (bytes == 0) bytes = 1;
    if (kind == MemKind::Heap) {
        const size_t rounded = (bytes + 255) & ~size_t(255);
        void *p = std::aligned_alloc(256, rounded);
        if (!p) return SA_E_NOMEM;
        out = MemBlock{p, rounded, -1, kind};
        return SA_OK;
    }
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    size_t best = g_free.size();
    for (size_t i = 0; i < g_free.size(); ++i) {
        const MemBlock &b = g_free[i];
        if (b.kind != kind || (kind == MemKind::Device && b.device != device)) continue;
        if (b.bytes < bytes) continue;
        if (best == g_free.size() || b.bytes < g_free[best].bytes) best = i;
    }
    if (best < g_free.size()) {
        out = g_free[best];
        g_free.erase(g_free.begin() + (std::ptrdiff_t) best);
        return SA_OK;
    }
    size_t rounded = kRound;
    while (rounded < bytes) rounded <<= 1;
    void *p = nullptr;
    if (!allocate(kind, device, rounded, &p)) {
        release_free(kind, device);
        if (!allocate(kind, device, rounded, &p)) return SA_E_NOMEM;
    }
    out = MemBlock{p, rounded, device, kind};
    return SA_OK;
}

void mem_put(MemBlock &b) {
    if (!b.ptr) return;
    if (b.kind == MemKind::Heap) {
        std::free(b.ptr);
    } else {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        g_free.push_back(b);
    }
    b = MemBlock{};
}

}  // namespace sa
