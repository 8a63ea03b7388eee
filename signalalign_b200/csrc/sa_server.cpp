// Serving loop: reads arrive one at a time and are aligned with continuous batching.
//
// A dispatcher thread owns the device side.  Each turn it (1) collects finished micro-batches
// (an event recorded after their kernels), copies each read's pairs and status to its ticket and
// returns the batch's memory to the pools; (2) admits waiting reads: as many as fit the band-cell
// budget (estimated from the read's size and the diagonal expansion) go into one new micro-batch,
// which is planned, uploaded and launched on a stream of its own, so it runs beside the batches
// already on the device.  A read that arrives while others are running waits only for budget and
// a free stream, not for them to finish.  Each read's computation depends on nothing but its own
// inputs, so its result is the same alone and in any mix.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "sa_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    // owned copies of the read's inputs
    std::string reference;
    std::vector<double> events;
    std::vector<int64_t> anchors;
    sa_read read;
    sa_params params;
    int64_t cells_estimate = 0;
    Clock::time_point submitted;
    // results
    bool done = false;
    sa_status status = SA_OK;
    std::vector<sa_aligned_pair> pairs;
    double log_likelihood = 0.0;
    double latency_ms = 0.0;
};

struct InFlight {
    sa_batch *batch = nullptr;
    int stream_index = -1;
    cudaEvent_t finished = nullptr;
    std::vector<int64_t> tickets;
    int64_t cells = 0;
};

bool same_params(const sa_params &a, const sa_params &b) { return std::memcmp(&a, &b, sizeof(sa_params)) == 0; }

}  // namespace

struct sa_server {
    int device = 0;
    int64_t budget_cells = 0;
    std::vector<cudaStream_t> streams;
    std::vector<bool> stream_busy;
    std::mutex mu;
    std::condition_variable cv_done;
    std::deque<int64_t> pending;
    std::unordered_map<int64_t, Request> requests;
    std::vector<InFlight> inflight;
    int64_t inflight_cells = 0;
    int64_t next_ticket = 1;
    bool stop = false;
    std::thread loop;

    void finish(InFlight &f) {
        sa_status st = sa_batch_download(f.batch, streams[f.stream_index]);
        const Clock::time_point now = Clock::now();
        std::lock_guard<std::mutex> lock(mu);
        for (size_t i = 0; i < f.tickets.size(); ++i) {
            Request &rq = requests[f.tickets[i]];
            rq.status = st ? st : sa_batch_read_status(f.batch, (int64_t) i);
            if (!rq.status) {
                const int64_t n = sa_batch_pair_count(f.batch, (int64_t) i);
                const sa_aligned_pair *pp = sa_batch_pairs(f.batch, (int64_t) i);
                rq.pairs.assign(pp, pp + (n > 0 ? n : 0));
                rq.log_likelihood = sa_batch_log_likelihood(f.batch, (int64_t) i);
            }
            rq.latency_ms = std::chrono::duration<double, std::milli>(now - rq.submitted).count();
            rq.done = true;
        }
        inflight_cells -= f.cells;
        stream_busy[f.stream_index] = false;
        cv_done.notify_all();
    }

    // one micro-batch of waiting reads (same parameters), within the budget; false if none fits
    bool admit() {
        std::vector<int64_t> take;
        std::vector<sa_read> reads;
        sa_params p;
        int64_t cells = 0;
        int si = -1;
        {
            std::lock_guard<std::mutex> lock(mu);
            if (pending.empty()) return false;
            for (size_t k = 0; k < stream_busy.size(); ++k)
                if (!stream_busy[k]) { si = (int) k; break; }
            if (si < 0) return false;
            p = requests[pending.front()].params;
            while (!pending.empty()) {
                const Request &rq = requests[pending.front()];
                if (!same_params(rq.params, p)) break;
                const bool first = take.empty() && inflight.empty();
                if (!first && inflight_cells + cells + rq.cells_estimate > budget_cells) break;
                cells += rq.cells_estimate;
                take.push_back(pending.front());
                reads.push_back(rq.read);
                pending.pop_front();
            }
            if (take.empty()) return false;
            stream_busy[si] = true;
            inflight_cells += cells;
        }
        InFlight f;
        f.stream_index = si;
        f.tickets = take;
        f.cells = cells;
        cudaStream_t s = streams[si];
        sa_status st = sa_batch_create(reads.data(), (int64_t) reads.size(), &p, &f.batch);
        if (!st) st = sa_batch_upload(f.batch, s);
        if (!st) st = sa_batch_run(f.batch, s);
        if (!st && (cudaEventCreateWithFlags(&f.finished, cudaEventDisableTiming) != cudaSuccess ||
                    cudaEventRecord(f.finished, s) != cudaSuccess))
            st = SA_E_CUDA;
        if (st) {
            const Clock::time_point now = Clock::now();
            std::lock_guard<std::mutex> lock(mu);
            for (int64_t t : take) {
                Request &rq = requests[t];
                rq.status = st;
                rq.done = true;
                rq.latency_ms = std::chrono::duration<double, std::milli>(now - rq.submitted).count();
            }
            inflight_cells -= cells;
            stream_busy[si] = false;
            if (f.finished) cudaEventDestroy(f.finished);
            sa_batch_destroy(f.batch);
            cv_done.notify_all();
            return true;
        }
        std::lock_guard<std::mutex> lock(mu);
        inflight.push_back(f);
        return true;
    }

    void run() {
        cudaSetDevice(device);
        for (;;) {
            bool worked = false;
            // finished micro-batches
            std::vector<InFlight> finished;
            {
                std::lock_guard<std::mutex> lock(mu);
                for (size_t k = 0; k < inflight.size();) {
                    if (cudaEventQuery(inflight[k].finished) == cudaSuccess) {
                        finished.push_back(inflight[k]);
                        inflight.erase(inflight.begin() + (std::ptrdiff_t) k);
                    } else {
                        ++k;
                    }
                }
            }
            for (InFlight &f : finished) {
                finish(f);
                cudaEventDestroy(f.finished);
                sa_batch_destroy(f.batch);
                worked = true;
            }
            while (admit()) worked = true;
            {
                std::lock_guard<std::mutex> lock(mu);
                if (stop && pending.empty() && inflight.empty()) break;
            }
            if (!worked) std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
};

extern "C" {

sa_status sa_server_create(int32_t device, int64_t max_inflight_cells, int32_t max_batches, sa_server **out) {
    if (!out || max_inflight_cells <= 0 || max_batches <= 0) return SA_E_ARG;
    *out = nullptr;
    auto *s = new (std::nothrow) sa_server();
    if (!s) return SA_E_NOMEM;
    s->device = device;
    s->budget_cells = max_inflight_cells;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) {
        delete s;
        return SA_E_CUDA;
    }
    for (int32_t k = 0; k < max_batches; ++k) {
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            for (cudaStream_t q : s->streams) cudaStreamDestroy(q);
            cudaSetDevice(prev);
            delete s;
            return SA_E_CUDA;
        }
        s->streams.push_back(st);
    }
    s->stream_busy.assign(max_batches, false);
    cudaSetDevice(prev);
    s->loop = std::thread([s]() { s->run(); });
    *out = s;
    return SA_OK;
}

sa_status sa_server_submit(sa_server *s, const sa_read *read, const sa_params *p, int64_t *ticket) {
    if (!s || !read || !p || !ticket) return SA_E_ARG;
    if (read->reference_length < 0 || read->n_events < 0 || read->n_anchors < 0 ||
        (read->reference_length > 0 && !read->reference) || (read->n_events > 0 && !read->events) ||
        (read->n_anchors > 0 && !read->anchors))
        return SA_E_ARG;
    Request rq;
    rq.reference.assign(read->reference ? read->reference : "", (size_t) read->reference_length);
    rq.events.assign(read->events, read->events + read->n_events * sa::kEventParams);
    rq.anchors.assign(read->anchors, read->anchors + 2 * read->n_anchors);
    rq.read = *read;
    rq.read.reference = rq.reference.c_str();
    rq.read.events = rq.events.data();
    rq.read.anchors = rq.anchors.data();
    rq.params = *p;
    rq.cells_estimate = (read->reference_length + read->n_events + 1) * (p->diagonal_expansion + 1);
    rq.submitted = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop) return SA_E_ARG;
    const int64_t t = s->next_ticket++;
    auto it = s->requests.emplace(t, std::move(rq)).first;
    // pointers into the stored copies (the map node does not move)
    it->second.read.reference = it->second.reference.c_str();
    it->second.read.events = it->second.events.data();
    it->second.read.anchors = it->second.anchors.data();
    s->pending.push_back(t);
    *ticket = t;
    return SA_OK;
}

sa_status sa_server_wait(sa_server *s, int64_t ticket, double timeout_ms) {
    if (!s) return SA_E_ARG;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return SA_E_ARG;
    const bool ok = s->cv_done.wait_for(lock, std::chrono::duration<double, std::milli>(timeout_ms),
                                        [&]() { return s->requests[ticket].done; });
    return ok ? SA_OK : SA_E_TIMEOUT;
}

sa_status sa_server_result(sa_server *s, int64_t ticket, int32_t *status, const sa_aligned_pair **pairs,
                           int64_t *n_pairs, double *log_likelihood, double *latency_ms) {
    if (!s || !status || !pairs || !n_pairs) return SA_E_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end() || !it->second.done) return SA_E_ARG;
    const Request &rq = it->second;
    *status = rq.status;
    *pairs = rq.pairs.data();
    *n_pairs = (int64_t) rq.pairs.size();
    if (log_likelihood) *log_likelihood = rq.log_likelihood;
    if (latency_ms) *latency_ms = rq.latency_ms;
    return SA_OK;
}

sa_status sa_server_release(sa_server *s, int64_t ticket) {
    if (!s) return SA_E_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end() || !it->second.done) return SA_E_ARG;
    s->requests.erase(it);
    return SA_OK;
}

void sa_server_destroy(sa_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    if (s->loop.joinable()) s->loop.join();
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    for (cudaStream_t q : s->streams) cudaStreamDestroy(q);
    cudaSetDevice(prev);
    delete s;
}

}  // extern "C"
