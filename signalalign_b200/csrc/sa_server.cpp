// Serving loop: reads arrive one at a time and are aligned with continuous batching.
//
// Host threads of two kinds own the device side.
//  * Admission threads (up to four, planning in parallel) admit waiting reads whenever a stream is
//    free: as many as fit the band-cell budget (estimated from the read's size and the diagonal
//    expansion) go into one new micro-batch, which is planned, uploaded and launched on a stream of
//    its own, so it runs beside the batches already on the device.  A read that arrives while others
//    are running waits only for budget and a free stream, not for them to finish.
//  * The completion thread finishes reads as the worker kernel publishes them: a micro-batch runs
//    with per-read completion, so the kernel group that ends a read's last traceback window gathers
//    the read's pairs and writes the read's record to mapped host memory; the thread sees the
//    record, copies that read's pairs on a side stream while the kernel runs on and hands the
//    result to the ticket, so a read does not wait for the longest read of its micro-batch.  When
//    a micro-batch's kernels end (an event recorded after them) it finishes the reads that got no
//    record (plain-form reads, plan errors, a run whose bounded wait gave up) from the batch's
//    download, frees the stream and returns the batch's memory to the pools.
// Planning and upload therefore never delay the hand-over of finished reads.  Each read's
// computation depends on nothing but its own inputs, so its result is the same alone and in any mix.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <algorithm>
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
    Clock::time_point submitted, admitted, launched;
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
    const sa::ReadDone *records = nullptr;   // per read, written by the worker kernel
    int32_t seq = 0;                         // the run whose records count
    std::vector<char> handled;               // per read: its ticket is finished
    size_t n_handled = 0;
};

bool same_params(const sa_params &a, const sa_params &b) { return std::memcmp(&a, &b, sizeof(sa_params)) == 0; }

}  // namespace

struct sa_server {
    int device = 0;
    int64_t budget_cells = 0;
    std::vector<cudaStream_t> streams;
    std::vector<bool> stream_busy;
    cudaStream_t fetch_stream = nullptr;     // copies of published reads
    sa::MemBlock staging;                    // pinned landing area of those copies (grows)
    cudaEvent_t origin = nullptr;            // device time zero of the batch log
    int64_t reads_early = 0, reads_at_end = 0, batches = 0;
    double admit_ms = 0.0, fetch_ms = 0.0, finish_ms = 0.0;   // host time by activity
    double plan_ms = 0.0, upload_ms = 0.0;   // parts of admit_ms
    std::vector<double> batch_log;           // per finished micro-batch: start ms, end ms, reads
    std::mutex mu;                           // guards everything above and below but the threads
    std::condition_variable cv_done;         // a read finished
    std::condition_variable cv_admit;        // a read arrived, a stream or budget came free, or stop
    uint64_t wake = 0;                       // bumped with every cv_admit notification
    std::deque<int64_t> pending;
    std::unordered_map<int64_t, Request> requests;
    // micro-batches on the device; an entry's fields belong to the completion thread once listed
    std::vector<std::unique_ptr<InFlight>> inflight;
    int64_t inflight_cells = 0;
    int64_t next_ticket = 1;
    bool stop = false, admission_over = false;
    int admitters_left = 0;
    std::vector<std::thread> admitters;
    std::thread completer;

    // hands a finished read's result to its ticket (mu held)
    void complete(int64_t ticket, sa_status st, std::vector<sa_aligned_pair> &&pairs, double ll,
                  Clock::time_point now) {
        Request &rq = requests[ticket];
        rq.status = st;
        if (!st) {
            rq.pairs = std::move(pairs);
            rq.log_likelihood = ll;
        }
        rq.latency_ms = std::chrono::duration<double, std::milli>(now - rq.submitted).count();
        rq.done = true;
    }

    void wake_admission() {
        // mu held
        ++wake;
        cv_admit.notify_all();
    }

    // reads of `f` the worker kernel has published since the last look (completion thread)
    bool poll(InFlight &f) {
        if (!f.records || f.seq <= 0 || f.n_handled == f.tickets.size()) return false;
        bool any = false;
        const Clock::time_point t0 = Clock::now();
        for (size_t i = 0; i < f.tickets.size(); ++i) {
            if (f.handled[i] || *reinterpret_cast<const volatile int32_t *>(&f.records[i].done) != f.seq) continue;
            std::atomic_thread_fence(std::memory_order_acquire);
            const sa::ReadDone rec = *const_cast<const sa::ReadDone *>(&f.records[i]);
            sa_status st = (sa_status) rec.status;
            std::vector<sa_aligned_pair> pairs;
            if (!st && rec.n_pairs > 0) {
                const size_t bytes = sizeof(sa_aligned_pair) * (size_t) rec.n_pairs;
                if (staging.bytes < bytes) {
                    sa::mem_put(staging);
                    st = sa::mem_get(sa::MemKind::Pinned, device, bytes, staging);
                }
                if (!st) st = sa::batch_fetch_read(f.batch, rec, static_cast<sa_aligned_pair *>(staging.ptr), fetch_stream);
                if (!st) {
                    const auto *src = static_cast<const sa_aligned_pair *>(staging.ptr);
                    pairs.assign(src, src + rec.n_pairs);
                }
            }
            const Clock::time_point now = Clock::now();
            {
                std::lock_guard<std::mutex> lock(mu);
                complete(f.tickets[i], st, std::move(pairs), rec.log_likelihood, now);
                ++reads_early;
            }
            cv_done.notify_all();
            f.handled[i] = 1;
            ++f.n_handled;
            any = true;
        }
        if (any) {
            std::lock_guard<std::mutex> lock(mu);
            fetch_ms += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        }
        return any;
    }

    // a micro-batch whose kernels ended (completion thread)
    void finish(InFlight &f) {
        // records the kernel wrote since the last poll are final now; the reads it did not publish
        // come from the batch's download
        poll(f);
        const Clock::time_point t_begin = Clock::now();
        const bool rest = f.n_handled < f.tickets.size();
        sa_status st = rest ? sa_batch_download(f.batch, streams[f.stream_index]) : SA_OK;
        double start_ms = 0.0, end_ms = 0.0;
        cudaEvent_t e0, e1;
        float t0 = 0.f, t1 = 0.f;
        if (sa::batch_run_events(f.batch, &e0, &e1) && cudaEventElapsedTime(&t0, origin, e0) == cudaSuccess &&
            cudaEventElapsedTime(&t1, origin, e1) == cudaSuccess) {
            start_ms = t0;
            end_ms = t1;
        } else {
            cudaGetLastError();
        }
        const Clock::time_point now = Clock::now();
        std::lock_guard<std::mutex> lock(mu);
        for (size_t i = 0; i < f.tickets.size(); ++i) {
            if (f.handled[i]) continue;
            const int64_t r = (int64_t) i;
            const sa_status rs = st ? st : sa_batch_read_status(f.batch, r);
            std::vector<sa_aligned_pair> pairs;
            if (!rs) {
                const int64_t n = sa_batch_pair_count(f.batch, r);
                const sa_aligned_pair *pp = sa_batch_pairs(f.batch, r);
                pairs.assign(pp, pp + (n > 0 ? n : 0));
            }
            complete(f.tickets[i], rs, std::move(pairs), rs ? 0.0 : sa_batch_log_likelihood(f.batch, r), now);
            ++reads_at_end;
        }
        ++batches;
        batch_log.push_back(start_ms);
        batch_log.push_back(end_ms);
        batch_log.push_back((double) f.tickets.size());
        inflight_cells -= f.cells;
        stream_busy[f.stream_index] = false;
        finish_ms += std::chrono::duration<double, std::milli>(Clock::now() - t_begin).count();
        cv_done.notify_all();
        wake_admission();
    }

    // one micro-batch of waiting reads (same parameters), within the budget; false if none fits
    // (admission thread)
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
                // a read above the whole budget goes alone onto an idle device
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
        const Clock::time_point t_admit = Clock::now();
        auto f = std::make_unique<InFlight>();
        f->stream_index = si;
        f->tickets = take;
        f->cells = cells;
        cudaStream_t s = streams[si];
        sa_status st = sa_batch_create(reads.data(), (int64_t) reads.size(), &p, &f->batch);
        if (!st) st = sa::batch_publish_reads(f->batch);
        if (!st) {
            f->records = sa::batch_read_records(f->batch);
            f->handled.assign(take.size(), 0);
        }
        const Clock::time_point t_plan = Clock::now();
        if (!st) st = sa_batch_upload(f->batch, s);
        const Clock::time_point t_upload = Clock::now();
        if (!st) st = sa_batch_run(f->batch, s);
        f->seq = sa::batch_run_seq(f->batch);
        if (!st && (cudaEventCreateWithFlags(&f->finished, cudaEventDisableTiming) != cudaSuccess ||
                    cudaEventRecord(f->finished, s) != cudaSuccess))
            st = SA_E_CUDA;
        const Clock::time_point t_launch = Clock::now();
        if (st) {
            // nothing of this micro-batch is on the device (a failed launch leaves the stream idle)
            cudaStreamSynchronize(s);
            cudaGetLastError();
            std::lock_guard<std::mutex> lock(mu);
            for (int64_t t : take) complete(t, st, {}, 0.0, t_launch);
            inflight_cells -= cells;
            stream_busy[si] = false;
            if (f->finished) cudaEventDestroy(f->finished);
            sa_batch_destroy(f->batch);
            cv_done.notify_all();
            return true;
        }
        std::lock_guard<std::mutex> lock(mu);
        for (int64_t t : take) {
            Request &rq = requests[t];
            rq.admitted = t_admit;
            rq.launched = t_launch;
        }
        admit_ms += std::chrono::duration<double, std::milli>(t_launch - t_admit).count();
        plan_ms += std::chrono::duration<double, std::milli>(t_plan - t_admit).count();
        upload_ms += std::chrono::duration<double, std::milli>(t_upload - t_plan).count();
        inflight.push_back(std::move(f));
        return true;
    }

    void admission_loop() {
        cudaSetDevice(device);
        for (;;) {
            uint64_t seen;
            {
                std::lock_guard<std::mutex> lock(mu);
                seen = wake;
            }
            if (admit()) continue;
            std::unique_lock<std::mutex> lock(mu);
            if (stop && pending.empty()) break;
            // woken by a submission, a finished micro-batch or stop (the time limit only bounds a
            // missed wake-up)
            cv_admit.wait_for(lock, std::chrono::milliseconds(2), [&]() { return wake != seen; });
        }
        std::lock_guard<std::mutex> lock(mu);
        if (--admitters_left == 0) admission_over = true;
    }

    void completion_loop() {
        cudaSetDevice(device);
        std::vector<InFlight *> cur;
        for (;;) {
            cur.clear();
            {
                std::lock_guard<std::mutex> lock(mu);
                for (auto &f : inflight) cur.push_back(f.get());
                if (cur.empty() && admission_over) break;
            }
            bool worked = false;
            for (InFlight *f : cur) worked = poll(*f) || worked;
            for (InFlight *f : cur) {
                if (cudaEventQuery(f->finished) != cudaSuccess) continue;
                finish(*f);
                cudaEventDestroy(f->finished);
                sa_batch_destroy(f->batch);
                std::lock_guard<std::mutex> lock(mu);
                for (size_t k = 0; k < inflight.size(); ++k)
                    if (inflight[k].get() == f) {
                        inflight.erase(inflight.begin() + (std::ptrdiff_t) k);
                        break;
                    }
                worked = true;
            }
            if (!worked) std::this_thread::sleep_for(std::chrono::microseconds(20));
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
    // the fetch landing area for reads of up to 256 k pairs before it first has to grow
    if (sa::mem_get(sa::MemKind::Pinned, device, sizeof(sa_aligned_pair) << 18, s->staging) != SA_OK) {
        for (cudaStream_t q : s->streams) cudaStreamDestroy(q);
        cudaSetDevice(prev);
        delete s;
        return SA_E_NOMEM;
    }
    if (cudaStreamCreateWithFlags(&s->fetch_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&s->origin) != cudaSuccess || cudaEventRecord(s->origin, s->streams[0]) != cudaSuccess) {
        for (cudaStream_t q : s->streams) cudaStreamDestroy(q);
        if (s->fetch_stream) cudaStreamDestroy(s->fetch_stream);
        if (s->origin) cudaEventDestroy(s->origin);
        sa::mem_put(s->staging);
        cudaSetDevice(prev);
        delete s;
        return SA_E_CUDA;
    }
    cudaSetDevice(prev);
    s->completer = std::thread([s]() { s->completion_loop(); });
    s->admitters_left = std::min<int32_t>(max_batches, 4);
    for (int k = 0; k < s->admitters_left; ++k) s->admitters.emplace_back([s]() { s->admission_loop(); });
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
    s->wake_admission();
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
        s->wake_admission();
    }
    // admission drains the queue (streams come free as the completion thread finishes batches),
    // then completion drains the device
    for (std::thread &t : s->admitters) t.join();
    if (s->completer.joinable()) s->completer.join();
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    for (cudaStream_t q : s->streams) cudaStreamDestroy(q);
    cudaStreamDestroy(s->fetch_stream);
    sa::mem_put(s->staging);
    cudaEventDestroy(s->origin);
    cudaSetDevice(prev);
    delete s;
}

sa_status sa_server_stats(sa_server *s, sa_server_counters *out) {
    if (!s || !out) return SA_E_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    out->reads_early = s->reads_early;
    out->reads_at_batch_end = s->reads_at_end;
    out->batches = s->batches;
    out->admit_ms = s->admit_ms;
    out->fetch_ms = s->fetch_ms;
    out->finish_ms = s->finish_ms;
    out->plan_ms = s->plan_ms;
    out->upload_ms = s->upload_ms;
    return SA_OK;
}

sa_status sa_server_read_timing(sa_server *s, int64_t ticket, double *queue_ms, double *launch_ms) {
    if (!s || !queue_ms || !launch_ms) return SA_E_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end() || !it->second.done) return SA_E_ARG;
    const Request &rq = it->second;
    const bool launched = rq.launched.time_since_epoch().count() != 0;
    *queue_ms = launched ? std::chrono::duration<double, std::milli>(rq.admitted - rq.submitted).count() : 0.0;
    *launch_ms = launched ? std::chrono::duration<double, std::milli>(rq.launched - rq.admitted).count() : 0.0;
    return SA_OK;
}

sa_status sa_server_batch_log(sa_server *s, double *out, int64_t capacity, int64_t *n_batches) {
    if (!s || !n_batches || capacity < 0 || (capacity > 0 && !out)) return SA_E_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    const int64_t n = (int64_t) s->batch_log.size() / 3;
    *n_batches = n;
    std::copy(s->batch_log.begin(), s->batch_log.begin() + 3 * std::min(n, capacity), out);
    return SA_OK;
}

}  // extern "C"
