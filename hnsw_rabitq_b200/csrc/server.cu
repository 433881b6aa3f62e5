// Serving loop over one GPU index: continuous batching of single-query
// requests with different k, ef, filter, tie order, precision and learned
// termination (no counterpart in the reference, whose callers run one
// searchKnn per query on their own threads, hnswlib/hnswalg.h:1269-1323).
//
// A scheduler thread owns the device side:
// * requests wait in arrival order; a batch is the oldest request plus every
//   waiting request with the same search configuration (k, ef, filter, flags,
//   precision, re-rank), up to max_batch;
// * admission is by footprint: each query of a configuration holds one warp
//   and that configuration's shared-memory layout (the kernel's per-warp
//   bytes) while its batch is in flight; a batch launches only while the
//   footprint in flight stays within the budget, and a finished batch frees
//   its share at once, so requests that arrive while others are on the GPU
//   are admitted as slots and memory free up;
// * each batch is one search launch on one of max_inflight CUDA streams with
//   its own pinned staging and device buffers (sized up front, grown
//   geometrically), so batches of different configurations overlap on the
//   device; completion is seen through a CUDA event per batch, polled from
//   the oldest batch in flight;
// * the scheduler releases the server lock while it copies and launches, so
//   submissions never wait for a launch (their arrival times stay exact);
// * latency is measured from submission to the moment the scheduler sees
//   the batch's results on the host.
// Tie-exact batches share the index's candidate-heap spill area, so at most
// one of them is in flight at a time.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "index_internal.h"

using namespace hnswgpu_host;
using Clock = std::chrono::steady_clock;

namespace {

struct Key {
    uint32_t k, ef, flags, precision, rerank;
    int32_t filter;
    bool operator<(const Key& o) const {
        return std::tie(k, ef, flags, precision, rerank, filter) <
               std::tie(o.k, o.ef, o.flags, o.precision, o.rerank, o.filter);
    }
};

// Buffer sizes grow geometrically: a reallocation frees device memory, and a
// free waits for the whole device, which stalls every batch in flight.
size_t grown(size_t need, size_t have) { return need <= have ? need : std::max(need, 2 * have); }

enum State { kPending = 0, kInflight = 1, kDone = 2, kFailed = 3 };

struct Ticket {
    Key key;
    std::vector<float> q;
    Clock::time_point t0;
    std::vector<uint64_t> labels;
    std::vector<float> dists;
    int32_t count = 0;
    double latency_us = 0;
    int state = kPending;
    int err = 0;
    std::string msg;
};

template <class T>
struct Pinned {
    T* p = nullptr;
    size_t n = 0;
    void ensure(size_t count) {
        if (count <= n) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        cuda_check(cudaMallocHost((void**)&p, count * sizeof(T)), "cudaMallocHost");
        n = count;
    }
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    Pinned<float> hq, hd;
    Pinned<uint64_t> hl;
    Pinned<int32_t> hc;
    DevBuf<float> dq, dd;
    DevBuf<uint64_t> dl;
    DevBuf<int32_t> dc;
    std::vector<uint64_t> tickets;
    Key key{};
    uint64_t footprint = 0;
    bool busy = false;
    bool exact = false;
};

}  // namespace

struct hnswgpu_server {
    hnswgpu_index* h = nullptr;
    hnswgpu_server_opts o{};
    uint64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    // Tickets by id.  A waiter keeps a pointer to its ticket while it waits:
    // element addresses survive the rehashing of later insertions.
    std::unordered_map<uint64_t, Ticket> tickets;
    // waiting requests by configuration, each queue in arrival (= id) order
    std::map<Key, std::deque<uint64_t>> queues;
    uint64_t npending = 0;
    std::deque<Slot*> inflight;  // busy slots in launch order
    std::vector<std::unique_ptr<Slot>> slots;
    std::vector<std::unique_ptr<DevBuf<uint8_t>>> filters;
    std::map<Key, uint64_t> footprint;  // per-query bytes of each configuration
    uint64_t next_ticket = 1, inflight_bytes = 0;
    bool exact_inflight = false;
    bool stop = false;
    std::thread worker;
    // statistics since the last reset
    std::vector<double> lat;
    uint64_t submitted = 0, completed = 0, batches = 0, batched_queries = 0;
};

namespace {

// Per-query shared-memory footprint of a configuration (also validates it).
uint64_t query_footprint(hnswgpu_server* s, const Key& key) {
    auto it = s->footprint.find(key);
    if (it != s->footprint.end()) return it->second;
    const uint8_t* allow = key.filter >= 0 ? s->filters[key.filter]->p : nullptr;
    hnswgpu::SearchParams p;
    {
        std::lock_guard<std::mutex> g(s->h->mu);
        set_device(s->h);
        if (key.precision) ensure_traversal_copy(s->h, key.precision);
        p = hnsw_params(s->h, nullptr, 1, key.k, key.ef, allow, nullptr, nullptr, nullptr, nullptr,
                        (key.flags & HNSWGPU_EXACT_TIES) != 0, key.precision, key.rerank, true);
        if ((key.flags & HNSWGPU_LEARNED_STOP) && !s->h->term_model.p)
            throw ApiError(HNSWGPU_ERR_STATE, "no termination model set");
    }
    const uint64_t f = (uint64_t)p.warp_smem;
    s->footprint[key] = f;
    return f;
}

// Stage a batch into a free slot and launch it.  Called by the worker with
// the server lock held; the lock is released around the copies and the
// search launch, so that submissions are not held up by them (only the
// worker thread touches slots).
void launch(hnswgpu_server* s, std::unique_lock<std::mutex>& lk, Slot& sl, const Key& key,
            const std::vector<uint64_t>& ids, uint64_t fq) {
    hnswgpu_index* h = s->h;
    const uint64_t n = ids.size(), dim = h->dim;
    sl.hq.ensure(grown(n * dim, sl.hq.n));
    sl.hl.ensure(grown(n * key.k, sl.hl.n));
    sl.hd.ensure(grown(n * key.k, sl.hd.n));
    sl.hc.ensure(grown(n, sl.hc.n));
    for (uint64_t i = 0; i < n; i++) {
        Ticket& t = s->tickets[ids[i]];
        std::memcpy(sl.hq.p + i * dim, t.q.data(), dim * sizeof(float));
        t.state = kInflight;
    }
    const uint8_t* allow = key.filter >= 0 ? s->filters[key.filter]->p : nullptr;
    // reserve the slot and the footprint before letting go of the lock
    sl.tickets = ids;
    sl.key = key;
    sl.footprint = fq * n;
    sl.exact = (key.flags & HNSWGPU_EXACT_TIES) != 0;
    sl.busy = true;
    s->inflight_bytes += sl.footprint;
    if (sl.exact) s->exact_inflight = true;
    s->batches++;
    s->batched_queries += n;
    s->inflight.push_back(&sl);
    lk.unlock();
    try {
        sl.dq.ensure(grown(n * dim, sl.dq.n));
        sl.dl.ensure(grown(n * key.k, sl.dl.n));
        sl.dd.ensure(grown(n * key.k, sl.dd.n));
        sl.dc.ensure(grown(n, sl.dc.n));
        cuda_check(cudaMemcpyAsync(sl.dq.p, sl.hq.p, n * dim * 4, cudaMemcpyHostToDevice, sl.st), "cudaMemcpyAsync");
        TermCfg term;
        if (key.flags & HNSWGPU_LEARNED_STOP) term.mode = 2;
        {
            std::lock_guard<std::mutex> g(h->mu);
            set_device(h);
            run_search(h, sl.dq.p, n, key.k, key.ef, allow, sl.dl.p, sl.dd.p, sl.dc.p, nullptr, sl.st,
                       (key.flags & HNSWGPU_EXACT_TIES) != 0, key.precision, key.rerank, &term, false);
        }
        cuda_check(cudaMemcpyAsync(sl.hl.p, sl.dl.p, n * key.k * 8, cudaMemcpyDeviceToHost, sl.st),
                   "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(sl.hd.p, sl.dd.p, n * key.k * 4, cudaMemcpyDeviceToHost, sl.st),
                   "cudaMemcpyAsync");
        cuda_check(cudaMemcpyAsync(sl.hc.p, sl.dc.p, n * 4, cudaMemcpyDeviceToHost, sl.st), "cudaMemcpyAsync");
        cuda_check(cudaEventRecord(sl.ev, sl.st), "cudaEventRecord");
    } catch (...) {
        lk.lock();
        s->inflight_bytes -= sl.footprint;
        if (sl.exact) s->exact_inflight = false;
        sl.busy = false;
        sl.tickets.clear();
        s->inflight.pop_back();
        throw;
    }
    lk.lock();
}

void finish(hnswgpu_server* s, Slot& sl, cudaError_t e) {
    const auto now = Clock::now();
    const uint32_t k = sl.key.k;
    for (size_t i = 0; i < sl.tickets.size(); i++) {
        Ticket& t = s->tickets[sl.tickets[i]];
        if (e != cudaSuccess) {
            t.state = kFailed;
            t.err = HNSWGPU_ERR_CUDA;
            t.msg = std::string("search batch failed: ") + cudaGetErrorString(e);
            continue;
        }
        t.labels.assign(sl.hl.p + i * k, sl.hl.p + (i + 1) * k);
        t.dists.assign(sl.hd.p + i * k, sl.hd.p + (i + 1) * k);
        t.count = sl.hc.p[i];
        t.latency_us = std::chrono::duration<double, std::micro>(now - t.t0).count();
        t.state = kDone;
        s->lat.push_back(t.latency_us);
        s->completed++;
    }
    s->inflight_bytes -= sl.footprint;
    if (sl.exact) s->exact_inflight = false;
    sl.busy = false;
    sl.tickets.clear();
}

void fail_tickets(hnswgpu_server* s, const std::vector<uint64_t>& ids, int code, const std::string& msg) {
    for (uint64_t id : ids) {
        Ticket& t = s->tickets[id];
        t.state = kFailed;
        t.err = code;
        t.msg = msg;
    }
}

// Next batch: the configuration of the oldest waiting request (skipping
// tie-exact ones while one is in flight), its waiting requests in arrival
// order up to max_batch and the footprint left in the budget.  Costs one look
// per configuration, however long the queues are.
bool try_launch(hnswgpu_server* s, std::unique_lock<std::mutex>& lk) {
    Slot* free_slot = nullptr;
    for (auto& sl : s->slots)
        if (!sl->busy) {
            free_slot = sl.get();
            break;
        }
    if (!free_slot || s->npending == 0) return false;
    std::deque<uint64_t>* q = nullptr;
    Key key{};
    for (auto& kv : s->queues) {
        if (kv.second.empty()) continue;
        if ((kv.first.flags & HNSWGPU_EXACT_TIES) && s->exact_inflight) continue;
        if (!q || kv.second.front() < q->front()) {
            q = &kv.second;
            key = kv.first;
        }
    }
    if (!q) return false;
    const uint64_t fq = s->footprint[key];
    const uint64_t room = s->budget > s->inflight_bytes ? (s->budget - s->inflight_bytes) / fq : 0;
    if (room == 0) return false;  // wait for a batch to finish
    const uint64_t cap = std::min<uint64_t>(room, s->o.max_batch);
    std::vector<uint64_t> ids;
    while (!q->empty() && ids.size() < cap) {
        ids.push_back(q->front());
        q->pop_front();
    }
    s->npending -= ids.size();
    try {
        launch(s, lk, *free_slot, key, ids, fq);
    } catch (const ApiError& e) {
        fail_tickets(s, ids, e.code, e.what());
        s->cv_done.notify_all();
    } catch (const std::exception& e) {
        fail_tickets(s, ids, HNSWGPU_ERR_NOMEM, e.what());
        s->cv_done.notify_all();
    }
    return true;
}

void worker_loop(hnswgpu_server* s) {
    cudaSetDevice(s->h->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        bool any_busy = false, progressed = false;
        // Batches mostly finish in launch order: poll from the oldest and
        // stop after two still running, so that a poll costs a few event
        // queries, not one per slot.
        int running = 0;
        for (size_t i = 0; i < s->inflight.size() && running < 2;) {
            Slot* sl = s->inflight[i];
            const cudaError_t e = cudaEventQuery(sl->ev);
            if (e == cudaErrorNotReady) {
                running++;
                i++;
                continue;
            }
            finish(s, *sl, e);
            s->inflight.erase(s->inflight.begin() + (std::ptrdiff_t)i);
            progressed = true;
        }
        any_busy = !s->inflight.empty();
        if (progressed) s->cv_done.notify_all();
        while (try_launch(s, lk)) any_busy = true;
        if (s->stop && s->npending == 0 && !any_busy) break;
        if (any_busy)
            s->cv_work.wait_for(lk, std::chrono::microseconds(10));
        else
            s->cv_work.wait(lk, [&] { return s->stop || s->npending != 0; });
    }
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

uint64_t submit_locked(hnswgpu_server* s, const float* query, const hnswgpu_request* r) {
    Key key{r->k, r->ef ? r->ef : (uint32_t)s->h->ef, r->flags & (HNSWGPU_LEARNED_STOP | HNSWGPU_EXACT_TIES),
            r->precision, r->rerank, r->filter};
    if (key.k == 0) throw ApiError(HNSWGPU_ERR_ARG, "k must be positive");
    if (key.filter >= (int32_t)s->filters.size() || key.filter < -1) throw ApiError(HNSWGPU_ERR_ARG, "unknown filter");
    if ((key.flags & HNSWGPU_LEARNED_STOP) && (key.flags & HNSWGPU_EXACT_TIES))
        throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "learned termination needs the id tie order");
    if (query_footprint(s, key) > s->budget)
        throw ApiError(HNSWGPU_ERR_UNSUPPORTED, "the request's shared-memory footprint exceeds the admission budget");
    const uint64_t id = s->next_ticket++;
    Ticket& t = s->tickets[id];
    t.key = key;
    t.q.assign(query, query + s->h->dim);
    t.t0 = Clock::now();
    s->queues[key].push_back(id);
    s->npending++;
    s->submitted++;
    return id;
}

}  // namespace

int hnswgpu_server_create(hnswgpu_index* h, const hnswgpu_server_opts* opts, hnswgpu_server** out) {
    return guarded([&] {
        if (!h || !out || h->is_bf) return fail(HNSWGPU_ERR_ARG, "a server needs an HNSW index");
        auto s = std::make_unique<hnswgpu_server>();
        s->h = h;
        if (opts) s->o = *opts;
        // 32 batches in flight: a batch lasts about one query's beam latency,
        // so concurrency, not batch size, bounds the served rate
        if (!s->o.max_inflight) s->o.max_inflight = 32;
        if (!s->o.max_batch) s->o.max_batch = 4096;
        set_device(h);
        int smem_per_sm = 0;
        cuda_check(cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, h->device),
                   "cudaDeviceGetAttribute");
        // default: the device's shared memory twice over (one wave running,
        // one queued behind it)
        s->budget = s->o.smem_budget ? s->o.smem_budget : 2ull * (uint64_t)h->num_sms * (uint64_t)smem_per_sm;
        // staging sized up front for batches of up to 256 queries with k <= 100,
        // so that serving rarely reallocates
        const uint64_t pq = std::min<uint64_t>(s->o.max_batch, 256), pk = 100;
        for (uint32_t i = 0; i < s->o.max_inflight; i++) {
            auto sl = std::make_unique<Slot>();
            cuda_check(cudaStreamCreateWithFlags(&sl->st, cudaStreamNonBlocking), "cudaStreamCreate");
            cuda_check(cudaEventCreateWithFlags(&sl->ev, cudaEventDisableTiming), "cudaEventCreate");
            sl->hq.ensure(pq * h->dim);
            sl->hl.ensure(pq * pk);
            sl->hd.ensure(pq * pk);
            sl->hc.ensure(pq);
            sl->dq.ensure(pq * h->dim);
            sl->dl.ensure(pq * pk);
            sl->dd.ensure(pq * pk);
            sl->dc.ensure(pq);
            s->slots.push_back(std::move(sl));
        }
        hnswgpu_server* raw = s.release();
        raw->worker = std::thread(worker_loop, raw);
        *out = raw;
        return HNSWGPU_OK;
    });
}

int hnswgpu_server_add_filter(hnswgpu_server* s, const uint8_t* allow, int32_t* out_id) {
    return guarded([&] {
        if (!s || !allow || !out_id) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        auto buf = std::make_unique<DevBuf<uint8_t>>();
        {
            std::lock_guard<std::mutex> g(s->h->mu);
            set_device(s->h);
            buf->alloc(std::max<uint64_t>(1, s->h->count));
            cuda_check(cudaMemcpy(buf->p, allow, s->h->count, cudaMemcpyHostToDevice), "cudaMemcpy");
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->filters.push_back(std::move(buf));
        *out_id = (int32_t)s->filters.size() - 1;
        return HNSWGPU_OK;
    });
}

int hnswgpu_server_submit(hnswgpu_server* s, const float* query, const hnswgpu_request* req, uint64_t* out_ticket) {
    return guarded([&] {
        if (!s || !query || !req || !out_ticket) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return fail(HNSWGPU_ERR_STATE, "server is shutting down");
        *out_ticket = submit_locked(s, query, req);
        s->cv_work.notify_one();
        return HNSWGPU_OK;
    });
}

int hnswgpu_server_wait(hnswgpu_server* s, uint64_t ticket, uint64_t* labels, float* dists, int32_t* count,
                        double* latency_us) {
    return guarded([&] {
        if (!s) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) return fail(HNSWGPU_ERR_ARG, "unknown ticket");
        const Ticket* tp = &it->second;
        s->cv_done.wait(lk, [&] { return tp->state >= kDone; });
        Ticket t = std::move(s->tickets[ticket]);
        s->tickets.erase(ticket);
        if (t.state == kFailed) return fail(t.err, t.msg);
        if (labels) std::memcpy(labels, t.labels.data(), t.labels.size() * 8);
        if (dists) std::memcpy(dists, t.dists.data(), t.dists.size() * 4);
        if (count) *count = t.count;
        if (latency_us) *latency_us = t.latency_us;
        return HNSWGPU_OK;
    });
}

int hnswgpu_server_replay(hnswgpu_server* s, const float* queries, uint64_t n, const hnswgpu_request* reqs,
                          const double* arrival_us, uint32_t k_stride, uint64_t* labels, float* dists,
                          int32_t* counts, double* latency_us) {
    return guarded([&] {
        if (!s || (n && (!queries || !reqs || !arrival_us || !labels || !dists || !counts)))
            return fail(HNSWGPU_ERR_ARG, "invalid argument");
        for (uint64_t i = 0; i < n; i++)
            if (reqs[i].k > k_stride) return fail(HNSWGPU_ERR_ARG, "a request's k exceeds k_stride");
        std::vector<uint64_t> ids(n);
        const uint64_t dim = s->h->dim;
        // open loop: each request is submitted at its arrival time
        const auto t0 = Clock::now();
        int err = HNSWGPU_OK;
        std::string msg;
        for (uint64_t i = 0; i < n; i++) {
            const auto due = t0 + std::chrono::duration_cast<Clock::duration>(
                                      std::chrono::duration<double, std::micro>(arrival_us[i]));
            while (Clock::now() < due) {
                const auto left = due - Clock::now();
                if (left > std::chrono::microseconds(200)) std::this_thread::sleep_for(left / 2);
            }
            std::lock_guard<std::mutex> lk(s->mu);
            try {
                ids[i] = submit_locked(s, queries + i * dim, &reqs[i]);
            } catch (const ApiError& e) {
                err = e.code;
                msg = e.what();
                n = i;
                break;
            }
            s->cv_work.notify_one();
        }
        for (uint64_t i = 0; i < n; i++) {
            std::unique_lock<std::mutex> lk(s->mu);
            Ticket& t = s->tickets.find(ids[i])->second;
            s->cv_done.wait(lk, [&] { return t.state >= kDone; });
            if (t.state == kFailed && err == HNSWGPU_OK) {
                err = t.err;
                msg = t.msg;
            }
            for (uint32_t j = 0; j < k_stride; j++) {
                labels[i * k_stride + j] = j < t.labels.size() ? t.labels[j] : ~0ull;
                dists[i * k_stride + j] = j < t.dists.size() ? t.dists[j] : __builtin_inff();
            }
            counts[i] = t.count;
            if (latency_us) latency_us[i] = t.latency_us;
            s->tickets.erase(ids[i]);
        }
        if (err != HNSWGPU_OK) return fail(err, msg);
        return HNSWGPU_OK;
    });
}

int hnswgpu_server_get_stats(hnswgpu_server* s, hnswgpu_server_stats* out, int reset) {
    return guarded([&] {
        if (!s || !out) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        std::lock_guard<std::mutex> lk(s->mu);
        out->submitted = s->submitted;
        out->completed = s->completed;
        out->batches = s->batches;
        out->mean_batch = s->batches ? (double)s->batched_queries / (double)s->batches : 0.0;
        out->p50_us = percentile(s->lat, 0.50);
        out->p99_us = percentile(s->lat, 0.99);
        double sum = 0, mx = 0;
        for (double v : s->lat) {
            sum += v;
            mx = std::max(mx, v);
        }
        out->mean_us = s->lat.empty() ? 0 : sum / (double)s->lat.size();
        out->max_us = mx;
        if (reset) {
            s->lat.clear();
            s->submitted = s->completed = s->batches = s->batched_queries = 0;
        }
        return HNSWGPU_OK;
    });
}

int hnswgpu_server_destroy(hnswgpu_server* s) {
    return guarded([&] {
        if (!s) return fail(HNSWGPU_ERR_ARG, "invalid argument");
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;
        }
        s->cv_work.notify_all();
        if (s->worker.joinable()) s->worker.join();
        cudaSetDevice(s->h->device);
        for (auto& sl : s->slots) {
            if (sl->st) cudaStreamSynchronize(sl->st);
            if (sl->ev) cudaEventDestroy(sl->ev);
            if (sl->st) cudaStreamDestroy(sl->st);
        }
        delete s;
        return HNSWGPU_OK;
    });
}
