// server.cu — K11: the serving loop. Replaces the reference's query caches (src/cpu.rs:16-89,
// src/gpu.rs:21-25, memoisation of repeated queries) with continuous batching against the
// device-resident index: requests of any size and k are queued, and each free slot takes every
// queued request of the same kind that fits and runs them as one batch.
//
// Slots. A slot is a view of the index (make_view: the index's device data shared, its own stream,
// status words and per-search scratch) driven by its own worker thread, so batches of different
// slots are on the device at the same time: one slot's uploads, kernels and read-backs overlap
// another's. A request that arrives while every slot is busy waits in the queue and joins the next
// batch of the first slot to free up (continuous batching, not a queue per request).
//
// Same result alone and in a mix. A query's result never depends on its batch: the FP32 scan's FMA
// order is fixed per (row, query), the tensor-core path re-scores its candidates in that same order
// and its certificate makes the result the exact top-k, and the IVF path fixes nprobe per batch
// (requests only share a batch with the same effective nprobe). A batch runs at its largest k and a
// request keeps the first k of its rows: the exact top-k is a prefix of the exact top-k′ for k ≤ k′.
//
// Admission by memory. Each slot may hold `slot_bytes` of per-batch device memory; a request's
// share is estimated from its queries and k (normalised queries, results, scan workspace, IVF
// slots). A batch only grows while its estimate fits, a request that cannot fit any batch is refused,
// and the queue is bounded in queries (NNDEX_ERR_ADMISSION: the caller may retry later).
//
// Admission by latency. With a latency budget, a request is also refused while the oldest queued
// request has waited longer than the budget (the queue is backed up: a newcomer would wait at least
// as long), or when the queries ahead of it would take longer than the budget to drain at the cost
// per query of large batches (a moving average over batches of at least a quarter of the batch
// limit: a long queue is served in such batches). Small batches cost far more per query, so their
// cost is not used: at light loads the queue is short and only its age matters. Under overload the
// queue stops growing at about one budget's worth of work, and the latency of admitted requests
// stays near the budget plus one batch instead of rising without limit.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "index.h"
#include "ivf.h"

namespace nndex {

namespace {

uint64_t now_ns() {
    return static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(
                                     std::chrono::steady_clock::now().time_since_epoch())
                                     .count());
}

struct Request {
    uint64_t ticket = 0;
    uint64_t nq = 0, kcap = 0;
    bool approx = false;    // answered through the IVF
    uint32_t nprobe = 0;    // effective lists probed (approx only)
    std::vector<float> q;   // nq × dims raw queries
    std::vector<uint64_t> idx;
    std::vector<float> sim;
    std::vector<uint64_t> cnt;
    int status = NNDEX_PENDING;
    std::string error;
    nndex_cuda_request_info info{};
};

}  // namespace

struct Server {
    CudaIndex* ix = nullptr;
    nndex_cuda_server_opts opts{};
    uint64_t max_chunks = 1;  // IVF: 4096-row chunks of the largest list (slot workspace estimate)
    std::vector<CudaIndex*> views;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
    uint64_t next_ticket = 1, next_batch = 1;
    bool stopping = false;
    nndex_cuda_server_stats st{};
    double spq = 0.0;      // moving average of one slot's wall seconds per query (0 until a batch ran)
    double spq_big = 0.0;  // the same over large batches (≥ a quarter of max_batch_queries) only

    // Device bytes a batch of nq queries at k (capped) needs in a slot.
    uint64_t batch_bytes(uint64_t nq, uint64_t kcap, bool approx, uint32_t nprobe) const {
        uint64_t per = (ix->dims + ix->ds) * 4 + kcap * 12;
        per += 160 * kcap * 8;                      // FP32 scan: one k-key slot per CTA and query
        per += 64 * std::max<uint64_t>(32, 2 * kcap) * 8;  // tensor-core pass 1 (k′ keys per row range)
        if (approx) {
            // FP32 list scan: k keys per (probed list, chunk); tensor-core list scan: k′ keys per
            // (probed list, chunk), the gathered BF16 query blocks, and the pass-2 row collection.
            const uint64_t kp = std::max<uint64_t>(32, 2 * kcap);
            per += (static_cast<uint64_t>(nprobe) * max_chunks * std::max(kp, kcap) + 4ull * nprobe) * 8;
            per += ix->ds * 2 + 8192ull * 4;
        }
        return nq * per;
    }
    void worker(uint32_t slot);
    ~Server();
};

// A batch runs at its largest k, and a search's cost grows with k (candidate widths, collections,
// merges): requests share a batch only within one class of k, so k = 1 and k = 10 requests never
// pay for a k = 100 neighbour.
static int k_class(uint64_t k) { return k <= 16 ? 0 : (k <= 128 ? 1 : 2); }

void Server::worker(uint32_t slot) {
    CudaIndex* v = views[slot];
    set_scratch_stream(v->stream);  // this slot's buffers grow in stream order (see set_scratch_stream)
    std::vector<float> qbuf;
    std::vector<uint64_t> bidx, bcnt;
    std::vector<float> bsim;
    const int mode = ix->normalized ? 2 : 0;  // batch normalisation (normalize_rows), as search_batch
    for (;;) {
        std::vector<std::shared_ptr<Request>> batch;
        uint64_t nq = 0, kmax = 0, batch_id = 0;
        bool approx = false;
        uint32_t nprobe = 0;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stopping || !queue.empty(); });
            if (queue.empty()) return;  // stopping, and nothing left to run
            approx = queue.front()->approx;
            nprobe = queue.front()->nprobe;
            const int kclass = k_class(queue.front()->kcap);
            for (auto it = queue.begin(); it != queue.end();) {
                const Request& r = **it;
                const uint64_t k2 = std::max(kmax, r.kcap);
                if (r.approx == approx && r.nprobe == nprobe && k_class(r.kcap) == kclass &&
                    nq + r.nq <= opts.max_batch_queries &&
                    batch_bytes(nq + r.nq, k2, approx, nprobe) <= opts.slot_bytes) {
                    nq += r.nq;
                    kmax = k2;
                    batch.push_back(*it);
                    it = queue.erase(it);
                } else if (nq >= opts.max_batch_queries) {
                    break;
                } else {
                    ++it;
                }
            }
            st.queued_queries -= nq;
            batch_id = next_batch++;
        }
        const uint64_t t_start = now_ns();
        qbuf.resize(nq * ix->dims);
        uint64_t off = 0;
        for (const auto& r : batch) {
            std::memcpy(qbuf.data() + off * ix->dims, r->q.data(), r->nq * ix->dims * sizeof(float));
            off += r->nq;
        }
        bidx.resize(nq * kmax);
        bsim.resize(nq * kmax);
        bcnt.resize(nq);
        v->approx_override = approx ? 1 : 0;
        v->ivf_scratch.nprobe = approx ? nprobe : 0;
        if (sync_check_enabled())
            std::fprintf(stderr, "nndex server: slot %u batch %llu: %llu queries from %zu requests, k %llu, approx %d\n",
                         slot, (unsigned long long)batch_id, (unsigned long long)nq, batch.size(),
                         (unsigned long long)kmax, approx ? 1 : 0);
        int code = v->search_host(qbuf.data(), nq, kmax, mode, bidx.data(), bsim.data(), bcnt.data());
        std::vector<int> codes(batch.size(), code);
        std::vector<std::string> msgs(batch.size(), code ? last_error() : "");
        if (code == NNDEX_OK) {
            off = 0;
            for (auto& r : batch) {
                r->idx.resize(r->nq * r->kcap);
                r->sim.resize(r->nq * r->kcap);
                r->cnt.resize(r->nq);
                for (uint64_t q = 0; q < r->nq; ++q) {
                    const uint64_t row = off + q;
                    for (uint64_t j = 0; j < r->kcap; ++j) {
                        r->idx[q * r->kcap + j] = bidx[row * kmax + j];
                        r->sim[q * r->kcap + j] = bsim[row * kmax + j];
                    }
                    r->cnt[q] = std::min<uint64_t>(bcnt[row], r->kcap);
                }
                off += r->nq;
            }
        } else {
            // Attribute the failure: every request of the batch on its own (a bad query fails only
            // its own request, as it would alone).
            if (sync_check_enabled())
                std::fprintf(stderr, "nndex server: batch %llu failed (%s); its requests run one by one\n",
                             (unsigned long long)batch_id, msgs[0].c_str());
            for (size_t i = 0; i < batch.size(); ++i) {
                auto& r = batch[i];
                r->idx.resize(r->nq * r->kcap);
                r->sim.resize(r->nq * r->kcap);
                r->cnt.resize(r->nq);
                codes[i] = v->search_host(r->q.data(), r->nq, r->kcap, mode, r->idx.data(), r->sim.data(),
                                          r->cnt.data());
                msgs[i] = codes[i] ? last_error() : "";
            }
        }
        const uint64_t t_done = now_ns();
        v->fetch_fallback_stats();  // the TF32 path's device-side re-run count
        const uint32_t path = v->stats.path;
        {
            std::lock_guard<std::mutex> lk(mu);
            const double per = static_cast<double>(t_done - t_start) * 1e-9 / static_cast<double>(nq);
            spq = spq > 0.0 ? 0.9 * spq + 0.1 * per : per;
            if (nq * 4 >= opts.max_batch_queries) spq_big = spq_big > 0.0 ? 0.9 * spq_big + 0.1 * per : per;
            st.us_per_query = spq * 1e6;
            st.fp32_fallback_queries += v->stats.fp32_fallback_queries;
            const double ms = static_cast<double>(t_done - t_start) * 1e-6;
            if (ms > st.slowest_batch_ms) {
                st.slowest_batch_ms = ms;
                st.slowest_batch_queries = static_cast<uint32_t>(nq);
                st.slowest_batch_k = static_cast<uint32_t>(kmax);
                st.slowest_batch_path = path;
                st.slowest_batch_approx = approx ? 1u : 0u;
            }
            for (size_t i = 0; i < batch.size(); ++i) {
                auto& r = batch[i];
                r->status = codes[i];
                r->error = msgs[i];
                r->info.start_ns = t_start;
                r->info.done_ns = t_done;
                r->info.batch_id = batch_id;
                r->info.batch_queries = static_cast<uint32_t>(nq);
                r->info.slot = slot;
                r->info.path = path;
                st.requests_done += 1;
                st.queries_done += r->nq;
            }
            st.batches += 1;
        }
        cv_done.notify_all();
    }
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu);
        stopping = true;
    }
    cv_work.notify_all();
    for (auto& t : workers)
        if (t.joinable()) t.join();
    for (CudaIndex* v : views) delete v;
}

}  // namespace nndex

struct nndex_cuda_server {
    nndex::Server* impl;
};

using namespace nndex;

extern "C" {

int nndex_cuda_server_start(nndex_cuda_index* index, const nndex_cuda_server_opts* opts, nndex_cuda_server** out) {
    clear_error();
    if (!index || !out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    *out = nullptr;
    CudaIndex* ix = index->impl;
    auto srv = std::make_unique<Server>();
    srv->ix = ix;
    nndex_cuda_server_opts o{};
    if (opts) o = *opts;
    if (o.slots == 0) o.slots = 2;
    if (o.max_batch_queries == 0) o.max_batch_queries = 4096;
    if (o.queue_capacity == 0) o.queue_capacity = 1ull << 20;
    cudaSetDevice(ix->device);
    if (o.slot_bytes == 0) {
        size_t free_b = 0, total_b = 0;
        cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
        if (e != cudaSuccess) return cuda_error(e, "cudaMemGetInfo");
        o.slot_bytes = static_cast<uint64_t>(free_b) / 2 / o.slots;
    }
    srv->opts = o;
    if (ix->ivf) srv->max_chunks = std::max<uint64_t>(1, (ix->ivf->max_list + 4095) / 4096);
    for (uint32_t i = 0; i < o.slots; ++i) {
        CudaIndex* v = nullptr;
        const int st = make_view(*ix, &v);
        if (st) return st;  // the views made so far are freed with srv
        srv->views.push_back(v);
    }
    srv->st.slots = o.slots;
    srv->st.max_batch_queries = o.max_batch_queries;
    srv->st.slot_bytes = o.slot_bytes;
    // Warm-up, before any request: every slot runs each kind of batch once (exact and, with an IVF,
    // approximate at the default nprobe; k = 1, 10 and 100; 16, 256 and the largest batch a slot
    // admits), on the index's first rows as queries. CUDA loads a kernel on its first launch (about
    // 130 ms for the first tensor-core batch), and a slot's buffers grow with its largest batch;
    // both would otherwise fall on the first requests of each kind while the other slots run on.
    const uint64_t wn = std::min<uint64_t>(o.max_batch_queries, ix->rows);
    if (wn) {
        std::vector<float> wq(wn * ix->dims);
        cudaError_t e = cudaMemcpy2D(wq.data(), ix->dims * sizeof(float), ix->d_base, ix->ds * sizeof(float),
                                     ix->dims * sizeof(float), wn, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_error(e, "server warm-up");
        const int mode = ix->normalized ? 2 : 0;
        Server* sv = srv.get();
        std::vector<std::thread> warm;
        for (uint32_t i = 0; i < o.slots; ++i)
            warm.emplace_back([sv, &wq, wn, mode, i] {
                CudaIndex* v = sv->views[i];
                const CudaIndex* x = sv->ix;
                cudaSetDevice(x->device);
                set_scratch_stream(v->stream);
                std::vector<uint64_t> bi, bc;
                std::vector<float> bs;
                for (int approx = 0; approx <= (x->ivf ? 1 : 0); ++approx)
                    for (uint64_t k : {1ull, 10ull, 100ull}) {
                        const uint64_t kc = std::min<uint64_t>(k, x->rows);
                        uint32_t np = 0;
                        if (approx) {
                            const uint64_t d = x->ivf_scratch.nprobe ? x->ivf_scratch.nprobe
                                                                     : ivf_choose_nprobe(x->ivf->nlist, kc, x->rows);
                            np = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(d, x->ivf->nlist)));
                        }
                        uint64_t top = wn;
                        while (top > 1 && sv->batch_bytes(top, kc, approx, np) > sv->opts.slot_bytes) top /= 2;
                        for (uint64_t n : {uint64_t{16}, uint64_t{256}, top}) {
                            const uint64_t nq = std::min<uint64_t>(n, top);
                            bi.resize(nq * kc);
                            bs.resize(nq * kc);
                            bc.resize(nq);
                            v->approx_override = approx;
                            v->ivf_scratch.nprobe = np;
                            v->search_host(wq.data(), nq, kc, mode, bi.data(), bs.data(), bc.data());
                        }
                    }
                v->approx_override = -1;
                v->ivf_scratch.nprobe = x->ivf_scratch.nprobe;
                clear_error();
            });
        for (auto& t : warm) t.join();
    }
    Server* s = srv.get();
    for (uint32_t i = 0; i < o.slots; ++i) s->workers.emplace_back([s, i] { s->worker(i); });
    *out = new nndex_cuda_server{srv.release()};
    return NNDEX_OK;
}

int nndex_cuda_server_submit(nndex_cuda_server* server, const float* host_queries, uint64_t query_rows,
                             uint64_t query_dims, uint64_t k, uint32_t flags, uint32_t nprobe, uint64_t* ticket) {
    clear_error();
    if (!server || !ticket) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    Server* s = server->impl;
    CudaIndex* ix = s->ix;
    // src/lib.rs:378-381: shape before k.
    if (query_rows == 0 || query_dims != ix->dims || !host_queries)
        return set_error(NNDEX_ERR_SHAPE_MISMATCH, "matrix shape mismatch: rows=%llu, dims=%llu, values=%llu",
                         (unsigned long long)query_rows, (unsigned long long)ix->dims,
                         (unsigned long long)(query_rows * query_dims));
    if (k == 0) return set_error(NNDEX_ERR_INVALID_TOPK, "top-k must be greater than zero");
    auto r = std::make_shared<Request>();
    r->nq = query_rows;
    r->kcap = std::min<uint64_t>(k, ix->rows);
    const bool ivf_ok = ix->ivf && ix->rows >= 256 && ix->ivf->nlist >= 4;
    r->approx = (flags & NNDEX_FLAG_APPROX) != 0 && ivf_ok;
    if (r->approx) {
        uint64_t np = nprobe ? nprobe
                             : (ix->ivf_scratch.nprobe ? ix->ivf_scratch.nprobe
                                                       : ivf_choose_nprobe(ix->ivf->nlist, r->kcap, ix->rows));
        r->nprobe = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(np, ix->ivf->nlist)));
    }
    if (r->nq > s->opts.max_batch_queries || s->batch_bytes(r->nq, r->kcap, r->approx, r->nprobe) > s->opts.slot_bytes) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.refused += 1;
        return set_error(NNDEX_ERR_ADMISSION,
                         "cuda execution error: request of %llu queries (k=%llu) does not fit one slot (%llu queries, "
                         "%llu bytes)",
                         (unsigned long long)r->nq, (unsigned long long)r->kcap,
                         (unsigned long long)s->opts.max_batch_queries, (unsigned long long)s->opts.slot_bytes);
    }
    r->q.assign(host_queries, host_queries + query_rows * query_dims);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: server stopped");
        if (s->st.queued_queries + r->nq > s->opts.queue_capacity) {
            s->st.refused += 1;
            return set_error(NNDEX_ERR_ADMISSION, "cuda execution error: queue full (%llu queries waiting)",
                             (unsigned long long)s->st.queued_queries);
        }
        if (s->opts.latency_budget_ms && !s->queue.empty()) {
            const double budget = static_cast<double>(s->opts.latency_budget_ms);
            const double age_ms = static_cast<double>(now_ns() - s->queue.front()->info.submit_ns) * 1e-6;
            // the wait ahead of this request at the cost per query of large batches (what a long
            // queue is served in)
            const double drain_ms = static_cast<double>(s->st.queued_queries + r->nq) * s->spq_big * 1e3 /
                                    static_cast<double>(s->opts.slots);
            if (age_ms > budget || drain_ms > budget) {
                s->st.refused += 1;
                s->st.refused_latency += 1;
                return set_error(NNDEX_ERR_ADMISSION,
                                 "cuda execution error: %llu queued queries (the oldest waiting %.1f ms, about %.1f ms "
                                 "to drain) exceed the %u ms latency budget",
                                 (unsigned long long)s->st.queued_queries, age_ms, drain_ms, s->opts.latency_budget_ms);
            }
        }
        r->ticket = s->next_ticket++;
        r->info.submit_ns = now_ns();
        s->queue.push_back(r);
        s->live.emplace(r->ticket, r);
        s->st.queued_queries += r->nq;
        s->st.max_queued_queries = std::max(s->st.max_queued_queries, s->st.queued_queries);
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return NNDEX_OK;
}

int nndex_cuda_server_poll(nndex_cuda_server* server, uint64_t ticket, int32_t timeout_ms, uint64_t* idx_out,
                           float* sim_out, uint64_t* counts_out, nndex_cuda_request_info* info) {
    clear_error();
    if (!server) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null server");
    Server* s = server->impl;
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->live.find(ticket);
        if (it == s->live.end())
            return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: unknown ticket %llu",
                             (unsigned long long)ticket);
        r = it->second;
        auto done = [&] { return r->status != NNDEX_PENDING; };
        if (!done()) {
            if (timeout_ms == 0) return NNDEX_PENDING;
            if (timeout_ms < 0)
                s->cv_done.wait(lk, done);
            else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
                return NNDEX_PENDING;
        }
        s->live.erase(ticket);
    }
    if (info) *info = r->info;
    if (r->status != NNDEX_OK) return set_error(r->status, "%s", r->error.c_str());
    if (idx_out) std::memcpy(idx_out, r->idx.data(), r->idx.size() * sizeof(uint64_t));
    if (sim_out) std::memcpy(sim_out, r->sim.data(), r->sim.size() * sizeof(float));
    if (counts_out) std::memcpy(counts_out, r->cnt.data(), r->cnt.size() * sizeof(uint64_t));
    return NNDEX_OK;
}

int nndex_cuda_server_stats_get(nndex_cuda_server* server, nndex_cuda_server_stats* out) {
    clear_error();
    if (!server || !out) return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: null argument");
    std::lock_guard<std::mutex> lk(server->impl->mu);
    *out = server->impl->st;
    return NNDEX_OK;
}

void nndex_cuda_server_stop(nndex_cuda_server* server) {
    if (!server) return;
    delete server->impl;
    delete server;
}

}  // extern "C"
