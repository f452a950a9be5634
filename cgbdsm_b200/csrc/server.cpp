// Serving loop over the multi-query engine (cgb_server_*).
//
// The reference has no serving path: it runs one query over one update file
// per process (main_calig.cpp:44-450).  Here the data graph, its index and
// every registered query stay resident on one device while requests arrive
// from any host thread:
//   update batch    edges to insert / delete; result = each registered
//                   query's positive / negative matches for that batch
//   register query  joins the running query set at the next batch boundary
//                   (it is matched in the same persistent launch as the
//                   others from then on); result = its query id
//   unregister      leaves at the next boundary
// Requests take effect in submission order (update batches must, for the
// counts to be the sequential ones).  Three threads:
//   client threads  copy the request (submit_*) and return a ticket
//   stager          admits update batches by HBM budget: a batch needs its
//                   edge pairs in a device staging ring (and its working set
//                   must fit the budget at all); it copies them into pinned
//                   memory and issues their H2D on a copy stream as soon as
//                   ring space frees up, so the copies of the next batches
//                   overlap the running batch's matching on the device
//   scheduler       applies requests in order: registrations immediately
//                   (between batches), batches through the engine once their
//                   copy event completed (the engine stream waits on it),
//                   then publishes counts and timestamps and frees the ring
//                   space.
// Results are per ticket (wait with a timeout); timestamps (ms since the
// server started): submitted, staged (admitted), started, done.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cgbdsm.h"
#include "staging_ring.h"

namespace {

// Device working set of one update batch per edge: pairs (8 B), two packed
// key buffers and the selected keys (24 B each direction), delta values,
// run keys and run lists (4 B each), flags; both orientations.
constexpr uint64_t kWorkBytesPerEdge = 2 * (3 * 8 + 4 * 4 + 1) + 8;

struct Req {
    uint64_t ticket = 0;
    uint32_t kind = 0;  // CGB_SERVER_BATCH / _REGISTER / _UNREGISTER
    std::vector<uint32_t> pairs;  // ins then del
    uint64_t n_ins = 0, n_del = 0;
    uint32_t qv = 0, qe = 0, query_id = 0;
    std::vector<uint32_t> qlabels, qedges;
    // staging
    bool staged = false;
    uint64_t ring_off = 0, ring_len = 0;
    cudaEvent_t copied = nullptr;
    // result
    bool done = false;
    int32_t status = CGB_OK;
    std::string err;
    std::vector<uint64_t> pos, neg;
    double t_submit = 0, t_staged = 0, t_start = 0, t_done = 0;
    uint32_t live_queries = 0;
    float device_ms = 0;
};

}  // namespace

struct cgb_server {
    cgb_server_config cfg{};
    cgb_mq* m = nullptr;
    int device = 0;
    std::string err;
    std::chrono::steady_clock::time_point t0;
    // staging ring (bytes): pinned host mirror + device
    cgb::StagingRing ring;
    unsigned char* h_ring = nullptr;
    unsigned char* d_ring = nullptr;
    cudaStream_t copy_stream = nullptr;
    uint64_t budget = 0, base_used = 0;
    // requests
    std::mutex mu;
    std::condition_variable cv_sched, cv_stage, cv_done;
    std::deque<std::shared_ptr<Req>> queue;        // not yet applied, in order
    std::map<uint64_t, std::shared_ptr<Req>> all;  // by ticket, until collected
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread sched, stager;
    uint32_t live = 0;
    // stats
    uint64_t batches_done = 0, edges_done = 0, rejected = 0;
    double busy_ms = 0;

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

uint64_t round16(uint64_t x) { return (x + 15) & ~15ull; }

void stager_loop(cgb_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        // the first update batch in order that is not staged yet
        std::shared_ptr<Req> r;
        for (auto& q : s->queue)
            if (q->kind == CGB_SERVER_BATCH && !q->staged) { r = q; break; }
        if (!r) { s->cv_stage.wait(lk); continue; }
        const uint64_t bytes = round16((r->n_ins + r->n_del) * 8);
        uint64_t off = 0;
        if (bytes && !s->ring.alloc(bytes, &off)) {
            if (bytes > s->ring.cap) {  // can never be staged: reject in order
                r->staged = true;
                r->status = CGB_ERR_LIMIT;
                r->err = "batch larger than the staging budget";
                s->cv_sched.notify_all();
                continue;
            }
            s->cv_stage.wait(lk);  // ring space frees as batches complete
            continue;
        }
        r->ring_off = off;
        r->ring_len = bytes;
        lk.unlock();
        if (bytes) {
            std::memcpy(s->h_ring + off, r->pairs.data(), (r->n_ins + r->n_del) * 8);
            cudaMemcpyAsync(s->d_ring + off, s->h_ring + off, (r->n_ins + r->n_del) * 8, cudaMemcpyHostToDevice,
                            s->copy_stream);
        }
        cudaEventCreateWithFlags(&r->copied, cudaEventDisableTiming);
        cudaEventRecord(r->copied, s->copy_stream);
        lk.lock();
        r->staged = true;
        r->t_staged = s->now_ms();
        s->cv_sched.notify_all();
    }
}

void complete(cgb_server* s, const std::shared_ptr<Req>& r) {
    r->t_done = s->now_ms();
    r->done = true;
    s->cv_done.notify_all();
}

void scheduler_loop(cgb_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        if (s->queue.empty()) { s->cv_sched.wait(lk); continue; }
        std::shared_ptr<Req> r = s->queue.front();
        if (r->kind == CGB_SERVER_REGISTER) {
            s->queue.pop_front();
            lk.unlock();
            uint32_t id = 0;
            cgb_status st = cgb_mq_register_query(s->m, r->qv, r->qlabels.data(), r->qe, r->qedges.data(), &id);
            lk.lock();
            r->t_start = s->now_ms();
            r->status = st;
            if (st == CGB_OK) { r->query_id = id; ++s->live; }
            else r->err = cgb_mq_last_error(s->m);
            complete(s, r);
            continue;
        }
        if (r->kind == CGB_SERVER_UNREGISTER) {
            s->queue.pop_front();
            lk.unlock();
            cgb_status st = cgb_mq_unregister_query(s->m, r->query_id);
            lk.lock();
            r->t_start = s->now_ms();
            r->status = st;
            if (st == CGB_OK) --s->live;
            else r->err = cgb_mq_last_error(s->m);
            complete(s, r);
            continue;
        }
        if (!r->staged) { s->cv_sched.wait(lk); continue; }
        s->queue.pop_front();
        s->cv_stage.notify_all();
        if (r->status != CGB_OK) {  // rejected by the stager
            ++s->rejected;
            complete(s, r);
            continue;
        }
        // the batch's device working set must fit the budget
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const uint64_t used = (uint64_t)(total_b - free_b);
        const uint64_t need = (r->n_ins + r->n_del) * kWorkBytesPerEdge;
        r->live_queries = s->live;
        r->t_start = s->now_ms();
        lk.unlock();
        cgb_status st = CGB_OK;
        std::string err;
        if (s->budget && used + need > s->budget + s->base_used) {
            st = CGB_ERR_LIMIT;
            err = "batch working set exceeds the HBM budget";
        } else {
            r->pos.assign(CGB_MQ_MAX_QUERIES, 0);
            r->neg.assign(CGB_MQ_MAX_QUERIES, 0);
            cudaStream_t es = (cudaStream_t)cgb_mq_stream(s->m);
            cudaStreamWaitEvent(es, r->copied, 0);
            const uint32_t* dp = (const uint32_t*)(s->d_ring + r->ring_off);
            st = cgb_mq_apply_batch_device(s->m, r->n_ins ? dp : nullptr, r->n_ins,
                                           r->n_del ? dp + 2 * r->n_ins : nullptr, r->n_del, nullptr,
                                           r->pos.data(), r->neg.data(), CGB_MQ_MAX_QUERIES);
            if (st != CGB_OK) err = cgb_mq_last_error(s->m);
            float t4[4] = {0, 0, 0, 0};
            cgb_mq_last_timings(s->m, t4);
            r->device_ms = t4[3];
        }
        if (r->copied) cudaEventDestroy(r->copied);
        r->copied = nullptr;
        lk.lock();
        s->ring.release(r->ring_off, r->ring_len);
        r->status = st;
        r->err = err;
        if (st == CGB_OK) {
            ++s->batches_done;
            s->edges_done += r->n_ins + r->n_del;
            s->busy_ms += r->device_ms;
        } else {
            ++s->rejected;
        }
        complete(s, r);
        s->cv_stage.notify_all();
    }
}

cgb_status submit(cgb_server* s, std::shared_ptr<Req> r, uint64_t* ticket) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return CGB_ERR_STATE;
    if (s->queue.size() >= (s->cfg.max_pending ? s->cfg.max_pending : 4096u)) return CGB_ERR_LIMIT;
    r->ticket = s->next_ticket++;
    r->t_submit = s->now_ms();
    s->queue.push_back(r);
    s->all[r->ticket] = r;
    *ticket = r->ticket;
    s->cv_sched.notify_all();
    s->cv_stage.notify_all();
    return CGB_OK;
}

}  // namespace

extern "C" {

void cgb_server_default_config(cgb_server_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cgb_mq_default_config(&cfg->mq);
}

cgb_status cgb_server_create(const cgb_server_config* cfg, uint32_t n, const uint32_t* labels, uint64_t num_edges,
                             const uint32_t* edges, cgb_server** out) {
    if (!out || !labels) return CGB_ERR_ARG;
    *out = nullptr;
    cgb_server* s = new cgb_server();
    if (cfg) s->cfg = *cfg;
    else cgb_server_default_config(&s->cfg);
    *out = s;
    s->device = s->cfg.mq.device;
    s->t0 = std::chrono::steady_clock::now();
    cgb_status st = cgb_mq_create(&s->cfg.mq, &s->m);
    if (st != CGB_OK) {
        s->err = s->m ? cgb_mq_last_error(s->m) : "engine creation failed";
        return st;
    }
    st = cgb_mq_load_graph(s->m, n, labels, num_edges, edges);
    if (st != CGB_OK) {
        s->err = cgb_mq_last_error(s->m);
        return st;
    }
    if (cudaSetDevice(s->device) != cudaSuccess) return CGB_ERR_CUDA;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return CGB_ERR_CUDA;
    // the budget covers what the server may add on top of the loaded index
    s->base_used = (uint64_t)(total_b - free_b);
    s->budget = s->cfg.hbm_budget_bytes ? s->cfg.hbm_budget_bytes : (uint64_t)(free_b * 0.9);
    s->ring.cap = round16(std::max<uint64_t>(s->cfg.staging_bytes ? s->cfg.staging_bytes : (64ull << 20), 1 << 20));
    if (s->ring.cap > s->budget) {
        s->err = "staging ring larger than the HBM budget";
        return CGB_ERR_LIMIT;
    }
    if (cudaMallocHost(&s->h_ring, s->ring.cap) != cudaSuccess || cudaMalloc(&s->d_ring, s->ring.cap) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
        s->err = "staging allocation failed";
        return CGB_ERR_OOM;
    }
    s->sched = std::thread(scheduler_loop, s);
    s->stager = std::thread(stager_loop, s);
    return CGB_OK;
}

void cgb_server_destroy(cgb_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_sched.notify_all();
        s->cv_stage.notify_all();
        s->cv_done.notify_all();
    }
    if (s->sched.joinable()) s->sched.join();
    if (s->stager.joinable()) s->stager.join();
    cudaSetDevice(s->device);
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    for (auto& kv : s->all)
        if (kv.second->copied) cudaEventDestroy(kv.second->copied);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->h_ring) cudaFreeHost(s->h_ring);
    if (s->d_ring) cudaFree(s->d_ring);
    if (s->m) cgb_mq_destroy(s->m);
    delete s;
}

const char* cgb_server_last_error(const cgb_server* s) { return s ? s->err.c_str() : "null handle"; }

cgb_status cgb_server_submit_batch(cgb_server* s, const uint32_t* ins, uint64_t n_ins, const uint32_t* del,
                                   uint64_t n_del, uint64_t* ticket) {
    if (!s || !ticket || (n_ins && !ins) || (n_del && !del)) return CGB_ERR_ARG;
    if (n_ins > (1ull << 31) || n_del > (1ull << 31)) return CGB_ERR_LIMIT;
    auto r = std::make_shared<Req>();
    r->kind = CGB_SERVER_BATCH;
    r->n_ins = n_ins;
    r->n_del = n_del;
    r->pairs.resize(2 * (n_ins + n_del));
    if (n_ins) std::memcpy(r->pairs.data(), ins, n_ins * 8);
    if (n_del) std::memcpy(r->pairs.data() + 2 * n_ins, del, n_del * 8);
    return submit(s, r, ticket);
}

cgb_status cgb_server_submit_register(cgb_server* s, uint32_t qv, const uint32_t* labels, uint32_t qe,
                                      const uint32_t* edges, uint64_t* ticket) {
    if (!s || !ticket || !labels || !edges || qv > 12 || qe > 66) return CGB_ERR_ARG;
    auto r = std::make_shared<Req>();
    r->kind = CGB_SERVER_REGISTER;
    r->qv = qv;
    r->qe = qe;
    r->qlabels.assign(labels, labels + qv);
    r->qedges.assign(edges, edges + 2 * qe);
    return submit(s, r, ticket);
}

cgb_status cgb_server_submit_unregister(cgb_server* s, uint32_t query_id, uint64_t* ticket) {
    if (!s || !ticket) return CGB_ERR_ARG;
    auto r = std::make_shared<Req>();
    r->kind = CGB_SERVER_UNREGISTER;
    r->query_id = query_id;
    return submit(s, r, ticket);
}

cgb_status cgb_server_wait(cgb_server* s, uint64_t ticket, uint32_t timeout_ms, cgb_server_result* res,
                           uint64_t* pos, uint64_t* neg, uint32_t cap) {
    if (!s) return CGB_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return CGB_ERR_ARG;
    std::shared_ptr<Req> r = it->second;
    if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->done || s->stop; }) ||
        !r->done)
        return CGB_ERR_TIMEOUT;
    if (res) {
        res->ticket = r->ticket;
        res->kind = r->kind;
        res->status = r->status;
        res->query_id = r->query_id;
        res->live_queries = r->live_queries;
        res->t_submit_ms = r->t_submit;
        res->t_staged_ms = r->t_staged;
        res->t_start_ms = r->t_start;
        res->t_done_ms = r->t_done;
        res->device_ms = r->device_ms;
    }
    for (uint32_t i = 0; i < cap && i < r->pos.size(); ++i) {
        if (pos) pos[i] = r->pos[i];
        if (neg) neg[i] = r->neg[i];
    }
    if (r->status != CGB_OK) s->err = r->err;
    s->all.erase(it);  // collected
    return CGB_OK;
}

cgb_status cgb_server_stats(const cgb_server* s, uint64_t* out8) {
    if (!s || !out8) return CGB_ERR_ARG;
    std::lock_guard<std::mutex> lk(const_cast<cgb_server*>(s)->mu);
    out8[0] = s->batches_done;
    out8[1] = s->edges_done;
    out8[2] = s->rejected;
    out8[3] = s->live;
    out8[4] = s->queue.size();
    out8[5] = s->ring.cap;
    out8[6] = s->budget;
    out8[7] = (uint64_t)(s->busy_ms * 1000.0);
    return CGB_OK;
}

}  // extern "C"
