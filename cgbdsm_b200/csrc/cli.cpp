// Drop-in command line for the reference's batched pipeline:
//     cgbdsm <query_path> <data_path> <update_path> <gpu_id> [batch_size]
// Argument meaning follows main_calig.cpp:42-69 (batch_size counts ints, two
// per edge; default UINT32_MAX = one batch).  Stage 1 (CaLiG producer) runs on
// a host thread ahead of Stage 2 (the GPU engine) with a bounded hand-off
// queue, as the reference's 2-stage pipeline does (main_calig.cpp:203-292).
// Prints "Num Positive Matches: N" and the reference's profiling summary
// (main_calig.cpp:400-438).
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cgbdsm.h"

namespace {

struct Batch {
    std::vector<uint64_t> ins, del, delta;
    std::vector<uint8_t> edge_ok;
    uint32_t dv = 0;
    double ms_ui = 0, ms_cu = 0, ms_pr = 0;
};

using Clock = std::chrono::high_resolution_clock;
double ms_since(Clock::time_point t0) { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s <query_path> <data_path> <update_path> <gpu_id> [batch_size]\n", argv[0]);
        return 1;
    }
    const char* qpath = argv[1];
    const char* dpath = argv[2];
    const char* upath = argv[3];
    const int gpu = std::atoi(argv[4]);
    const uint32_t batch_size = argc > 5 ? (uint32_t)std::strtoul(argv[5], nullptr, 10) : UINT32_MAX;

    cgb_producer* prod = nullptr;
    auto t_open = Clock::now();
    cgb_status st = cgb_producer_open(qpath, dpath, upath, batch_size, 0, &prod);
    if (st != CGB_OK) {
        std::fprintf(stderr, "error: %s\n", prod ? cgb_producer_last_error(prod) : "producer");
        cgb_producer_close(prod);
        return 2;
    }
    const uint32_t nb = cgb_producer_num_batches(prod);
    std::printf("Stage 1 index built in %.1f ms, num_batches: %u\n", ms_since(t_open), nb);

    cgb_config cfg;
    cgb_default_config(&cfg);
    cfg.device = gpu;
    cgb_handle* h = nullptr;
    st = cgb_create(&cfg, &h);
    if (st == CGB_OK) st = cgb_load_query_file(h, qpath);
    const uint64_t* init = nullptr;
    uint64_t n_init = 0;
    uint32_t dv0 = 0;
    if (st == CGB_OK) st = cgb_producer_initial(prod, &init, &n_init, &dv0);
    if (st == CGB_OK) st = cgb_build_index(h, init, n_init, dv0);
    if (st != CGB_OK) {
        std::fprintf(stderr, "error: %s\n", h ? cgb_last_error(h) : "engine");
        cgb_destroy(h);
        cgb_producer_close(prod);
        return 3;
    }
    if (nb == 0) {
        std::printf("No updates to process.\n");
        cgb_destroy(h);
        cgb_producer_close(prod);
        return 0;
    }

    // ---- Stage 1 thread ----
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Batch> q;
    bool s1_done = false, s1_error = false;
    std::string s1_err;
    const size_t max_ahead = 2;
    double s1_ui = 0, s1_cu = 0, s1_pr = 0;
    std::thread s1([&] {
        for (uint32_t b = 0; b < nb; ++b) {
            cgb_batch_keys k;
            if (cgb_producer_next(prod, &k) != CGB_OK) {
                std::lock_guard<std::mutex> lk(mu);
                s1_error = true;
                s1_err = cgb_producer_last_error(prod);
                break;
            }
            Batch bt;
            bt.ins.assign(k.ins, k.ins + k.n_ins);
            bt.del.assign(k.del, k.del + k.n_del);
            bt.delta.assign(k.delta, k.delta + k.n_delta);
            bt.edge_ok.assign(k.edge_ok, k.edge_ok + k.qe);
            bt.dv = k.dv_count;
            bt.ms_ui = k.ms_update_index;
            bt.ms_cu = k.ms_construct_update;
            bt.ms_pr = k.ms_prepare;
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return q.size() < max_ahead; });
            q.push_back(std::move(bt));
            cv.notify_all();
        }
        std::lock_guard<std::mutex> lk(mu);
        s1_done = true;
        cv.notify_all();
    });

    // ---- Stage 2: GPU ----
    unsigned long long matches = 0;
    double s2_update = 0, s2_delta = 0, s2_match = 0, s2_wall = 0, wait_ms = 0;
    auto t_pipe = Clock::now();
    int rc = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        Batch bt;
        {
            auto w0 = Clock::now();
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return !q.empty() || s1_done || s1_error; });
            wait_ms += ms_since(w0);
            if (q.empty()) {
                std::fprintf(stderr, "error: stage 1 stopped: %s\n", s1_err.c_str());
                rc = 4;
                break;
            }
            bt = std::move(q.front());
            q.pop_front();
            cv.notify_all();
        }
        s1_ui += bt.ms_ui;
        s1_cu += bt.ms_cu;
        s1_pr += bt.ms_pr;
        uint64_t c = 0;
        auto t0 = Clock::now();
        st = cgb_apply_batch(h, bt.dv, bt.ins.data(), bt.ins.size(), bt.del.data(), bt.del.size(), bt.delta.data(),
                             bt.delta.size(), bt.edge_ok.data(), &c);
        s2_wall += ms_since(t0);
        if (st != CGB_OK) {
            std::fprintf(stderr, "error: batch %u: %s\n", b, cgb_last_error(h));
            rc = 5;
            break;
        }
        float t4[4];
        cgb_last_timings(h, t4);
        s2_update += t4[0];
        s2_delta += t4[1];
        s2_match += t4[2];
        matches += c;
    }
    {
        std::unique_lock<std::mutex> lk(mu);
        q.clear();
        s1_error = s1_error || rc != 0;
        cv.notify_all();
    }
    if (rc != 0) {
        // let stage 1 finish its current batch, then stop
        s1.detach();
        cgb_destroy(h);
        return rc;
    }
    s1.join();
    const double total_ms = ms_since(t_pipe);
    std::printf("Incremental Matching (2-Stage Pipeline): %.1f ms\n", total_ms);
    std::printf("Num Positive Matches: %llu\n", matches);
    const double s1_total = s1_ui + s1_cu + s1_pr;
    const double s2_total = s2_wall;
    std::printf("\n========== 2-Stage Pipeline Profiling Summary ==========\n");
    std::printf("Total batches: %u\n", nb);
    std::printf("\n--- Stage 1 (CPU: updateIndex + ConstructUpdate + PrepareUpdate) ---\n");
    std::printf("[S1] updateIndex:        %.3f ms\n", s1_ui);
    std::printf("[S1] ConstructUpdate:    %.3f ms\n", s1_cu);
    std::printf("[S1] PrepareUpdate:      %.3f ms\n", s1_pr);
    std::printf("[S1] TOTAL:              %.3f ms\n", s1_total);
    std::printf("\n--- Stage 2 (GPU: Transfer + Match) ---\n");
    std::printf("[S2] TransferUpdateAll:  %.3f ms (device; includes the previous batch's delta merge-back)\n",
                s2_update);
    std::printf("[S2] TransferUpdateIdx:  %.3f ms (device)\n", s2_delta);
    std::printf("[S2] Matching:           %.3f ms (device)\n", s2_match);
    std::printf("[S2] TOTAL:              %.3f ms (host wall, incl. copies)\n", s2_total);
    std::printf("\n--- Sync Waits ---\n");
    std::printf("[Sync] S2 wait for S1:   %.3f ms\n", wait_ms);
    std::printf("\n--- Bottleneck = max(S1, S2) ---\n");
    std::printf("S1 avg/batch: %.3f ms\n", s1_total / nb);
    std::printf("S2 avg/batch: %.3f ms\n", s2_total / nb);
    std::printf("===================================================\n");
    cgb_destroy(h);
    cgb_producer_close(prod);
    return 0;
}
