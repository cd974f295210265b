/*
 * gw_ref_bench.cpp -- BENCHMARK INFRASTRUCTURE (the CPU reference arm).
 *
 * Times GraphWalker's own CPU engine (src/engine/graphwalker.hpp) and walk
 * class, compiled unmodified from the reference tree with its native glibc
 * rand_r, on a preprocessed graph.  The app below mirrors
 * apps/rwdomination.cpp (RandomWalkwithJump, per-vertex visit counter
 * incremented without atomics in updateInfo, walks placed block by block
 * with source = start vertex) but starts one walk on every `stride`-th vertex
 * so that one engine run is a bounded sample of the one-walk-per-vertex
 * workload; the engine object (and its in-memory block cache) is reused
 * across runs, so runs after the first see the graph resident in RAM, as
 * the GPU engine sees it resident in HBM.
 *
 * Usage: gw_ref_bench <graph base> <blocksize_kb> <N> <L> <stride>
 *                     <warmup> <steps> <execthreads> [rule]
 *   rule 0 = RandomWalkwithJump (rwdomination), 1 = RandomWalkwithStop (msppr)
 * Prints one line per timed run: "step <i> walks <n> steps <visits> sec <t>".
 */
#include <chrono>
#include <cmath>
#include <fstream>
#include <string>

#include "api/graphwalker_basic_includes.hpp"
#include "walks/randomwalkwithjump.hpp"

class BenchDomination : public RandomWalkwithJump {
public:
    unsigned *vertex_value = nullptr;
    vid_t stride = 1;
    wid_t started = 0;

    void startWalksbyApp(WalkManager &walk_manager) {
        tid_t nthreads = get_option_int("execthreads", omp_get_max_threads());
        omp_set_num_threads(nthreads);
        started = 0;
#pragma omp parallel for schedule(static) reduction(+ : started)
        for (bid_t p = 0; p < nblocks; p++) {
            wid_t n = 0;
            vid_t first = (blocks[p] + stride - 1) / stride * stride;
            for (vid_t v = first; v < blocks[p + 1]; v += stride) {
                WalkDataType walk = walk_manager.encode(v, v - blocks[p], 0);
                walk_manager.moveWalk(walk, p, omp_get_thread_num(), v - blocks[p]);
                n++;
            }
            walk_manager.walknum[p] = n;
            walk_manager.minstep[p] = n ? 0 : 0xffff;
            started += n;
        }
        walk_manager.walksum = started;
    }

    void updateInfo(vid_t s, vid_t dstId, tid_t threadid, hid_t hop) {
        vertex_value[dstId]++;  // as apps/rwdomination.cpp:65 (no atomics)
    }
};

int main(int argc, const char **argv) {
    if (argc < 9) {
        fprintf(stderr, "usage: %s graph blocksize_kb N L stride warmup steps execthreads\n", argv[0]);
        return 2;
    }
    set_argc(argc, argv);
    metrics m("gw_ref_bench");
    std::string graph = argv[1];
    unsigned long long blocksize_kb = strtoull(argv[2], nullptr, 10);
    vid_t N = (vid_t)strtoul(argv[3], nullptr, 10);
    hid_t L = (hid_t)atoi(argv[4]);
    vid_t stride = (vid_t)strtoul(argv[5], nullptr, 10);
    int warmup = atoi(argv[6]), steps = atoi(argv[7]);

    BenchDomination app;
    app.initializeRW(N, 1, L);
    app.stride = stride ? stride : 1;
    app.vertex_value = new unsigned[N]();
    bid_t nblocks = convert_if_notexists(graph, blocksize_kb);
    graphwalker_engine engine(graph, blocksize_kb, nblocks, nblocks, m);
    for (int i = 0; i < warmup + steps; ++i) {
        std::fill(app.vertex_value, app.vertex_value + N, 0u);
        auto t0 = std::chrono::steady_clock::now();
        engine.run(app, 0.2f);
        auto t1 = std::chrono::steady_clock::now();
        unsigned long long visits = 0;
        for (vid_t v = 0; v < N; ++v) visits += app.vertex_value[v];
        if (i >= warmup)
            printf("step %d walks %llu steps %llu sec %.6f\n", i - warmup, (unsigned long long)app.started,
                   visits, std::chrono::duration<double>(t1 - t0).count());
        fflush(stdout);
    }
    return 0;
}
