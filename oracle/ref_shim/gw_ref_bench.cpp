/*
 * gw_ref_bench.cpp -- BENCHMARK INFRASTRUCTURE (the CPU reference arm).
 *
 * Times GraphWalker's own CPU engine (src/engine/graphwalker.hpp) and walk
 * classes, compiled unmodified from the reference tree with its native glibc
 * rand_r, on a preprocessed graph.  The engine object (and its in-memory
 * block cache) is reused across runs, so runs after the first see the graph
 * resident in RAM, as the GPU engine sees it resident in HBM.
 *
 * Apps:
 *   rwd   -- mirrors apps/rwdomination.cpp: RandomWalkwithJump, a per-vertex
 *            visit counter incremented without atomics in updateInfo, walks
 *            placed block by block with source = start vertex; one walk on
 *            every `stride`-th vertex (a bounded sample of one walk per vertex).
 *   msppr -- mirrors apps/msppr.cpp's placement (walkspersource walks on each
 *            of `numsources` sources starting at firstsource, source field =
 *            source index) with RandomWalkwithStop; the per-visit sink is a
 *            per-thread counter as in apps/kk_ppr.cpp, because msppr's
 *            DiscreteDistribution::add is not thread-safe.
 *
 * Usage: gw_ref_bench <graph base> <blocksize_kb> <N> <L> <stride> <warmup>
 *                     <steps> <execthreads> [rwd | msppr <firstsource>
 *                     <numsources> <walkspersource>]
 * Prints one line per timed run:
 *   "step <i> walks <n> steps <visits> sec <t> threads_after <k>"
 * threads_after is omp_get_max_threads() when the run returns.  The engine's
 * exec_updates sets the OpenMP thread count to 1 for a block with fewer than
 * 100 walks and never restores it (graphwalker.hpp:260), so k == 1 with
 * execthreads > 1 means that fallback fired during the run and the rest of
 * the run was single-threaded.  Each run starts again at execthreads (the
 * apps' startWalksbyApp calls omp_set_num_threads, as the reference's apps do).
 */
#include <chrono>
#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "api/graphwalker_basic_includes.hpp"
#include "walks/randomwalkwithjump.hpp"
#include "walks/randomwalkwithstop.hpp"

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

class BenchMsppr : public RandomWalkwithStop {
public:
    vid_t firstsource = 0, numsources = 1;
    wid_t walkspersource = 1;
    std::vector<unsigned long long> visits;  // per thread, padded
    wid_t started = 0;

    void startWalksbyApp(WalkManager &walk_manager) {
        tid_t nthreads = get_option_int("execthreads", omp_get_max_threads());
        omp_set_num_threads(nthreads);
        visits.assign((size_t)nthreads * 16, 0);
        // apps/msppr.cpp:41-69: sources block by block, source field = source index
        bid_t p = getblock(firstsource);
        vid_t sts = firstsource, ens = blocks[p + 1];
        vid_t count = numsources;
        walk_manager.walksum = 0;
        while (count > 0) {
            if (ens > firstsource + numsources) ens = firstsource + numsources;
            vid_t nums = ens - sts;
            count -= nums;
            walk_manager.minstep[p] = 0;
            walk_manager.walknum[p] = nums * walkspersource;
#pragma omp parallel for schedule(static)
            for (vid_t s = 0; s < nums; s++) {
                vid_t cur = s + sts - blocks[p];
                WalkDataType walk = walk_manager.encode(s + sts - firstsource, cur, 0);
                for (wid_t j = 0; j < walkspersource; j++)
                    walk_manager.moveWalk(walk, p, omp_get_thread_num(), cur);
            }
            walk_manager.walksum += walk_manager.walknum[p];
            p++;
            sts = ens;
            ens = blocks[p + 1];
        }
        started = walk_manager.walksum;
    }

    void updateInfo(vid_t s, vid_t dstId, tid_t threadid, hid_t hop) { visits[(size_t)threadid * 16]++; }

    unsigned long long total_visits() const {
        unsigned long long t = 0;
        for (size_t i = 0; i < visits.size(); i += 16) t += visits[i];
        return t;
    }
};

int main(int argc, const char **argv) {
    if (argc < 9) {
        fprintf(stderr, "usage: %s graph blocksize_kb N L stride warmup steps execthreads [rwd|msppr first num wps]\n",
                argv[0]);
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
    const std::string app = argc > 10 ? argv[10] : "rwd";

    bid_t nblocks = convert_if_notexists(graph, blocksize_kb);
    graphwalker_engine engine(graph, blocksize_kb, nblocks, nblocks, m);
    if (app == "msppr") {
        if (argc < 14) return 2;
        BenchMsppr prog;
        prog.firstsource = (vid_t)strtoul(argv[11], nullptr, 10);
        prog.numsources = (vid_t)strtoul(argv[12], nullptr, 10);
        prog.walkspersource = strtoull(argv[13], nullptr, 10);
        prog.initializeRW(prog.numsources * prog.walkspersource, L);
        for (int i = 0; i < warmup + steps; ++i) {
            auto t0 = std::chrono::steady_clock::now();
            engine.run(prog, 0.2f);
            auto t1 = std::chrono::steady_clock::now();
            if (i >= warmup)
                printf("step %d walks %llu steps %llu sec %.6f threads_after %d\n", i - warmup,
                       (unsigned long long)prog.started, prog.total_visits(),
                       std::chrono::duration<double>(t1 - t0).count(), omp_get_max_threads());
            fflush(stdout);
        }
        return 0;
    }
    BenchDomination prog;
    prog.initializeRW(N, 1, L);
    prog.stride = stride ? stride : 1;
    prog.vertex_value = new unsigned[N]();
    for (int i = 0; i < warmup + steps; ++i) {
        std::fill(prog.vertex_value, prog.vertex_value + N, 0u);
        auto t0 = std::chrono::steady_clock::now();
        engine.run(prog, 0.2f);
        auto t1 = std::chrono::steady_clock::now();
        unsigned long long visits = 0;
        for (vid_t v = 0; v < N; ++v) visits += prog.vertex_value[v];
        if (i >= warmup)
            printf("step %d walks %llu steps %llu sec %.6f threads_after %d\n", i - warmup,
                   (unsigned long long)prog.started, visits, std::chrono::duration<double>(t1 - t0).count(),
                   omp_get_max_threads());
        fflush(stdout);
    }
    return 0;
}
