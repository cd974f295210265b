/*
 * gw_ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Builds GraphWalker's own engine (src/engine/graphwalker.hpp), walk manager
 * (src/walks/walk.hpp) and one of its walk classes, unmodified, from the
 * reference tree, with one change made from the outside: every `rand_r`
 * call the walk classes make (randomwalkwithjump.hpp:37-50 and siblings) is
 * routed to a Philox4x32-10 stream keyed on (seed, walk key, hop, draw
 * index), so that its trajectories become reproducible and can be compared
 * bit for bit with the CUDA walk kernels.
 *
 * The shim relies on a property of every live walk class: the app's
 * updateInfo(s, dst, tid, hop) is called immediately before that hop's
 * rand_r draws, on the same thread (randomwalkwithjump.hpp:42,
 * randomwalkwithstop.hpp:32, randomwalkwithprob.hpp:32,
 * randomwalkwithrestartwithjoint.hpp:40).  The app below records
 * {key = s, hop, draw = 0} in thread-local state there, and the shimmed
 * rand_r returns word[draw++] >> 1 of Philox(key=seed, ctr=(s, hop, 0, 0)).
 *
 * Build: oracle/Makefile (RULE=0..3 selects the walk class; the stop and
 * prob classes share an include guard, so each class is its own binary).
 *
 * Usage: gw_ref_shim_<rule> <graph base> <blocksize_kb> <walks file> <out file>
 *                           <L> <seed_hex> <njump> <nmblocks> <prob>
 *                           <nkeys> <stride> [execthreads <n>]
 *   walks file: uint64 n, then n records {uint32 block, uint32 pad, uint64 word}
 *   out file  : uint32 status, uint32 nv, uint32 counts[nv],
 *               uint32 paths[nkeys * stride] (0xffffffff = no visit),
 *               uint64 closure
 *   paths[s * stride + hop] records the vertex a walk with source field s
 *   visited at hop (the simrank sink, apps/simrank.cpp:59-69).
 */
#include <cstdlib>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <cmath>
#include <atomic>
#include <string>
#include <vector>
#include <map>
#include <queue>
#include <fstream>
#include <sstream>
#include <iostream>
#include <omp.h>
#include <assert.h>
#include <fcntl.h>
#include <unistd.h>
#include <dirent.h>
#include <errno.h>
#include <sys/stat.h>
#include <sys/time.h>
#include <sys/types.h>
#include <sys/mman.h>
#include <zlib.h>

extern "C" {
#include "../gw_oracle.h"
}

static uint64_t g_seed = 0;
static thread_local uint32_t tl_key = 0, tl_hop = 0, tl_draw = 0;
static std::atomic<uint32_t> g_status{0};

static int gw_shim_rand_r(unsigned *) {
    if (tl_draw >= 4) {
        g_status |= 8u; /* more than four draws in one hop: not expected */
        return 0;
    }
    uint32_t ctr[4] = {tl_key, tl_hop, 0u, 0u};
    uint32_t key[2] = {(uint32_t)g_seed, (uint32_t)(g_seed >> 32)};
    uint32_t out[4];
    gwo_philox4x32_10(ctr, key, out);
    return (int)(out[tl_draw++] >> 1);
}
#define rand_r(s) gw_shim_rand_r(s)

#include "api/graphwalker_basic_includes.hpp"

#if GW_SHIM_RULE == 0
#include "walks/randomwalkwithjump.hpp"
typedef RandomWalkwithJump ShimBase;
#elif GW_SHIM_RULE == 1
#include "walks/randomwalkwithstop.hpp"
typedef RandomWalkwithStop ShimBase;
#elif GW_SHIM_RULE == 2
#include "walks/randomwalkwithprob.hpp"
typedef RandomWalkwithProb ShimBase;
#elif GW_SHIM_RULE == 3
#include "walks/randomwalkwithrestartwithjoint.hpp"
typedef RandomWalkwithRestartwithJoint ShimBase;
#else
#error "GW_SHIM_RULE must be 0..3"
#endif

struct ShimWalk {
    uint32_t block;
    uint32_t pad;
    uint64_t word;
};

class ShimApp : public ShimBase {
public:
    std::vector<ShimWalk> start;
    uint32_t nv = 0;
    uint32_t nkeys = 0, stride = 0;
    hid_t Lcap = 0;
    std::vector<std::atomic<uint32_t>> counts;
    std::vector<std::atomic<uint32_t>> paths;
    std::atomic<uint64_t> closure{0};

    void setup(uint32_t _nv, uint32_t _nkeys, uint32_t _stride, hid_t _L) {
        nv = _nv;
        nkeys = _nkeys;
        stride = _stride;
        Lcap = _L;
        counts = std::vector<std::atomic<uint32_t>>(nv);
        for (auto &c : counts) c = 0;
        paths = std::vector<std::atomic<uint32_t>>((size_t)nkeys * stride);
        for (auto &c : paths) c = 0xffffffffu;
    }

    void startWalksbyApp(WalkManager &wm) {
        for (const ShimWalk &w : start) {
            uint32_t p = w.block;
            wm.moveWalk(w.word, p, 0, wm.getCurrentId(w.word));
            wm.walknum[p]++;
            hid_t h = wm.getHop(w.word);
            if (wm.minstep[p] > h) wm.minstep[p] = h;
        }
        wm.walksum = start.size();
    }

    void updateInfo(vid_t s, vid_t dstId, tid_t threadid, hid_t hop) {
        tl_key = s;
        tl_hop = hop;
        tl_draw = 0;
        if (dstId < nv) counts[dstId].fetch_add(1, std::memory_order_relaxed);
        else g_status |= 1u;
        if (s < nkeys && hop < stride) paths[(size_t)s * stride + hop].store(dstId);
        if ((int)hop >= (int)Lcap - 1 && dstId == s) closure.fetch_add(1);
    }
};

int main(int argc, const char **argv) {
    if (argc < 12) {
        fprintf(stderr, "usage: %s graph blocksize_kb walks out L seed_hex njump nmblocks prob nkeys stride [execthreads n]\n", argv[0]);
        return 2;
    }
    set_argc(argc, argv);
    metrics m("gw_ref_shim");
    std::string graph = argv[1];
    unsigned long long blocksize_kb = strtoull(argv[2], nullptr, 10);
    const char *walks_path = argv[3];
    const char *out_path = argv[4];
    hid_t L = (hid_t)atoi(argv[5]);
    g_seed = strtoull(argv[6], nullptr, 16);
    uint32_t njump = (uint32_t)strtoul(argv[7], nullptr, 10);
    bid_t nmblocks = (bid_t)atoi(argv[8]);
    float prob = (float)atof(argv[9]);
    uint32_t nkeys = (uint32_t)strtoul(argv[10], nullptr, 10);
    uint32_t stride = (uint32_t)strtoul(argv[11], nullptr, 10);

    ShimApp app;
    FILE *wf = fopen(walks_path, "rb");
    if (!wf) { perror("walks"); return 3; }
    uint64_t n = 0;
    if (fread(&n, 8, 1, wf) != 1) return 3;
    app.start.resize(n);
    if (n && fread(app.start.data(), sizeof(ShimWalk), n, wf) != n) return 3;
    fclose(wf);

    bid_t nblocks = convert_if_notexists(graph, blocksize_kb);
    if (nmblocks == 0 || nmblocks > nblocks) nmblocks = nblocks;

#if GW_SHIM_RULE == 0
    app.initializeRW(njump, n, L);
#else
    app.initializeRW(n, L);
    (void)njump;
#endif
    graphwalker_engine engine(graph, blocksize_kb, nblocks, nmblocks, m);
    app.setup(engine.num_vertices(), nkeys, stride, L);
    engine.run(app, prob);

    FILE *of = fopen(out_path, "wb");
    if (!of) { perror("out"); return 4; }
    uint32_t st = g_status.load();
    fwrite(&st, 4, 1, of);
    fwrite(&app.nv, 4, 1, of);
    for (auto &c : app.counts) { uint32_t x = c.load(); fwrite(&x, 4, 1, of); }
    for (auto &c : app.paths) { uint32_t x = c.load(); fwrite(&x, 4, 1, of); }
    uint64_t cl = app.closure.load();
    fwrite(&cl, 8, 1, of);
    fclose(of);
    return 0;
}
