/*
 * A GraphWalker-style program built on the drop-in headers
 * (graphwalker_b200/compat) and the B200 engine, used by tests/test_compat.py.
 * It places the walks of a walks file into the WalkManager pools, runs
 * graphwalker_engine::run, and records what its updateInfo receives -- in the
 * output format of oracle/ref_shim/gw_ref_shim.cpp, so the result can be
 * compared with the reference engine's golden vectors.
 *
 * Usage: gw_compat_app <graph base> <blocksize_kb> <walks file> <out file> <L>
 *                      <seed> <njump> <nkeys> <stride> [key value ...]
 * RULE (compile-time): 0 jump, 1 stop, 2 prob, 3 restart.
 */
#include <atomic>
#include <cstdio>
#include <vector>

#include "api/graphwalker_basic_includes.hpp"
#include "walks/randomwalkwithjump.hpp"
#include "walks/randomwalkwithprob.hpp"
#include "walks/randomwalkwithrestartwithjoint.hpp"
#include "walks/randomwalkwithstop.hpp"

#if GW_APP_RULE == 0
typedef RandomWalkwithJump Base;
#elif GW_APP_RULE == 1
typedef RandomWalkwithStop Base;
#elif GW_APP_RULE == 2
typedef RandomWalkwithProb Base;
#else
typedef RandomWalkwithRestartwithJoint Base;
#endif

struct StartWalk {
  uint32_t block, pad;
  uint64_t word;
};

class App : public Base {
 public:
  std::vector<StartWalk> start;
  uint32_t nv = 0, nkeys = 0, stride = 0;
  hid_t Lcap = 0;
  std::vector<std::atomic<uint32_t>> counts, paths;
  std::atomic<uint64_t> closure{0};

  void setup(uint32_t _nv, uint32_t _nkeys, uint32_t _stride, hid_t _L) {
    nv = _nv;
    nkeys = _nkeys;
    stride = _stride;
    Lcap = _L;
    counts = std::vector<std::atomic<uint32_t>>(nv);
    for (auto& c : counts) c = 0;
    paths = std::vector<std::atomic<uint32_t>>((size_t)nkeys * stride);
    for (auto& c : paths) c = 0xffffffffu;
  }
  void startWalksbyApp(WalkManager& wm) {
    for (const StartWalk& w : start) {
      wm.moveWalk(w.word, w.block, 0, wm.getCurrentId(w.word));
      wm.walknum[w.block]++;
      wm.setMinStep(w.block, wm.getHop(w.word));
    }
    wm.walksum = start.size();
  }
  void updateInfo(vid_t s, vid_t dst, tid_t t, hid_t hop) {
    if (dst < nv) counts[dst].fetch_add(1, std::memory_order_relaxed);
    if (s < nkeys && hop < stride) paths[(size_t)s * stride + hop].store(dst);
    if ((int)hop >= (int)Lcap - 1 && dst == s) closure.fetch_add(1);
  }
};

int main(int argc, const char** argv) {
  if (argc < 10) {
    fprintf(stderr, "usage: %s graph blocksize_kb walks out L seed njump nkeys stride [key value ...]\n", argv[0]);
    return 2;
  }
  set_argc(argc, argv);
  metrics m("gw_compat_app");
  std::string graph = argv[1];
  unsigned long long blocksize_kb = strtoull(argv[2], nullptr, 10);
  hid_t L = (hid_t)atoi(argv[5]);
  uint32_t njump = (uint32_t)strtoul(argv[7], nullptr, 10);
  uint32_t nkeys = (uint32_t)strtoul(argv[8], nullptr, 10), stride = (uint32_t)strtoul(argv[9], nullptr, 10);
  App app;
  FILE* wf = fopen(argv[3], "rb");
  if (!wf) return 3;
  uint64_t n = 0;
  if (fread(&n, 8, 1, wf) != 1) return 3;
  app.start.resize(n);
  if (n && fread(app.start.data(), sizeof(StartWalk), n, wf) != n) return 3;
  fclose(wf);
  bid_t nblocks = convert_if_notexists(graph, blocksize_kb);
#if GW_APP_RULE == 0
  app.initializeRW(njump, n, L);
#else
  app.initializeRW(n, L);
  (void)njump;
#endif
  graphwalker_engine engine(graph, blocksize_kb, nblocks, nblocks, m);
  app.setup(engine.num_vertices(), nkeys, stride, L);
  engine.run(app, 0.2f);
  metrics_report(m);
  FILE* of = fopen(argv[4], "wb");
  uint32_t st = 0;
  fwrite(&st, 4, 1, of);
  fwrite(&app.nv, 4, 1, of);
  for (auto& c : app.counts) { uint32_t x = c.load(); fwrite(&x, 4, 1, of); }
  for (auto& c : app.paths) { uint32_t x = c.load(); fwrite(&x, 4, 1, of); }
  uint64_t cl = app.closure.load();
  fwrite(&cl, 8, 1, of);
  fclose(of);
  return 0;
}
