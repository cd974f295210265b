// reachability -- the reference's apps/reachability.cpp, which no longer
// builds against the reference's own engine (it uses the earlier interval
// API), rewritten on the live API that the drop-in headers provide.
//
// Same options and defaults as the reference app: file, a, b, R (walks), L
// (steps per walk), tail, prob, shardsize (the block size in KB; 0 = sized
// from the walk count).  R walks start at a (RandomWalkwithRestart); the
// answer is whether any of their visits reaches b.  Output, as the reference
// app's: "Reachability from <a> to <b> = <0|1>", then the metrics report.
#include <atomic>
#include <iostream>
#include <string>

#include "api/graphwalker_basic_includes.hpp"
#include "walks/randomwalkwithrestart.hpp"

class Reachability : public RandomWalkwithRestart {
 public:
  vid_t a = 0, b = 0;
  std::atomic<bool> ans{false};

  void initializeApp(vid_t _a, vid_t _b, wid_t _R, hid_t _L, float _tail) {
    a = _a;
    b = _b;
    initializeRW(a, _R, _L, _tail);
  }

  void startWalksbyApp(WalkManager& walk_manager) {
    logstream(LOG_INFO) << "Start " << nwalks << " walks of length " << nsteps << " from a : " << std::endl;
    const bid_t p = getblock(a);
    if (p >= nblocks) logstream(LOG_FATAL) << "a = " << a << " is not a vertex of the graph" << std::endl;
    const vid_t cur = a - blocks[p];
    const WalkDataType walk = walk_manager.encode(a, cur, 0);
    for (wid_t j = 0; j < nwalks; ++j) walk_manager.moveWalk(walk, p, 0, cur);
    walk_manager.walknum[p] += nwalks;
    walk_manager.minstep[p] = 0;
    walk_manager.walksum = nwalks;
  }

  void updateInfo(vid_t sourId, vid_t dstId, tid_t threadid, hid_t hop) {
    if (dstId == b) ans.store(true, std::memory_order_relaxed);
  }
};

int main(int argc, const char** argv) {
  set_argc(argc, argv);
  metrics m("reachability");
  std::string filename = get_option_string("file", "../DataSet/LiveJournal/soc-LiveJournal1.txt");
  unsigned a = get_option_int("a", 1);
  unsigned b = get_option_int("b", 2);
  unsigned R = get_option_int("R", 1000);
  unsigned L = get_option_int("L", 100);
  float tail = get_option_float("tail", 0);
  float prob = get_option_float("prob", 0.2);
  unsigned long long shardsize = get_option_long("shardsize", 0);

  Reachability program;
  program.initializeApp(a, b, R, L, tail);
  if (shardsize == 0) shardsize = program.compBlockSize(R);
  bid_t nblocks = convert_if_notexists(filename, shardsize);
  graphwalker_engine engine(filename, shardsize, nblocks, nblocks, m);
  engine.run(program, prob);
  std::cout << "Reachability from " << a << " to " << b << " = " << program.ans.load() << std::endl;
  metrics_report(m);
  return 0;
}
