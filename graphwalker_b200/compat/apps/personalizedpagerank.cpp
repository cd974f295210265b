// personalizedpagerank -- the reference's apps/personalizedpagerank.cpp,
// which no longer builds against the reference's own engine (it uses the
// earlier interval API: getInterval, pwalks, before/after_exec_interval),
// rewritten on the live API that the drop-in headers provide.
//
// Same options and defaults as the reference app: file, nvertices, source,
// R (walks), L (steps per walk), tail, prob, shardsize (the block size in KB).
// R walks start at `source` (RandomWalkwithRestart: restart at the source on
// the 0.15 branch and at dangling vertices, L visits per walk) and every visit
// is counted per vertex.  Output, as the reference app's: the counts as
// uint32 per vertex in <file>_GraphWalker/4B.vvalue, then the metrics report.
#include <fcntl.h>
#include <unistd.h>

#include <atomic>
#include <string>
#include <vector>

#include "api/graphwalker_basic_includes.hpp"
#include "walks/randomwalkwithrestart.hpp"

typedef unsigned VertexDataType;

class PersonalizedPageRank : public RandomWalkwithRestart {
 public:
  vid_t N = 0;
  std::vector<std::atomic<VertexDataType>> visits;

  static std::string filename_vertex_data(const std::string& base) {
    return base + "_GraphWalker/" + std::to_string(sizeof(VertexDataType)) + "B.vvalue";
  }

  void initializeApp(vid_t _N, vid_t _source, wid_t _R, hid_t _L, float _tail) {
    N = _N;
    visits = std::vector<std::atomic<VertexDataType>>(N);
    for (auto& x : visits) x.store(0, std::memory_order_relaxed);
    initializeRW(_source, _R, _L, _tail);
  }

  // all R walks at the source, hop 0, in the source's block
  void startWalksbyApp(WalkManager& walk_manager) {
    logstream(LOG_INFO) << "Start walks ! Total walk number = " << nwalks << std::endl;
    const bid_t p = getblock(source);
    if (p >= nblocks) logstream(LOG_FATAL) << "source " << source << " is not a vertex of the graph" << std::endl;
    const vid_t cur = source - blocks[p];
    const WalkDataType walk = walk_manager.encode(source, cur, 0);
    for (wid_t j = 0; j < nwalks; ++j) walk_manager.moveWalk(walk, p, 0, cur);
    walk_manager.walknum[p] += nwalks;
    walk_manager.minstep[p] = 0;
    walk_manager.walksum = nwalks;
  }

  void updateInfo(vid_t sourId, vid_t dstId, tid_t threadid, hid_t hop) {
    if (dstId < N) visits[dstId].fetch_add(1, std::memory_order_relaxed);
  }

  void write_vertex_values(const std::string& base) const {
    std::vector<VertexDataType> out(N);
    for (vid_t v = 0; v < N; ++v) out[v] = visits[v].load(std::memory_order_relaxed);
    int f = open(filename_vertex_data(base).c_str(), O_WRONLY | O_CREAT | O_TRUNC, S_IROTH | S_IWOTH | S_IWUSR | S_IRUSR);
    if (f < 0) logstream(LOG_FATAL) << "could not open " << filename_vertex_data(base) << std::endl;
    pwritea(f, out.data(), sizeof(VertexDataType) * N, 0);
    close(f);
  }
};

int main(int argc, const char** argv) {
  set_argc(argc, argv);
  metrics m("personalizedpagerank");
  std::string filename = get_option_string("file", "../DataSet/LiveJournal/soc-LiveJournal1.txt");
  unsigned nvertices = get_option_int("nvertices", 4847571);
  unsigned source = get_option_int("source", 0);
  unsigned R = get_option_int("R", 2000);
  unsigned L = get_option_int("L", 10);
  float tail = get_option_float("tail", 0);
  float prob = get_option_float("prob", 0.2);
  unsigned long long shardsize = get_option_long("shardsize", 128);

  bid_t nblocks = convert_if_notexists(filename, shardsize);
  PersonalizedPageRank program;
  program.initializeApp(nvertices, source, R, L, tail);
  graphwalker_engine engine(filename, shardsize, nblocks, nblocks, m);
  engine.run(program, prob);
  program.write_vertex_values(filename);
  metrics_report(m);
  return 0;
}
