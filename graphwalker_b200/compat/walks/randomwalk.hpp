// Drop-in GraphWalker API: the RandomWalk base class apps derive from.
// Members and virtuals as in the reference (src/walks/randomwalk.hpp:16-116).
// Four hooks tell the device engine how to run a program: the walk class
// (gw_rule), its length (gw_length), the jump range (gw_njump), and what to
// do with per-vertex visit counts when the engine counts on the device
// (gw_deliver_counts, used with the `gw_sink count` knob).
#ifndef RANDOMWALK
#define RANDOMWALK

#include <cmath>
#include <fstream>
#include <string>

#include "api/datatype.hpp"
#include "graphwalker_b200.h"
#include "walks/walk.hpp"

class RandomWalk {
 public:
  bid_t nblocks = 0;
  vid_t* blocks = nullptr;
  wid_t R = 0;
  hid_t L = 0;

  virtual ~RandomWalk() {}

  virtual void startWalksbyApp(WalkManager& walk_manager) {
    logstream(LOG_ERROR) << "No definition of function : startWalksbyApp!" << std::endl;
  }
  virtual void updateInfo(vid_t s, vid_t dstId, tid_t threadid, hid_t hop) {
    logstream(LOG_ERROR) << "No definition of function : updateInfo!" << std::endl;
  }
  // The per-walk host update of the reference; the device engine runs the
  // walk class's rule itself and never calls this.
  virtual void updateByWalk(WalkDataType walk, wid_t walkid, bid_t exec_block, eid_t*& beg_pos, vid_t*& csr,
                            WalkManager& walk_manager) {
    logstream(LOG_ERROR) << "No definition of function : updateByWalk!" << std::endl;
  }
  virtual wid_t before_exec_block(bid_t exec_block, vid_t window_st, vid_t window_en, WalkManager& walk_manager) {
    return 0;
  }
  virtual void after_exec_block(bid_t exec_block, vid_t window_st, vid_t window_en, WalkManager& walk_manager) {}
  virtual void compUtilization(eid_t total_edges) {}

  virtual void initializeRW(wid_t _R, hid_t _L) {
    R = _R;
    L = _L;
  }
  virtual void startWalks(WalkManager& walk_manager, bid_t _nblocks, vid_t* _blocks, std::string base_filename) {
    nblocks = _nblocks;
    blocks = _blocks;
    startWalksbyApp(walk_manager);
  }
  // first p with v < blocks[p+1]; nblocks when v is past the last block
  virtual unsigned getblock(vid_t v) { return gw_getblock(blocks, nblocks, v); }
  virtual bool hasFinishedWalk(WalkManager& walk_manager) { return walk_manager.walksum > 0; }
  // 2^(11 + number of decimal digits of nwalks) KB
  virtual unsigned long long compBlockSize(wid_t nwalks) {
    unsigned long long kb = gw_comp_block_size(nwalks);
    logstream(LOG_DEBUG) << "Determined blocksize_kb = " << kb << std::endl;
    return kb;
  }
  virtual bid_t compNmblocks(unsigned long long blocksize_kb) {
    bid_t n = gw_comp_nmblocks(blocksize_kb, MEM_BUDGET);
    logstream(LOG_DEBUG) << "Computed nmblocks = " << n << std::endl;
    return n;
  }

  // ---- device-engine hooks ----
  virtual int gw_rule() const { return -1; }  // not a walk class the engine runs
  virtual hid_t gw_length() const { return L; }
  virtual vid_t gw_njump() const { return 0; }
  // Visits per walk the device records for the host replay of updateInfo.
  virtual uint32_t gw_max_visits() const { return gw_length() ? gw_length() : 1; }
  // Counts mode: hands per-vertex visit counts to the program.  The default
  // replays them through updateInfo(0, v, 0, 0) once per visit, which is
  // exact for programs whose updateInfo depends on the vertex alone.
  virtual void gw_deliver_counts(const uint32_t* counts, vid_t n) {
    for (vid_t v = 0; v < n; ++v)
      for (uint32_t c = 0; c < counts[v]; ++c) updateInfo(0, v, 0, 0);
  }
};

#endif
