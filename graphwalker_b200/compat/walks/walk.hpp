// Drop-in GraphWalker API: WalkManager -- the walk codec, the per-block
// pools the apps fill in startWalksbyApp, and the per-block counters.
// Public members and methods as in the reference (src/walks/walk.hpp:17-267).
// The pools stay on the host only until graphwalker_engine::run hands them to
// the device engine (gw_walks_add); block scheduling then runs on the device
// engine's own counters.
#ifndef DEF_GRAPHWALKER_WALK
#define DEF_GRAPHWALKER_WALK

#include <sys/stat.h>

#include <cassert>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "api/filename.hpp"
#include "metrics/metrics.hpp"
#include "walks/walkbuffer.hpp"

class WalkManager {
 protected:
  std::string base_filename;
  bid_t nblocks;
  tid_t nthreads;
  metrics& m;

 public:
  wid_t* walknum;   // walks pending per block
  wid_t* dwalknum;  // walks spilled to disk per block (always 0 here)
  hid_t* minstep;   // lowest hop pending per block
  WalkBuffer** pwalks;
  bid_t curp = 0;
  WalkDataType* curwalks = nullptr;
  wid_t walksum;
  bool* ismodified;

  WalkManager(metrics& _m, bid_t _nblocks, tid_t _nthreads, std::string _base_filename)
      : base_filename(_base_filename), nblocks(_nblocks), nthreads(_nthreads ? _nthreads : 1), m(_m) {
    pwalks = new WalkBuffer*[nthreads];
    for (tid_t i = 0; i < nthreads; i++) pwalks[i] = new WalkBuffer[nblocks];
    walknum = (wid_t*)calloc(nblocks, sizeof(wid_t));
    dwalknum = (wid_t*)calloc(nblocks, sizeof(wid_t));
    minstep = (hid_t*)malloc(nblocks * sizeof(hid_t));
    memset(minstep, 0xff, nblocks * sizeof(hid_t));
    ismodified = (bool*)calloc(nblocks, sizeof(bool));
    walksum = 0;
    mkdir((base_filename + "_GraphWalker/walks/").c_str(), 0777);
  }

  ~WalkManager() {
    for (tid_t t = 0; t < nthreads; t++) delete[] pwalks[t];
    delete[] pwalks;
    free(walknum);
    free(dwalknum);
    free(minstep);
    free(ismodified);
  }

  tid_t num_threads() const { return nthreads; }
  bid_t num_blocks() const { return nblocks; }

  // (source & 0xffffff) << 40 | (current & 0x3ffffff) << 14 | (hop & 0x3fff)
  WalkDataType encode(vid_t sourceId, vid_t currentId, hid_t hop) {
    assert(hop < 16384);
    return (((WalkDataType)sourceId & 0xffffff) << 40) | (((WalkDataType)currentId & 0x3ffffff) << 14) |
           ((WalkDataType)hop & 0x3fff);
  }
  vid_t getSourceId(WalkDataType walk) { return (vid_t)(walk >> 40) & 0xffffff; }
  vid_t getCurrentId(WalkDataType walk) { return (vid_t)(walk >> 14) & 0x3ffffff; }
  hid_t getHop(WalkDataType walk) { return (hid_t)(walk & 0x3fff); }
  WalkDataType reencode(WalkDataType walk, vid_t toVertex) {
    return encode(getSourceId(walk), toVertex, getHop(walk));
  }

  // Appends a walk to the buffer of (thread t, block p), with its current
  // vertex made relative to block p.
  void moveWalk(WalkDataType walk, bid_t p, tid_t t, vid_t toVertex) {
    assert(t < nthreads && p < nblocks);
    pwalks[t][p].push_back(reencode(walk, toVertex));
  }

  // Pool of block p in the reference's getCurrentWalks order (buffers of
  // thread 0, 1, ...); the buffers are emptied.
  std::vector<WalkDataType> takeWalks(bid_t p) {
    std::vector<WalkDataType> out;
    for (tid_t t = 0; t < nthreads; t++) {
      WalkBuffer& b = pwalks[t][p];
      out.insert(out.end(), b.walks, b.walks + b.size_w);
      b.clear();
    }
    return out;
  }

  wid_t getCurrentWalks(bid_t p) {
    std::vector<WalkDataType> w = takeWalks(p);
    curwalks = (WalkDataType*)malloc((w.size() ? w.size() : 1) * sizeof(WalkDataType));
    if (!w.empty()) memcpy(curwalks, w.data(), w.size() * sizeof(WalkDataType));
    curp = p;
    dwalknum[p] = 0;
    return w.size();
  }

  void setMinStep(bid_t p, hid_t hop) {
    if (minstep[p] > hop) minstep[p] = hop;
  }

  void updateWalkNum(bid_t p) {
    wid_t forward = 0;
    for (bid_t b = 0; b < nblocks; b++) {
      if (!ismodified[b] || b == p) continue;
      ismodified[b] = false;
      wid_t n = dwalknum[b];
      for (tid_t t = 0; t < nthreads; t++) n += pwalks[t][b].size_w;
      forward += n - walknum[b];
      walknum[b] = n;
    }
    walksum += forward;
    walksum -= walknum[p];
    walknum[p] = 0;
    minstep[p] = 0xffff;
    free(curwalks);
    curwalks = nullptr;
  }

  bid_t blockWithMaxWalks() {
    wid_t maxw = 0;
    bid_t maxp = 0;
    for (bid_t p = 0; p < nblocks; p++)
      if (maxw < walknum[p]) {
        maxw = walknum[p];
        maxp = p;
      }
    return maxp;
  }
  bid_t blockWithMinStep() {
    hid_t mins = 0xffff;
    bid_t minp = 0;
    for (bid_t p = 0; p < nblocks; p++)
      if (mins > minstep[p]) {
        mins = minstep[p];
        minp = p;
      }
    return walknum[minp] > 0 ? minp : blockWithMaxWalks();
  }
  bid_t blockWithMaxWeight() {
    float maxwt = 0;
    bid_t maxp = 0;
    for (bid_t p = 0; p < nblocks; p++)
      if (minstep[p] && maxwt < (float)walknum[p] / minstep[p]) {
        maxwt = (float)walknum[p] / minstep[p];
        maxp = p;
      }
    return maxp;
  }
  bid_t blockWithRandom() { return rand() % nblocks; }
  bid_t chooseBlock(float prob) {
    const float cc = ((float)rand()) / RAND_MAX;
    return cc < prob ? blockWithMinStep() : blockWithMaxWalks();
  }
};

#endif
