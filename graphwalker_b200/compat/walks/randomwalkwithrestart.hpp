// Drop-in GraphWalker API: RandomWalkwithRestart, the walk class of the
// reference's personalizedpagerank and reachability apps
// (src/walks/randomwalkwithrestart.hpp:16-62).  The reference's copy is
// written against its earlier interval API and no longer builds with its own
// engine; this one keeps its members and initializeRW signature on the live
// API.
//
// The walk (randomwalkwithrestart.hpp:40-51): per hop, with probability 0.85
// move to a uniform out-neighbour, otherwise -- or at a dangling vertex -- go
// back to the walk's source; a walk makes nsteps visits (hops 0 .. nsteps-1).
// The draws are consumed as in every live class (test, then neighbour).  The
// device engine runs it as GW_RULE_RESTART with segment length nsteps + 1: a
// walk that starts at hop 0 ends when its hop count reaches nsteps, after
// exactly these visits.  Walks must start at hop 0.
//
// `tail` (the share of walks whose end the reference's interval engine did
// not wait for) has no counterpart in an engine that runs every walk to its
// end: only tail = 0, the apps' default, is accepted.
#ifndef RANDOMWALKWITHRESTART
#define RANDOMWALKWITHRESTART

#include "logger/logger.hpp"
#include "walks/randomwalk.hpp"

class RandomWalkwithRestart : public RandomWalk {
 public:
  vid_t source = 0;
  wid_t nwalks = 0;
  hid_t nsteps = 0;
  float tail = 0.f;
  wid_t tailwalknum = 0;

  void initializeRW(vid_t _source, wid_t _nwalks, hid_t _nsteps, float _tail) {
    source = _source;
    nwalks = _nwalks;
    nsteps = _nsteps;
    tail = _tail;
    tailwalknum = (wid_t)(nwalks * tail);
    if (tail != 0.f) logstream(LOG_FATAL) << "RandomWalkwithRestart: only tail = 0 is supported" << std::endl;
    if (nsteps == 0 || nsteps == 0xffff)
      logstream(LOG_FATAL) << "RandomWalkwithRestart: nsteps must lie in [1, 65534]" << std::endl;
    R = nwalks;
    L = nsteps;
  }
  int gw_rule() const { return GW_RULE_RESTART; }
  hid_t gw_length() const { return (hid_t)(nsteps + 1); }
  uint32_t gw_max_visits() const { return nsteps; }
};

#endif
