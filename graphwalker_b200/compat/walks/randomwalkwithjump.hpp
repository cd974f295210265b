// Drop-in GraphWalker API: RandomWalkwithJump (the reference's
// src/walks/randomwalkwithjump.hpp:16-62).  Per hop: with probability 0.85
// (draw test) move to a uniform out-neighbour, otherwise -- or at a dangling
// vertex -- jump to a uniform vertex in [0, N); walks run exactly L hops.
// The device engine runs this rule as GW_RULE_JUMP.
#ifndef RANDOMWALKWITHJUMP
#define RANDOMWALKWITHJUMP

#include "walks/randomwalk.hpp"

class RandomWalkwithJump : public RandomWalk {
 public:
  vid_t N = 0;

  void initializeRW(vid_t _N, wid_t _R, hid_t _L) {
    N = _N;
    R = _R;
    L = _L;
  }
  int gw_rule() const { return GW_RULE_JUMP; }
  vid_t gw_njump() const { return N; }
};

#endif
