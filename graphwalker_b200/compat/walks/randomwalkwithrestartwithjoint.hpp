// Drop-in GraphWalker API: RandomWalkwithRestartwithJoint (the reference's
// src/walks/randomwalkwithrestartwithjoint.hpp:16-61).  Per hop: with
// probability 0.85 move to a uniform out-neighbour, otherwise -- or at a
// dangling vertex -- go back to the walk's source; a walk ends when its hop
// count reaches L-1 modulo L (SimRank places replica i at hop i*L).  The class
// keeps its own R and L, shadowing RandomWalk's, as the reference's does.
// The device engine runs it as GW_RULE_RESTART.
#ifndef RANDOMWALKWITHRESTARTWITHJOINT
#define RANDOMWALKWITHRESTARTWITHJOINT

#include "walks/randomwalk.hpp"

class RandomWalkwithRestartwithJoint : public RandomWalk {
 public:
  wid_t R = 0;
  hid_t L = 0;

  void initializeRW(wid_t _R, hid_t _L) {
    R = _R;
    L = _L;
  }
  int gw_rule() const { return GW_RULE_RESTART; }
  hid_t gw_length() const { return L; }
};

#endif
