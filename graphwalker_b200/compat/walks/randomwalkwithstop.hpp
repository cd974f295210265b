// Drop-in GraphWalker API: RandomWalkwithStop (the reference's
// src/walks/randomwalkwithstop.hpp:16-52).  Per hop: with probability 0.85
// move to a uniform out-neighbour, otherwise -- or at a dangling vertex --
// the walk ends; at most L hops.  The device engine runs it as GW_RULE_STOP.
#ifndef RANDOMWALKWITHSTOP
#define RANDOMWALKWITHSTOP

#include "walks/randomwalk.hpp"

class RandomWalkwithStop : public RandomWalk {
 public:
  int gw_rule() const { return GW_RULE_STOP; }
};

#endif
