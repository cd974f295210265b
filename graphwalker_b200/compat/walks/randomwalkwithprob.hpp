// Drop-in GraphWalker API: RandomWalkwithProb (the reference's
// src/walks/randomwalkwithprob.hpp:16-57): as RandomWalkwithStop without the
// L cap.  (The reference reuses RandomWalkwithStop's include guard here, so
// the two headers cannot be included together there; here they can.)
// The device engine runs it as GW_RULE_PROB; the host replay records up to
// gw_max_visits() visits per walk (512).
#ifndef RANDOMWALKWITHPROB
#define RANDOMWALKWITHPROB

#include "walks/randomwalk.hpp"

class RandomWalkwithProb : public RandomWalk {
 public:
  int gw_rule() const { return GW_RULE_PROB; }
  uint32_t gw_max_visits() const { return 512; }
};

#endif
