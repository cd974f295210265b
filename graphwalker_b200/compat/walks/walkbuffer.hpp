// Drop-in GraphWalker API: a per-(thread, block) buffer of 64-bit walks.
// Same public members as the reference's WalkBuffer (src/walks/walkbuffer.hpp:8-40).
// It grows instead of spilling to pool_<b>.walks files: the walks go to the
// device when the engine runs, so there is no host pool to bound.
#ifndef DEF_WALK_BUFFER
#define DEF_WALK_BUFFER

#include <vector>

#include "api/datatype.hpp"

class WalkBuffer {
 public:
  bool malloced = false;
  wid_t size_w = 0;
  WalkDataType* walks = nullptr;

  WalkDataType& operator[](int i) { return walks[i]; }

  void push_back(WalkDataType w) {
    if (size_w == store_.size()) store_.resize(store_.empty() ? WALK_BUFFER_SIZE : store_.size() * 2);
    store_[size_w++] = w;
    walks = store_.data();
    malloced = true;
  }
  void clear() { size_w = 0; }

 private:
  std::vector<WalkDataType> store_;
};

#endif
