// Drop-in GraphWalker API: DiscreteDistribution, msppr's per-source visit
// sketch (the reference's src/walks/discretedistribution.hpp:9-95).
// Same calls (add, filter, getTop).  Counts here are exact 32-bit counts per
// vertex and add() may be called from several threads at once; the
// reference keeps at most 1000 16-bit counters, which wrap at 65,535 and are
// thinned by filter(2) when full.  getTop orders by count, then by vertex id.
#ifndef DEF_DISCRETE_DISTRIBUTION
#define DEF_DISCRETE_DISTRIBUTION

#include <algorithm>
#include <mutex>
#include <unordered_map>
#include <utility>
#include <vector>

#include "api/datatype.hpp"

const unsigned capacity = 1000;

struct IdCount {
  vid_t id;
  uint32_t count;
  IdCount(vid_t _id, uint32_t _count) : id(_id), count(_count) {}
  bool operator<(const IdCount ic) const { return count > ic.count; }
};

class DiscreteDistribution {
 public:
  void add(vid_t id) {
    std::lock_guard<std::mutex> g(mu_);
    ++counts_[id];
  }
  void add(vid_t id, uint32_t n) {
    std::lock_guard<std::mutex> g(mu_);
    counts_[id] += n;
  }
  // Drops ids seen fewer than mincount times and lowers the others by
  // mincount - 1 (the reference's thinning step).
  void filter(uint16_t mincount) {
    std::lock_guard<std::mutex> g(mu_);
    for (auto it = counts_.begin(); it != counts_.end();) {
      if (it->second >= mincount) {
        it->second -= mincount - 1;
        ++it;
      } else {
        it = counts_.erase(it);
      }
    }
  }
  std::vector<IdCount> top(unsigned ntop) {
    std::lock_guard<std::mutex> g(mu_);
    std::vector<IdCount> v;
    v.reserve(counts_.size());
    for (auto& kv : counts_) v.emplace_back(kv.first, kv.second);
    auto order = [](const IdCount& a, const IdCount& b) {
      return a.count != b.count ? a.count > b.count : a.id < b.id;
    };
    const size_t k = std::min<size_t>(ntop, v.size());
    std::partial_sort(v.begin(), v.begin() + k, v.end(), order);
    v.erase(v.begin() + k, v.end());
    return v;
  }
  void getTop(unsigned ntop) {
    std::vector<IdCount> t = top(ntop);
    logstream(LOG_INFO) << "Top " << ntop << " visitfrequencies - " << std::endl;
    for (size_t i = 0; i < t.size(); ++i)
      logstream(LOG_INFO) << i << "-\t" << t[i].id << ":\t " << t[i].count << std::endl;
  }
  size_t distinct() {
    std::lock_guard<std::mutex> g(mu_);
    return counts_.size();
  }
  uint32_t count(vid_t id) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = counts_.find(id);
    return it == counts_.end() ? 0 : it->second;
  }

 private:
  std::mutex mu_;
  std::unordered_map<vid_t, uint32_t> counts_;
};

#endif
