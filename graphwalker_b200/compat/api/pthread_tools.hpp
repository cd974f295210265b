// Drop-in GraphWalker API: the one pthread wrapper apps may use (mutex).
#ifndef GW_COMPAT_PTHREAD_TOOLS_HPP
#define GW_COMPAT_PTHREAD_TOOLS_HPP
#include <mutex>
namespace graphchi {
class mutex {
  std::mutex m_;
 public:
  void lock() { m_.lock(); }
  void unlock() { m_.unlock(); }
  bool try_lock() { return m_.try_lock(); }
};
}  // namespace graphchi
using graphchi::mutex;
#endif
