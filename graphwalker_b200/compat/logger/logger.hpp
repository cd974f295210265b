// Drop-in GraphWalker API: the stream logger.
// logstream(LEVEL) << ...; as in the reference's src/logger/logger.hpp:71-217
// (levels, a compile-time OUTPUTLEVEL filter, LOG_FATAL throws).
#ifndef GW_COMPAT_LOGGER_HPP
#define GW_COMPAT_LOGGER_HPP

#include <iostream>
#include <mutex>
#include <sstream>
#include <string>

#define LOG_NONE 5
#define LOG_FATAL 4
#define LOG_ERROR 3
#define LOG_WARNING 2
#define LOG_INFO 1
#define LOG_DEBUG 0

#ifndef OUTPUTLEVEL
#define OUTPUTLEVEL LOG_INFO
#endif

namespace gw_compat {

// Collects one log line and writes it (under a lock) when the statement ends.
class log_line {
 public:
  log_line(int level, const char* file, const char* fn, int line) : level_(level) {
    if (level_ >= OUTPUTLEVEL) {
      static const char* names[] = {"DEBUG", "INFO", "WARNING", "ERROR", "FATAL"};
      const char* base = file;
      for (const char* p = file; *p; ++p)
        if (*p == '/') base = p + 1;
      ss_ << names[level_ < 5 ? level_ : 4] << ":\t" << base << "(" << fn << ":" << line << "): ";
    }
  }
  log_line(const log_line&) = delete;
  ~log_line() noexcept(false) {
    if (level_ >= OUTPUTLEVEL) {
      static std::mutex mu;
      std::lock_guard<std::mutex> g(mu);
      std::cerr << ss_.str() << std::flush;
    }
    if (level_ == LOG_FATAL) throw std::string("log fatal");
  }
  template <typename T>
  log_line& operator<<(const T& x) {
    if (level_ >= OUTPUTLEVEL) ss_ << x;
    return *this;
  }
  log_line& operator<<(std::ostream& (*manip)(std::ostream&)) {
    if (level_ >= OUTPUTLEVEL) ss_ << manip;
    return *this;
  }

 private:
  int level_;
  std::ostringstream ss_;
};

}  // namespace gw_compat

#define logstream(lvl) gw_compat::log_line(lvl, __FILE__, __func__, __LINE__)

#endif
