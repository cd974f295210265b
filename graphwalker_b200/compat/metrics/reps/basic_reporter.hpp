// Drop-in GraphWalker API: console metrics reporter.
#ifndef DEF_GRAPHCHI_BASIC_REPORTER
#define DEF_GRAPHCHI_BASIC_REPORTER

#include <cstdio>

#include "metrics/metrics.hpp"

class basic_reporter : public imetrics_reporter {
 public:
  void do_report(std::string name, std::string ident, std::map<std::string, metrics_entry>& entries) {
    printf("\n=== REPORT FOR %s(%s) ===\n", name.c_str(), ident.c_str());
    for (auto& kv : entries) {
      const metrics_entry& e = kv.second;
      switch (e.valtype) {
        case STRING: printf("%s:\t%s\n", kv.first.c_str(), e.stringval.c_str()); break;
        case VECTOR: break;
        case TIME:
          printf("%s:\t%.6f s (count %zu, min %.6f, max %.6f)\n", kv.first.c_str(), e.value, e.count,
                 e.count ? e.minvalue : 0.0, e.count ? e.maxvalue : 0.0);
          break;
        default: printf("%s:\t%.6g\n", kv.first.c_str(), e.value);
      }
    }
  }
};

#endif
