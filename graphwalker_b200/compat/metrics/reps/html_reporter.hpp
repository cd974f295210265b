// Drop-in GraphWalker API: HTML metrics reporter (a plain table).
#ifndef DEF_GRAPHCHI_HTML_REPORTER
#define DEF_GRAPHCHI_HTML_REPORTER

#include <cstdio>

#include "metrics/metrics.hpp"

class html_reporter : public imetrics_reporter {
  std::string filename;

 public:
  explicit html_reporter(std::string fname) : filename(fname) {}
  void do_report(std::string name, std::string ident, std::map<std::string, metrics_entry>& entries) {
    FILE* f = fopen(filename.c_str(), "w");
    if (!f) return;
    fprintf(f, "<html><body><h1>%s %s</h1><table>\n", name.c_str(), ident.c_str());
    for (auto& kv : entries) {
      if (kv.second.valtype == STRING)
        fprintf(f, "<tr><td>%s</td><td>%s</td></tr>\n", kv.first.c_str(), kv.second.stringval.c_str());
      else if (kv.second.valtype != VECTOR)
        fprintf(f, "<tr><td>%s</td><td>%g</td></tr>\n", kv.first.c_str(), kv.second.value);
    }
    fprintf(f, "</table></body></html>\n");
    fclose(f);
  }
};

#endif
