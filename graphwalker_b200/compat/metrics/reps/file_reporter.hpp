// Drop-in GraphWalker API: file metrics reporter.
// Writes <file> with `<ident>.<key>=<value>` lines and appends one row to
// <file>.statistics with the reference's columns (reps/file_reporter.hpp:66-92):
// 00_runtime, 1_chooseBlock, 2_findSubGraph, 3_getCurrentWalks,
// [4_writeWalks2Disk], 5_exec_updates, 6_updateWalkNum value and count,
// g_loadSubGraph count, nblocks -- so scripts that parse old rows still work.
#ifndef DEF_GRAPHCHI_FILE_REPORTER
#define DEF_GRAPHCHI_FILE_REPORTER

#include <cstdio>
#include <fstream>

#include "metrics/metrics.hpp"

class file_reporter : public imetrics_reporter {
  std::string filename;

 public:
  explicit file_reporter(std::string fname) : filename(fname) {}

  void do_report(std::string name, std::string ident, std::map<std::string, metrics_entry>& entries) {
    FILE* f = fopen(filename.c_str(), "w");
    if (!f) return;
    if (ident != name) fprintf(f, "[%s:%s]\n", name.c_str(), ident.c_str());
    else fprintf(f, "[%s]\n", name.c_str());
    std::ofstream stats((filename + ".statistics").c_str(), std::ofstream::out | std::ofstream::app);
    for (auto& kv : entries) {
      const std::string& k = kv.first;
      const metrics_entry& e = kv.second;
      if (k == "00_runtime" || k == "1_chooseBlock" || k == "2_findSubGraph" || k == "3_getCurrentWalks" ||
          k == "4_writeWalks2Disk" || k == "5_exec_updates")
        stats << e.value << "  \t  ";
      else if (k == "6_updateWalkNum")
        stats << e.value << "  \t  " << e.count << "  \t  ";
      else if (k == "g_loadSubGraph")
        stats << e.count << "  \t  ";
      else if (k == "nblocks")
        stats << e.value << std::endl;
      switch (e.valtype) {
        case INTEGER:
          fprintf(f, "%s.%s=%ld\n", ident.c_str(), k.c_str(), (long)e.value);
          fprintf(f, "%s.%s.count=%zu\n", ident.c_str(), k.c_str(), e.count);
          break;
        case REAL:
        case TIME:
          fprintf(f, "%s.%s=%lf\n", ident.c_str(), k.c_str(), e.value);
          fprintf(f, "%s.%s.count=%zu\n", ident.c_str(), k.c_str(), e.count);
          fprintf(f, "%s.%s.min=%lf\n", ident.c_str(), k.c_str(), e.count ? e.minvalue : 0.0);
          fprintf(f, "%s.%s.max=%lf\n", ident.c_str(), k.c_str(), e.count ? e.maxvalue : 0.0);
          fprintf(f, "%s.%s.avg=%lf\n", ident.c_str(), k.c_str(), e.count ? e.cumvalue / e.count : 0.0);
          break;
        case STRING: fprintf(f, "%s.%s=%s\n", ident.c_str(), k.c_str(), e.stringval.c_str()); break;
        case VECTOR: break;
      }
    }
    fclose(f);
  }
};

#endif
