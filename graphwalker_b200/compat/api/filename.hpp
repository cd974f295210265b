// Drop-in GraphWalker API: on-disk names under <base>_GraphWalker/
// (the reference's src/api/filename.hpp:16-76).
#ifndef GW_COMPAT_FILENAME_HPP
#define GW_COMPAT_FILENAME_HPP

#include <cstdlib>
#include <sstream>
#include <string>

#include "api/datatype.hpp"

static inline std::string fidname(std::string base, bid_t p) {
  return base + "_GraphWalker/graphinfo/file_" + std::to_string(p);
}

static inline std::string walksname(std::string base, bid_t p) {
  return base + "_GraphWalker/walks/pool_" + std::to_string(p) + ".walks";
}

static inline std::string filerangename(std::string base, uint16_t filesize_GB) {
  return base + "_GraphWalker/filesize_" + std::to_string(filesize_GB) + "GB.filerange";
}

static inline std::string blockrangename(std::string base, unsigned long long blocksize_KB) {
  return base + "_GraphWalker/blocksize_" + std::to_string(blocksize_KB) + "KB.blockrange";
}

static inline std::string nverticesname(std::string base) { return base + "_GraphWalker/N.nvertices"; }

// Configuration file, $GRAPHCHI_ROOT aware.
static inline std::string configname() {
  const char* root = getenv("GRAPHCHI_ROOT");
  return root ? std::string(root) + "/conf/graphchi.cnf" : std::string("conf/graphwalker.cnf");
}

static inline std::string configlocalname() {
  const char* root = getenv("GRAPHCHI_ROOT");
  return root ? std::string(root) + "/conf/graphwalker.local.cnf" : std::string("conf/graphwalker.local.cnf");
}

#endif
