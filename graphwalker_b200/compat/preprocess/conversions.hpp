// Drop-in GraphWalker API: preprocessing of a text edge list into the
// preprocessed CSR layout, and block ranges (the reference's
// src/preprocess/conversions.hpp:42-404).
//
// convert_to_csr reads "<from> <to>" lines (separators tab, comma or space;
// '#' and '%' lines are comments), drops self-loops, keeps duplicate edges
// and keeps the file's order of a vertex's out-edges.  The reference requires
// the file to be sorted by source; here a stable sort by source is applied,
// which leaves a sorted file unchanged.  The parsing runs on the GPU
// (gw_convert_edgelist).  Block ranges follow compute_block
// (gw_compute_blocks in the C ABI).
#ifndef GRAPHWALKER_CONVERSIONS_DEF
#define GRAPHWALKER_CONVERSIONS_DEF

#include <dirent.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <sys/types.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "api/datatype.hpp"
#include "api/cmdopts.hpp"
#include "api/filename.hpp"
#include "api/io.hpp"
#include "graphwalker_b200.h"
#include "logger/logger.hpp"

static inline int rm_dir(std::string path) {
  DIR* d = opendir(path.c_str());
  if (!d) return -1;
  struct dirent* e;
  while ((e = readdir(d)) != nullptr) {
    if (!strcmp(e->d_name, ".") || !strcmp(e->d_name, "..")) continue;
    const std::string sub = path + "/" + e->d_name;
    struct stat st;
    if (lstat(sub.c_str(), &st) != 0) continue;
    if (S_ISDIR(st.st_mode)) rm_dir(sub);
    else unlink(sub.c_str());
  }
  closedir(d);
  return rmdir(path.c_str());
}

// Lines of a range file minus one; 0 when the file does not exist.
static inline bid_t gw_count_ranges(const std::string& f) {
  FILE* fp = fopen(f.c_str(), "r");
  if (!fp) return 0;
  bid_t lines = 0;
  int c;
  while ((c = fgetc(fp)) != EOF)
    if (c == '\n') ++lines;
  fclose(fp);
  return lines ? lines - 1 : 0;
}

static inline bid_t find_filerange(std::string base, uint16_t filesize_GB) {
  return gw_count_ranges(filerangename(base, filesize_GB));
}

static inline bid_t find_blockrange(std::string base, unsigned long long blocksize_kb) {
  return gw_count_ranges(blockrangename(base, blocksize_kb));
}

static inline bid_t convert_to_csr(std::string filename, uint16_t filesize_GB) {
  // The text is parsed and grouped on the GPU (gw_convert_edgelist), which
  // writes the same files as the reference's loop (one CSR file: a 1024 GB
  // file size never splits them).
  (void)filesize_GB;
  gw_convert_stats st;
  const gw_status s = gw_convert_edgelist(filename.c_str(), 0, get_option_int("gw_device", 0), &st);
  if (s != GW_OK) {
    logstream(LOG_FATAL) << "convert_to_csr(" << filename << "): " << gw_last_error(nullptr) << std::endl;
    return 0;
  }
  logstream(LOG_INFO) << "nverts = " << st.nvertices << ", nedges = " << st.edges << " (" << st.lines << " lines, "
                      << st.ms_total << " ms)" << std::endl;
  return 1;
}

static inline bid_t compute_block(std::string filename, unsigned long long blocksize_kb) {
  const std::string f = fidname(filename, 0) + ".beg_pos";
  FILE* in = fopen(f.c_str(), "rb");
  if (!in) {
    logstream(LOG_FATAL) << "Could not load :" << f << std::endl;
    return 0;
  }
  fseek(in, 0, SEEK_END);
  const uint64_t entries = (uint64_t)ftell(in) / 8;
  fseek(in, 0, SEEK_SET);
  std::vector<uint64_t> rowptr(entries);
  if (fread(rowptr.data(), 8, entries, in) != entries) logstream(LOG_FATAL) << "short read of " << f << std::endl;
  fclose(in);
  const uint32_t nv = (uint32_t)(entries - 1);
  std::vector<uint32_t> blocks((size_t)nv + 2);
  const uint32_t n = gw_compute_blocks(rowptr.data(), nv, blocksize_kb, blocks.data(), (uint32_t)blocks.size());
  std::ofstream o(blockrangename(filename, blocksize_kb).c_str());
  for (uint32_t i = 0; i < n; ++i) o << blocks[i] << std::endl;
  return n - 1;
}

static inline bid_t convert_if_notexists(std::string basefilename, unsigned long long blocksize_kb) {
  if (find_filerange(basefilename, FILE_SIZE) > 0) {
    logstream(LOG_INFO) << "Found preprocessed files for " << basefilename << std::endl;
  } else {
    logstream(LOG_INFO) << "Did not find preprocessed shards for " << basefilename << ", creating them" << std::endl;
    convert_to_csr(basefilename, FILE_SIZE);
  }
  assert(blocksize_kb > 0);
  bid_t nblocks = find_blockrange(basefilename, blocksize_kb);
  if (nblocks == 0) nblocks = compute_block(basefilename, blocksize_kb);
  logstream(LOG_INFO) << "blocksize = " << blocksize_kb << "KB, num blocks = " << nblocks << std::endl;
  return nblocks;
}

#endif
