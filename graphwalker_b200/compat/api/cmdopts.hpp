// Drop-in GraphWalker API: command-line and configuration-file knobs.
//
// Semantics of the reference (src/api/cmdopts.hpp:87-218,
// src/api/configfile.hpp:81-117): set_argc loads conf/graphwalker.local.cnf,
// else conf/graphwalker.cnf ($GRAPHCHI_ROOT aware; a missing file is fatal),
// then overlays every --key=value argument; get_option_* returns the value
// following the last `key value` pair on the command line, else the
// configuration value, else the default.
//
// Engine knobs of this implementation go through the same mechanism:
//   seed            Philox key of the walk draws            (default 42)
//   gw_walk_id      "index": walk id = pool position (default);
//                   "source": walk id = source field (the keying of the
//                   reference's shimmed test build)
//   gw_sink         "replay": record each walk's visits on the device and
//                   call the program's updateInfo for every visit (default);
//                   "count": count visits per vertex on the device and hand
//                   the counts to RandomWalk::gw_deliver_counts
//   gw_mode         "resident" (default) | "blocked"
//   gw_residency    "hbm" (default) | "stream"
//   gw_mapped_walks streamed blocks with at most this many pending walks are
//                   read in place from pinned host memory, not copied:
//                   "auto" (default, per block one walk per 128 bytes of its
//                   CSR) | a number | 0 (copy every block)
//                   (gw_set_mapped_block_walks)
//   gw_pool_budget_mb device MB the blocked engine's walk pools may hold; past
//                   it pools move to pinned host memory and come back when
//                   their block runs (default 0: no limit; gw_set_pool_budget)
//   gw_chunk        walks per device run in replay mode (default 4194304)
//   gw_device       CUDA device ordinal (default 0)
//   gw_edge_records "auto" (default): 16-byte edge records when they fit in
//                   half of the free device memory | "on" | "off"
//                   (gw_set_edge_records)
//   gw_rng          "philox" (default): the deterministic mode, the draws of
//                   hop h from Philox(seed; walk id, h) in the reference's
//                   order | "native": one Philox block per two hops
//                   (gw_walk_params.rng = GW_RNG_NATIVE)
#ifndef GRAPHWALKER_CMDOPTS_DEF
#define GRAPHWALKER_CMDOPTS_DEF

#include <stdint.h>

#include <cassert>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <string>

#include "api/configfile.hpp"
#include "api/filename.hpp"

#ifdef __GNUC__
#define VARIABLE_IS_NOT_USED __attribute__((unused))
#else
#define VARIABLE_IS_NOT_USED
#endif

namespace gw_compat {
struct cmdline {
  int argc = 0;
  char** argv = nullptr;
  bool configured = false;
  std::map<std::string, std::string> conf;
  static cmdline& get() {
    static cmdline c;
    return c;
  }
  const char* find(const char* name) const {
    for (int i = argc - 2; i >= 0; --i)
      if (strcmp(argv[i], name) == 0) return argv[i + 1];
    return nullptr;
  }
};
}  // namespace gw_compat

static void VARIABLE_IS_NOT_USED set_conf(std::string key, std::string value) {
  gw_compat::cmdline::get().conf[key] = value;
}

static void VARIABLE_IS_NOT_USED set_argc(int argc, const char** argv) {
  gw_compat::cmdline& c = gw_compat::cmdline::get();
  c.argc = argc;
  c.argv = (char**)argv;
  c.configured = true;
  c.conf = loadconfig(configlocalname(), configname());
  for (int i = 1; i < argc; ++i) {
    std::string arg = argv[i];
    if (arg.rfind("--", 0) != 0) continue;
    arg = arg.substr(2);
    const size_t eq = arg.find('=');
    if (eq == std::string::npos) continue;
    std::cout << "[" << arg.substr(0, eq) << "] => [" << arg.substr(eq + 1) << "]" << std::endl;
    c.conf[arg.substr(0, eq)] = arg.substr(eq + 1);
  }
}

static inline void gw_check_cmd_init() {
  if (!gw_compat::cmdline::get().configured) {
    std::cout << "ERROR: command line options not initialized." << std::endl;
    std::cout << "       You need to call set_argc() in the beginning of the program." << std::endl;
  }
}

static std::string VARIABLE_IS_NOT_USED get_option_string(const char* name, std::string dflt) {
  gw_check_cmd_init();
  gw_compat::cmdline& c = gw_compat::cmdline::get();
  if (const char* v = c.find(name)) return v;
  auto it = c.conf.find(name);
  return it != c.conf.end() ? it->second : dflt;
}

static std::string VARIABLE_IS_NOT_USED get_option_string(const char* name) {
  gw_check_cmd_init();
  gw_compat::cmdline& c = gw_compat::cmdline::get();
  if (const char* v = c.find(name)) return v;
  auto it = c.conf.find(name);
  if (it == c.conf.end()) {
    std::cout << "ERROR: could not find option " << name << " from config.";
    assert(false);
    return "ERROR";
  }
  return it->second;
}

static int VARIABLE_IS_NOT_USED get_option_int(const char* name, int dflt) {
  gw_check_cmd_init();
  gw_compat::cmdline& c = gw_compat::cmdline::get();
  if (const char* v = c.find(name)) return atoi(v);
  auto it = c.conf.find(name);
  return it != c.conf.end() ? atoi(it->second.c_str()) : dflt;
}

static int VARIABLE_IS_NOT_USED get_option_int(const char* name) {
  return atoi(get_option_string(name).c_str());
}

static uint64_t VARIABLE_IS_NOT_USED get_option_long(const char* name, uint64_t dflt) {
  gw_check_cmd_init();
  gw_compat::cmdline& c = gw_compat::cmdline::get();
  if (const char* v = c.find(name)) return atol(v);
  auto it = c.conf.find(name);
  return it != c.conf.end() ? (uint64_t)atol(it->second.c_str()) : dflt;
}

static float VARIABLE_IS_NOT_USED get_option_float(const char* name, float dflt) {
  gw_check_cmd_init();
  gw_compat::cmdline& c = gw_compat::cmdline::get();
  if (const char* v = c.find(name)) return (float)atof(v);
  auto it = c.conf.find(name);
  return it != c.conf.end() ? (float)atof(it->second.c_str()) : dflt;
}

#endif
