// Drop-in GraphWalker API: graphwalker_engine on the B200 engine.
//
// Same constructor and run() as the reference (src/engine/graphwalker.hpp:74,
// 272-311).  run() lets the program place its walks (startWalks), hands the
// pools to the device engine (gw_walks_add), runs the program's walk class
// there (gw_run) and gives the program its visits:
//   gw_sink replay (default): each walk's visited vertices are recorded on the
//     device and the program's updateInfo(source, vertex, thread, hop) is
//     called for every visit, walk by walk, on `execthreads` OpenMP threads;
//   gw_sink count: visits are counted per vertex on the device and handed to
//     RandomWalk::gw_deliver_counts.
// Timers keep the reference's names (0_startWalks, 00_runtime,
// 2_findSubGraph = graph upload, 3_getCurrentWalks = pool hand-over,
// 5_exec_updates = device time, 7_replay = updateInfo calls).
#ifndef DEF_GRAPHCHWALKER_ENGINE
#define DEF_GRAPHCHWALKER_ENGINE

#include <omp.h>
#include <sys/time.h>

#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "api/cmdopts.hpp"
#include "api/filename.hpp"
#include "graphwalker_b200.h"
#include "logger/logger.hpp"
#include "metrics/metrics.hpp"
#include "walks/randomwalk.hpp"

class graphwalker_engine {
 public:
  std::string base_filename;
  unsigned long long blocksize_kb;
  bid_t nblocks;
  vid_t nvertices;
  tid_t exec_threads;
  vid_t* blocks = nullptr;
  timeval start;
  bid_t nmblocks;
  bid_t exec_block = 0;
  metrics& m;
  WalkManager* walk_manager = nullptr;
  gw_ctx* ctx = nullptr;

  graphwalker_engine(std::string _base_filename, unsigned long long _blocksize_kb, bid_t _nblocks, bid_t _nmblocks,
                     metrics& _m)
      : base_filename(_base_filename), blocksize_kb(_blocksize_kb), nblocks(_nblocks), nmblocks(_nmblocks), m(_m) {
    exec_threads = (tid_t)get_option_int("execthreads", omp_get_max_threads());
    omp_set_num_threads(exec_threads);
    const std::string residency = get_option_string("gw_residency", "hbm");
    gw_graph_desc d;
    d.base_filename = base_filename.c_str();
    d.blocksize_kb = blocksize_kb;
    d.nmblocks = nmblocks;
    d.residency = residency == "stream" ? GW_STREAM_PINNED : GW_RESIDENT_HBM;
    d.device = get_option_int("gw_device", 0);
    m.start_time("2_findSubGraph");
    if (gw_open(&d, &ctx) != GW_OK)
      logstream(LOG_FATAL) << "graphwalker_engine: " << gw_last_error(nullptr) << std::endl;
    m.stop_time("2_findSubGraph");
    const uint64_t pool_mb = get_option_long("gw_pool_budget_mb", 0);
    if (gw_set_pool_budget(ctx, pool_mb << 20) != GW_OK)
      logstream(LOG_FATAL) << "graphwalker_engine: " << gw_last_error(ctx) << std::endl;
    const std::string mapped = get_option_string("gw_mapped_walks", "auto");
    if (gw_set_mapped_block_walks(ctx, mapped == "auto" ? GW_MAPPED_AUTO : strtoull(mapped.c_str(), nullptr, 10)) !=
        GW_OK)
      logstream(LOG_FATAL) << "graphwalker_engine: " << gw_last_error(ctx) << std::endl;
    const std::string erec = get_option_string("gw_edge_records", "auto");
    uint32_t erec_built = 0;
    if (gw_set_edge_records(ctx, erec == "on" ? GW_EDGE_RECORDS_ON : erec == "off" ? GW_EDGE_RECORDS_OFF
                                                                                     : GW_EDGE_RECORDS_AUTO,
                            &erec_built) != GW_OK)
      logstream(LOG_FATAL) << "graphwalker_engine: " << gw_last_error(ctx) << std::endl;
    m.set("gpu_edge_records", std::string(erec_built ? "on" : "off"));
    uint32_t nv = 0, nb = 0;
    uint64_t ne = 0;
    gw_graph_info(ctx, &nv, &ne, &nb);
    if (nb != nblocks)
      logstream(LOG_WARNING) << "block range has " << nb << " blocks, caller said " << nblocks << std::endl;
    nblocks = nb;
    blocks = (vid_t*)malloc((nblocks + 1) * sizeof(vid_t));
    gw_get_blocks(ctx, blocks, nblocks + 1);
    nvertices = blocks[nblocks];
    walk_manager = new WalkManager(m, nblocks, exec_threads, base_filename);
    m.set("file", base_filename);
    m.set("engine", std::string("graphwalker_b200"));
    m.set("nblocks", (size_t)nblocks);
    logstream(LOG_INFO) << "engine: " << gw_version() << ", " << nvertices << " vertices, " << ne << " edges, "
                        << nblocks << " blocks, " << (int)exec_threads << " host threads" << std::endl;
  }

  virtual ~graphwalker_engine() {
    delete walk_manager;
    free(blocks);
    gw_close(ctx);
  }

  virtual size_t num_vertices() { return blocks[nblocks]; }

  double runtime() {
    timeval end;
    gettimeofday(&end, nullptr);
    return end.tv_sec - start.tv_sec + ((double)(end.tv_usec - start.tv_usec)) / 1.0E6;
  }

  void run(RandomWalk& userprogram, float prob) {
    m.start_time("0_startWalks");
    userprogram.startWalks(*walk_manager, nblocks, blocks, base_filename);
    m.stop_time("0_startWalks");
    gettimeofday(&start, nullptr);
    m.start_time("00_runtime");
    const int rule = userprogram.gw_rule();
    if (rule < 0)
      logstream(LOG_FATAL) << "the program does not derive from RandomWalkwithJump/Stop/Prob/RestartwithJoint"
                           << std::endl;
    gw_walk_params p;
    memset(&p, 0, sizeof p);
    p.rule = (uint32_t)rule;
    p.L = userprogram.gw_length();
    p.njump = userprogram.gw_njump();
    p.jump_prob = 0.15;
    p.seed = get_option_long("seed", 42);
    p.prob = prob;
    p.mode = get_option_string("gw_mode", "resident") == "blocked" ? GW_MODE_BLOCKED : GW_MODE_RESIDENT;
    // gw_rng philox (default): the deterministic mode, bit-exact to the
    // reference engine with its rand_r routed to the same Philox stream;
    // gw_rng native: one Philox block per two hops (checked statistically)
    const std::string rng = get_option_string("gw_rng", "philox");
    if (rng != "philox" && rng != "native")
      logstream(LOG_FATAL) << "gw_rng must be philox or native, not " << rng << std::endl;
    p.rng = rng == "native" ? GW_RNG_NATIVE : GW_RNG_PHILOX;
    const bool by_source = get_option_string("gw_walk_id", "index") == "source";
    const bool count_sink = get_option_string("gw_sink", "replay") == "count";

    m.start_time("3_getCurrentWalks");
    std::vector<std::vector<WalkDataType>> pools(nblocks);
    wid_t total = 0;
    for (bid_t b = 0; b < nblocks; ++b) {
      pools[b] = walk_manager->takeWalks(b);
      total += pools[b].size();
    }
    m.stop_time("3_getCurrentWalks");
    std::vector<uint32_t> ids;
    if (!by_source) {  // distinct walk ids: the position in pool order
      ids.resize(total);
      for (wid_t i = 0; i < total; ++i) ids[i] = (uint32_t)i;
    }

    if (count_sink) {
      check(gw_walks_clear(ctx));
      wid_t off = 0;
      for (bid_t b = 0; b < nblocks; ++b) {
        check(gw_walks_add(ctx, b, pools[b].data(), by_source ? nullptr : ids.data() + off, pools[b].size()));
        off += pools[b].size();
      }
      p.sink = GW_SINK_VERTEX_COUNT;
      check(gw_run(ctx, &p));
      add_device_time();
      std::vector<uint32_t> counts(nvertices);
      check(gw_read_counts(ctx, counts.data(), counts.size()));
      m.start_time("7_replay");
      userprogram.gw_deliver_counts(counts.data(), nvertices);
      m.stop_time("7_replay");
    } else {
      replay(userprogram, p, pools, ids, total);
    }
    for (bid_t b = 0; b < nblocks; ++b) {
      walk_manager->walknum[b] = 0;
      walk_manager->minstep[b] = 0xffff;
    }
    walk_manager->walksum = 0;
    m.stop_time("00_runtime");
  }

 private:
  void check(gw_status s) {
    if (s != GW_OK) logstream(LOG_FATAL) << "graphwalker_engine: " << gw_last_error(ctx) << std::endl;
  }

  void add_device_time() {
    gw_run_stats st;
    gw_read_stats(ctx, &st);
    m.add_time("5_exec_updates", st.ms_total * 1e-3);
    if (st.block_loads) m.add("g_loadSubGraph", (double)st.block_loads, INTEGER);
    // the device's own counters, in the same metrics map (graphwalker_metrics.txt)
    m.add("gpu_walks", (double)st.walks, INTEGER);
    m.add("gpu_supersteps", (double)st.supersteps, INTEGER);
    m.add("gpu_block_loads", (double)st.block_loads, INTEGER);
    m.add("gpu_bytes_h2d", (double)st.bytes_h2d, INTEGER);
    m.add("gpu_ms_walk", st.ms_walk);
    m.add("gpu_ms_partition", st.ms_partition);
    m.add("gpu_ms_copy_wait", st.ms_copy_wait);
    m.add("gpu_blocks_read_in_place", (double)st.mapped_supersteps, INTEGER);
    m.add("gpu_pools_spilled", (double)st.pools_spilled, INTEGER);
    m.add("gpu_pools_refilled", (double)st.pools_refilled, INTEGER);
  }

  // Runs the walks in chunks that record paths on the device, then calls
  // updateInfo for every recorded visit.
  void replay(RandomWalk& prog, gw_walk_params p, const std::vector<std::vector<WalkDataType>>& pools,
              const std::vector<uint32_t>& ids, wid_t total) {
    const uint32_t stride = prog.gw_max_visits();
    uint64_t chunk = get_option_long("gw_chunk", 1ull << 22);
    const uint64_t cap = (1ull << 30) / stride;  // at most 4 GB of paths per chunk
    if (chunk > cap) chunk = cap ? cap : 1;
    p.sink = GW_SINK_PATH_RECORD;
    p.path_stride = stride;
    p.mode = GW_MODE_RESIDENT;
    std::vector<uint32_t> paths, lens;
    std::vector<const WalkDataType*> words;
    bid_t b = 0;
    size_t in_b = 0;
    wid_t done = 0;
    while (done < total) {
      check(gw_walks_clear(ctx));
      words.clear();
      uint64_t n = 0;
      while (n < chunk && b < nblocks) {
        const size_t avail = pools[b].size() - in_b;
        const size_t take = (size_t)std::min<uint64_t>(avail, chunk - n);
        if (take) {
          check(gw_walks_add(ctx, b, pools[b].data() + in_b, ids.empty() ? nullptr : ids.data() + done + n, take));
          for (size_t i = 0; i < take; ++i) words.push_back(pools[b].data() + in_b + i);
        }
        n += take;
        in_b += take;
        if (in_b == pools[b].size()) {
          ++b;
          in_b = 0;
        }
      }
      check(gw_run(ctx, &p));
      add_device_time();
      paths.resize(n * stride);
      lens.resize(n);
      check(gw_read_paths(ctx, paths.data(), lens.data(), n));
      m.start_time("7_replay");
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < (int64_t)n; ++i) {
        const WalkDataType w = *words[i];
        const vid_t s = (vid_t)(w >> 40) & 0xffffff;
        const hid_t h0 = (hid_t)(w & 0x3fff);
        const tid_t t = (tid_t)omp_get_thread_num();
        for (uint32_t k = 0; k < lens[i]; ++k) prog.updateInfo(s, paths[i * stride + k], t, (hid_t)(h0 + k));
      }
      m.stop_time("7_replay");
      done += n;
    }
  }
};

#endif
