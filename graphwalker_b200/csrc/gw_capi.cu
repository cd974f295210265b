// gw_capi.cu -- the C ABI (include/graphwalker_b200.h): graph loading, walk
// pools, resident-mode runs and the device-pointer entry points.
#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>

#include "gw_ctx.h"

namespace {

thread_local std::string t_last_error;

gw_status set_thread_error(gw_status code, const std::string& msg) {
  t_last_error = msg;
  return code;
}

std::string graph_file(const std::string& base, const char* suffix) {
  // fidname(base, 0) + suffix (src/api/filename.hpp:16-22)
  return base + "_GraphWalker/graphinfo/file_0" + suffix;
}

std::string blockrange_file(const std::string& base, uint64_t kb) {
  // blockrangename (src/api/filename.hpp:39-44)
  return base + "_GraphWalker/blocksize_" + std::to_string(kb) + "KB.blockrange";
}

// Reads a whole binary file into a pinned host buffer.
gw_status read_pinned(gw_ctx* ctx, const std::string& path, gw_hostbuf* out, size_t* bytes) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return ctx->fail(GW_E_IO, "cannot open %s: %s", path.c_str(), strerror(errno));
  struct stat st;
  if (fstat(fileno(f), &st) != 0) {
    fclose(f);
    return ctx->fail(GW_E_IO, "cannot stat %s", path.c_str());
  }
  const size_t n = (size_t)st.st_size;
  cudaError_t e = out->ensure(n);
  if (e != cudaSuccess) {
    fclose(f);
    return ctx->fail(GW_E_NOMEM, "pinned allocation of %zu bytes: %s", n, cudaGetErrorString(e));
  }
  size_t got = 0;
  while (got < n) {
    size_t r = fread(static_cast<char*>(out->p) + got, 1, n - got, f);
    if (r == 0) break;
    got += r;
  }
  if (n && gw::fault_now(GW_FAULT_FILE_READ)) got = n / 2;  // an injected short read
  fclose(f);
  if (got != n) return ctx->fail(GW_E_IO, "short read of %s (%zu of %zu bytes)", path.c_str(), got, n);
  *bytes = n;
  return GW_OK;
}

gw_status init_ctx(gw_ctx* ctx, int device) {
  ctx->device = device;
  GW_CUDA(ctx, cudaSetDevice(device), "cudaSetDevice");
  GW_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
  GW_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "stream");
  GW_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->aux_stream, cudaStreamNonBlocking), "stream");
  GW_CUDA(ctx, ctx->d_status.ensure(sizeof(uint32_t)), "status alloc");
  GW_CUDA(ctx, ctx->h_status.ensure(sizeof(uint32_t)), "status alloc");
  GW_CUDA(ctx, cudaMemsetAsync(ctx->d_status.p, 0, sizeof(uint32_t), ctx->stream), "memset");
  const char* env = getenv("GW_EDGE_RECORDS");
  ctx->erec_mode = env && strcmp(env, "0") == 0 ? GW_EDGE_RECORDS_OFF : GW_EDGE_RECORDS_AUTO;
  return GW_OK;
}

// Builds or drops the edge records of a graph as ctx->erec_mode and the
// residency say (see gw_set_edge_records).
gw_status apply_edge_records(gw_ctx* ctx) {
  if (ctx->residency != GW_RESIDENT_HBM || ctx->erec_mode == GW_EDGE_RECORDS_OFF) {
    ctx->d_erec.release();
    return GW_OK;
  }
  const size_t bytes = (size_t)ctx->ne * sizeof(ulonglong2);
  if (ctx->d_erec.p && ctx->d_erec.bytes >= bytes) return GW_OK;
  GW_CUDA(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (ctx->erec_mode == GW_EDGE_RECORDS_AUTO) {
    size_t free_b = 0, total_b = 0;
    GW_CUDA(ctx, cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    if (bytes > free_b / 2) return GW_OK;
  }
  if (ctx->d_erec.ensure(bytes) != cudaSuccess) {
    cudaGetLastError();  // an allocation failure is not sticky
    ctx->d_erec.release();
    if (ctx->erec_mode == GW_EDGE_RECORDS_ON)
      return ctx->fail(GW_E_NOMEM, "edge records: %zu bytes do not fit on the device", bytes);
    return GW_OK;
  }
  GW_CUDA(ctx, gw::launch_build_erec(ctx->d_colidx.as<uint32_t>(), ctx->d_vrec.as<unsigned long long>(), ctx->ne,
                                     ctx->nv, ctx->d_erec.as<ulonglong2>(), ctx->stream), "build_erec");
  GW_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "build_erec");
  return GW_OK;
}

// Uploads the CSR (host pointers, pinned or not) and builds the packed
// vertex records.  Streamed residency keeps the CSR in pinned host memory and
// only the row pointer (8 bytes per vertex) in HBM: blocks then stream their
// column slices alone, and a block read in place fetches only its columns
// over the host link.
gw_status install_graph(gw_ctx* ctx, const uint64_t* rowptr, const uint32_t* colidx,
                        uint32_t nv, const uint32_t* blocks, uint32_t nblocks) {
  ctx->nv = nv;
  ctx->ne = rowptr[nv];
  ctx->nblocks = nblocks;
  ctx->blocks.assign(blocks, blocks + nblocks + 1);
  if (nblocks == 0 || ctx->blocks[nblocks] != nv)
    return ctx->fail(GW_E_INVALID, "block range must end at nvertices (%u), ends at %u", nv,
                     nblocks ? ctx->blocks[nblocks] : 0);
  for (uint32_t b = 0; b < nblocks; ++b)
    if (ctx->blocks[b] > ctx->blocks[b + 1]) return ctx->fail(GW_E_INVALID, "block range not sorted");
  const size_t rp_bytes = ((size_t)nv + 1) * sizeof(uint64_t);
  const size_t ci_bytes = (size_t)ctx->ne * sizeof(uint32_t);
  GW_CUDA(ctx, ctx->d_blocks.ensure((nblocks + 1) * sizeof(uint32_t)), "blocks alloc");
  GW_CUDA(ctx, cudaMemcpyAsync(ctx->d_blocks.p, blocks, (nblocks + 1) * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, ctx->stream), "blocks copy");
  if (ctx->residency == GW_STREAM_PINNED) {
    if (ctx->h_rowptr.p != rowptr) {
      GW_CUDA(ctx, ctx->h_rowptr.ensure(rp_bytes), "pinned rowptr");
      memcpy(ctx->h_rowptr.p, rowptr, rp_bytes);
    }
    if (ctx->h_colidx.p != colidx) {
      GW_CUDA(ctx, ctx->h_colidx.ensure(ci_bytes), "pinned colidx");
      memcpy(ctx->h_colidx.p, colidx, ci_bytes);
    }
    GW_CUDA(ctx, ctx->d_rowptr.ensure(rp_bytes), "rowptr alloc");
    GW_CUDA(ctx, cudaMemcpyAsync(ctx->d_rowptr.p, ctx->h_rowptr.p, rp_bytes, cudaMemcpyHostToDevice,
                                 ctx->stream), "rowptr copy");
  } else {
    GW_CUDA(ctx, ctx->d_rowptr.ensure(rp_bytes), "rowptr alloc");
    GW_CUDA(ctx, ctx->d_colidx.ensure(ci_bytes), "colidx alloc");
    GW_CUDA(ctx, ctx->d_vrec.ensure(gw::vrec_bytes(nv)), "vrec alloc");
    GW_CUDA(ctx, cudaMemcpyAsync(ctx->d_rowptr.p, rowptr, rp_bytes, cudaMemcpyHostToDevice,
                                 ctx->stream), "rowptr copy");
    GW_CUDA(ctx, cudaMemcpyAsync(ctx->d_colidx.p, colidx, ci_bytes, cudaMemcpyHostToDevice,
                                 ctx->stream), "colidx copy");
    GW_CUDA(ctx, gw::launch_build_vrec(ctx->d_rowptr.as<unsigned long long>(), nv,
                                       ctx->d_vrec.as<unsigned long long>(), ctx->stream),
            "build_vrec");
  }
  GW_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "graph upload");
  ctx->pool_words.assign(nblocks, {});
  ctx->pool_ids.assign(nblocks, {});
  return GW_OK;
}

// By default a context reserves L2 for its visit counters (persisting access
// policy window, see gw_set_l2_persisting); GW_L2_PERSIST=0 disables it.
void default_l2_persisting(gw_ctx* ctx) {
  const char* env = getenv("GW_L2_PERSIST");
  if (env && strcmp(env, "0") == 0) return;
  gw_set_l2_persisting(ctx, (uint64_t)ctx->nv * sizeof(uint32_t));
  ctx->err.clear();  // a device without persisting L2 simply runs without it
}

uint32_t prob_to_u32(double x) {
  if (x <= 0.0) return 0;
  const double v = std::floor(x * 4294967296.0 + 0.5);
  return v >= 4294967295.0 ? 0xffffffffu : (uint32_t)v;
}

}  // namespace

namespace gw {

gw_status make_walk_args(gw_ctx* ctx, const gw_walk_params* p, WalkArgs* a) {
  if (!p) return ctx->fail(GW_E_INVALID, "params is NULL");
  if (p->rule > GW_RULE_PPR) return ctx->fail(GW_E_INVALID, "unknown rule %u", p->rule);
  if (p->sink > GW_SINK_CLOSURE_COUNT) return ctx->fail(GW_E_INVALID, "unknown sink %u", p->sink);
  if (p->rule == GW_RULE_RESTART && p->L == 0)
    return ctx->fail(GW_E_INVALID, "the restart rule needs L >= 1");
  if (p->sink == GW_SINK_PATH_RECORD && p->path_stride == 0)
    return ctx->fail(GW_E_INVALID, "PATH_RECORD needs path_stride >= 1");
  if (!(p->jump_prob >= 0.0 && p->jump_prob <= 1.0))
    return ctx->fail(GW_E_INVALID, "jump_prob must lie in [0, 1]");
  a->hints = (p->cache_hints & GW_HINT_EXPLICIT) ? (p->cache_hints & 15u) : kDefaultHints;
  a->L = p->L;
  a->thr = gw_continue_threshold(p->jump_prob);
  a->njump = p->njump ? p->njump : ctx->nv;
  if (a->njump == 0) return ctx->fail(GW_E_INVALID, "empty graph");
  a->max_hops = p->max_hops ? p->max_hops : 65535u;
  a->seed_lo = (uint32_t)p->seed;
  a->seed_hi = (uint32_t)(p->seed >> 32);
  a->path_stride = p->path_stride;
  a->lo = 0;
  a->hi = ctx->nv;
  if (p->rng > GW_RNG_NATIVE) return ctx->fail(GW_E_INVALID, "unknown rng %u", p->rng);
  a->native = p->rng == GW_RNG_NATIVE ? 1u : 0u;
  return GW_OK;
}

cudaError_t enqueue_status_read(gw_ctx* ctx, cudaStream_t stream) {
  cudaError_t e = cudaMemcpyAsync(ctx->h_status.p, ctx->d_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_status.p, 0, sizeof(uint32_t), stream);
  return e;
}

gw_status take_status(gw_ctx* ctx, cudaStream_t stream) {
  GW_CUDA(ctx, enqueue_status_read(ctx, stream), "status read");
  GW_CUDA(ctx, cudaStreamSynchronize(stream), "synchronize");
  return read_status(ctx);
}

gw_status read_status(gw_ctx* ctx) { return status_of(ctx, *ctx->h_status.as<uint32_t>()); }

gw_status status_of(gw_ctx* ctx, uint32_t st) {
  if (st & kStBounds) return ctx->fail(GW_E_BOUNDS, "a walk reached a vertex id >= %u", ctx->nv);
  if (st & kStOverflow) return ctx->fail(GW_E_OVERFLOW, "a walk made more visits than path_stride");
  if (st & kStHops) return ctx->fail(GW_E_OVERFLOW, "an uncapped walk exceeded max_hops");
  return GW_OK;
}

namespace {
std::atomic<uint32_t> g_fault_kind{GW_FAULT_NONE};
std::atomic<int64_t> g_fault_countdown{0};
}  // namespace

bool fault_now(uint32_t kind) {
  if (g_fault_kind.load(std::memory_order_relaxed) != kind) return false;
  if (g_fault_countdown.fetch_sub(1) != 1) return false;
  g_fault_kind.store(GW_FAULT_NONE);  // fires once
  return true;
}

// Errors of entry points that have no context (gw_last_error(NULL)).
gw_status thread_error(gw_status code, const std::string& msg) { return set_thread_error(code, msg); }

// Grid of a resident walk launch over n walks: the autotuned CTAs per SM
// (gw_walk_autotune), or 0 for the kernel's full occupancy.
int resident_grid(gw_ctx* ctx, uint64_t n) {
  if (ctx->walk_ctas_per_sm <= 0) return 0;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const uint64_t need = (n + kWalkThreads - 1) / kWalkThreads, full = (uint64_t)sms * ctx->walk_ctas_per_sm;
  return (int)(need < full ? (need ? need : 1) : full);
}

}  // namespace gw

extern "C" {

const char* gw_version(void) { return "graphwalker_b200 0.1 (sm_100a)"; }

uint64_t gw_encode(uint32_t source, uint32_t current, uint32_t hop) {
  return (((uint64_t)source & 0xffffffu) << 40) | (((uint64_t)current & 0x3ffffffu) << 14) |
         ((uint64_t)hop & 0x3fffu);
}
uint32_t gw_get_source(uint64_t w) { return (uint32_t)(w >> 40) & 0xffffffu; }
uint32_t gw_get_current(uint64_t w) { return (uint32_t)(w >> 14) & 0x3ffffffu; }
uint32_t gw_get_hop(uint64_t w) { return (uint32_t)(w & 0x3fffu); }

uint32_t gw_continue_threshold(double p) {
  // passes(r) == ((float)r / RAND_MAX > p) with the quotient in float, as in
  // randomwalkwithjump.hpp:45; monotone in r, so bisect for the first pass.
  auto passes = [p](uint32_t r) {
    volatile float q = (float)(int32_t)r / 2147483647;
    return (double)q > p;
  };
  if (!passes(0x7fffffffu)) return 0x80000000u;
  uint32_t lo = 0, hi = 0x7fffffffu;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (passes(mid)) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

uint32_t gw_getblock(const uint32_t* blocks, uint32_t nblocks, uint32_t v) {
  uint32_t lo = 0, hi = nblocks;  // first p with v < blocks[p+1]
  while (lo < hi) {
    const uint32_t mid = (lo + hi) / 2;
    if (v < blocks[mid + 1]) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

uint32_t gw_compute_blocks(const uint64_t* rowptr, uint32_t nvertices, uint64_t blocksize_kb,
                           uint32_t* blocks, uint32_t cap) {
  // compute_block (conversions.hpp:300-364): a block closes before the vertex
  // whose edges would push it past blocksize_kb*1024/4 edges; a vertex whose
  // own degree exceeds that budget becomes a block of its own.
  const uint64_t budget = blocksize_kb * 1024 / sizeof(uint32_t);
  const uint64_t entries = (uint64_t)nvertices + 1;
  uint32_t n = 0;
  uint64_t start_edge = 0;
  if (cap < 1) return 0;
  blocks[n++] = 0;
  for (uint64_t v = 1; v < entries; ++v) {
    if (rowptr[v] - start_edge <= budget) continue;
    const bool lone = rowptr[v] - rowptr[v - 1] > budget;
    if (n + (lone ? 2 : 1) > cap) return 0;
    blocks[n++] = (uint32_t)(v - 1);
    if (lone) {
      blocks[n++] = (uint32_t)v;
      start_edge = rowptr[v];
    } else {
      start_edge = rowptr[v - 1];
    }
  }
  if (n + 1 > cap) return 0;
  blocks[n++] = nvertices;
  return n;
}

uint64_t gw_comp_block_size(uint64_t nwalks) {
  int digits = 0;  // RandomWalk::compBlockSize (randomwalk.hpp:96-105)
  while (nwalks) {
    ++digits;
    nwalks /= 10;
  }
  return 1ull << (11 + digits);
}

uint32_t gw_comp_nmblocks(uint64_t blocksize_kb, uint64_t mem_budget_kb) {
  if (blocksize_kb == 0) return 0;
  if (mem_budget_kb == 0) mem_budget_kb = 44ull * 1024 * 1024;  // MEM_BUDGET, datatype.hpp:13
  return (uint32_t)(mem_budget_kb / blocksize_kb);
}

gw_status gw_open(const gw_graph_desc* desc, gw_ctx** out) {
  if (!desc || !out || !desc->base_filename) return set_thread_error(GW_E_INVALID, "gw_open: NULL argument");
  *out = nullptr;
  gw_ctx* ctx = new gw_ctx();
  ctx->residency = desc->residency;
  ctx->nmblocks = desc->nmblocks ? desc->nmblocks : 2;
  gw_status s = init_ctx(ctx, desc->device);
  const std::string base = desc->base_filename;
  size_t rp_bytes = 0, ci_bytes = 0;
  if (s == GW_OK) s = read_pinned(ctx, graph_file(base, ".beg_pos"), &ctx->h_rowptr, &rp_bytes);
  if (s == GW_OK) s = read_pinned(ctx, graph_file(base, ".csr"), &ctx->h_colidx, &ci_bytes);
  if (s == GW_OK && (rp_bytes < 16 || rp_bytes % 8 || ci_bytes % 4))
    s = ctx->fail(GW_E_IO, "malformed CSR files under %s_GraphWalker", base.c_str());
  std::vector<uint32_t> blocks;
  uint32_t nv = 0;
  if (s == GW_OK) {
    nv = (uint32_t)(rp_bytes / 8 - 1);
    const uint64_t* rp = ctx->h_rowptr.as<uint64_t>();
    if (rp[nv] != ci_bytes / 4)
      s = ctx->fail(GW_E_IO, "beg_pos ends at %llu but the csr holds %zu edges",
                    (unsigned long long)rp[nv], ci_bytes / 4);
  }
  if (s == GW_OK) {
    const std::string brf = blockrange_file(base, desc->blocksize_kb);
    std::ifstream in(brf);
    if (in.good()) {
      uint64_t x;
      while (in >> x) blocks.push_back((uint32_t)x);
    } else {
      // convert_if_notexists computes and writes the block range when absent
      std::vector<uint32_t> tmp((size_t)nv + 2);
      uint32_t cnt = gw_compute_blocks(ctx->h_rowptr.as<uint64_t>(), nv, desc->blocksize_kb,
                                       tmp.data(), (uint32_t)tmp.size());
      blocks.assign(tmp.begin(), tmp.begin() + cnt);
      std::ofstream o(brf);
      for (uint32_t b : blocks) o << b << "\n";
    }
    if (blocks.size() < 2) s = ctx->fail(GW_E_IO, "empty block range %s", brf.c_str());
  }
  if (s == GW_OK)
    s = install_graph(ctx, ctx->h_rowptr.as<uint64_t>(), ctx->h_colidx.as<uint32_t>(), nv,
                      blocks.data(), (uint32_t)blocks.size() - 1);
  if (s == GW_OK && ctx->residency != GW_STREAM_PINNED) {
    ctx->h_rowptr.release();
    ctx->h_colidx.release();
  }
  if (s == GW_OK) s = apply_edge_records(ctx);
  if (s != GW_OK) {
    set_thread_error(s, ctx->err);
    gw_close(ctx);
    return s;
  }
  default_l2_persisting(ctx);
  *out = ctx;
  return GW_OK;
}

gw_status gw_open_csr(const uint64_t* rowptr, const uint32_t* colidx, uint32_t nvertices,
                      const uint32_t* blocks, uint32_t nblocks, uint32_t residency,
                      int32_t device, gw_ctx** out) {
  if (!out || !rowptr || !blocks || (!colidx && rowptr[nvertices] > 0))
    return set_thread_error(GW_E_INVALID, "gw_open_csr: NULL argument");
  *out = nullptr;
  gw_ctx* ctx = new gw_ctx();
  ctx->residency = residency;
  gw_status s = init_ctx(ctx, device);
  static const uint32_t kNoEdges = 0;
  if (s == GW_OK)
    s = install_graph(ctx, rowptr, colidx ? colidx : &kNoEdges, nvertices, blocks, nblocks);
  if (s == GW_OK) s = apply_edge_records(ctx);
  if (s != GW_OK) {
    set_thread_error(s, ctx->err);
    gw_close(ctx);
    return s;
  }
  default_l2_persisting(ctx);
  *out = ctx;
  return GW_OK;
}

gw_status gw_open_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, double a, double b,
                       double c, uint64_t blocksize_kb, int32_t device, gw_ctx** out) {
  if (!out || scale == 0 || scale > 31 || blocksize_kb == 0)
    return set_thread_error(GW_E_INVALID, "gw_open_rmat: bad argument");
  *out = nullptr;
  gw_ctx* ctx = new gw_ctx();
  gw_status s = init_ctx(ctx, device);
  unsigned long long* rowptr = nullptr;
  uint32_t* colidx = nullptr;
  uint64_t kept = 0;
  const uint32_t nv = 1u << scale;
  if (s == GW_OK) {
    cudaError_t e = gw::rmat_build_csr(scale, (uint64_t)edge_factor << scale, seed,
                                       prob_to_u32(a), prob_to_u32(a + b), prob_to_u32(a + b + c),
                                       &rowptr, &colidx, &kept, ctx->stream);
    if (e != cudaSuccess) s = ctx->cuda_fail(e, "rmat_build_csr");
  }
  std::vector<uint64_t> h_rowptr;
  std::vector<uint32_t> blocks;
  if (s == GW_OK) {
    ctx->d_rowptr.p = rowptr;
    ctx->d_rowptr.bytes = ((size_t)nv + 1) * 8;
    ctx->d_colidx.p = colidx;
    ctx->d_colidx.bytes = kept * 4;
    h_rowptr.resize((size_t)nv + 1);
    cudaError_t e = cudaMemcpy(h_rowptr.data(), rowptr, h_rowptr.size() * 8, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) s = ctx->cuda_fail(e, "rowptr readback");
  }
  if (s == GW_OK) {
    blocks.resize((size_t)nv + 2);
    uint32_t cnt = gw_compute_blocks(h_rowptr.data(), nv, blocksize_kb, blocks.data(),
                                     (uint32_t)blocks.size());
    blocks.resize(cnt);
    ctx->nv = nv;
    ctx->ne = kept;
    ctx->nblocks = cnt - 1;
    ctx->blocks = blocks;
    ctx->pool_words.assign(ctx->nblocks, {});
    ctx->pool_ids.assign(ctx->nblocks, {});
    cudaError_t e = ctx->d_blocks.ensure(cnt * sizeof(uint32_t));
    if (e == cudaSuccess)
      e = cudaMemcpy(ctx->d_blocks.p, blocks.data(), cnt * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = ctx->d_vrec.ensure(gw::vrec_bytes(nv));
    if (e == cudaSuccess)
      e = gw::launch_build_vrec(rowptr, nv, ctx->d_vrec.as<unsigned long long>(), ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) s = ctx->cuda_fail(e, "rmat install");
  }
  if (s == GW_OK) s = apply_edge_records(ctx);
  if (s != GW_OK) {
    set_thread_error(s, ctx->err);
    gw_close(ctx);
    return s;
  }
  default_l2_persisting(ctx);
  *out = ctx;
  return GW_OK;
}

gw_status gw_close(gw_ctx* ctx) {
  if (!ctx) return GW_OK;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  if (ctx->aux_stream) cudaStreamSynchronize(ctx->aux_stream);
  if (ctx->l2_persist_bytes) gw_set_l2_persisting(ctx, 0);
  gw::pipe_release(ctx);
  for (gw_devbuf* b : {&ctx->d_rowptr, &ctx->d_colidx, &ctx->d_vrec, &ctx->d_erec, &ctx->d_meet, &ctx->d_sr_rows, &ctx->d_blocks,
                       &ctx->d_status,
                       &ctx->d_walks, &ctx->d_words, &ctx->d_ids, &ctx->d_counts, &ctx->d_paths,
                       &ctx->d_plen, &ctx->d_closure, &ctx->d_pool_offsets, &ctx->d_dest,
                       &ctx->d_tile_hist, &ctx->d_tile_off, &ctx->d_totals, &ctx->d_minhop,
                       &ctx->d_scan_temp, &ctx->d_out_ptr, &ctx->d_out_base, &ctx->d_q_sources,
                       &ctx->d_q_prefix, &ctx->d_q_idbase, &ctx->d_q_toff, &ctx->d_q_tmask, &ctx->d_q_tables,
                       &ctx->d_q_full, &ctx->d_q_ids, &ctx->d_q_counts, &ctx->d_q_visits,
                       &ctx->d_q_cursor, &ctx->d_q_segs, &ctx->d_q_cand})
    b->release();
  for (gw_devbuf& b : ctx->pools) b.release();
  ctx->h_rowptr.release();
  ctx->h_colidx.release();
  ctx->h_status.release();
  ctx->pool_arena.release();
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->aux_stream) cudaStreamDestroy(ctx->aux_stream);
  delete ctx;
  return GW_OK;
}

const char* gw_last_error(gw_ctx* ctx) { return ctx ? ctx->err.c_str() : t_last_error.c_str(); }

gw_status gw_graph_info(gw_ctx* ctx, uint32_t* nvertices, uint64_t* nedges, uint32_t* nblocks) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  if (nvertices) *nvertices = ctx->nv;
  if (nedges) *nedges = ctx->ne;
  if (nblocks) *nblocks = ctx->nblocks;
  return GW_OK;
}

gw_status gw_get_blocks(gw_ctx* ctx, uint32_t* blocks, uint32_t cap) {
  if (!ctx || !blocks) return set_thread_error(GW_E_INVALID, "NULL argument");
  if (cap < ctx->nblocks + 1) return ctx->fail(GW_E_INVALID, "need room for %u entries", ctx->nblocks + 1);
  std::copy(ctx->blocks.begin(), ctx->blocks.end(), blocks);
  return GW_OK;
}

gw_status gw_export_csr(gw_ctx* ctx, uint64_t* rowptr, uint32_t* colidx) {
  if (!ctx || !rowptr) return set_thread_error(GW_E_INVALID, "NULL argument");
  const size_t rp = ((size_t)ctx->nv + 1) * 8, ci = (size_t)ctx->ne * 4;
  if (ctx->residency == GW_STREAM_PINNED) {
    memcpy(rowptr, ctx->h_rowptr.p, rp);
    if (colidx) memcpy(colidx, ctx->h_colidx.p, ci);
    return GW_OK;
  }
  GW_CUDA(ctx, cudaMemcpy(rowptr, ctx->d_rowptr.p, rp, cudaMemcpyDeviceToHost), "rowptr export");
  if (colidx && ci)
    GW_CUDA(ctx, cudaMemcpy(colidx, ctx->d_colidx.p, ci, cudaMemcpyDeviceToHost), "colidx export");
  return GW_OK;
}

gw_status gw_set_residency(gw_ctx* ctx, uint32_t residency, uint32_t nmblocks) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  if (residency > GW_STREAM_PINNED) return ctx->fail(GW_E_INVALID, "unknown residency %u", residency);
  if (nmblocks) ctx->nmblocks = nmblocks;
  if (residency == ctx->residency) return GW_OK;
  const size_t rp = ((size_t)ctx->nv + 1) * 8, ci = (size_t)ctx->ne * 4;
  GW_CUDA(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (residency == GW_STREAM_PINNED) {
    GW_CUDA(ctx, ctx->h_rowptr.ensure(rp), "pinned rowptr");
    GW_CUDA(ctx, ctx->h_colidx.ensure(ci), "pinned colidx");
    GW_CUDA(ctx, cudaMemcpy(ctx->h_rowptr.p, ctx->d_rowptr.p, rp, cudaMemcpyDeviceToHost), "rowptr to host");
    if (ci) GW_CUDA(ctx, cudaMemcpy(ctx->h_colidx.p, ctx->d_colidx.p, ci, cudaMemcpyDeviceToHost), "colidx to host");
    ctx->d_colidx.release();  // the row pointer stays in HBM
    ctx->d_vrec.release();
    ctx->d_erec.release();
  } else {
    GW_CUDA(ctx, ctx->d_rowptr.ensure(rp), "rowptr alloc");
    GW_CUDA(ctx, ctx->d_colidx.ensure(ci), "colidx alloc");
    GW_CUDA(ctx, ctx->d_vrec.ensure(gw::vrec_bytes(ctx->nv)), "vrec alloc");
    GW_CUDA(ctx, cudaMemcpy(ctx->d_rowptr.p, ctx->h_rowptr.p, rp, cudaMemcpyHostToDevice), "rowptr to device");
    if (ci) GW_CUDA(ctx, cudaMemcpy(ctx->d_colidx.p, ctx->h_colidx.p, ci, cudaMemcpyHostToDevice), "colidx to device");
    GW_CUDA(ctx, gw::launch_build_vrec(ctx->d_rowptr.as<unsigned long long>(), ctx->nv,
                                       ctx->d_vrec.as<unsigned long long>(), ctx->stream), "build_vrec");
    GW_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    ctx->h_rowptr.release();
    ctx->h_colidx.release();
  }
  ctx->residency = residency;
  return apply_edge_records(ctx);
}

gw_status gw_set_pool_budget(gw_ctx* ctx, uint64_t bytes) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  ctx->pool_budget = bytes;
  return GW_OK;
}

gw_status gw_set_mapped_block_walks(gw_ctx* ctx, uint64_t max_walks) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  ctx->mapped_max_walks = max_walks;
  return GW_OK;
}

gw_status gw_simrank_meet(gw_ctx* ctx, const uint32_t* d_paths_a, const uint32_t* d_paths_b, uint32_t R,
                          uint32_t L, uint64_t* meet, void* stream) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  if (!meet || (R && L && (!d_paths_a || !d_paths_b))) return ctx->fail(GW_E_INVALID, "gw_simrank_meet: NULL argument");
  if (R > 65535u * 64u) return ctx->fail(GW_E_INVALID, "gw_simrank_meet: R = %u exceeds 4194240", R);
  if (L == 0) return GW_OK;
  GW_CUDA(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  GW_CUDA(ctx, ctx->d_meet.ensure((size_t)L * sizeof(unsigned long long)), "meet alloc");
  GW_CUDA(ctx, gw::launch_simrank_meet(d_paths_a, d_paths_b, nullptr, 1, R, L, ctx->d_meet.as<unsigned long long>(),
                                       st),
          "simrank_meet");
  GW_CUDA(ctx, cudaMemcpyAsync(meet, ctx->d_meet.p, (size_t)L * sizeof(uint64_t), cudaMemcpyDeviceToHost, st),
          "meet copy");
  GW_CUDA(ctx, cudaStreamSynchronize(st), "synchronize");
  return GW_OK;
}

gw_status gw_simrank_batch(gw_ctx* ctx, const gw_walk_params* params, const uint32_t* a, const uint32_t* b,
                           uint32_t nq, uint32_t R, double decay, uint64_t* meet, double* scores) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  if (!params || (nq && (!a || !b || !scores))) return ctx->fail(GW_E_INVALID, "gw_simrank_batch: NULL argument");
  if (params->rule != GW_RULE_RESTART)
    return ctx->fail(GW_E_INVALID, "SimRank walks use the restart rule (RandomWalkwithRestartwithJoint)");
  if (ctx->residency != GW_RESIDENT_HBM) return ctx->fail(GW_E_STATE, "gw_simrank_batch needs a resident graph");
  const uint32_t L = params->L;
  if (L == 0 || R == 0 || R > 65535u * 64u || nq > (1u << 31))
    return ctx->fail(GW_E_INVALID, "gw_simrank_batch: need L > 0, 0 < R <= 4194240, nq <= 2^31");
  if (nq == 0) return GW_OK;
  gw_walk_params pp = *params;  // the walks record their paths, L positions per replica
  pp.sink = GW_SINK_PATH_RECORD;
  pp.path_stride = L;
  gw::WalkArgs wa;
  gw_status s = gw::make_walk_args(ctx, &pp, &wa);
  if (s != GW_OK) return s;
  // the distinct vertices of the batch, R walks each (the app's placement, simrank.cpp:30-57)
  std::vector<uint32_t> verts(a, a + nq);
  verts.insert(verts.end(), b, b + nq);
  std::sort(verts.begin(), verts.end());
  verts.erase(std::unique(verts.begin(), verts.end()), verts.end());
  for (uint32_t v : verts)
    if (v >= ctx->nv) return ctx->fail(GW_E_INVALID, "SimRank vertex %u >= nvertices", v);
  const uint64_t n = (uint64_t)verts.size() * R;
  if ((uint64_t)(R - 1) * L >= (1ull << 32)) return ctx->fail(GW_E_INVALID, "R * L exceeds the 32-bit hop field");
  std::vector<unsigned long long> rows(2 * (size_t)nq);
  auto row_of = [&](uint32_t v) {
    return (unsigned long long)(std::lower_bound(verts.begin(), verts.end(), v) - verts.begin()) * R * L;
  };
  for (uint32_t q = 0; q < nq; ++q) {
    rows[2 * q] = row_of(a[q]);
    rows[2 * q + 1] = row_of(b[q]);
  }
  GW_CUDA(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  cudaStream_t st = ctx->stream;
  GW_CUDA(ctx, ctx->d_walks.ensure(n * sizeof(gw_walk_rec)), "walk alloc");
  GW_CUDA(ctx, ctx->d_paths.ensure(n * L * 4), "paths alloc");
  GW_CUDA(ctx, ctx->d_plen.ensure(n * 4), "plen alloc");
  GW_CUDA(ctx, ctx->d_sr_rows.ensure(rows.size() * 8 + verts.size() * 4), "rows alloc");
  uint32_t* d_verts = reinterpret_cast<uint32_t*>(ctx->d_sr_rows.as<char>() + rows.size() * 8);
  GW_CUDA(ctx, ctx->d_meet.ensure((size_t)nq * L * 8), "meet alloc");
  GW_CUDA(ctx, cudaMemcpyAsync(d_verts, verts.data(), verts.size() * 4, cudaMemcpyHostToDevice, st), "vertex upload");
  GW_CUDA(ctx, gw::launch_simrank_walks(d_verts, (uint32_t)verts.size(), R, L, ctx->d_walks.as<gw_walk_rec>(), st),
          "simrank placement");
  GW_CUDA(ctx, cudaMemcpyAsync(ctx->d_sr_rows.p, rows.data(), rows.size() * 8, cudaMemcpyHostToDevice, st),
          "rows upload");
  GW_CUDA(ctx, cudaMemsetAsync(ctx->d_paths.p, 0xff, n * L * 4, st), "paths clear");
  gw::SinkView sv{};
  sv.paths = ctx->d_paths.as<uint32_t>();
  sv.plen = ctx->d_plen.as<uint32_t>();
  GW_CUDA(ctx, gw::launch_walk_resident(GW_RULE_RESTART, GW_SINK_PATH_RECORD, false, ctx->d_walks.as<gw_walk_rec>(),
                                        n, ctx->view(), wa, sv, ctx->d_status.as<uint32_t>(), 0, st, nullptr),
          "simrank walks");
  GW_CUDA(ctx, gw::launch_simrank_meet(ctx->d_paths.as<uint32_t>(), ctx->d_paths.as<uint32_t>(),
                                       ctx->d_sr_rows.as<unsigned long long>(), nq, R, L,
                                       ctx->d_meet.as<unsigned long long>(), st),
          "simrank meet");
  std::vector<uint64_t> m((size_t)nq * L);
  GW_CUDA(ctx, cudaMemcpyAsync(m.data(), ctx->d_meet.p, m.size() * 8, cudaMemcpyDeviceToHost, st), "meet copy");
  s = gw::take_status(ctx, st);  // synchronises the stream
  if (s != GW_OK) return s;
  const double rr = (double)R * (double)R;
  for (uint32_t q = 0; q < nq; ++q) {
    double sc = 0.0, w = 1.0;
    for (uint32_t l = 0; l < L; ++l, w *= decay) sc += (double)m[(size_t)q * L + l] * w;
    scores[q] = sc / rr;
  }
  if (meet) std::copy(m.begin(), m.end(), meet);
  ctx->have_run = false;  // the path buffers now hold SimRank walks, not a gw_run's
  return GW_OK;
}

gw_status gw_inject_fault(uint32_t kind, uint32_t after) {
  if (kind > GW_FAULT_FILE_READ) return set_thread_error(GW_E_INVALID, "unknown fault kind");
  gw::g_fault_kind.store(GW_FAULT_NONE);
  gw::g_fault_countdown.store((int64_t)after + 1);
  gw::g_fault_kind.store(kind);
  return GW_OK;
}

gw_status gw_set_edge_records(gw_ctx* ctx, uint32_t mode, uint32_t* built) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  if (mode > GW_EDGE_RECORDS_AUTO) return ctx->fail(GW_E_INVALID, "unknown edge-record mode %u", mode);
  ctx->erec_mode = mode;
  if (mode == GW_EDGE_RECORDS_OFF) ctx->d_erec.release();
  const gw_status s = apply_edge_records(ctx);
  if (built) *built = ctx->view().erec ? 1u : 0u;
  return s;
}

gw_status gw_walks_clear(gw_ctx* ctx) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  for (auto& p : ctx->pool_words) p.clear();
  for (auto& p : ctx->pool_ids) p.clear();
  ctx->pools_have_ids = false;
  return GW_OK;
}

gw_status gw_walks_add(gw_ctx* ctx, uint32_t block, const uint64_t* words, const uint32_t* ids,
                       size_t n) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  if (block >= ctx->nblocks) return ctx->fail(GW_E_INVALID, "block %u >= nblocks %u", block, ctx->nblocks);
  if (n == 0) return GW_OK;
  if (!words) return ctx->fail(GW_E_INVALID, "words is NULL");
  auto& pw = ctx->pool_words[block];
  auto& pi = ctx->pool_ids[block];
  if (ids && !ctx->pools_have_ids) {
    // earlier walks default to their source field
    for (uint32_t b = 0; b < ctx->nblocks; ++b) {
      auto& ids_b = ctx->pool_ids[b];
      ids_b.resize(ctx->pool_words[b].size());
      for (size_t i = 0; i < ids_b.size(); ++i) ids_b[i] = gw_get_source(ctx->pool_words[b][i]);
    }
    ctx->pools_have_ids = true;
  }
  pw.insert(pw.end(), words, words + n);
  if (ctx->pools_have_ids) {
    if (ids) pi.insert(pi.end(), ids, ids + n);
    else
      for (size_t i = 0; i < n; ++i) pi.push_back(gw_get_source(words[i]));
  }
  return GW_OK;
}

gw_status gw_walks_count(gw_ctx* ctx, uint64_t* per_block, uint64_t* total) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  uint64_t t = 0;
  for (uint32_t b = 0; b < ctx->nblocks; ++b) {
    if (per_block) per_block[b] = ctx->pool_words[b].size();
    t += ctx->pool_words[b].size();
  }
  if (total) *total = t;
  return GW_OK;
}

gw_status gw_run(gw_ctx* ctx, const gw_walk_params* params) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  gw::WalkArgs a;
  gw_status s = gw::make_walk_args(ctx, params, &a);
  if (s != GW_OK) return s;
  if (params->mode == GW_MODE_BLOCKED || ctx->residency == GW_STREAM_PINNED)
    return gw::run_blocked(ctx, params);
  if (params->mode != GW_MODE_RESIDENT) return ctx->fail(GW_E_INVALID, "unknown mode %u", params->mode);

  // Upload the pools in block order and decode them into walk records.
  uint64_t n = 0;
  for (auto& p : ctx->pool_words) n += p.size();
  cudaStream_t st = ctx->stream;
  GW_CUDA(ctx, ctx->d_walks.ensure(n * sizeof(gw_walk_rec)), "walk alloc");
  GW_CUDA(ctx, ctx->d_words.ensure(n * sizeof(uint64_t)), "word alloc");
  if (ctx->pools_have_ids) GW_CUDA(ctx, ctx->d_ids.ensure(n * sizeof(uint32_t)), "id alloc");
  uint64_t off = 0;
  for (uint32_t b = 0; b < ctx->nblocks; ++b) {
    const size_t m = ctx->pool_words[b].size();
    if (!m) continue;
    uint64_t* w = ctx->d_words.as<uint64_t>() + off;
    uint32_t* ids = ctx->pools_have_ids ? ctx->d_ids.as<uint32_t>() + off : nullptr;
    GW_CUDA(ctx, cudaMemcpyAsync(w, ctx->pool_words[b].data(), m * 8, cudaMemcpyHostToDevice, st),
            "walk upload");
    if (ids)
      GW_CUDA(ctx, cudaMemcpyAsync(ids, ctx->pool_ids[b].data(), m * 4, cudaMemcpyHostToDevice, st),
              "id upload");
    GW_CUDA(ctx, gw::launch_unpack_words(w, ids, m, ctx->blocks[b],
                                         ctx->d_walks.as<gw_walk_rec>() + off, st), "unpack");
    off += m;
  }
  // Sinks.
  gw::SinkView sv{};
  GW_CUDA(ctx, ctx->d_counts.ensure((size_t)ctx->nv * 4), "counts alloc");
  GW_CUDA(ctx, cudaMemsetAsync(ctx->d_counts.p, 0, (size_t)ctx->nv * 4, st), "counts clear");
  sv.counts = ctx->d_counts.as<uint32_t>();
  if (params->sink == GW_SINK_PATH_RECORD) {
    GW_CUDA(ctx, ctx->d_paths.ensure(n * params->path_stride * 4), "paths alloc");
    GW_CUDA(ctx, ctx->d_plen.ensure(n * 4), "plen alloc");
    GW_CUDA(ctx, cudaMemsetAsync(ctx->d_paths.p, 0xff, n * params->path_stride * 4, st), "paths clear");
    sv.paths = ctx->d_paths.as<uint32_t>();
    sv.plen = ctx->d_plen.as<uint32_t>();
  }
  GW_CUDA(ctx, ctx->d_closure.ensure(8), "closure alloc");
  GW_CUDA(ctx, cudaMemsetAsync(ctx->d_closure.p, 0, 8, st), "closure clear");
  sv.closure = ctx->d_closure.as<unsigned long long>();

  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  cudaAccessPolicyWindow win;
  const bool use_win = params->sink == GW_SINK_VERTEX_COUNT && ctx->counts_window(sv.counts, &win);
  cudaError_t e = gw::launch_walk_resident((int)params->rule, (int)params->sink, params->aggregate != 0,
                                           ctx->d_walks.as<gw_walk_rec>(), n, ctx->view(), a, sv,
                                           ctx->d_status.as<uint32_t>(), gw::resident_grid(ctx, n), st,
                                           use_win ? &win : nullptr);
  cudaEventRecord(e1, st);
  if (e != cudaSuccess) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ctx->cuda_fail(e, "walk kernel launch");
  }
  s = gw::take_status(ctx, st);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->stats = gw_run_stats{};
  ctx->stats.walks = n;
  ctx->stats.ms_total = ms;
  ctx->stats.ms_walk = ms;
  ctx->last_nwalks = n;
  ctx->last_stride = params->path_stride;
  ctx->last_sink = params->sink;
  ctx->have_run = true;
  return s;
}

gw_status gw_read_counts(gw_ctx* ctx, uint32_t* counts, size_t n) {
  if (!ctx || !counts) return set_thread_error(GW_E_INVALID, "NULL argument");
  if (!ctx->have_run) return ctx->fail(GW_E_STATE, "no run yet");
  if (n > ctx->nv) n = ctx->nv;
  GW_CUDA(ctx, cudaMemcpy(counts, ctx->d_counts.p, n * 4, cudaMemcpyDeviceToHost), "counts read");
  return GW_OK;
}

gw_status gw_read_paths(gw_ctx* ctx, uint32_t* paths, uint32_t* lens, size_t nwalks) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  if (!ctx->have_run || ctx->last_sink != GW_SINK_PATH_RECORD)
    return ctx->fail(GW_E_STATE, "the last run did not record paths");
  if (nwalks > ctx->last_nwalks) nwalks = ctx->last_nwalks;
  if (paths)
    GW_CUDA(ctx, cudaMemcpy(paths, ctx->d_paths.p, nwalks * ctx->last_stride * 4, cudaMemcpyDeviceToHost),
            "paths read");
  if (lens) GW_CUDA(ctx, cudaMemcpy(lens, ctx->d_plen.p, nwalks * 4, cudaMemcpyDeviceToHost), "lens read");
  return GW_OK;
}

gw_status gw_read_closure(gw_ctx* ctx, uint64_t* closure) {
  if (!ctx || !closure) return set_thread_error(GW_E_INVALID, "NULL argument");
  if (!ctx->have_run) return ctx->fail(GW_E_STATE, "no run yet");
  GW_CUDA(ctx, cudaMemcpy(closure, ctx->d_closure.p, 8, cudaMemcpyDeviceToHost), "closure read");
  return GW_OK;
}

gw_status gw_read_stats(gw_ctx* ctx, gw_run_stats* stats) {
  if (!ctx || !stats) return set_thread_error(GW_E_INVALID, "NULL argument");
  *stats = ctx->stats;
  return GW_OK;
}

gw_status gw_read_pool(gw_ctx* ctx, uint32_t block, gw_walk_rec* out, size_t cap, uint64_t* n) {
  if (!ctx || !n) return set_thread_error(GW_E_INVALID, "NULL argument");
  if (block >= ctx->nblocks) return ctx->fail(GW_E_INVALID, "block %u >= nblocks", block);
  const uint64_t size = block < ctx->pool_size.size() ? ctx->pool_size[block] : 0;
  *n = size;
  const uint64_t m = std::min<uint64_t>(size, cap);
  if (!m || !out) return GW_OK;
  // the part moved to host memory comes first (older walks), then the device part
  const uint64_t hn = block < ctx->pool_host_n.size() ? std::min<uint64_t>(ctx->pool_host_n[block], m) : 0;
  if (hn) {
    GW_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "pool read");
    const gw_walk_rec* arena = ctx->pool_arena.as<gw_walk_rec>();
    for (uint64_t i = 0; i * gw_ctx::kPoolChunk < hn; ++i) {
      const uint64_t c = ctx->pool_chunks[block][i], k = std::min(gw_ctx::kPoolChunk, hn - i * gw_ctx::kPoolChunk);
      std::copy(arena + c * gw_ctx::kPoolChunk, arena + c * gw_ctx::kPoolChunk + k, out + i * gw_ctx::kPoolChunk);
    }
  }
  if (m > hn)
    GW_CUDA(ctx, cudaMemcpy(out + hn, ctx->pools[block].p, (m - hn) * sizeof(gw_walk_rec), cudaMemcpyDeviceToHost),
            "pool read");
  return GW_OK;
}

gw_status gw_run_pools(gw_ctx* ctx, const gw_walk_params* params, const uint64_t* words,
                       const uint64_t* pool_offsets, const uint32_t* ids, uint32_t* counts) {
  if (!ctx || !params || !pool_offsets || !counts) return set_thread_error(GW_E_INVALID, "NULL argument");
  if (params->sink != GW_SINK_VERTEX_COUNT && params->sink != GW_SINK_NONE)
    return ctx->fail(GW_E_INVALID, "gw_run_pools returns vertex counts only");
  if (ctx->residency != GW_RESIDENT_HBM) return ctx->fail(GW_E_STATE, "gw_run_pools needs a resident graph");
  gw::WalkArgs a;
  gw_status s = gw::make_walk_args(ctx, params, &a);
  if (s != GW_OK) return s;
  const uint64_t n = pool_offsets[ctx->nblocks];
  if (n && !words) return ctx->fail(GW_E_INVALID, "words is NULL");
  // Chunks of the host words (gw::chunk_bounds) are copied on the copy stream
  // while the walk kernel of the previous chunk runs.  The chunk kernels
  // alternate between two compute streams, so a chunk's walks start while the
  // previous kernel's last walks finish instead of after them (the walks of
  // different chunks share only the visit counters, updated atomically).
  const std::vector<uint64_t> chunk_lo = gw::chunk_bounds(n);
  const uint64_t nchunks = chunk_lo.size() - 1;
  GW_CUDA(ctx, ctx->d_walks.ensure(n * sizeof(gw_walk_rec)), "walk alloc");
  GW_CUDA(ctx, ctx->d_words.ensure(n * 8), "word alloc");
  if (ids) GW_CUDA(ctx, ctx->d_ids.ensure(n * 4), "id alloc");
  GW_CUDA(ctx, ctx->d_pool_offsets.ensure((ctx->nblocks + 1) * 8), "offsets alloc");
  GW_CUDA(ctx, ctx->d_counts.ensure((size_t)ctx->nv * 4), "counts alloc");
  cudaStream_t cs = ctx->stream, xs = ctx->copy_stream;
  GW_CUDA(ctx, cudaMemcpyAsync(ctx->d_pool_offsets.p, pool_offsets, (ctx->nblocks + 1) * 8,
                               cudaMemcpyHostToDevice, cs), "offsets copy");
  GW_CUDA(ctx, cudaMemsetAsync(ctx->d_counts.p, 0, (size_t)ctx->nv * 4, cs), "counts clear");
  gw::SinkView sv{};
  sv.counts = ctx->d_counts.as<uint32_t>();
  std::vector<cudaEvent_t> ready(nchunks);
  for (auto& ev : ready) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  cudaEvent_t start_ev, aux_done;
  cudaEventCreateWithFlags(&start_ev, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&aux_done, cudaEventDisableTiming);
  cudaStream_t as = ctx->aux_stream;
  cudaEventRecord(start_ev, cs);  // copies and kernels must not overtake earlier work on cs
  cudaStreamWaitEvent(xs, start_ev, 0);
  cudaStreamWaitEvent(as, start_ev, 0);
  cudaError_t e = cudaSuccess;
  for (uint64_t c = 0; c < nchunks && e == cudaSuccess; ++c) {
    const uint64_t lo = chunk_lo[c], m = chunk_lo[c + 1] - lo;
    e = cudaMemcpyAsync(ctx->d_words.as<uint64_t>() + lo, words + lo, m * 8, cudaMemcpyHostToDevice, xs);
    if (e == cudaSuccess && ids)
      e = cudaMemcpyAsync(ctx->d_ids.as<uint32_t>() + lo, ids + lo, m * 4, cudaMemcpyHostToDevice, xs);
    if (e == cudaSuccess) e = cudaEventRecord(ready[c], xs);
  }
  for (uint64_t c = 0; c < nchunks && e == cudaSuccess; ++c) {
    const uint64_t lo = chunk_lo[c], m = chunk_lo[c + 1] - lo;
    const cudaStream_t ks = (c & 1) ? as : cs;
    e = cudaStreamWaitEvent(ks, ready[c], 0);
    if (e == cudaSuccess)
      e = gw::launch_unpack_pools(ctx->d_words.as<uint64_t>() + lo,
                                  ids ? ctx->d_ids.as<uint32_t>() + lo : nullptr, lo, m,
                                  ctx->d_pool_offsets.as<uint64_t>(), ctx->d_blocks.as<uint32_t>(),
                                  ctx->nblocks, ctx->d_walks.as<gw_walk_rec>() + lo, ks);
    cudaAccessPolicyWindow win;
    const bool use_win = params->sink == GW_SINK_VERTEX_COUNT && ctx->counts_window(sv.counts, &win);
    if (e == cudaSuccess)
      e = gw::launch_walk_resident((int)params->rule, (int)params->sink, params->aggregate != 0,
                                   ctx->d_walks.as<gw_walk_rec>() + lo, m, ctx->view(), a, sv,
                                   ctx->d_status.as<uint32_t>(), gw::resident_grid(ctx, m), ks,
                                   use_win ? &win : nullptr);
  }
  // the counts are complete once both compute streams are done
  cudaEventRecord(aux_done, as);
  cudaStreamWaitEvent(cs, aux_done, 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(counts, ctx->d_counts.p, (size_t)ctx->nv * 4, cudaMemcpyDeviceToHost, cs);
  for (auto& ev : ready) cudaEventDestroy(ev);
  cudaEventDestroy(start_ev);
  cudaEventDestroy(aux_done);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "gw_run_pools");
  s = gw::take_status(ctx, cs);
  ctx->last_nwalks = n;
  ctx->last_sink = params->sink;
  ctx->have_run = true;
  ctx->stats = gw_run_stats{};
  ctx->stats.walks = n;
  return s;
}

gw_status gw_walk_device(gw_ctx* ctx, const gw_walk_params* params, const gw_walk_rec* d_walks,
                         uint64_t n, uint32_t* d_counts, uint32_t* d_paths, uint32_t* d_plen,
                         unsigned long long* d_closure, void* stream) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  if (ctx->residency != GW_RESIDENT_HBM) return ctx->fail(GW_E_STATE, "gw_walk_device needs a resident graph");
  gw::WalkArgs a;
  gw_status s = gw::make_walk_args(ctx, params, &a);
  if (s != GW_OK) return s;
  gw::SinkView sv{};
  sv.counts = d_counts;
  sv.paths = d_paths;
  sv.plen = d_plen;
  sv.closure = d_closure;
  if (n && !d_walks) return ctx->fail(GW_E_INVALID, "d_walks is NULL");
  if (params->sink == GW_SINK_VERTEX_COUNT && !d_counts) return ctx->fail(GW_E_INVALID, "d_counts is NULL");
  if (params->sink == GW_SINK_PATH_RECORD && (!d_paths || !d_plen))
    return ctx->fail(GW_E_INVALID, "d_paths/d_plen is NULL");
  if (params->sink == GW_SINK_CLOSURE_COUNT && !d_closure) return ctx->fail(GW_E_INVALID, "d_closure is NULL");
  cudaStream_t st = (cudaStream_t)stream;  // NULL = the default stream
  cudaAccessPolicyWindow win;
  const bool use_win = params->sink == GW_SINK_VERTEX_COUNT && ctx->counts_window(d_counts, &win);
  cudaError_t e = gw::launch_walk_resident((int)params->rule, (int)params->sink, params->aggregate != 0,
                                           d_walks, n, ctx->view(), a, sv,
                                           ctx->d_status.as<uint32_t>(), gw::resident_grid(ctx, n), st,
                                           use_win ? &win : nullptr);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "walk kernel launch");
  return GW_OK;
}

gw_status gw_walk_autotune(gw_ctx* ctx, const gw_walk_params* params, const gw_walk_rec* d_walks, uint64_t n,
                           uint32_t* ctas_per_sm) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  if (ctx->residency != GW_RESIDENT_HBM) return ctx->fail(GW_E_STATE, "gw_walk_autotune needs a resident graph");
  if (!d_walks || n == 0) return ctx->fail(GW_E_INVALID, "gw_walk_autotune: no walks");
  gw_walk_params pp = *params;  // counts into a scratch array; other sinks cost the same per step
  pp.sink = GW_SINK_VERTEX_COUNT;
  gw::WalkArgs a;
  gw_status s = gw::make_walk_args(ctx, &pp, &a);
  if (s != GW_OK) return s;
  GW_CUDA(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  GW_CUDA(ctx, ctx->d_counts.ensure((size_t)ctx->nv * 4), "counts alloc");
  gw::SinkView sv{};
  sv.counts = ctx->d_counts.as<uint32_t>();
  cudaStream_t st = ctx->stream;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int full = gw::walk_resident_grid((int)pp.rule, (int)pp.sink, pp.aggregate != 0, (uint64_t)sms * 64 * 1024);
  const int max_per_sm = std::max(1, full / sms);
  cudaAccessPolicyWindow win;
  const bool use_win = ctx->counts_window(sv.counts, &win);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best = max_per_sm;
  float best_ms = 1e30f;
  // a quarter to full occupancy: a random-miss-bound kernel often runs best
  // well below full occupancy, where fewer requests queue at the DRAM
  for (int c = std::max(1, max_per_sm / 4); c <= max_per_sm; ++c) {
    ctx->walk_ctas_per_sm = c;
    float sum = 0.f;
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(e0, st);
      cudaError_t e = gw::launch_walk_resident((int)pp.rule, (int)pp.sink, pp.aggregate != 0, d_walks, n, ctx->view(),
                                               a, sv, ctx->d_status.as<uint32_t>(), gw::resident_grid(ctx, n), st,
                                               use_win ? &win : nullptr);
      cudaEventRecord(e1, st);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        ctx->walk_ctas_per_sm = 0;
        return ctx->cuda_fail(e, "autotune launch");
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep) sum += ms;  // the first run warms up
    }
    if (sum < best_ms) {
      best_ms = sum;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->walk_ctas_per_sm = best == max_per_sm ? 0 : best;  // full occupancy is the default shape
  if (ctas_per_sm) *ctas_per_sm = (uint32_t)best;
  return gw::take_status(ctx, st);
}

gw_status gw_set_l2_fetch_granularity(gw_ctx* ctx, uint32_t bytes, uint32_t* previous) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  size_t old = 0;
  GW_CUDA(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  GW_CUDA(ctx, cudaDeviceGetLimit(&old, cudaLimitMaxL2FetchGranularity), "get L2 fetch granularity");
  if (previous) *previous = (uint32_t)old;
  if (bytes) {
    if (bytes > 128 || (bytes & (bytes - 1))) return ctx->fail(GW_E_INVALID, "granularity must be a power of two <= 128");
    GW_CUDA(ctx, cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, bytes), "set L2 fetch granularity");
  }
  return GW_OK;
}

gw_status gw_set_l2_persisting(gw_ctx* ctx, uint64_t bytes) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  GW_CUDA(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  int max_persist = 0;
  GW_CUDA(ctx, cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, ctx->device),
          "max persisting L2");
  int max_window = 0;
  GW_CUDA(ctx, cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, ctx->device),
          "max access policy window");
  ctx->max_window_bytes = (size_t)std::max(max_window, 0);
  const uint64_t b = std::min<uint64_t>(bytes, (uint64_t)max_persist);
  GW_CUDA(ctx, cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, (size_t)b), "persisting L2 limit");
  if (b == 0) GW_CUDA(ctx, cudaCtxResetPersistingL2Cache(), "reset persisting L2");
  ctx->l2_persist_bytes = b;
  return GW_OK;
}

gw_status gw_unpack_words_device(gw_ctx* ctx, uint32_t block, const uint64_t* d_words,
                                 const uint32_t* d_ids, uint64_t n, gw_walk_rec* d_out,
                                 void* stream) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  if (block >= ctx->nblocks) return ctx->fail(GW_E_INVALID, "block %u >= nblocks", block);
  cudaStream_t st = (cudaStream_t)stream;  // NULL = the default stream
  GW_CUDA(ctx, gw::launch_unpack_words(d_words, d_ids, n, ctx->blocks[block], d_out, st), "unpack");
  return GW_OK;
}

gw_status gw_pack_words_device(gw_ctx* ctx, const gw_walk_rec* d_walks, uint64_t n,
                               uint64_t* d_words, uint32_t* d_blocks, void* stream) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  cudaStream_t st = (cudaStream_t)stream;  // NULL = the default stream
  GW_CUDA(ctx, gw::launch_pack_words(d_walks, n, ctx->d_blocks.as<uint32_t>(), ctx->nblocks, d_words,
                                     d_blocks, st), "pack");
  return GW_OK;
}

gw_status gw_sync(gw_ctx* ctx, void* stream) {
  if (!ctx) return set_thread_error(GW_E_INVALID, "NULL context");
  return gw::take_status(ctx, (cudaStream_t)stream);
}

gw_status gw_probe_gather(gw_ctx* ctx, const uint32_t* d_buf, uint64_t n_words, uint64_t loads,
                          int iters, double* bytes_per_s) {
  if (!ctx || !d_buf || !bytes_per_s || n_words < 64 || iters < 1)
    return set_thread_error(GW_E_INVALID, "gw_probe_gather: bad argument");
  cudaStream_t st = ctx->stream;
  gw_devbuf sink;
  GW_CUDA(ctx, sink.ensure(8), "sink alloc");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  gw::launch_gather_probe(d_buf, n_words, loads, sink.as<unsigned long long>(), st);  // warm-up
  float best = 1e30f;
  for (int it = 0; it < iters; ++it) {
    cudaEventRecord(e0, st);
    gw::launch_gather_probe(d_buf, n_words, loads, sink.as<unsigned long long>(), st);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  sink.release();
  if (e != cudaSuccess) return ctx->cuda_fail(e, "gather probe");
  *bytes_per_s = (double)loads * 32.0 / (best * 1e-3);
  return GW_OK;
}

gw_status gw_probe_red(gw_ctx* ctx, uint32_t* d_counters, uint64_t n_words, uint64_t ops, int iters,
                       double* ops_per_s) {
  if (!ctx || !d_counters || !ops_per_s || n_words == 0 || ops == 0 || iters < 1)
    return set_thread_error(GW_E_INVALID, "gw_probe_red: bad argument");
  uint64_t words = 1;  // counters used: n_words rounded down to a power of two
  while (words * 2 <= n_words && words < (1ull << 32)) words *= 2;
  cudaStream_t st = ctx->stream;
  cudaEvent_t e0, e1;
  GW_CUDA(ctx, cudaEventCreate(&e0), "event");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return ctx->fail(GW_E_CUDA, "event");
  }
  cudaError_t e = gw::launch_red_probe(d_counters, (uint32_t)(words - 1), ops, st);  // warm-up
  float best = 1e30f;
  for (int it = 0; it < iters && e == cudaSuccess; ++it) {
    cudaEventRecord(e0, st);
    e = gw::launch_red_probe(d_counters, (uint32_t)(words - 1), ops, st);
    cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "red probe");
  *ops_per_s = (double)ops / (best * 1e-3);
  return GW_OK;
}

}  // extern "C"
