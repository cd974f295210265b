// gw_exact.cu -- expected visits per vertex of one walk from a source, in
// FP64, by propagating the exact per-hop distribution over the resident
// graph (the truncated power series behind PPR / RWR estimates).
//
// x_0 = e_src.  Each hop: a vertex with out-edges passes x[v]*q/deg to every
// out-neighbour (q = the exact probability that a 31-bit draw passes the
// continuation test); the rest -- x[v]*(1-q), or all of x[v] at a dangling
// vertex -- follows the rule's else-branch: back to the source (restart; the
// PPR rule only at dangling vertices), spread uniformly (jump), or ends (stop).
// Visits accumulate x_h for every hop the rule visits (L hops for the capped
// rules, L-1 per restart segment, until the mass vanishes for the uncapped
// rule).  The neighbour choice is taken as exactly uniform; the walks'
// r % deg has a bias below deg / 2^31.
#include <vector>

#include "gw_ctx.h"

namespace gw {
namespace {

constexpr int kExactThreads = 256;

// one warp per vertex: lanes stride over its out-edges
__global__ void __launch_bounds__(kExactThreads)
    exact_hop_kernel(const double* __restrict__ x, double* __restrict__ y, double* __restrict__ visits,
                     double* __restrict__ sums, GraphView g, double q, int rule, bool capped_jump_to_src) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  double to_src = 0.0, to_uniform = 0.0, mass = 0.0;
  for (uint64_t v = warp; v < g.nv; v += nwarps) {
    const double xv = x[v];
    if (xv == 0.0) continue;
    if (lane == 0) {
      visits[v] += xv;
      mass += xv;
    }
    const unsigned long long b = g.rowptr[v], deg = g.rowptr[v + 1] - b;
    double fail;
    if (deg > 0) {
      const double share = xv * q / (double)deg;
      for (unsigned long long e = lane; e < deg; e += 32) atomicAdd(y + g.colidx[b + e], share);
      fail = xv * (1.0 - q);
    } else {
      fail = xv;
    }
    if (lane == 0) {
      if (rule == GW_RULE_RESTART) to_src += fail;
      else if (rule == GW_RULE_PPR && deg == 0) to_src += fail;
      else if (rule == GW_RULE_JUMP) to_uniform += fail;
    }
  }
  (void)capped_jump_to_src;
  if (lane == 0) {
    if (to_src != 0.0) atomicAdd(sums + 0, to_src);
    if (to_uniform != 0.0) atomicAdd(sums + 1, to_uniform);
    if (mass != 0.0) atomicAdd(sums + 2, mass);
  }
}

// y[src] += to_src; y[v] += to_uniform / njump for v < njump; x := 0
__global__ void exact_fold_kernel(double* __restrict__ y, double* __restrict__ x, const double* __restrict__ sums,
                                  uint32_t nv, uint32_t src, uint32_t njump) {
  const double u = sums[1] / (double)njump;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (uint64_t)gridDim.x * blockDim.x) {
    double add = (v < njump) ? u : 0.0;
    if (v == src) add += sums[0];
    if (add != 0.0) y[v] += add;
    x[v] = 0.0;
  }
}

}  // namespace
}  // namespace gw

extern "C" gw_status gw_expected_visits(gw_ctx* ctx, const gw_walk_params* params, uint32_t source, double* out) {
  if (!ctx) return GW_E_INVALID;
  if (ctx->residency != GW_RESIDENT_HBM) return ctx->fail(GW_E_STATE, "needs a resident graph");
  if (!out || source >= ctx->nv) return ctx->fail(GW_E_INVALID, "bad source or NULL output");
  gw::WalkArgs a;
  gw_status s = gw::make_walk_args(ctx, params, &a);
  if (s != GW_OK) return s;
  const double q = (double)(0x80000000u - a.thr) / 2147483648.0;
  const int rule = (int)params->rule;
  uint32_t hops;
  if (rule == GW_RULE_RESTART) hops = params->L > 1 ? params->L - 1 : 1;
  else if (rule == GW_RULE_PROB) hops = a.max_hops;
  else hops = params->L;
  const size_t nv = ctx->nv;
  gw_devbuf bx, by, bvis, bsum;
  GW_CUDA(ctx, bx.ensure(nv * 8), "alloc");
  GW_CUDA(ctx, by.ensure(nv * 8), "alloc");
  GW_CUDA(ctx, bvis.ensure(nv * 8), "alloc");
  GW_CUDA(ctx, bsum.ensure(3 * 8), "alloc");
  cudaStream_t st = ctx->stream;
  double* x = bx.as<double>();
  double* y = by.as<double>();
  GW_CUDA(ctx, cudaMemsetAsync(x, 0, nv * 8, st), "clear");
  GW_CUDA(ctx, cudaMemsetAsync(y, 0, nv * 8, st), "clear");
  GW_CUDA(ctx, cudaMemsetAsync(bvis.p, 0, nv * 8, st), "clear");
  const double one = 1.0;
  GW_CUDA(ctx, cudaMemcpyAsync(x + source, &one, 8, cudaMemcpyHostToDevice, st), "seed");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = sms * 8;
  double sums[3];
  for (uint32_t h = 0; h < hops; ++h) {
    GW_CUDA(ctx, cudaMemsetAsync(bsum.p, 0, 3 * 8, st), "clear");
    gw::exact_hop_kernel<<<grid, gw::kExactThreads, 0, st>>>(x, y, bvis.as<double>(), bsum.as<double>(), ctx->view(),
                                                             q, rule, false);
    GW_CUDA(ctx, cudaGetLastError(), "exact hop");
    gw::exact_fold_kernel<<<grid, 256, 0, st>>>(y, x, bsum.as<double>(), ctx->nv, source, a.njump);
    GW_CUDA(ctx, cudaGetLastError(), "exact fold");
    std::swap(x, y);
    if (rule == GW_RULE_PROB && (h & 15) == 15) {  // the uncapped rule stops when the mass is gone
      GW_CUDA(ctx, cudaMemcpyAsync(sums, bsum.p, 3 * 8, cudaMemcpyDeviceToHost, st), "mass");
      GW_CUDA(ctx, cudaStreamSynchronize(st), "sync");
      if (sums[2] < 1e-16) break;
    }
  }
  GW_CUDA(ctx, cudaMemcpyAsync(out, bvis.p, nv * 8, cudaMemcpyDeviceToHost, st), "visits out");
  GW_CUDA(ctx, cudaStreamSynchronize(st), "sync");
  return GW_OK;
}
