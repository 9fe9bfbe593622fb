// brandes.cu -- exact unweighted betweenness (Brandes) with many sources in
// flight per launch.
//
// Reference: priv/zog/src/centrality.zig:687-798 (ArrayGraph branch).  For
// every live source s (ascending) the reference runs a BFS that fills
// dist[] and the path counts sigma[] (`sigma[w] += sigma[v]` for every arc
// v->w with dist[w] == dist[v]+1, duplicates counted, :745-767), then walks the
// BFS order backwards accumulating delta[u] += sigma[u]/sigma[v] * (1+delta[v])
// over predecessors and adds delta[v] to the score of every v != s (:769-787).
//
// B200 design: a batch of 64 sources advances level by level in lock-step.
// Per vertex the batch keeps 64-bit masks (visited, frontier of the current
// level) and, per (vertex, source) pair, dist (u32), sigma (u64) and
// q = (1+delta)/sigma (f64) in vertex-major rows of 64, so one warp owns one
// vertex and each lane owns sources lane and lane+32.
//   forward (pull): a vertex w with unvisited sources scans its in-neighbours
//     32 at a time (one coalesced index load, one mask gather per lane), keeps
//     only neighbours whose frontier mask meets w's unvisited mask, and lanes
//     add the matching sigma[v][b] -- no atomics, deterministic, and the sums
//     are exact integers (wrapping modulo 2^64 like the reference's usize);
//   backward (pull over successors): at level l a vertex v with sources at
//     depth l gathers q[w][b] of successors w at depth l+1 (mask test first),
//     so delta[v][b] = sigma[v][b] * sum q[w][b] -- the reference's
//     sum of sigma_v/sigma_w * (1+delta_w), reassociated -- and the warp adds
//     sum_b delta[v][b] to BC[v] (only v's own warp touches BC[v]).
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace zogcu {

constexpr int kBcBatch = 64;
constexpr int kBcThreads = 256;

__device__ __forceinline__ unsigned long long shfl_u64(unsigned long long v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}

template <typename OffT>
__global__ void __launch_bounds__(kBcThreads) bc_forward_kernel(
    uint32_t V, const OffT* __restrict__ off, const uint32_t* __restrict__ col,
    const unsigned long long* __restrict__ front_cur, unsigned long long* __restrict__ front_nxt,
    unsigned long long* __restrict__ visited, unsigned long long* __restrict__ sigma, uint32_t* __restrict__ dist,
    unsigned long long full, uint32_t level, unsigned int* __restrict__ flags) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = (uint64_t)gridDim.x * (kBcThreads / 32);
  bool any_ovf = false;
  for (uint64_t w = blockIdx.x * (uint64_t)(kBcThreads / 32) + (threadIdx.x >> 5); w < V; w += nwarps) {
    const unsigned long long vis = visited[w];
    const unsigned long long cand = full & ~vis;
    unsigned long long newmask = 0;
    if (cand) {
      const OffT b = __ldg(off + w), e = __ldg(off + w + 1);
      unsigned long long acc0 = 0, acc1 = 0;
      bool got0 = false, got1 = false;
      for (OffT j0 = b; j0 < e; j0 += 32) {
        const OffT j = j0 + lane;
        uint32_t v = 0;
        unsigned long long m = 0;
        if (j < e) {
          v = __ldg(col + j);
          m = __ldg(front_cur + v) & cand;
        }
        unsigned bal = __ballot_sync(0xffffffffu, m != 0);
        while (bal) {
          const int k = __ffs(bal) - 1;
          bal &= bal - 1;
          const uint32_t vk = __shfl_sync(0xffffffffu, v, k);
          const unsigned long long mk = shfl_u64(m, k);
          if ((mk >> lane) & 1ull) {
            const unsigned long long s = sigma[(uint64_t)vk * kBcBatch + lane];
            const unsigned long long n = acc0 + s;
            any_ovf |= n < acc0;
            acc0 = n;
            got0 = true;
          }
          if ((mk >> (lane + 32)) & 1ull) {
            const unsigned long long s = sigma[(uint64_t)vk * kBcBatch + lane + 32];
            const unsigned long long n = acc1 + s;
            any_ovf |= n < acc1;
            acc1 = n;
            got1 = true;
          }
        }
      }
      newmask = (unsigned long long)__ballot_sync(0xffffffffu, got0) |
                ((unsigned long long)__ballot_sync(0xffffffffu, got1) << 32);
      if (got0) {
        sigma[w * kBcBatch + lane] = acc0;
        dist[w * kBcBatch + lane] = level + 1;
      }
      if (got1) {
        sigma[w * kBcBatch + lane + 32] = acc1;
        dist[w * kBcBatch + lane + 32] = level + 1;
      }
    }
    if (lane == 0) {
      front_nxt[w] = newmask;
      if (newmask) {
        visited[w] = vis | newmask;
        flags[0] = 1u;
      }
    }
  }
  if (__any_sync(0xffffffffu, any_ovf) && lane == 0) flags[1] = 1u;
}

template <typename OffT>
__global__ void __launch_bounds__(kBcThreads) bc_backward_kernel(
    uint32_t V, const OffT* __restrict__ off, const uint32_t* __restrict__ col,
    const unsigned long long* __restrict__ mask_nxt, unsigned long long* __restrict__ mask_cur,
    const uint32_t* __restrict__ dist, const unsigned long long* __restrict__ sigma, double* __restrict__ q,
    double* __restrict__ bc, uint32_t level, int last_level) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = (uint64_t)gridDim.x * (kBcThreads / 32);
  for (uint64_t v = blockIdx.x * (uint64_t)(kBcThreads / 32) + (threadIdx.x >> 5); v < V; v += nwarps) {
    const bool a0 = dist[v * kBcBatch + lane] == level;
    const bool a1 = dist[v * kBcBatch + lane + 32] == level;
    const unsigned long long act =
        (unsigned long long)__ballot_sync(0xffffffffu, a0) | ((unsigned long long)__ballot_sync(0xffffffffu, a1) << 32);
    if (lane == 0) mask_cur[v] = act;
    if (!act) continue;
    double acc0 = 0.0, acc1 = 0.0;
    if (!last_level) {
      const OffT b = __ldg(off + v), e = __ldg(off + v + 1);
      for (OffT j0 = b; j0 < e; j0 += 32) {
        const OffT j = j0 + lane;
        uint32_t w = 0;
        unsigned long long g = 0;
        if (j < e) {
          w = __ldg(col + j);
          g = __ldg(mask_nxt + w) & act;
        }
        unsigned bal = __ballot_sync(0xffffffffu, g != 0);
        while (bal) {
          const int k = __ffs(bal) - 1;
          bal &= bal - 1;
          const uint32_t wk = __shfl_sync(0xffffffffu, w, k);
          const unsigned long long gk = shfl_u64(g, k);
          if ((gk >> lane) & 1ull) acc0 += q[(uint64_t)wk * kBcBatch + lane];
          if ((gk >> (lane + 32)) & 1ull) acc1 += q[(uint64_t)wk * kBcBatch + lane + 32];
        }
      }
    }
    double dsum = 0.0;
    if (a0) {
      const double sv = (double)sigma[v * kBcBatch + lane];
      const double d = __dmul_rn(sv, acc0);
      q[v * kBcBatch + lane] = __ddiv_rn(1.0 + d, sv);
      dsum += d;
    }
    if (a1) {
      const double sv = (double)sigma[v * kBcBatch + lane + 32];
      const double d = __dmul_rn(sv, acc1);
      q[v * kBcBatch + lane + 32] = __ddiv_rn(1.0 + d, sv);
      dsum += d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
    if (lane == 0) bc[v] += dsum;
  }
}

__global__ void bc_seed_kernel(const uint32_t* __restrict__ sources, int nb, unsigned long long* visited,
                               unsigned long long* front, unsigned long long* sigma, uint32_t* dist) {
  const int b = threadIdx.x;
  if (b < nb) {
    const uint64_t s = sources[b];
    atomicOr(visited + s, 1ull << b);
    atomicOr(front + s, 1ull << b);
    sigma[s * kBcBatch + b] = 1ull;
    dist[s * kBcBatch + b] = 0u;
  }
}

static int bc_grid(uint32_t V) {
  const uint64_t warps = V;
  uint64_t blocks = (warps + (kBcThreads / 32) - 1) / (kBcThreads / 32);
  const uint64_t cap = (uint64_t)sm_count() * (2048 / kBcThreads) * 4;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

struct BcWork {
  DevBuf visited, fa, fb, sigma, dist, q, flags, src;
  int alloc(uint32_t V, uint64_t ns, cudaStream_t s, bool need_q) {
    const size_t Vs = std::max<uint32_t>(V, 1);
    ZOGCU_TRY(visited.alloc(Vs * 8, s));
    ZOGCU_TRY(fa.alloc(Vs * 8, s));
    ZOGCU_TRY(fb.alloc(Vs * 8, s));
    ZOGCU_TRY(sigma.alloc(Vs * 8 * kBcBatch, s));
    ZOGCU_TRY(dist.alloc(Vs * 4 * kBcBatch, s));
    if (need_q) ZOGCU_TRY(q.alloc(Vs * 8 * kBcBatch, s));
    ZOGCU_TRY(flags.alloc(16, s));
    ZOGCU_TRY(src.alloc(std::max<uint64_t>(ns, 1) * 4, s));
    return ZOGCU_OK;
  }
};

// Forward phase of one batch; returns the deepest level reached in *depth.
template <typename OffT>
static int bc_forward_batch(const Graph* g, const OffT* in_off, BcWork& W, uint64_t first, int nb,
                            cudaStream_t s, uint32_t* depth, bool* overflow, uint64_t* launches,
                            unsigned int* h_flags) {
  const uint32_t V = g->V;
  const int grid = bc_grid(V);
  const unsigned long long full = nb == 64 ? ~0ull : ((1ull << nb) - 1);
  ZOGCU_CUDA(cudaMemsetAsync(W.visited.ptr, 0, (size_t)V * 8, s));
  ZOGCU_CUDA(cudaMemsetAsync(W.fa.ptr, 0, (size_t)V * 8, s));
  ZOGCU_CUDA(cudaMemsetAsync(W.dist.ptr, 0xFF, (size_t)V * 4 * kBcBatch, s));
  ZOGCU_CUDA(cudaMemsetAsync(W.flags.ptr, 0, 16, s));
  bc_seed_kernel<<<1, 64, 0, s>>>(W.src.as<uint32_t>() + first, nb, W.visited.as<unsigned long long>(),
                                  W.fa.as<unsigned long long>(), W.sigma.as<unsigned long long>(),
                                  W.dist.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  *launches += 1;
  unsigned long long* cur = W.fa.as<unsigned long long>();
  unsigned long long* nxt = W.fb.as<unsigned long long>();
  uint32_t level = 0;
  for (;;) {
    ZOGCU_CUDA(cudaMemsetAsync(W.flags.ptr, 0, 4, s));
    bc_forward_kernel<OffT><<<grid, kBcThreads, 0, s>>>(V, in_off, g->in_col.as<uint32_t>(), cur, nxt,
                                                        W.visited.as<unsigned long long>(),
                                                        W.sigma.as<unsigned long long>(), W.dist.as<uint32_t>(),
                                                        full, level, W.flags.as<unsigned int>());
    ZOGCU_CUDA(cudaGetLastError());
    *launches += 1;
    ZOGCU_CUDA(cudaMemcpyAsync(h_flags, W.flags.ptr, 8, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    if (h_flags[1]) *overflow = true;
    if (!h_flags[0]) break;
    ++level;
    std::swap(cur, nxt);
  }
  *depth = level;
  return ZOGCU_OK;
}

template <typename OffT>
static int run_betweenness(Graph* g, const OffT* in_off, const OffT* out_off, const std::vector<uint32_t>& sources,
                           double* d_bc, cudaStream_t s, zogcu_stats* stats) {
  const uint32_t V = g->V;
  const uint64_t ns = sources.size();
  BcWork W;
  ZOGCU_TRY(W.alloc(V, ns, s, true));
  if (ns) ZOGCU_CUDA(cudaMemcpyAsync(W.src.ptr, sources.data(), ns * 4, cudaMemcpyHostToDevice, s));
  unsigned int* h_flags = nullptr;
  ZOGCU_CUDA(cudaMallocHost(&h_flags, 16));
  struct HostFree {
    unsigned int* p;
    ~HostFree() { cudaFreeHost(p); }
  } hf{h_flags};
  const int grid = bc_grid(V);
  bool overflow = false;
  uint32_t max_depth = 0;
  uint64_t launches = 0;
  for (uint64_t first = 0; first < ns; first += kBcBatch) {
    const int nb = (int)std::min<uint64_t>(kBcBatch, ns - first);
    uint32_t depth = 0;
    ZOGCU_TRY(bc_forward_batch<OffT>(g, in_off, W, first, nb, s, &depth, &overflow, &launches, h_flags));
    max_depth = std::max(max_depth, depth);
    // backward: levels depth .. 1 (the sources sit at level 0 and are excluded)
    unsigned long long* mnxt = W.fa.as<unsigned long long>();
    unsigned long long* mcur = W.fb.as<unsigned long long>();
    ZOGCU_CUDA(cudaMemsetAsync(mnxt, 0, (size_t)V * 8, s));
    for (uint32_t l = depth; l >= 1; --l) {
      bc_backward_kernel<OffT><<<grid, kBcThreads, 0, s>>>(V, out_off, g->out_col.as<uint32_t>(), mnxt, mcur,
                                                           W.dist.as<uint32_t>(), W.sigma.as<unsigned long long>(),
                                                           W.q.as<double>(), d_bc, l, l == depth ? 1 : 0);
      ZOGCU_CUDA(cudaGetLastError());
      ++launches;
      std::swap(mnxt, mcur);
    }
  }
  if (stats) {
    stats->sources = ns;
    stats->max_depth = max_depth;
    stats->sigma_overflow = overflow ? 1u : 0u;
    stats->launches = launches;
  }
  return ZOGCU_OK;
}

static std::vector<uint32_t> live_sources(Graph* g) {
  std::vector<uint32_t> src;
  if (!g->has_deleted) {
    src.resize(g->V);
    for (uint32_t v = 0; v < g->V; ++v) src[v] = v;
    return src;
  }
  std::vector<uint32_t> deg(g->V);
  cudaMemcpy(deg.data(), g->out_deg.ptr, (size_t)g->V * 4, cudaMemcpyDeviceToHost);
  for (uint32_t v = 0; v < g->V; ++v)
    if (deg[v] != kDeletedDegree) src.push_back(v);
  return src;
}

}  // namespace zogcu

using namespace zogcu;

extern "C" {

int zogcu_betweenness_unweighted_ex(zogcu_graph* G, const zogcu_bc_opts* opts, double* out_scores,
                                    zogcu_stats* stats) {
  if (!G) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graph is null");
  if (opts && opts->struct_size != sizeof(zogcu_bc_opts))
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "zogcu_bc_opts.struct_size mismatch");
  Graph* g = &G->g;
  const uint32_t V = g->V;
  if (!out_scores && V) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out_scores is null");
  ZOGCU_CUDA(cudaSetDevice(g->device));
  if (stats) std::memset(stats, 0, sizeof(*stats));
  std::vector<uint32_t> sources;
  if (opts && opts->sources) {
    sources.assign(opts->sources, opts->sources + opts->num_sources);
    for (uint32_t s : sources)
      if (s >= V) return fail(ZOGCU_ERR_NODE_NOT_FOUND, "source id >= node capacity");
  } else {
    sources = live_sources(g);
  }
  const bool dev_out = opts && opts->device_pointers;
  StreamGuard sg;
  ZOGCU_TRY(sg.init(opts ? opts->stream : nullptr));
  DevBuf bc;
  ZOGCU_TRY(bc.alloc((size_t)std::max<uint32_t>(V, 1) * 8, sg.s));
  ZOGCU_CUDA(cudaMemsetAsync(bc.ptr, 0, (size_t)std::max<uint32_t>(V, 1) * 8, sg.s));
  EventTimer tm;
  ZOGCU_TRY(tm.start(sg.s));
  if (V) {
    if (g->offsets32)
      ZOGCU_TRY(run_betweenness<uint32_t>(g, g->in_off32.as<uint32_t>(), g->out_off32.as<uint32_t>(), sources,
                                          bc.as<double>(), sg.s, stats));
    else
      ZOGCU_TRY(run_betweenness<uint64_t>(g, g->in_off64.as<uint64_t>(), g->out_off64.as<uint64_t>(), sources,
                                          bc.as<double>(), sg.s, stats));
  }
  ZOGCU_TRY(tm.stop(sg.s));
  if (V)
    ZOGCU_CUDA(cudaMemcpyAsync(out_scores, bc.ptr, (size_t)V * 8,
                               dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, sg.s));
  ZOGCU_CUDA(cudaStreamSynchronize(sg.s));
  if (stats) stats->elapsed_ms = tm.ms();
  return ZOGCU_OK;
}

int zogcu_betweenness_unweighted(zogcu_graph* G, double* out_scores, zogcu_stats* stats) {
  return zogcu_betweenness_unweighted_ex(G, nullptr, out_scores, stats);
}

int zogcu_bfs_sigma(zogcu_graph* G, const uint32_t* sources, uint64_t num_sources, uint32_t* dist_out,
                    uint64_t* sigma_out, uint32_t* overflow) {
  if (!G) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graph is null");
  if (num_sources && !sources) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "sources is null");
  Graph* g = &G->g;
  const uint32_t V = g->V;
  for (uint64_t i = 0; i < num_sources; ++i)
    if (sources[i] >= V) return fail(ZOGCU_ERR_NODE_NOT_FOUND, "source id >= node capacity");
  ZOGCU_CUDA(cudaSetDevice(g->device));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(nullptr));
  BcWork W;
  ZOGCU_TRY(W.alloc(V, num_sources, sg.s, false));
  if (num_sources) ZOGCU_CUDA(cudaMemcpyAsync(W.src.ptr, sources, num_sources * 4, cudaMemcpyHostToDevice, sg.s));
  unsigned int* h_flags = nullptr;
  ZOGCU_CUDA(cudaMallocHost(&h_flags, 16));
  std::vector<uint32_t> hd((size_t)V * kBcBatch);
  std::vector<unsigned long long> hs((size_t)V * kBcBatch);
  bool ovf = false;
  uint64_t launches = 0;
  int rc = ZOGCU_OK;
  for (uint64_t first = 0; first < num_sources && rc == ZOGCU_OK; first += kBcBatch) {
    const int nb = (int)std::min<uint64_t>(kBcBatch, num_sources - first);
    uint32_t depth = 0;
    rc = g->offsets32 ? bc_forward_batch<uint32_t>(g, g->in_off32.as<uint32_t>(), W, first, nb, sg.s, &depth, &ovf,
                                                   &launches, h_flags)
                      : bc_forward_batch<uint64_t>(g, g->in_off64.as<uint64_t>(), W, first, nb, sg.s, &depth, &ovf,
                                                   &launches, h_flags);
    if (rc != ZOGCU_OK) break;
    if (cudaMemcpy(hd.data(), W.dist.ptr, hd.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hs.data(), W.sigma.ptr, hs.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = fail(ZOGCU_ERR_CUDA, "copy of BFS state failed");
      break;
    }
    for (int b = 0; b < nb; ++b) {
      for (uint32_t v = 0; v < V; ++v) {
        const uint32_t d = hd[(size_t)v * kBcBatch + b];
        if (dist_out) dist_out[(first + b) * V + v] = d;
        if (sigma_out) sigma_out[(first + b) * V + v] = (d == kUnreached) ? 0ull : hs[(size_t)v * kBcBatch + b];
      }
    }
  }
  cudaFreeHost(h_flags);
  if (overflow) *overflow = ovf ? 1u : 0u;
  return rc;
}

}  // extern "C"
