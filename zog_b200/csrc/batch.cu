// batch.cu -- PageRank of many graphs of uneven sizes in one persistent launch.
//
// Each graph is solved exactly as zogcu_pagerank solves it alone
// (priv/zog/src/centrality.zig:858-965: uniform start, sink = sum over
// dangling nodes of x/n, x' = (1-d)/n + d (sink + sum_{u in in(v)} x[u]/deg(u)),
// stop once the L1 step is below tol, the returned vector is the last one
// computed; n = 0 gives zeros and n = 1 gives 1.0 without iterating).
//
// B200 design:
//   * a batch concatenates the graphs' device CSRs once (local 32-bit
//     offsets and node ids, plus a per-graph descriptor);
//   * one persistent kernel: thread-block clusters take whole graphs from a
//     queue (largest first) and run every power iteration of a graph inside
//     the cluster.  The cluster's CTAs split the rows; after each iteration
//     they reduce the L1 step and the next sink through distributed shared
//     memory (fixed order, so every CTA sees the same totals and takes the
//     same branch) and meet at the hardware cluster barrier, which also makes
//     the iteration's global writes visible to the whole cluster.  There are
//     no spin-waits and no inter-cluster dependencies;
//   * degree-binned rows: rows of in-degree <= T are summed by one thread in
//     the reference's ascending order; longer rows by a warp (lanes stride the
//     arcs, shuffle tree);
//   * the CTA size, cluster size and bin threshold T are chosen by an
//     autotuner that times the candidates on the batch itself (first call;
//     ZOGCU_BATCH_CONFIG forces one), and the chosen launch (queue reset +
//     persistent kernel) is captured once in a CUDA graph and replayed.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>
#include <tuple>
#include <vector>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace zogcu {
namespace {

// Degree bins: rows of in-degree <= kBins[b] are summed by one thread; the
// longer rows of every graph are listed per bin (built at batch creation).
constexpr uint32_t kBins[] = {8, 16, 32};
constexpr int kNumBins = 3;

struct BatchGraph {
  uint64_t off_base;   // first offset of this graph in the concatenated offsets (V+1 entries)
  uint64_t col_base;   // first arc
  uint64_t node_base;  // node 0 of this graph in the node arrays
  uint32_t V;          // node capacity
  uint32_t n_live;
  uint64_t long_base[kNumBins];  // first entry of this graph's long rows, per bin
  uint32_t n_long[kNumBins];
  uint32_t pad;
};

struct BatchConfig {
  int threads;   // CTA size
  int cluster;   // CTAs per cluster (one graph at a time per cluster)
  int bin;       // index into kBins
};
constexpr BatchConfig kBatchConfigs[] = {
    {512, 1, 1}, {1024, 1, 1}, {1024, 2, 1}, {1024, 4, 1}, {512, 4, 0}, {1024, 8, 2},
};
constexpr int kNumBatchConfigs = sizeof(kBatchConfigs) / sizeof(kBatchConfigs[0]);

struct BatchArgs {
  const BatchGraph* graphs;
  const uint32_t* order;  // graph ids, largest first
  uint32_t count;
  const uint32_t* off;    // local in-CSR offsets
  const uint32_t* col;    // local source ids (ascending per row)
  const uint32_t* deg;    // out-degree, kDeletedDegree on deleted slots
  double* xa;
  double* xb;
  double* ca;
  double* cb;
  double* out;            // result, concatenated node order
  uint64_t* iters;        // per graph
  double* resid;          // per graph
  uint32_t* next;         // queue head
  const uint32_t* long_rows;  // rows above the bin, per graph (local ids)
  double damping;
  uint64_t max_iter;
  double tol;
  uint32_t bin;           // in-degree bound of the one-thread rows
  int bin_index;
};

// Sum of (a, b) over the CTA, then over the cluster, in a fixed order; every
// thread of every CTA of the cluster returns the same totals.  Ends with the
// cluster barrier, so writes made before the call are visible cluster-wide.
template <int THREADS>
__device__ __forceinline__ void cluster_sum2(double& a, double& b, double (*s_warp)[2], double* s_part) {
  cg::cluster_group cluster = cg::this_cluster();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    s_warp[warp][0] = a;
    s_warp[warp][1] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int w = 0; w < THREADS / 32; ++w) {
      ta += s_warp[w][0];
      tb += s_warp[w][1];
    }
    s_part[0] = ta;
    s_part[1] = tb;
  }
  cluster.sync();
  const unsigned n = cluster.num_blocks();
  double ta = 0.0, tb = 0.0;
  for (unsigned r = 0; r < n; ++r) {
    const double* p = cluster.map_shared_rank(s_part, r);
    ta += p[0];
    tb += p[1];
  }
  a = ta;
  b = tb;
  cluster.sync();  // every CTA has read the partials before they change
}

template <bool MULTI>
__device__ __forceinline__ double ld_shared_vec(const double* p);

// x' for row v from its in-sum s; accumulates |x' - x| and the dangling mass.
template <bool MULTI>
__device__ __forceinline__ void pr_epilogue(const BatchArgs& A, uint64_t node, uint32_t deg, double s, double tele,
                                            double sink, double n_f, const double* x, double* xn, double* cn,
                                            double& l1, double& dang) {
  const double v = __dadd_rn(tele, __dmul_rn(A.damping, __dadd_rn(sink, s)));
  l1 += fabs(v - ld_shared_vec<MULTI>(x + node));
  xn[node] = v;
  if (deg == 0) {
    cn[node] = 0.0;
    dang += __ddiv_rn(v, n_f);
  } else {
    cn[node] = __ddiv_rn(v, (double)deg);
  }
}

// Loads of x and c, which other CTAs of the cluster wrote in the previous
// iteration, go to L2 (ld.global.cg) when the cluster has several CTAs.
template <bool MULTI>
__device__ __forceinline__ double ld_shared_vec(const double* p) {
  if (MULTI) return __ldcg(p);
  return *p;
}

template <int THREADS, bool MULTI>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_batch_pagerank(BatchArgs A) {
  cg::cluster_group cluster = cg::this_cluster();
  const unsigned crank = cluster.block_rank(), ncta = cluster.num_blocks();
  __shared__ uint32_t s_gi;
  __shared__ double s_warp[THREADS / 32][2];
  __shared__ double s_part[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t tid = crank * THREADS + threadIdx.x;  // thread index within the cluster
  const uint32_t nthreads = ncta * THREADS;
  const uint32_t gwarp = crank * (THREADS / 32) + warp, nwarps = ncta * (THREADS / 32);
  for (;;) {
    if (crank == 0 && threadIdx.x == 0) s_gi = atomicAdd(A.next, 1u);
    cluster.sync();
    const uint32_t gi = *cluster.map_shared_rank(&s_gi, 0);
    cluster.sync();  // every CTA has read the index before rank 0 takes the next
    if (gi >= A.count) break;
    const uint32_t gid = A.order[gi];
    const BatchGraph G = A.graphs[gid];
    const uint32_t* off = A.off + G.off_base;
    const uint32_t* col = A.col + G.col_base;
    const uint32_t* deg = A.deg + G.node_base;
    double* out = A.out + G.node_base;
    const uint32_t V = G.V;
    const uint32_t* longs = A.long_rows + G.long_base[A.bin_index];
    const uint32_t n_long = G.n_long[A.bin_index];
    if (G.n_live <= 1) {  // centrality.zig:875-879
      for (uint32_t v = tid; v < V; v += nthreads) out[v] = (G.n_live == 1 && deg[v] != kDeletedDegree) ? 1.0 : 0.0;
      if (tid == 0) {
        A.iters[gid] = 0;
        A.resid[gid] = 0.0;
      }
      continue;
    }
    const double n_f = (double)G.n_live;
    const double x_init = 1.0 / n_f;
    const double tele = (1.0 - A.damping) / n_f;
    double* xc = A.xa + G.node_base;
    double* xn = A.xb + G.node_base;
    double* cc = A.ca + G.node_base;
    double* cn = A.cb + G.node_base;
    // uniform start (centrality.zig:912-918); contributions c = x/deg
    double l1 = 0.0, sink = 0.0;
    for (uint32_t v = tid; v < V; v += nthreads) {
      const uint32_t d = deg[v];
      double x = 0.0, c = 0.0;
      if (d != kDeletedDegree) {
        x = x_init;
        if (d == 0) sink += __ddiv_rn(x, n_f);
        else c = __ddiv_rn(x, (double)d);
      }
      xc[v] = x;
      cc[v] = c;
    }
    cluster_sum2<THREADS>(l1, sink, s_warp, s_part);
    uint64_t it = 0;
    l1 = 0.0;
    while (it < A.max_iter) {
      double l1p = 0.0, dang = 0.0;
      // short rows: one thread each, arcs in the reference's order
      for (uint32_t v = tid; v < V; v += nthreads) {
        const uint32_t d = deg[v];
        if (d == kDeletedDegree) {
          xn[v] = 0.0;
          cn[v] = 0.0;
          continue;
        }
        const uint32_t b = off[v], e = off[v + 1];
        if (e - b > A.bin) continue;
        double s = 0.0;
#pragma unroll 4
        for (uint32_t j = b; j < e; ++j) s = __dadd_rn(s, ld_shared_vec<MULTI>(cc + col[j]));
        pr_epilogue<MULTI>(A, v, d, s, tele, sink, n_f, xc, xn, cn, l1p, dang);
      }
      // long rows (listed at batch creation): one warp each
      for (uint32_t k = gwarp; k < n_long; k += nwarps) {
        const uint32_t v = longs[k];
        const uint32_t b = off[v], e = off[v + 1];
        const uint32_t d = deg[v];
        double s = 0.0;
        for (uint32_t j = b + lane; j < e; j += 32) s += ld_shared_vec<MULTI>(cc + col[j]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) pr_epilogue<MULTI>(A, v, d, s, tele, sink, n_f, xc, xn, cn, l1p, dang);
      }
      cluster_sum2<THREADS>(l1p, dang, s_warp, s_part);
      l1 = l1p;
      sink = dang;
      double* t = xc;
      xc = xn;
      xn = t;
      t = cc;
      cc = cn;
      cn = t;
      ++it;
      if (l1 < A.tol) break;  // centrality.zig:957, after the swap
    }
    for (uint32_t v = tid; v < V; v += nthreads) out[v] = ld_shared_vec<MULTI>(xc + v);
    if (tid == 0) {
      A.iters[gid] = it;
      A.resid[gid] = l1;
    }
  }
}

}  // namespace
}  // namespace zogcu

using namespace zogcu;

struct zogcu_batch {
  int device = 0;
  uint32_t count = 0;
  uint64_t total_nodes = 0, total_arcs = 0;
  std::vector<uint64_t> node_offsets;  // count + 1
  std::vector<uint32_t> nodes_of;      // node capacity of each graph
  std::vector<uint64_t> arcs_of;       // stored arcs of each graph
  int grid_clusters[16] = {0};         // persistent grid of each configuration (clusters)
  DevArray graphs, order, off, col, deg;
  DevArray xa, xb, ca, cb, out, iters, resid, next, long_rows;
  int config = -1;
  std::mutex mu;
  // CUDA graphs of the persistent launch, by (config, damping, max_iter, tol)
  std::map<std::tuple<int, double, uint64_t, double>, cudaGraphExec_t> execs;
  ~zogcu_batch() {
    for (auto& kv : execs) cudaGraphExecDestroy(kv.second);
  }
};

namespace zogcu {
namespace {

// Launches the persistent kernel with `cluster` CTAs per cluster (query = the
// number of co-resident clusters is computed into *clusters instead; it is
// done once per configuration, outside any stream capture).
template <int THREADS>
int launch_batch(zogcu_batch* B, const BatchArgs& A, int cluster, int* clusters, bool query, cudaStream_t s) {
  auto kern = cluster > 1 ? k_batch_pagerank<THREADS, true> : k_batch_pagerank<THREADS, false>;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(cluster);
  if (query) {
    int n = 0;
    ZOGCU_CUDA(cudaOccupancyMaxActiveClusters(&n, kern, &cfg));
    if (n < 1) return fail(ZOGCU_ERR_CUDA, "batched PageRank: no cluster fits on the device");
    // persistent grid: every co-resident cluster, but no more clusters than graphs
    *clusters = std::min<int>(n, (int)std::max<uint32_t>(B->count, 1));
    return ZOGCU_OK;
  }
  cfg.gridDim = dim3(*clusters * cluster);
  ZOGCU_CUDA(cudaMemsetAsync(B->next.ptr, 0, 4, s));
  ZOGCU_CUDA(cudaLaunchKernelEx(&cfg, kern, A));
  return ZOGCU_OK;
}

int launch_config(zogcu_batch* B, const BatchArgs& A0, int c, cudaStream_t s) {
  BatchArgs A = A0;
  A.bin_index = kBatchConfigs[c].bin;
  A.bin = kBins[A.bin_index];
  const int cl = kBatchConfigs[c].cluster;
  for (int pass = B->grid_clusters[c] > 0 ? 1 : 0; pass < 2; ++pass) {
    const bool query = pass == 0;
    switch (kBatchConfigs[c].threads) {
      case 512: ZOGCU_TRY(launch_batch<512>(B, A, cl, &B->grid_clusters[c], query, s)); break;
      case 1024: ZOGCU_TRY(launch_batch<1024>(B, A, cl, &B->grid_clusters[c], query, s)); break;
      default: return fail(ZOGCU_ERR_INTERNAL, "bad batch configuration");
    }
  }
  return ZOGCU_OK;
}

// Sizes every configuration's persistent grid (outside stream capture).
int size_grids(zogcu_batch* B) {
  for (int c = 0; c < kNumBatchConfigs; ++c) {
    if (B->grid_clusters[c] > 0) continue;
    BatchArgs A{};
    const int cl = kBatchConfigs[c].cluster;
    switch (kBatchConfigs[c].threads) {
      case 512: ZOGCU_TRY(launch_batch<512>(B, A, cl, &B->grid_clusters[c], true, nullptr)); break;
      case 1024: ZOGCU_TRY(launch_batch<1024>(B, A, cl, &B->grid_clusters[c], true, nullptr)); break;
      default: return fail(ZOGCU_ERR_INTERNAL, "bad batch configuration");
    }
  }
  return ZOGCU_OK;
}

BatchArgs batch_args(zogcu_batch* B, double damping, uint64_t max_iter, double tol) {
  BatchArgs A{};
  A.graphs = B->graphs.as<BatchGraph>();
  A.order = B->order.as<uint32_t>();
  A.count = B->count;
  A.off = B->off.as<uint32_t>();
  A.col = B->col.as<uint32_t>();
  A.deg = B->deg.as<uint32_t>();
  A.xa = B->xa.as<double>();
  A.xb = B->xb.as<double>();
  A.ca = B->ca.as<double>();
  A.cb = B->cb.as<double>();
  A.out = B->out.as<double>();
  A.iters = B->iters.as<uint64_t>();
  A.resid = B->resid.as<double>();
  A.next = B->next.as<uint32_t>();
  A.long_rows = B->long_rows.as<uint32_t>();
  A.damping = damping;
  A.max_iter = max_iter;
  A.tol = tol;
  return A;
}

// Times every configuration on the batch itself (a few fixed iterations,
// tol 0) and keeps the fastest; ZOGCU_BATCH_CONFIG forces one.
int batch_autotune(zogcu_batch* B, double damping, cudaStream_t s) {
  if (B->config >= 0) return ZOGCU_OK;
  if (const char* e = std::getenv("ZOGCU_BATCH_CONFIG")) {
    const int c = std::atoi(e);
    if (c >= 0 && c < kNumBatchConfigs) {
      B->config = c;
      return ZOGCU_OK;
    }
  }
  EventTimer tm;
  float best = 1e30f;
  int best_c = 1;
  const BatchArgs A = batch_args(B, damping, 4, 0.0);
  for (int c = 0; c < kNumBatchConfigs; ++c) {
    ZOGCU_TRY(launch_config(B, A, c, s));  // warm-up
    ZOGCU_TRY(tm.start(s));
    ZOGCU_TRY(launch_config(B, A, c, s));
    ZOGCU_TRY(tm.stop(s));
    const float ms = tm.ms();
    if (ms > 0.f && ms < best) {
      best = ms;
      best_c = c;
    }
  }
  B->config = best_c;
  return ZOGCU_OK;
}

}  // namespace
}  // namespace zogcu

extern "C" {

int zogcu_batch_create(zogcu_graph* const* graphs, uint32_t count, zogcu_batch** out) {
  if (!out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  if (count && !graphs) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graphs is null");
  int dev;
  ZOGCU_TRY(ensure_device(&dev));
  std::unique_ptr<zogcu_batch> B(new (std::nothrow) zogcu_batch());
  if (!B) return fail(ZOGCU_ERR_OUT_OF_MEMORY, "host allocation failed");
  B->device = dev;
  B->count = count;
  std::vector<BatchGraph> meta(count);
  uint64_t nodes = 0, arcs = 0, offs = 0;
  B->node_offsets.assign(1, 0);
  for (uint32_t i = 0; i < count; ++i) {
    if (!graphs[i]) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "a graph of the batch is null");
    const Graph& g = graphs[i]->g;
    if (g.device != dev) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "every graph of a batch must be on one device");
    if (!g.offsets32) return fail(ZOGCU_ERR_TOO_LARGE, "a graph of the batch has 2^32 or more arcs");
    meta[i] = BatchGraph{};
    meta[i].off_base = offs;
    meta[i].col_base = arcs;
    meta[i].node_base = nodes;
    meta[i].V = g.V;
    meta[i].n_live = (uint32_t)g.n_live;
    B->nodes_of.push_back(g.V);
    B->arcs_of.push_back(g.E);
    offs += (uint64_t)g.V + 1;
    arcs += g.E;
    nodes += g.V;
    B->node_offsets.push_back(nodes);
  }
  B->total_nodes = nodes;
  B->total_arcs = arcs;
  ZOGCU_TRY(B->graphs.alloc(std::max<size_t>(count, 1) * sizeof(BatchGraph)));
  ZOGCU_TRY(B->order.alloc(std::max<size_t>(count, 1) * 4));
  ZOGCU_TRY(B->off.alloc(std::max<uint64_t>(offs, 1) * 4));
  ZOGCU_TRY(B->col.alloc(std::max<uint64_t>(arcs, 1) * 4));
  ZOGCU_TRY(B->deg.alloc(std::max<uint64_t>(nodes, 1) * 4));
  for (DevArray* a : {&B->xa, &B->xb, &B->ca, &B->cb, &B->out}) ZOGCU_TRY(a->alloc(std::max<uint64_t>(nodes, 1) * 8));
  ZOGCU_TRY(B->iters.alloc(std::max<size_t>(count, 1) * 8));
  ZOGCU_TRY(B->resid.alloc(std::max<size_t>(count, 1) * 8));
  ZOGCU_TRY(B->next.alloc(16));
  for (uint32_t i = 0; i < count; ++i) {
    const Graph& g = graphs[i]->g;
    ZOGCU_CUDA(cudaMemcpy(B->off.as<uint32_t>() + meta[i].off_base, g.in_off32.ptr, ((size_t)g.V + 1) * 4,
                          cudaMemcpyDeviceToDevice));
    if (g.E)
      ZOGCU_CUDA(cudaMemcpy(B->col.as<uint32_t>() + meta[i].col_base, g.in_col.ptr, (size_t)g.E * 4,
                            cudaMemcpyDeviceToDevice));
    if (g.V)
      ZOGCU_CUDA(cudaMemcpy(B->deg.as<uint32_t>() + meta[i].node_base, g.out_deg.ptr, (size_t)g.V * 4,
                            cudaMemcpyDeviceToDevice));
  }
  // rows above each degree bin (live rows only), per graph
  {
    std::vector<uint32_t> h_off(offs), h_deg(nodes), longs;
    if (offs) ZOGCU_CUDA(cudaMemcpy(h_off.data(), B->off.ptr, offs * 4, cudaMemcpyDeviceToHost));
    if (nodes) ZOGCU_CUDA(cudaMemcpy(h_deg.data(), B->deg.ptr, nodes * 4, cudaMemcpyDeviceToHost));
    for (int b = 0; b < kNumBins; ++b)
      for (uint32_t i = 0; i < count; ++i) {
        meta[i].long_base[b] = longs.size();
        const uint32_t* o = h_off.data() + meta[i].off_base;
        const uint32_t* d = h_deg.data() + meta[i].node_base;
        for (uint32_t v = 0; v < meta[i].V; ++v)
          if (d[v] != kDeletedDegree && o[v + 1] - o[v] > kBins[b]) longs.push_back(v);
        meta[i].n_long[b] = (uint32_t)(longs.size() - meta[i].long_base[b]);
      }
    ZOGCU_TRY(B->long_rows.alloc(std::max<size_t>(longs.size(), 1) * 4));
    if (!longs.empty())
      ZOGCU_CUDA(cudaMemcpy(B->long_rows.ptr, longs.data(), longs.size() * 4, cudaMemcpyHostToDevice));
  }
  // largest graphs first, so the last graphs to start are the short ones
  std::vector<uint32_t> order(count);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    const uint64_t wa = meta[a].V + (uint64_t)graphs[a]->g.E, wb = meta[b].V + (uint64_t)graphs[b]->g.E;
    return wa > wb;
  });
  if (count) {
    ZOGCU_CUDA(cudaMemcpy(B->graphs.ptr, meta.data(), count * sizeof(BatchGraph), cudaMemcpyHostToDevice));
    ZOGCU_CUDA(cudaMemcpy(B->order.ptr, order.data(), count * 4, cudaMemcpyHostToDevice));
  }
  *out = B.release();
  return ZOGCU_OK;
}

int zogcu_batch_destroy(zogcu_batch* B) {
  if (!B) return ZOGCU_OK;
  cudaSetDevice(B->device);
  delete B;
  return ZOGCU_OK;
}

int zogcu_batch_info(const zogcu_batch* B, uint32_t* count, uint64_t* total_nodes, uint64_t* total_arcs,
                     uint64_t* node_offsets) {
  if (!B) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "batch is null");
  if (count) *count = B->count;
  if (total_nodes) *total_nodes = B->total_nodes;
  if (total_arcs) *total_arcs = B->total_arcs;
  if (node_offsets) std::memcpy(node_offsets, B->node_offsets.data(), B->node_offsets.size() * 8);
  return ZOGCU_OK;
}

int zogcu_batch_pagerank(zogcu_batch* B, double damping, uint64_t max_iterations, double tolerance,
                         const zogcu_batch_opts* opts, double* out_scores, uint64_t* iterations,
                         zogcu_stats* stats) {
  if (!B) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "batch is null");
  if (opts && opts->struct_size != sizeof(zogcu_batch_opts))
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "zogcu_batch_opts.struct_size mismatch");
  if (!out_scores && B->total_nodes) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out_scores is null");
  if (stats) std::memset(stats, 0, sizeof(*stats));
  std::lock_guard<std::mutex> lock(B->mu);
  ZOGCU_CUDA(cudaSetDevice(B->device));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(opts ? opts->stream : nullptr));
  const bool dev_ptrs = opts && opts->device_pointers;
  if (B->count == 0) return ZOGCU_OK;
  ZOGCU_TRY(size_grids(B));
  int cfg = opts && opts->config >= 0 && opts->config < kNumBatchConfigs ? opts->config : -1;
  if (cfg < 0) {
    ZOGCU_TRY(batch_autotune(B, damping, sg.s));
    cfg = B->config;
  }
  const BatchArgs A = batch_args(B, damping, max_iterations, tolerance);
  // the persistent launch as a CUDA graph, captured once per parameter set
  const auto key = std::make_tuple(cfg, damping, max_iterations, tolerance);
  auto it = B->execs.find(key);
  if (it == B->execs.end()) {
    cudaStream_t cap;
    ZOGCU_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    int rc = ZOGCU_OK;
    if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      rc = fail(ZOGCU_ERR_CUDA, "batched PageRank: stream capture failed to start");
    } else {
      rc = launch_config(B, A, cfg, cap);
      const cudaError_t e = cudaStreamEndCapture(cap, &graph);
      if (rc == ZOGCU_OK && e != cudaSuccess) rc = fail(ZOGCU_ERR_CUDA, "batched PageRank: stream capture failed");
    }
    cudaGraphExec_t exec = nullptr;
    if (rc == ZOGCU_OK && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
      rc = fail(ZOGCU_ERR_CUDA, "batched PageRank: graph instantiation failed");
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    if (rc != ZOGCU_OK) return rc;
    it = B->execs.emplace(key, exec).first;
  }
  EventTimer tm;
  ZOGCU_TRY(tm.start(sg.s));
  ZOGCU_CUDA(cudaGraphLaunch(it->second, sg.s));
  ZOGCU_TRY(tm.stop(sg.s));
  ZOGCU_CUDA(cudaMemcpyAsync(out_scores, B->out.ptr, B->total_nodes * 8,
                             dev_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, sg.s));
  std::vector<uint64_t> its(B->count);
  ZOGCU_CUDA(cudaMemcpyAsync(its.data(), B->iters.ptr, (size_t)B->count * 8, cudaMemcpyDeviceToHost, sg.s));
  ZOGCU_CUDA(cudaStreamSynchronize(sg.s));
  if (iterations) std::memcpy(iterations, its.data(), its.size() * 8);
  if (stats) {
    stats->iterations = its.empty() ? 0 : *std::max_element(its.begin(), its.end());
    stats->elapsed_ms = tm.ms();
    // per iteration of graph g: arc indices, offsets, and x / c reads and writes
    double bytes = 0.0;
    for (uint32_t g = 0; g < B->count; ++g)
      bytes += (double)its[g] * (4.0 * (double)B->arcs_of[g] + 4.0 * ((double)B->nodes_of[g] + 1) +
                                 36.0 * (double)B->nodes_of[g]);
    stats->bytes_moved = bytes;
    stats->launches = 1;
    stats->kernel_config = (uint32_t)cfg;
  }
  return ZOGCU_OK;
}

}  // extern "C"
