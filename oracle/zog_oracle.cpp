// zog_oracle.cpp -- CPU oracle for the PageRank and unweighted Brandes hot paths.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, loop for loop, the reference
// Zig code of code-shoily/zog so that the CUDA library (zog_b200/csrc) can be
// checked against it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load it; the CUDA product path never links or calls it.
//
// What is restated, with the reference lines each part follows:
//   * ArrayGraph(void, f64): SoA node/edge arrays, head-insertion adjacency,
//     tombstones, successor iteration      priv/zog/src/models/array_graph.zig:13-38,
//                                          :62-108 (addNode/addEdge), :110-146
//                                          (removeEdge/removeNode), :150-192
//                                          (successors), :206-213, :268-284
//   * collectNodes (ascending live ids)    priv/zog/src/utils.zig:42-48
//   * pagerank, ArrayGraph branch          priv/zog/src/centrality.zig:858-965
//   * betweennessUnweighted, ArrayGraph    priv/zog/src/centrality.zig:687-798
//   * extractScores (missing -> 0.0)       lib/zog/.Elixir.Zog.ResourceGraph.zig:72-80
//   * NIF graph build in list order        lib/zog/.Elixir.Zog.ResourceGraph.zig:26-35
//   * edge-list reader + addParsedEdges    lib/zog/.Elixir.Zog.ResourceGraph.zig:859-990
//
// Summation orders are kept exactly as in the Zig loops, and the file is built
// with -ffp-contract=off, so results equal the reference's bit for bit on the
// same graph (Zig's default float mode does not contract a*b+c either).
//
// Extensions used only to check the CUDA library (no reference counterpart):
//   * og_bfs: per-source dist / sigma intermediates (sigma kept as the
//     reference's wrapping usize, plus an overflow flag);
//   * og_betweenness_sources: the same per-source loop over a source subset;
//   * og_pagerank_csr / og_betweenness_csr_sources: the same hot loops driven
//     from CSR arrays, for graphs too large to hold as a linked-list ArrayGraph;
//   * og_pagerank_ext: the generalised iteration with a start vector and a
//     teleport vector (personalised PageRank), uniform dangling mass;
//   * og_rmat: the seeded R-MAT generator whose definition the CUDA generator
//     shares (counter-based SplitMix64; see rmat_edge below);
//   * og_betweenness_weighted: the weighted (Dijkstra) Brandes of
//     centrality.zig:528-682, restated loop for loop like the unweighted one;
//   * og_ba / og_ws: the seeded Barabasi-Albert and Watts-Strogatz generators
//     (generator.ex:132-253 models), written independently of the library's.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>

#include <omp.h>
#include <parallel/algorithm>

namespace {

constexpr uint32_t kNull = 0xFFFFFFFFu;  // stands for Zig's `null` in ?u32

// ---------------------------------------------------------------------------
// ArrayGraph(void, f64)            array_graph.zig:13-38
// ---------------------------------------------------------------------------
struct ArrayGraph {
  // nodes (MultiArrayList(Node)): first_edge ?u32, is_deleted bool
  std::vector<uint32_t> first_edge;
  std::vector<uint8_t> node_deleted;
  // edges (MultiArrayList(Edge)): to u32, data f64, next_edge ?u32, is_deleted
  std::vector<uint32_t> to;
  std::vector<double> data;
  std::vector<uint32_t> next_edge;
  std::vector<uint8_t> edge_deleted;
  size_t live_nodes = 0;
  size_t live_edges = 0;

  uint32_t add_node() {  // array_graph.zig:62-71
    uint32_t idx = (uint32_t)first_edge.size();
    first_edge.push_back(kNull);
    node_deleted.push_back(0);
    live_nodes += 1;
    return idx;
  }
  bool has_node(uint32_t id) const {  // array_graph.zig:210-213
    if (id >= first_edge.size()) return false;
    return !node_deleted[id];
  }
  int add_edge(uint32_t from, uint32_t t, double w) {  // array_graph.zig:88-108
    if (!has_node(from) || !has_node(t)) return -1;    // error.NodeNotFound
    uint32_t edge_idx = (uint32_t)to.size();
    uint32_t prev_first = first_edge[from];
    to.push_back(t);
    data.push_back(w);
    next_edge.push_back(prev_first);
    edge_deleted.push_back(0);
    first_edge[from] = edge_idx;  // head insertion
    live_edges += 1;
    return 0;
  }
  int remove_edge(uint32_t from, uint32_t t) {  // array_graph.zig:110-126
    if (!has_node(from) || !has_node(t)) return -1;
    uint32_t curr = first_edge[from];
    while (curr != kNull) {
      if (!edge_deleted[curr] && to[curr] == t) {
        edge_deleted[curr] = 1;
        live_edges -= 1;
      }
      curr = next_edge[curr];
    }
    return 0;
  }
  int remove_node(uint32_t id) {  // array_graph.zig:128-152
    if (!has_node(id)) return -1;
    node_deleted[id] = 1;
    live_nodes -= 1;
    uint32_t curr = first_edge[id];
    while (curr != kNull) {
      if (!edge_deleted[curr]) live_edges -= 1;
      edge_deleted[curr] = 1;
      curr = next_edge[curr];
    }
    for (size_t idx = 0; idx < to.size(); ++idx) {
      if (to[idx] == id && !edge_deleted[idx]) {
        edge_deleted[idx] = 1;
        live_edges -= 1;
      }
    }
    return 0;
  }
  size_t node_capacity() const { return first_edge.size(); }  // :206

  // SuccessorIterator.next (array_graph.zig:164-180): skips tombstoned edges
  // and edges whose destination node is deleted.
  template <class F>
  void for_each_successor(uint32_t id, F&& f) const {
    uint32_t idx = first_edge[id];
    while (idx != kNull) {
      uint32_t nxt = next_edge[idx];
      if (!edge_deleted[idx]) {
        uint32_t dest = to[idx];
        if (!node_deleted[dest]) f(dest);
      }
      idx = nxt;
    }
  }
  // the same walk, also handing over the edge's f64 data (the weight)
  template <class F>
  void for_each_successor_edge(uint32_t id, F&& f) const {
    uint32_t idx = first_edge[id];
    while (idx != kNull) {
      uint32_t nxt = next_edge[idx];
      if (!edge_deleted[idx]) {
        uint32_t dest = to[idx];
        if (!node_deleted[dest]) f(dest, data[idx]);
      }
      idx = nxt;
    }
  }
  // utils.collectNodes (utils.zig:42-48) via nodeIds (array_graph.zig:268-284)
  std::vector<uint32_t> collect_nodes() const {
    std::vector<uint32_t> nodes;
    nodes.reserve(live_nodes);
    for (size_t i = 0; i < first_edge.size(); ++i)
      if (!node_deleted[i]) nodes.push_back((uint32_t)i);
    return nodes;
  }
};

// ---------------------------------------------------------------------------
// pagerank, ArrayGraph branch      centrality.zig:858-965
// ---------------------------------------------------------------------------
void pagerank_arraygraph(const ArrayGraph& g, double damping, uint64_t max_iter,
                         double tol, double* out, uint64_t* iters_out,
                         double* l1_out) {
  const size_t V = g.node_capacity();
  std::vector<uint32_t> nodes = g.collect_nodes();
  const size_t n = nodes.size();
  for (size_t i = 0; i < V; ++i) out[i] = 0.0;  // extractScores: missing -> 0.0
  *iters_out = 0;
  *l1_out = 0.0;
  if (n == 0) return;                       // :875
  if (n == 1) { out[nodes[0]] = 1.0; return; }  // :876-879

  // in_neighbors (:881-899): appended while iterating nodes ascending, so each
  // list holds sources in ascending id order.
  std::vector<std::vector<uint32_t>> in_neighbors(V);
  for (uint32_t from : nodes)
    g.for_each_successor(from, [&](uint32_t t) { in_neighbors[t].push_back(from); });
  // out_degrees (:901-910)
  std::vector<uint64_t> out_degrees(V, 0);
  for (uint32_t node : nodes) g.for_each_successor(node, [&](uint32_t) { out_degrees[node] += 1; });

  const double n_f = (double)n;
  const double initial_rank = 1.0 / n_f;
  std::vector<double> ranks(V, 0.0), new_ranks(V, 0.0);
  for (uint32_t node : nodes) ranks[node] = initial_rank;  // :912-918

  uint64_t iteration = 0;
  double l1_norm = 0.0;
  while (iteration < max_iter) {  // :924-958
    double sink_sum = 0.0;
    for (uint32_t node : nodes)
      if (out_degrees[node] == 0) sink_sum += ranks[node] / n_f;
    for (uint32_t node : nodes) {
      double rank_sum = 0.0;
      for (uint32_t nb : in_neighbors[node]) {
        uint64_t deg = out_degrees[nb];
        if (deg > 0) rank_sum += ranks[nb] / (double)deg;
      }
      new_ranks[node] = (1.0 - damping) / n_f + damping * (sink_sum + rank_sum);
    }
    l1_norm = 0.0;
    for (uint32_t node : nodes) l1_norm += std::fabs(new_ranks[node] - ranks[node]);
    std::swap(ranks, new_ranks);
    iteration += 1;
    if (l1_norm < tol) break;
  }
  for (uint32_t node : nodes) out[node] = ranks[node];  // :960-964
  *iters_out = iteration;
  *l1_out = l1_norm;
}

// ---------------------------------------------------------------------------
// katz (centrality.zig:1190-1251) and alphaCentrality (:1262-1321): plain
// in-neighbour sums (buildInNeighbors order, utils.zig:52-74: sources
// ascending), L1 step, swap, stop when the step < tol.
// ---------------------------------------------------------------------------
void linear_centrality(const ArrayGraph& g, double alpha, double beta, double start, uint64_t max_iter,
                       double tol, double* out, uint64_t* iters_out, double* l1_out) {
  const size_t V = g.node_capacity();
  std::vector<uint32_t> nodes = g.collect_nodes();
  for (size_t i = 0; i < V; ++i) out[i] = 0.0;
  *iters_out = 0;
  *l1_out = 0.0;
  if (nodes.empty()) return;
  std::vector<std::vector<uint32_t>> in_nb(V);
  for (uint32_t from : nodes) g.for_each_successor(from, [&](uint32_t t) { in_nb[t].push_back(from); });
  std::vector<double> curr(V, 0.0), next(V, 0.0);
  for (uint32_t v : nodes) curr[v] = start;
  uint64_t it = 0;
  double l1 = 0.0;
  while (it < max_iter) {
    for (uint32_t v : nodes) {
      double sum = 0.0;
      for (uint32_t u : in_nb[v]) sum += curr[u];
      next[v] = alpha * sum + beta;  // beta = 0 for alpha centrality
    }
    l1 = 0.0;
    for (uint32_t v : nodes) l1 += std::fabs(next[v] - curr[v]);
    std::swap(curr, next);
    it += 1;
    if (l1 < tol) break;
  }
  for (uint32_t v : nodes) out[v] = curr[v];
  *iters_out = it;
  *l1_out = l1;
}

// eigenvector (centrality.zig:1050-1180): start 1 + i/1000 (i = position in
// the ascending live-node list), new = sum of in-neighbours, L2-normalise,
// degenerate zero vector -> uniform 1/sqrt(n), oscillation test against the
// vector two steps back (-> normalised average), stop when the L2 step < tol,
// else rotate; after max_iterations return the last vector.  The reference
// sums the squared norm in hash-map order; this restatement sums in node
// order.  *how: 0 = converged or max_iterations, 1 = oscillation, 2 = zero.
void eigenvector_arraygraph(const ArrayGraph& g, uint64_t max_iter, double tol, double* out,
                            uint64_t* iters_out, int* how) {
  const size_t V = g.node_capacity();
  std::vector<uint32_t> nodes = g.collect_nodes();
  const size_t n = nodes.size();
  for (size_t i = 0; i < V; ++i) out[i] = 0.0;
  *iters_out = 0;
  *how = 0;
  if (n <= 1) {
    for (uint32_t v : nodes) out[v] = 1.0;
    return;
  }
  std::vector<std::vector<uint32_t>> in_nb(V);
  for (uint32_t from : nodes) g.for_each_successor(from, [&](uint32_t t) { in_nb[t].push_back(from); });
  std::vector<double> curr(V, 0.0), pp(V, 0.0), nw(V, 0.0);
  bool have_pp = false;
  for (size_t i = 0; i < n; ++i) curr[nodes[i]] = 1.0 + (double)i / 1000.0;
  uint64_t it = 0;
  while (it < max_iter) {
    for (uint32_t v : nodes) {
      double sum = 0.0;
      for (uint32_t u : in_nb[v]) sum += curr[u];
      nw[v] = sum;
    }
    double l2 = 0.0;
    for (uint32_t v : nodes) l2 += nw[v] * nw[v];
    if (l2 > 0.0) {
      const double norm = std::sqrt(l2);
      for (uint32_t v : nodes) nw[v] /= norm;
    }
    if (l2 == 0.0) {
      const double u = 1.0 / std::sqrt((double)n);
      for (uint32_t v : nodes) out[v] = u;
      *iters_out = it + 1;
      *how = 2;
      return;
    }
    double d = 0.0;
    for (uint32_t v : nodes) d += (nw[v] - curr[v]) * (nw[v] - curr[v]);
    if (d > 0.0) d = std::sqrt(d);
    if (have_pp) {
      double d2 = 0.0;
      for (uint32_t v : nodes) d2 += (nw[v] - pp[v]) * (nw[v] - pp[v]);
      if (d2 > 0.0) d2 = std::sqrt(d2);
      if (d2 < tol) {
        double a2 = 0.0;
        for (uint32_t v : nodes) {
          out[v] = (nw[v] + curr[v]) / 2.0;
          a2 += out[v] * out[v];
        }
        if (a2 > 0.0) {
          const double an = std::sqrt(a2);
          for (uint32_t v : nodes) out[v] /= an;
        }
        *iters_out = it + 1;
        *how = 1;
        return;
      }
    }
    if (d < tol) {
      for (uint32_t v : nodes) out[v] = nw[v];
      *iters_out = it + 1;
      return;
    }
    std::swap(pp, curr);  // prev_prev <- curr
    std::swap(curr, nw);  // curr <- new
    have_pp = true;
    it += 1;
  }
  for (uint32_t v : nodes) out[v] = curr[v];
  *iters_out = it;
}

// ---------------------------------------------------------------------------
// betweenness (weighted, f64), ArrayGraph branch   centrality.zig:528-682
// (betweennessF64 :1355-1357: Weight = f64, zero = 0.0, add = a + b,
// compare = std.math.order).  The heap is a binary min-heap on the distance;
// the reference's std.PriorityQueue pops equal distances in its own order,
// which with positive weights changes only the summation order of delta.
// ---------------------------------------------------------------------------
void betweenness_weighted_arraygraph(const ArrayGraph& g, const uint32_t* sources, size_t ns, double* out,
                                     uint32_t* overflow_out) {
  const size_t V = g.node_capacity();
  std::vector<double> dist(V);
  std::vector<uint8_t> has_dist(V);  // ?f64: 0 = null
  std::vector<uint64_t> sigma(V);
  std::vector<double> delta(V);
  std::vector<std::vector<uint32_t>> preds(V);
  std::vector<std::pair<double, uint32_t>> heap;  // (d, node)
  std::vector<uint32_t> stack;
  std::vector<double> scores(V, 0.0);
  uint32_t overflow = 0;
  auto cmp = [](const std::pair<double, uint32_t>& a, const std::pair<double, uint32_t>& b) {
    return a.first > b.first;  // min-heap on d
  };
  for (size_t si = 0; si < ns; ++si) {
    const uint32_t s = sources[si];
    std::fill(has_dist.begin(), has_dist.end(), 0);  // :592-599
    std::fill(sigma.begin(), sigma.end(), 0);
    std::fill(delta.begin(), delta.end(), 0.0);
    for (auto& p : preds) p.clear();
    heap.clear();
    stack.clear();
    dist[s] = 0.0;  // :602-605
    has_dist[s] = 1;
    sigma[s] = 1;
    heap.push_back({0.0, s});
    std::push_heap(heap.begin(), heap.end(), cmp);
    while (!heap.empty()) {  // :607-642
      std::pop_heap(heap.begin(), heap.end(), cmp);
      const double d_v = heap.back().first;
      const uint32_t v = heap.back().second;
      heap.pop_back();
      const double current_best = has_dist[v] ? dist[v] : d_v;
      if (d_v > current_best) continue;  // compare(d_v, current_best) == .gt
      stack.push_back(v);
      g.for_each_successor_edge(v, [&](uint32_t w, double weight) {
        const double new_dist = d_v + weight;
        if (has_dist[w]) {
          const double old_dist = dist[w];
          if (new_dist < old_dist) {
            dist[w] = new_dist;
            sigma[w] = sigma[v];
            preds[w].clear();
            preds[w].push_back(v);
            heap.push_back({new_dist, w});
            std::push_heap(heap.begin(), heap.end(), cmp);
          } else if (new_dist == old_dist) {
            const uint64_t before = sigma[w];
            sigma[w] += sigma[v];  // usize add; wraps like a ReleaseFast build
            if (sigma[w] < before) overflow = 1;
            preds[w].push_back(v);
          }
        } else {
          dist[w] = new_dist;
          has_dist[w] = 1;
          sigma[w] = sigma[v];
          preds[w].push_back(v);
          heap.push_back({new_dist, w});
          std::push_heap(heap.begin(), heap.end(), cmp);
        }
      });
    }
    size_t i = stack.size();  // :645-662
    while (i > 0) {
      i -= 1;
      const uint32_t v = stack[i];
      const double sigma_v_f = (double)sigma[v];
      const double delta_v = delta[v];
      for (uint32_t u : preds[v]) {
        const double sigma_u_f = (double)sigma[u];
        const double c = (sigma_u_f / sigma_v_f) * (1.0 + delta_v);
        delta[u] += c;
      }
      if (v != s) scores[v] += delta_v;
    }
  }
  for (size_t v = 0; v < V; ++v) out[v] = g.has_node((uint32_t)v) ? scores[v] : 0.0;  // :664-671, extractScores
  if (overflow_out) *overflow_out = overflow;
}

// ---------------------------------------------------------------------------
// betweennessUnweighted, ArrayGraph branch   centrality.zig:687-798
// Runs the per-source body for the given sources (all live nodes ascending
// for the reference call).
// ---------------------------------------------------------------------------
void betweenness_arraygraph(const ArrayGraph& g, const uint32_t* sources, size_t ns,
                            double* out, uint32_t* overflow_out) {
  const size_t V = g.node_capacity();
  std::vector<uint32_t> dist(V);
  std::vector<uint64_t> sigma(V);
  std::vector<double> delta(V);
  std::vector<std::vector<uint32_t>> preds(V);
  std::vector<uint32_t> queue, stack;
  std::vector<double> scores(V, 0.0);
  uint32_t overflow = 0;

  for (size_t si = 0; si < ns; ++si) {
    const uint32_t s = sources[si];
    std::fill(dist.begin(), dist.end(), kNull);  // :731-738
    std::fill(sigma.begin(), sigma.end(), 0);
    std::fill(delta.begin(), delta.end(), 0.0);
    for (auto& p : preds) p.clear();
    queue.clear();
    stack.clear();

    dist[s] = 0;  // :741-743
    sigma[s] = 1;
    queue.push_back(s);
    size_t head = 0;
    while (head < queue.size()) {  // :745-767
      const uint32_t v = queue[head++];
      stack.push_back(v);
      const uint32_t d_v = dist[v];
      g.for_each_successor(v, [&](uint32_t w) {
        if (dist[w] == kNull) {
          dist[w] = d_v + 1;
          queue.push_back(w);
        }
        if (dist[w] == d_v + 1) {
          uint64_t before = sigma[w];
          sigma[w] += sigma[v];  // usize add; wraps like a ReleaseFast build
          if (sigma[w] < before) overflow = 1;
          preds[w].push_back(v);
        }
      });
    }
    size_t i = stack.size();  // :769-787
    while (i > 0) {
      i -= 1;
      const uint32_t v = stack[i];
      const double sigma_v_f = (double)sigma[v];
      const double delta_v = delta[v];
      for (uint32_t u : preds[v]) {
        const double sigma_u_f = (double)sigma[u];
        const double c = (sigma_u_f / sigma_v_f) * (1.0 + delta_v);
        delta[u] += c;
      }
      if (v != s) scores[v] += delta_v;
    }
  }
  for (size_t i = 0; i < V; ++i) out[i] = g.has_node((uint32_t)i) ? scores[i] : 0.0;  // :790-797
  if (overflow_out) *overflow_out = overflow;
}

// ---------------------------------------------------------------------------
// Seeded R-MAT generator shared by the oracle and the CUDA generator.
//   key      = splitmix64(seed)
//   r(i, k)  = splitmix64(key ^ (i << 6 | k))          level k of edge i
//   u        = r >> 11  (53-bit integer), compared with integer thresholds
//              floor(a*2^53), floor((a+b)*2^53), floor((a+b+c)*2^53)
//   quadrant 0:(0,0) 1:(0,1) 2:(1,0) 3:(1,1) appended MSB first to (src,dst).
// SplitMix64 is the public-domain mixer of Steele, Lea and Flood (2014) in the
// form published by S. Vigna.
// ---------------------------------------------------------------------------
inline uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct RmatThresholds { uint64_t ta, tab, tabc; };

RmatThresholds rmat_thresholds(double a, double b, double c) {
  const double two53 = 9007199254740992.0;
  return {(uint64_t)std::floor(a * two53), (uint64_t)std::floor((a + b) * two53),
          (uint64_t)std::floor((a + b + c) * two53)};
}

inline void rmat_edge(uint64_t key, uint64_t i, int scale, RmatThresholds t,
                      uint32_t* src, uint32_t* dst) {
  uint32_t s = 0, d = 0;
  for (int k = 0; k < scale; ++k) {
    uint64_t u = splitmix64(key ^ ((i << 6) | (uint64_t)k)) >> 11;
    uint32_t q = u < t.ta ? 0u : (u < t.tab ? 1u : (u < t.tabc ? 2u : 3u));
    s = (s << 1) | (q >> 1);
    d = (d << 1) | (q & 1u);
  }
  *src = s;
  *dst = d;
}

struct EdgeList {
  uint32_t V = 0;
  std::vector<uint32_t> from, to;
};

}  // namespace

extern "C" {

// ---- ArrayGraph handle ------------------------------------------------------
void* og_new(uint32_t node_count) {  // NIF buildGraph: addNode x n (.zig:26-35)
  auto* g = new ArrayGraph();
  g->first_edge.reserve(node_count);
  for (uint32_t i = 0; i < node_count; ++i) g->add_node();
  return g;
}
void og_free(void* h) { delete (ArrayGraph*)h; }
int og_add_edge(void* h, uint32_t from, uint32_t to, double w) {
  return ((ArrayGraph*)h)->add_edge(from, to, w);
}
int og_add_edges(void* h, const uint32_t* from, const uint32_t* to, const double* w, uint64_t m) {
  auto* g = (ArrayGraph*)h;  // NIF buildGraph edge loop in list order
  g->to.reserve(g->to.size() + m);
  g->data.reserve(g->data.size() + m);
  g->next_edge.reserve(g->next_edge.size() + m);
  g->edge_deleted.reserve(g->edge_deleted.size() + m);
  for (uint64_t i = 0; i < m; ++i)
    if (g->add_edge(from[i], to[i], w ? w[i] : 1.0) != 0) return -1;
  return 0;
}
int og_remove_edge(void* h, uint32_t from, uint32_t to) { return ((ArrayGraph*)h)->remove_edge(from, to); }
int og_remove_node(void* h, uint32_t id) { return ((ArrayGraph*)h)->remove_node(id); }
uint64_t og_node_capacity(void* h) { return ((ArrayGraph*)h)->node_capacity(); }
uint64_t og_edge_capacity(void* h) { return ((ArrayGraph*)h)->to.size(); }
uint64_t og_live_nodes(void* h) { return ((ArrayGraph*)h)->live_nodes; }
uint64_t og_live_edges(void* h) { return ((ArrayGraph*)h)->live_edges; }

// Raw ArrayGraph slices (what a NIF holding the resource can pass across the
// C ABI): null first_edge / next_edge are written as 0xFFFFFFFF.
void og_export(void* h, uint32_t* first_edge, uint8_t* node_deleted, uint32_t* to,
               uint32_t* next_edge, uint8_t* edge_deleted, double* data) {
  auto* g = (ArrayGraph*)h;
  size_t V = g->node_capacity(), E = g->to.size();
  if (first_edge) std::memcpy(first_edge, g->first_edge.data(), V * 4);
  if (node_deleted) std::memcpy(node_deleted, g->node_deleted.data(), V);
  if (to) std::memcpy(to, g->to.data(), E * 4);
  if (next_edge) std::memcpy(next_edge, g->next_edge.data(), E * 4);
  if (edge_deleted) std::memcpy(edge_deleted, g->edge_deleted.data(), E);
  if (data) std::memcpy(data, g->data.data(), E * 8);
}

// Successor lists in iteration order (reverse insertion), as a CSR.
void og_successor_csr(void* h, uint64_t* off, uint32_t* col) {
  auto* g = (ArrayGraph*)h;
  size_t V = g->node_capacity();
  uint64_t k = 0;
  for (size_t v = 0; v < V; ++v) {
    off[v] = k;
    if (g->node_deleted[v]) continue;
    g->for_each_successor((uint32_t)v, [&](uint32_t w) { col[k++] = w; });
  }
  off[V] = k;
}

// ---- algorithms on the ArrayGraph ---------------------------------------
void og_pagerank(void* h, double damping, uint64_t max_iter, double tol, double* out,
                 uint64_t* iters, double* l1) {
  pagerank_arraygraph(*(ArrayGraph*)h, damping, max_iter, tol, out, iters, l1);
}

void og_katz(void* h, double alpha, double beta, uint64_t max_iter, double tol, double* out, uint64_t* iters,
             double* l1) {
  linear_centrality(*(ArrayGraph*)h, alpha, beta, beta, max_iter, tol, out, iters, l1);
}
void og_alpha_centrality(void* h, double alpha, double initial, uint64_t max_iter, double tol, double* out,
                         uint64_t* iters, double* l1) {
  linear_centrality(*(ArrayGraph*)h, alpha, 0.0, initial, max_iter, tol, out, iters, l1);
}
void og_eigenvector(void* h, uint64_t max_iter, double tol, double* out, uint64_t* iters, int* how) {
  eigenvector_arraygraph(*(ArrayGraph*)h, max_iter, tol, out, iters, how);
}

void og_betweenness_unweighted(void* h, double* out, uint32_t* overflow) {
  auto* g = (ArrayGraph*)h;
  std::vector<uint32_t> nodes = g->collect_nodes();  // sources: nodeIds ascending (:728)
  betweenness_arraygraph(*g, nodes.data(), nodes.size(), out, overflow);
}

void og_betweenness_sources(void* h, const uint32_t* sources, uint64_t ns, double* out,
                            uint32_t* overflow) {
  betweenness_arraygraph(*(ArrayGraph*)h, sources, ns, out, overflow);
}

// nif_betweenness_f64 (.zig:123-132): every live node ascending, or a subset.
void og_betweenness_weighted(void* h, const uint32_t* sources, uint64_t ns, double* out, uint32_t* overflow) {
  auto* g = (ArrayGraph*)h;
  if (sources) {
    betweenness_weighted_arraygraph(*g, sources, ns, out, overflow);
  } else {
    std::vector<uint32_t> nodes = g->collect_nodes();
    betweenness_weighted_arraygraph(*g, nodes.data(), nodes.size(), out, overflow);
  }
}

// BFS intermediates of one source (centrality.zig:741-767): dist (0xFFFFFFFF =
// unreached) and sigma as the reference's wrapping usize.
void og_bfs(void* h, uint32_t s, uint32_t* dist_out, uint64_t* sigma_out, uint32_t* overflow) {
  auto* g = (ArrayGraph*)h;
  size_t V = g->node_capacity();
  std::vector<uint32_t> dist(V, kNull);
  std::vector<uint64_t> sigma(V, 0);
  std::vector<uint32_t> queue;
  uint32_t ovf = 0;
  dist[s] = 0;
  sigma[s] = 1;
  queue.push_back(s);
  size_t head = 0;
  while (head < queue.size()) {
    uint32_t v = queue[head++];
    uint32_t d_v = dist[v];
    g->for_each_successor(v, [&](uint32_t w) {
      if (dist[w] == kNull) { dist[w] = d_v + 1; queue.push_back(w); }
      if (dist[w] == d_v + 1) {
        uint64_t before = sigma[w];
        sigma[w] += sigma[v];
        if (sigma[w] < before) ovf = 1;
      }
    });
  }
  std::memcpy(dist_out, dist.data(), V * 4);
  std::memcpy(sigma_out, sigma.data(), V * 8);
  if (overflow) *overflow = ovf;
}

// ---- CSR-driven restatements for large graphs -----------------------------
// The PageRank hot loop of centrality.zig:924-958 over in_neighbors given as a
// CSR (rows hold sources ascending, the order :893-899 produces) and the
// out-degree array.  `live` may be null (all nodes live).  Returns the number of
// iterations run; `secs` receives the wall time of the iteration loop only.
uint64_t og_pagerank_csr(uint32_t V, const uint64_t* in_off, const uint32_t* in_col,
                         const uint32_t* outdeg, const uint8_t* live, double damping,
                         uint64_t max_iter, double tol, double* out, double* l1_out,
                         double* secs) {
  std::vector<uint32_t> nodes;
  nodes.reserve(V);
  for (uint32_t i = 0; i < V; ++i)
    if (!live || live[i]) nodes.push_back(i);
  const size_t n = nodes.size();
  for (uint32_t i = 0; i < V; ++i) out[i] = 0.0;
  *l1_out = 0.0;
  if (secs) *secs = 0.0;
  if (n == 0) return 0;
  if (n == 1) { out[nodes[0]] = 1.0; return 0; }
  const double n_f = (double)n;
  std::vector<double> ranks(V, 0.0), new_ranks(V, 0.0);
  for (uint32_t node : nodes) ranks[node] = 1.0 / n_f;
  auto t0 = std::chrono::steady_clock::now();
  uint64_t iteration = 0;
  double l1_norm = 0.0;
  while (iteration < max_iter) {
    double sink_sum = 0.0;
    for (uint32_t node : nodes)
      if (outdeg[node] == 0) sink_sum += ranks[node] / n_f;
    for (uint32_t node : nodes) {
      double rank_sum = 0.0;
      for (uint64_t j = in_off[node]; j < in_off[node + 1]; ++j) {
        uint32_t nb = in_col[j];
        uint64_t deg = outdeg[nb];
        if (deg > 0) rank_sum += ranks[nb] / (double)deg;
      }
      new_ranks[node] = (1.0 - damping) / n_f + damping * (sink_sum + rank_sum);
    }
    l1_norm = 0.0;
    for (uint32_t node : nodes) l1_norm += std::fabs(new_ranks[node] - ranks[node]);
    std::swap(ranks, new_ranks);
    iteration += 1;
    if (l1_norm < tol) break;
  }
  auto t1 = std::chrono::steady_clock::now();
  if (secs) *secs = std::chrono::duration<double>(t1 - t0).count();
  for (uint32_t node : nodes) out[node] = ranks[node];
  *l1_out = l1_norm;
  return iteration;
}

// The same iteration with the row loop spread over `threads` host threads
// (extension, no reference counterpart; <= 0 = all OpenMP threads).  Each row
// is still summed by one thread in ascending in_col order, and the two global
// sums -- the dangling mass and the L1 step -- are still taken in ascending
// node order by one thread.  The L1 pass of iteration k also accumulates the
// dangling mass of iteration k+1, which reads the same new ranks in the same
// order as the separate loop of centrality.zig:926-931, so every iterate is
// bit for bit the single-threaded og_pagerank_csr's.  x0 (null = uniform 1/n)
// and p (null = the reference's uniform teleport) generalise it like
// og_pagerank_ext; with both null and every node live it is the reference loop.
uint64_t og_pagerank_csr_mt(uint32_t V, const uint64_t* in_off, const uint32_t* in_col,
                            const uint32_t* outdeg, const double* x0, const double* p, double damping,
                            uint64_t max_iter, double tol, double* out, double* l1_out, double* secs,
                            int threads) {
  for (uint32_t i = 0; i < V; ++i) out[i] = 0.0;
  *l1_out = 0.0;
  if (secs) *secs = 0.0;
  if (V == 0) return 0;
  if (V == 1 && !x0 && !p) { out[0] = 1.0; return 0; }
  const int nt = threads > 0 ? threads : omp_get_max_threads();
  const double n_f = (double)V;
  std::vector<double> ranks(V), new_ranks(V, 0.0);
  for (uint32_t i = 0; i < V; ++i) ranks[i] = x0 ? x0[i] : 1.0 / n_f;
  auto t0 = std::chrono::steady_clock::now();
  double sink_sum = 0.0;
  for (uint32_t node = 0; node < V; ++node)
    if (outdeg[node] == 0) sink_sum += ranks[node] / n_f;
  uint64_t iteration = 0;
  double l1_norm = 0.0;
  while (iteration < max_iter) {
    const double sink = sink_sum;
    const double* rk = ranks.data();
    double* nr = new_ranks.data();
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nt)
    for (int64_t node = 0; node < (int64_t)V; ++node) {
      double rank_sum = 0.0;
      for (uint64_t j = in_off[node]; j < in_off[node + 1]; ++j) {
        const uint32_t nb = in_col[j];
        const uint64_t deg = outdeg[nb];
        if (deg > 0) rank_sum += rk[nb] / (double)deg;
      }
      const double tele = p ? (1.0 - damping) * p[node] : (1.0 - damping) / n_f;
      nr[node] = tele + damping * (sink + rank_sum);
    }
    l1_norm = 0.0;
    sink_sum = 0.0;
    for (uint32_t node = 0; node < V; ++node) {
      l1_norm += std::fabs(nr[node] - rk[node]);
      if (outdeg[node] == 0) sink_sum += nr[node] / n_f;
    }
    std::swap(ranks, new_ranks);
    iteration += 1;
    if (l1_norm < tol) break;
  }
  auto t1 = std::chrono::steady_clock::now();
  if (secs) *secs = std::chrono::duration<double>(t1 - t0).count();
  for (uint32_t i = 0; i < V; ++i) out[i] = ranks[i];
  *l1_out = l1_norm;
  return iteration;
}

// Per-source BFS distances and path counts (centrality.zig:740-767 restated,
// the dist / sigma half of the Brandes body) for many sources at once, the
// sources spread over host threads (extension for checking the CUDA library).
// Row k of dist_out / sigma_out (V entries each) belongs to sources[k]; sigma
// wraps like the reference's usize and overflow_out[k] records a wrap.
void og_bfs_csr_many(uint32_t V, const uint64_t* off, const uint32_t* col, const uint32_t* sources,
                     uint64_t ns, uint32_t* dist_out, uint64_t* sigma_out, uint8_t* overflow_out,
                     int threads) {
  const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
  {
    std::vector<uint32_t> queue;
    queue.reserve(V);
#pragma omp for schedule(dynamic, 1)
    for (int64_t k = 0; k < (int64_t)ns; ++k) {
      uint32_t* dist = dist_out + (size_t)k * V;
      uint64_t* sigma = sigma_out + (size_t)k * V;
      for (uint32_t v = 0; v < V; ++v) { dist[v] = kNull; sigma[v] = 0; }
      uint8_t ovf = 0;
      const uint32_t s = sources[k];
      dist[s] = 0;
      sigma[s] = 1;
      queue.clear();
      queue.push_back(s);
      size_t head = 0;
      while (head < queue.size()) {
        const uint32_t v = queue[head++];
        const uint32_t d_v = dist[v];
        for (uint64_t j = off[v]; j < off[v + 1]; ++j) {
          const uint32_t w = col[j];
          if (dist[w] == kNull) { dist[w] = d_v + 1; queue.push_back(w); }
          if (dist[w] == d_v + 1) {
            const uint64_t before = sigma[w];
            sigma[w] += sigma[v];
            if (sigma[w] < before) ovf = 1;
          }
        }
      }
      overflow_out[k] = ovf;
    }
  }
}

// The betweenness loop of og_betweenness_csr_sources with the sources split
// over host threads in contiguous runs (extension for checking the CUDA
// library at full size).  Each thread keeps its own score vector, added in
// thread order at the end; the per-source dependencies are the reference's,
// only the order in which sources' dependencies are summed into a score
// differs, so scores agree with the single-threaded loop to rounding.
void og_betweenness_csr_sources(uint32_t V, const uint64_t* off, const uint32_t* col,
                                const uint32_t* sources, uint64_t ns, double* out,
                                uint32_t* overflow_out, double* secs);
void og_betweenness_csr_sources_mt(uint32_t V, const uint64_t* off, const uint32_t* col,
                                   const uint32_t* sources, uint64_t ns, double* out,
                                   uint32_t* overflow_out, int threads) {
  const int nt = threads > 0 ? threads : omp_get_max_threads();
  std::vector<std::vector<double>> part(nt);
  std::vector<uint32_t> ovf_t(nt, 0);
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num();
    const uint64_t lo = ns * t / nt, hi = ns * (t + 1) / nt;
    double secs = 0.0;
    part[t].assign(V, 0.0);
    if (hi > lo)
      og_betweenness_csr_sources(V, off, col, sources + lo, hi - lo, part[t].data(), &ovf_t[t], &secs);
  }
  for (uint32_t v = 0; v < V; ++v) out[v] = 0.0;
  uint32_t ovf = 0;
  for (int t = 0; t < nt; ++t) {
    for (uint32_t v = 0; v < V; ++v) out[v] += part[t][v];
    ovf |= ovf_t[t];
  }
  if (overflow_out) *overflow_out = ovf;
}

// Generalised iteration (extension, no reference counterpart): start vector x0
// (null = uniform 1/n), teleport vector p (null = uniform (1-d)/n, the
// reference's teleport); dangling mass is redistributed uniformly as in the
// reference.  new = (1-d)*p[v] + d*(sink + rank_sum) when p is given.
uint64_t og_pagerank_ext(uint32_t V, const uint64_t* in_off, const uint32_t* in_col,
                         const uint32_t* outdeg, const double* x0, const double* p,
                         double damping, uint64_t max_iter, double tol, double* out,
                         double* l1_out) {
  const double n_f = (double)V;
  std::vector<double> ranks(V), new_ranks(V, 0.0);
  for (uint32_t i = 0; i < V; ++i) ranks[i] = x0 ? x0[i] : 1.0 / n_f;
  uint64_t iteration = 0;
  double l1_norm = 0.0;
  while (iteration < max_iter) {
    double sink_sum = 0.0;
    for (uint32_t node = 0; node < V; ++node)
      if (outdeg[node] == 0) sink_sum += ranks[node] / n_f;
    for (uint32_t node = 0; node < V; ++node) {
      double rank_sum = 0.0;
      for (uint64_t j = in_off[node]; j < in_off[node + 1]; ++j) {
        uint32_t nb = in_col[j];
        if (outdeg[nb] > 0) rank_sum += ranks[nb] / (double)outdeg[nb];
      }
      double tele = p ? (1.0 - damping) * p[node] : (1.0 - damping) / n_f;
      new_ranks[node] = tele + damping * (sink_sum + rank_sum);
    }
    l1_norm = 0.0;
    for (uint32_t node = 0; node < V; ++node) l1_norm += std::fabs(new_ranks[node] - ranks[node]);
    std::swap(ranks, new_ranks);
    iteration += 1;
    if (l1_norm < tol) break;
  }
  for (uint32_t i = 0; i < V; ++i) out[i] = ranks[i];
  *l1_out = l1_norm;
  return iteration;
}

// The betweenness per-source body (centrality.zig:728-788) driven from a
// successor CSR (rows in successor-iteration order).  `secs` = wall time.
void og_betweenness_csr_sources(uint32_t V, const uint64_t* off, const uint32_t* col,
                                const uint32_t* sources, uint64_t ns, double* out,
                                uint32_t* overflow_out, double* secs) {
  std::vector<uint32_t> dist(V);
  std::vector<uint64_t> sigma(V);
  std::vector<double> delta(V);
  std::vector<std::vector<uint32_t>> preds(V);
  std::vector<uint32_t> queue, stack;
  std::vector<double> scores(V, 0.0);
  uint32_t overflow = 0;
  auto t0 = std::chrono::steady_clock::now();
  for (uint64_t si = 0; si < ns; ++si) {
    const uint32_t s = sources[si];
    std::fill(dist.begin(), dist.end(), kNull);
    std::fill(sigma.begin(), sigma.end(), 0);
    std::fill(delta.begin(), delta.end(), 0.0);
    for (auto& p : preds) p.clear();
    queue.clear();
    stack.clear();
    dist[s] = 0;
    sigma[s] = 1;
    queue.push_back(s);
    size_t head = 0;
    while (head < queue.size()) {
      const uint32_t v = queue[head++];
      stack.push_back(v);
      const uint32_t d_v = dist[v];
      for (uint64_t j = off[v]; j < off[v + 1]; ++j) {
        const uint32_t w = col[j];
        if (dist[w] == kNull) { dist[w] = d_v + 1; queue.push_back(w); }
        if (dist[w] == d_v + 1) {
          uint64_t before = sigma[w];
          sigma[w] += sigma[v];
          if (sigma[w] < before) overflow = 1;
          preds[w].push_back(v);
        }
      }
    }
    size_t i = stack.size();
    while (i > 0) {
      i -= 1;
      const uint32_t v = stack[i];
      const double sigma_v_f = (double)sigma[v];
      const double delta_v = delta[v];
      for (uint32_t u : preds[v]) {
        const double c = ((double)sigma[u] / sigma_v_f) * (1.0 + delta_v);
        delta[u] += c;
      }
      if (v != s) scores[v] += delta_v;
    }
  }
  auto t1 = std::chrono::steady_clock::now();
  if (secs) *secs = std::chrono::duration<double>(t1 - t0).count();
  std::memcpy(out, scores.data(), (size_t)V * 8);
  if (overflow_out) *overflow_out = overflow;
}

// ---- R-MAT ------------------------------------------------------------------
// Generates ef * 2^scale raw edges, then (directed) drops self-loops and
// duplicate (src,dst) pairs and sorts by (src,dst); (undirected) canonicalises
// to (lo,hi), drops self-loops and duplicate pairs, sorts, and emits the arcs
// lo->hi, hi->lo per pair in that order -- the insertion order the undirected
// edge-list reader uses (.zig:868-893).  Returns a handle.
void* og_rmat(int scale, int edge_factor, uint64_t seed, double a, double b, double c,
              int directed) {
  auto* el = new EdgeList();
  el->V = 1u << scale;
  const uint64_t M = (uint64_t)edge_factor << scale;
  RmatThresholds t = rmat_thresholds(a, b, c);
  const uint64_t key = splitmix64(seed);
  // Input generation only (not a restated reference algorithm): parallel over
  // edges with a sentinel for self-loops, then a parallel sort.
  const uint64_t kLoop = ~0ull;
  std::vector<uint64_t> packed(M);
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)M; ++ii) {
    uint32_t s, d;
    rmat_edge(key, (uint64_t)ii, scale, t, &s, &d);
    if (!directed && s > d) std::swap(s, d);
    packed[ii] = (s == d) ? kLoop : (((uint64_t)s << 32) | d);
  }
  __gnu_parallel::sort(packed.begin(), packed.end());
  packed.erase(std::unique(packed.begin(), packed.end()), packed.end());
  if (!packed.empty() && packed.back() == kLoop) packed.pop_back();
  size_t m = packed.size();
  if (directed) {
    el->from.resize(m);
    el->to.resize(m);
    for (size_t i = 0; i < m; ++i) {
      el->from[i] = (uint32_t)(packed[i] >> 32);
      el->to[i] = (uint32_t)packed[i];
    }
  } else {
    el->from.resize(2 * m);
    el->to.resize(2 * m);
    for (size_t i = 0; i < m; ++i) {
      uint32_t lo = (uint32_t)(packed[i] >> 32), hi = (uint32_t)packed[i];
      el->from[2 * i] = lo; el->to[2 * i] = hi;
      el->from[2 * i + 1] = hi; el->to[2 * i + 1] = lo;
    }
  }
  return el;
}
// ---- Barabasi-Albert and Watts-Strogatz (benchmark / training inputs) --------
// The model definitions of generator.ex:132-198 and :210-253 with a seeded
// SplitMix64 stream (state advanced by the golden gamma, output mixed) in
// place of :rand.  below(n) = high 64 bits of next() * n; uniform() =
// (next() >> 11) * 2^-53.
//   BA: clique on 0..m-1 (pairs u < v in order); the degree list holds each
//       clique node m-1 times (node 0 once when m = 1).  Node u = m..n-1 draws
//       list entries until it has m distinct targets, adds u->v for them in
//       ascending order, then appends u, the targets, and u m-1 more times.
//   WS: ring lattice u -- u+j mod n (j = 1..k/2); each lattice slot (u, j)
//       draws one uniform; below beta, and if (u, u+j) is still joined, it is
//       rewired to (u, w) with w drawn until w != u and not joined to u
//       (skipped when u is joined to every other node).  Edges in sorted
//       (lo, hi) order.
// Undirected: both arcs per edge, forward first.
namespace {
struct Sm64Stream {
  uint64_t s;
  uint64_t next() {
    const uint64_t r = splitmix64(s);
    s += 0x9E3779B97F4A7C15ull;
    return r;
  }
  uint64_t below(uint64_t n) { return (uint64_t)(((unsigned __int128)next() * n) >> 64); }
  double uniform() { return (double)(next() >> 11) * 0x1p-53; }
};
void el_push(EdgeList* el, uint32_t u, uint32_t v, bool directed) {
  el->from.push_back(u);
  el->to.push_back(v);
  if (!directed) {
    el->from.push_back(v);
    el->to.push_back(u);
  }
}
}  // namespace

void* og_ba(uint32_t n, uint32_t m, uint64_t seed, int directed) {
  auto* el = new EdgeList();
  el->V = n;
  Sm64Stream rng{seed};
  for (uint32_t u = 0; u < m; ++u)
    for (uint32_t v = u + 1; v < m; ++v) el_push(el, u, v, directed != 0);
  std::vector<uint32_t> pool;
  for (uint32_t u = 0; u < m; ++u)
    for (uint32_t c = 1; c < m; ++c) pool.push_back(u);
  if (m == 1) pool.push_back(0);
  for (uint32_t u = m; u < n; ++u) {
    std::vector<uint32_t> chosen;
    while (chosen.size() < m) {
      const uint32_t v = pool[rng.below(pool.size())];
      bool dup = false;
      for (uint32_t x : chosen) dup |= x == v;
      if (!dup) chosen.push_back(v);
    }
    std::sort(chosen.begin(), chosen.end());
    for (uint32_t v : chosen) el_push(el, u, v, directed != 0);
    pool.push_back(u);
    pool.insert(pool.end(), chosen.begin(), chosen.end());
    for (uint32_t c = 1; c < m; ++c) pool.push_back(u);
  }
  return el;
}

void* og_ws(uint32_t n, uint32_t k, double beta, uint64_t seed, int directed) {
  auto* el = new EdgeList();
  el->V = n;
  Sm64Stream rng{seed};
  std::vector<std::set<uint32_t>> adj(n);
  for (uint32_t u = 0; u < n; ++u)
    for (uint32_t j = 1; j <= k / 2; ++j) {
      const uint32_t v = (u + j) % n;
      adj[u].insert(v);
      adj[v].insert(u);
    }
  for (uint32_t u = 0; u < n; ++u)
    for (uint32_t j = 1; j <= k / 2; ++j) {
      const uint32_t v = (u + j) % n;
      const double r = rng.uniform();
      if (!(r < beta) || !adj[u].count(v) || adj[u].size() + 1 >= n) continue;
      uint32_t w = (uint32_t)rng.below(n);
      while (w == u || adj[u].count(w)) w = (uint32_t)rng.below(n);
      adj[u].erase(v);
      adj[v].erase(u);
      adj[u].insert(w);
      adj[w].insert(u);
    }
  for (uint32_t u = 0; u < n; ++u)
    for (uint32_t v : adj[u])
      if (u < v) el_push(el, u, v, directed != 0);
  return el;
}

uint64_t og_edges_count(void* h) { return ((EdgeList*)h)->from.size(); }
uint32_t og_edges_nodes(void* h) { return ((EdgeList*)h)->V; }
void og_edges_copy(void* h, uint32_t* from, uint32_t* to) {
  auto* el = (EdgeList*)h;
  std::memcpy(from, el->from.data(), el->from.size() * 4);
  std::memcpy(to, el->to.data(), el->to.size() * 4);
}
void og_edges_free(void* h) { delete (EdgeList*)h; }

// in_neighbors CSR (rows = sources ascending, the order centrality.zig:893-899
// builds) and out-degrees from an edge list given in (src, dst)-sorted or any
// source-ascending order: a stable counting sort by destination.
void og_in_csr(uint32_t V, const uint32_t* from, const uint32_t* to, uint64_t E, uint64_t* off,
               uint32_t* col, uint32_t* outdeg) {
  std::vector<uint64_t> cnt((size_t)V + 1, 0);
  for (uint32_t v = 0; v < V; ++v) outdeg[v] = 0;
  for (uint64_t i = 0; i < E; ++i) { cnt[to[i] + 1]++; outdeg[from[i]]++; }
  for (uint32_t v = 0; v < V; ++v) cnt[v + 1] += cnt[v];
  for (uint32_t v = 0; v <= V; ++v) off[v] = cnt[v];
  // sources ascending within a row: scatter edges ordered by source
  std::vector<uint64_t> order(E);
  {
    std::vector<uint64_t> sc((size_t)V + 1, 0);
    for (uint64_t i = 0; i < E; ++i) sc[from[i] + 1]++;
    for (uint32_t v = 0; v < V; ++v) sc[v + 1] += sc[v];
    for (uint64_t i = 0; i < E; ++i) order[sc[from[i]]++] = i;
  }
  for (uint64_t k = 0; k < E; ++k) {
    const uint64_t i = order[k];
    col[cnt[to[i]]++] = from[i];
  }
}
// Raw (pre-dedupe) R-MAT endpoints of edges [i0, i0+m): lets tests compare the
// CUDA generator with this one element by element.
void og_rmat_raw(int scale, uint64_t seed, double a, double b, double c, uint64_t i0,
                 uint64_t m, uint32_t* src, uint32_t* dst) {
  RmatThresholds t = rmat_thresholds(a, b, c);
  const uint64_t key = splitmix64(seed);
  for (uint64_t i = 0; i < m; ++i) rmat_edge(key, i0 + i, scale, t, src + i, dst + i);
}

// ---- edge-list reader (nif_read_edgelist, .zig:896-990) ---------------------
// Parses the file like the NIF: skips blank and '#' lines, a "source target"
// header, splits on space/tab/comma, weight defaults to 1.0 (also when it does
// not parse).  integer_labels: ids parsed as u32 (lines that fail are skipped),
// next_id = max+1.  Otherwise labels get ids in order of first appearance.
// Builds an ArrayGraph with next_id nodes and adds edges with addParsedEdges
// (.zig:859-894).  Returns the graph handle (null on I/O error); *next_id_out
// receives the node count; label bytes are joined with '\n' into *labels_out
// (caller frees with og_free_buf).
void* og_read_edgelist(const char* path, int directed, int integer_labels,
                       uint32_t* next_id_out, char** labels_out, uint64_t* labels_len) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return nullptr;
  struct PE { uint32_t from, to; double w; };
  std::vector<PE> edges;
  std::unordered_map<std::string, uint32_t> label_to_id;
  std::vector<std::string> labels;
  uint32_t next_id = 0;
  std::string line;
  auto is_trim = [](char ch) { return ch == ' ' || ch == '\t' || ch == '\r'; };
  auto is_sep = [](char ch) { return ch == ' ' || ch == '\t' || ch == ','; };
  auto get_id = [&](const std::string& lbl) {
    auto it = label_to_id.find(lbl);
    if (it != label_to_id.end()) return it->second;
    uint32_t id = next_id++;
    label_to_id.emplace(lbl, id);
    labels.push_back(lbl);
    return id;
  };
  auto parse_u32 = [](const std::string& s, uint32_t* v) {
    if (s.empty()) return false;
    uint64_t acc = 0;
    size_t i = 0;
    if (s[0] == '+') { i = 1; if (s.size() == 1) return false; }
    for (; i < s.size(); ++i) {
      if (s[i] == '_') continue;
      if (s[i] < '0' || s[i] > '9') return false;
      acc = acc * 10 + (uint64_t)(s[i] - '0');
      if (acc > 0xFFFFFFFFull) return false;
    }
    *v = (uint32_t)acc;
    return true;
  };
  auto ieq = [](const std::string& a, const char* b) {
    size_t n = std::strlen(b);
    if (a.size() != n) return false;
    for (size_t i = 0; i < n; ++i)
      if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i])) return false;
    return true;
  };
  while (std::getline(f, line)) {
    size_t b0 = 0, e0 = line.size();
    while (b0 < e0 && is_trim(line[b0])) ++b0;
    while (e0 > b0 && is_trim(line[e0 - 1])) --e0;
    if (b0 == e0 || line[b0] == '#') continue;
    std::vector<std::string> parts;
    size_t i = b0;
    while (i < e0 && parts.size() < 3) {
      while (i < e0 && is_sep(line[i])) ++i;
      size_t j = i;
      while (j < e0 && !is_sep(line[j])) ++j;
      if (j > i) parts.emplace_back(line.substr(i, j - i));
      i = j;
    }
    if (parts.size() < 2) continue;
    if (ieq(parts[0], "source") && ieq(parts[1], "target")) continue;
    double w = 1.0;
    if (parts.size() >= 3) {
      char* endp = nullptr;
      double pw = std::strtod(parts[2].c_str(), &endp);
      if (endp && *endp == '\0' && endp != parts[2].c_str()) w = pw;
    }
    uint32_t s = 0, d = 0;
    if (integer_labels) {
      if (!parse_u32(parts[0], &s) || !parse_u32(parts[1], &d)) continue;
      uint32_t mx = std::max(s, d);
      if (mx >= next_id) next_id = mx + 1;
    } else {
      s = get_id(parts[0]);
      d = get_id(parts[1]);
    }
    edges.push_back({s, d, w});
  }
  auto* g = new ArrayGraph();
  for (uint32_t k = 0; k < next_id; ++k) g->add_node();
  if (directed) {
    for (auto& e : edges) g->add_edge(e.from, e.to, e.w);
  } else {
    std::stable_sort(edges.begin(), edges.end(), [](const PE& x, const PE& y) {
      uint32_t xl = std::min(x.from, x.to), xh = std::max(x.from, x.to);
      uint32_t yl = std::min(y.from, y.to), yh = std::max(y.from, y.to);
      if (xl != yl) return xl < yl;
      return xh < yh;
    });
    uint32_t plo = kNull, phi = kNull;
    for (auto& e : edges) {
      uint32_t lo = std::min(e.from, e.to), hi = std::max(e.from, e.to);
      if (lo == plo && hi == phi) continue;
      g->add_edge(e.from, e.to, e.w);
      if (e.from != e.to) g->add_edge(e.to, e.from, e.w);
      plo = lo;
      phi = hi;
    }
  }
  *next_id_out = next_id;
  std::string joined;
  for (size_t k = 0; k < labels.size(); ++k) {
    if (k) joined.push_back('\n');
    joined += labels[k];
  }
  *labels_len = joined.size();
  *labels_out = (char*)std::malloc(joined.size() + 1);
  std::memcpy(*labels_out, joined.c_str(), joined.size() + 1);
  return g;
}
void og_free_buf(char* p) { std::free(p); }

}  // extern "C"
