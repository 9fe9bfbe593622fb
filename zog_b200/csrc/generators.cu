// generators.cu -- seeded Barabasi-Albert and Watts-Strogatz graphs (benchmark
// and training inputs), following the model definitions of the reference's
// generators (lib/zog/generator.ex:132-198 and :210-253) with a seeded
// SplitMix64 stream instead of the unseeded :rand:
//   BA: a clique on nodes 0..m-1 (edges u<v in order), a node list holding
//       every clique node m-1 times; then each new node u picks m distinct
//       targets uniformly from that list (probability proportional to degree),
//       adds u->v for the targets in ascending order, and appends u, the
//       targets and m-1 more copies of u to the list.
//   WS: a ring lattice (each u joined to u+1..u+k/2 mod n), then every
//       lattice edge (u, u+j) is rewired with probability beta to (u, w) with
//       w uniform, not u and not already joined to u; edges are added in
//       sorted (lo, hi) order.
// Undirected graphs store both arcs of each edge (forward first), as the SoA
// builder does (lib/zog/soa.ex:111-128).
#include <algorithm>
#include <set>
#include <vector>

#include "common.cuh"

namespace zogcu {
namespace {

struct SplitMix {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  uint64_t below(uint64_t n) { return (uint64_t)(((unsigned __int128)next() * n) >> 64); }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

void push_edge(std::vector<uint32_t>& f, std::vector<uint32_t>& t, uint32_t u, uint32_t v, bool directed) {
  f.push_back(u);
  t.push_back(v);
  if (!directed) {
    f.push_back(v);
    t.push_back(u);
  }
}

}  // namespace
}  // namespace zogcu

using namespace zogcu;

extern "C" int zogcu_graph_generate_ba(uint32_t n, uint32_t m, uint64_t seed, int directed, zogcu_graph** out) {
  if (!out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  if (m < 1 || n <= m) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "Barabasi-Albert needs n > m >= 1");
  SplitMix rng{seed};
  std::vector<uint32_t> f, t;
  const uint64_t arcs = ((uint64_t)m * (m - 1) / 2 + (uint64_t)(n - m) * m) * (directed ? 1 : 2);
  if (arcs >= 0xFFFFFFFFull) return fail(ZOGCU_ERR_TOO_LARGE, "too many arcs");
  f.reserve(arcs);
  t.reserve(arcs);
  for (uint32_t u = 0; u + 1 < m; ++u)
    for (uint32_t v = u + 1; v < m; ++v) push_edge(f, t, u, v, directed != 0);
  std::vector<uint32_t> deg_list;
  deg_list.reserve((size_t)2 * m * n);
  if (m > 1) {
    for (uint32_t u = 0; u < m; ++u)
      for (uint32_t k = 0; k + 1 < m; ++k) deg_list.push_back(u);
  } else {
    deg_list.push_back(0);
  }
  std::vector<uint32_t> targets;
  for (uint32_t u = m; u < n; ++u) {
    targets.clear();
    while (targets.size() < m) {
      const uint32_t v = deg_list[rng.below(deg_list.size())];
      if (std::find(targets.begin(), targets.end(), v) == targets.end()) targets.push_back(v);
    }
    std::sort(targets.begin(), targets.end());
    for (uint32_t v : targets) push_edge(f, t, u, v, directed != 0);
    deg_list.push_back(u);
    for (uint32_t v : targets) deg_list.push_back(v);
    for (uint32_t k = 0; k + 1 < m; ++k) deg_list.push_back(u);
  }
  return zogcu_graph_create_from_edges(n, f.data(), t.data(), nullptr, f.size(), out);
}

extern "C" int zogcu_graph_generate_ws(uint32_t n, uint32_t k, double beta, uint64_t seed, int directed,
                                       zogcu_graph** out) {
  if (!out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  if (k % 2 != 0 || k < 2 || k >= n) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "k must be even, 2 <= k < n");
  if (!(beta >= 0.0 && beta <= 1.0)) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "beta must be in [0, 1]");
  SplitMix rng{seed};
  const uint32_t half = k / 2;
  // adjacency sets for the "not already joined" test of the rewiring step
  std::vector<std::vector<uint32_t>> nb(n);
  auto has = [&](uint32_t a, uint32_t b) {
    const auto& l = nb[a];
    return std::find(l.begin(), l.end(), b) != l.end();
  };
  auto add = [&](uint32_t a, uint32_t b) {
    nb[a].push_back(b);
    nb[b].push_back(a);
  };
  auto del = [&](uint32_t a, uint32_t b) {
    auto& la = nb[a];
    la.erase(std::find(la.begin(), la.end(), b));
    auto& lb = nb[b];
    lb.erase(std::find(lb.begin(), lb.end(), a));
  };
  for (uint32_t u = 0; u < n; ++u)
    for (uint32_t j = 1; j <= half; ++j) {
      const uint32_t v = (u + j) % n;
      if (!has(u, v)) add(u, v);
    }
  for (uint32_t u = 0; u < n; ++u)
    for (uint32_t j = 1; j <= half; ++j) {
      const uint32_t v = (u + j) % n;
      if (rng.uniform() < beta && has(u, v)) {
        if (nb[u].size() + 1 >= n) continue;  // u is joined to everyone: nothing to rewire to
        uint32_t w;
        do {
          w = (uint32_t)rng.below(n);
        } while (w == u || has(u, w));
        del(u, v);
        add(u, w);
      }
    }
  std::vector<std::pair<uint32_t, uint32_t>> edges;
  for (uint32_t u = 0; u < n; ++u)
    for (uint32_t v : nb[u])
      if (u < v) edges.emplace_back(u, v);
  std::sort(edges.begin(), edges.end());
  std::vector<uint32_t> f, t;
  f.reserve(edges.size() * 2);
  t.reserve(edges.size() * 2);
  for (auto& e : edges) push_edge(f, t, e.first, e.second, directed != 0);
  return zogcu_graph_create_from_edges(n, f.data(), t.data(), nullptr, f.size(), out);
}
