// wbrandes.cu -- weighted Brandes betweenness on the device.
//
// Reference: priv/zog/src/centrality.zig:528-682 (`betweenness`, ArrayGraph
// branch, called through betweennessF64 :1355-1357 by nif_betweenness_f64).
// Per source s, in ascending id order, a Dijkstra pass with a lazy-deletion
// binary heap computes f64 distances (new = d_v + w, compared with
// std.math.order: exact equality is a tie), shortest-path counts sigma
// (usize; a tie adds, a strict improvement resets) and predecessor lists; the
// reverse settle order then accumulates delta[u] += (sigma_u/sigma_v)(1+delta_v)
// over predecessors and adds delta_v to the score of every v != s.
//
// With positive weights every predecessor of v on a shortest path has a
// strictly smaller distance, so the distances are the fixed point
// D(w) = min over arcs v->w of fl(D(v) + w), sigma(w) is the sum of sigma(v)
// over the arcs with fl(D(v) + w) == D(w) (multi-arcs counted), and neither
// depends on the order in which the heap pops ties -- which lets a parallel
// algorithm reproduce them exactly:
//   1. distances: Bellman-Ford rounds over a per-node frontier mask with a
//      64-bit atomic min on the bit pattern of non-negative doubles (ordered
//      like the values);
//   2. sigma: the shortest-path DAG is swept in topological rounds (each node
//      counts its DAG in-arcs; the last predecessor to add its sigma makes the
//      node ready for the next round), which also numbers the rounds;
//   3. delta: rounds in reverse, each node pulling (sigma_v / sigma_w)(1 +
//      delta_w) from its DAG successors -- the reference's per-term value.
// 32 sources run side by side: node-major rows of 32 (distance, sigma, delta,
// round, in-count), lane b = source b.  Work items are (node, 256-arc chunk of
// its out-arcs), one warp each, so a hub's arcs spread over many warps (R-MAT's
// hubs are the low ids -- the first sources); chunk partials of delta and of
// the scores are added atomically.  The frontier / ready masks rotate through
// three buffers (read, write, clear for the next round).  Rounds are chained
// launches with device flags (a launch whose round has no work returns at
// once); the host checks the flags every 32 launches.  No kernel waits on
// another.
//
// An arc of effective length zero on a shortest path (fl(D + w) == D, for
// w <= 0 or w below half an ulp of D) would make the reference's sigma depend
// on its heap's tie order; weights must be positive and finite, and such an
// arc is reported as an error instead of guessed at.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace zogcu {
namespace {

constexpr int kWb = 32;                                     // sources per batch
constexpr unsigned long long kInf = 0x7FF0000000000000ull;  // +inf
constexpr uint32_t kNoRound = 0xFFFFFFFFu;
constexpr int kWbChain = 32;                                // launches between host checks
constexpr int kWbMaxLanes = 8;                              // batch lanes (streams with host threads)

struct EventGuardWb {
  cudaEvent_t e = nullptr;
  int init() {
    ZOGCU_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return ZOGCU_OK;
  }
  ~EventGuardWb() {
    if (e) cudaEventDestroy(e);
  }
};
constexpr uint32_t kWbChunk = 256;                          // arcs per work item

enum : int { kFlagZeroArc = 0, kFlagOverflow = 1, kFlagBadWeight = 2, kFlagMaxRound = 3, kFlags = 4 };

__device__ __forceinline__ double wt_of(const double* __restrict__ w, uint32_t j) { return w ? __ldg(w + j) : 1.0; }

__global__ void k_wb_check_weights(const double* __restrict__ w, uint64_t E, uint32_t* __restrict__ flags) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < E; j += (uint64_t)gridDim.x * blockDim.x) {
    const double x = w[j];
    if (!(x > 0.0) || !(x <= 1.7976931348623157e308)) atomicOr(flags + kFlagBadWeight, 1u);
  }
}

__global__ void k_wb_init(uint32_t V, unsigned long long* __restrict__ dist, unsigned long long* __restrict__ sigma,
                          double* __restrict__ delta, uint32_t* __restrict__ round, uint32_t* __restrict__ cnt,
                          uint32_t* __restrict__ mask0, uint32_t* __restrict__ mask1) {
  const uint64_t n = (uint64_t)V * kWb;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    dist[i] = kInf;
    sigma[i] = 0;
    delta[i] = 0.0;
    round[i] = kNoRound;
    cnt[i] = 0;
    if (i < V) {
      mask0[i] = 0;
      mask1[i] = 0;
    }
  }
}

// Lane b < ns: distance 0, sigma 1 and round 0 at its source, which joins the
// first frontier / ready set.
__global__ void k_wb_seed(const uint32_t* __restrict__ src, uint32_t ns, unsigned long long* __restrict__ dist,
                          unsigned long long* __restrict__ sigma, uint32_t* __restrict__ round,
                          uint32_t* __restrict__ mask0) {
  const uint32_t b = threadIdx.x;
  if (b < ns) {
    const uint32_t s = src[b];
    dist[(size_t)s * kWb + b] = 0ull;  // +0.0
    sigma[(size_t)s * kWb + b] = 1ull;
    round[(size_t)s * kWb + b] = 0;
    atomicOr(mask0 + s, 1u << b);
  }
}

// Work item t: node tnode[t], arcs [tbeg[t], min(tbeg[t] + kWbChunk, off[node+1])).

// Phase 1, round k: relax the out-arcs of every (node, source) in the frontier.
__global__ void __launch_bounds__(256) k_wb_relax(const uint32_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                  const double* __restrict__ w, const uint32_t* __restrict__ tnode,
                                                  const uint32_t* __restrict__ tbeg, uint32_t ntasks,
                                                  unsigned long long* __restrict__ dist,
                                                  const uint32_t* __restrict__ mcur, uint32_t* __restrict__ mnext,
                                                  uint32_t* __restrict__ mclear, uint32_t V,
                                                  uint32_t* __restrict__ work, uint32_t k) {
  if (*(volatile uint32_t*)(work + k) == 0) return;
  const int lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) mclear[i] = 0;
  bool any = false;
  for (uint32_t t = gw; t < ntasks; t += nw) {
    const uint32_t v = tnode[t];
    const uint32_t m = mcur[v];
    if (m == 0) continue;
    const bool on = (m >> lane) & 1u;
    const double dv = on ? __longlong_as_double((long long)dist[(size_t)v * kWb + lane]) : 0.0;
    const uint32_t b = tbeg[t], e = min(b + kWbChunk, off[v + 1]);
    for (uint32_t j = b; j < e; ++j) {
      const uint32_t u = __ldg(col + j);
      const double wt = wt_of(w, j);
      if (on) {
        const unsigned long long nd = (unsigned long long)__double_as_longlong(__dadd_rn(dv, wt));
        const unsigned long long old = atomicMin(dist + (size_t)u * kWb + lane, nd);
        if (nd < old) {
          atomicOr(mnext + u, 1u << lane);
          any = true;
        }
      }
    }
  }
  if (__any_sync(0xffffffffu, any) && lane == 0) work[k + 1] = 1u;
}

// Phase 2a: DAG in-arc counts (and the zero-length check).
__global__ void __launch_bounds__(256) k_wb_dagcount(const uint32_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                     const double* __restrict__ w, const uint32_t* __restrict__ tnode,
                                                     const uint32_t* __restrict__ tbeg, uint32_t ntasks,
                                                     const unsigned long long* __restrict__ dist,
                                                     uint32_t* __restrict__ cnt, uint32_t* __restrict__ flags) {
  const int lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntasks; t += nw) {
    const uint32_t v = tnode[t];
    const unsigned long long dvb = dist[(size_t)v * kWb + lane];
    const bool on = dvb != kInf;
    if (!__any_sync(0xffffffffu, on)) continue;
    const double dv = __longlong_as_double((long long)dvb);
    const uint32_t b = tbeg[t], e = min(b + kWbChunk, off[v + 1]);
    for (uint32_t j = b; j < e; ++j) {
      const uint32_t u = __ldg(col + j);
      const double wt = wt_of(w, j);
      if (on) {
        const unsigned long long nd = (unsigned long long)__double_as_longlong(__dadd_rn(dv, wt));
        const unsigned long long du = dist[(size_t)u * kWb + lane];
        if (nd == du) {
          atomicAdd(cnt + (size_t)u * kWb + lane, 1u);
          if (du == dvb) atomicOr(flags + kFlagZeroArc, 1u);
        }
      }
    }
  }
}

// Phase 2b, round k: ready nodes add their sigma along DAG arcs; a node whose
// last DAG predecessor has added becomes ready in round k + 1.
__global__ void __launch_bounds__(256) k_wb_sigma(const uint32_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                  const double* __restrict__ w, const uint32_t* __restrict__ tnode,
                                                  const uint32_t* __restrict__ tbeg, uint32_t ntasks,
                                                  const unsigned long long* __restrict__ dist,
                                                  unsigned long long* __restrict__ sigma, uint32_t* __restrict__ cnt,
                                                  uint32_t* __restrict__ round, const uint32_t* __restrict__ mcur,
                                                  uint32_t* __restrict__ mnext, uint32_t* __restrict__ mclear,
                                                  uint32_t V, uint32_t* __restrict__ work,
                                                  uint32_t* __restrict__ flags, uint32_t k) {
  if (*(volatile uint32_t*)(work + k) == 0) return;
  const int lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) mclear[i] = 0;
  bool any = false;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntasks; t += nw) {
    const uint32_t v = tnode[t];
    const uint32_t m = mcur[v];
    if (m == 0) continue;
    const bool on = (m >> lane) & 1u;
    const unsigned long long sv = on ? sigma[(size_t)v * kWb + lane] : 0ull;
    const double dv = on ? __longlong_as_double((long long)dist[(size_t)v * kWb + lane]) : 0.0;
    const uint32_t b = tbeg[t], e = min(b + kWbChunk, off[v + 1]);
    for (uint32_t j = b; j < e; ++j) {
      const uint32_t u = __ldg(col + j);
      const double wt = wt_of(w, j);
      if (on) {
        const unsigned long long nd = (unsigned long long)__double_as_longlong(__dadd_rn(dv, wt));
        const size_t iu = (size_t)u * kWb + lane;
        if (nd == dist[iu]) {
          const unsigned long long old = atomicAdd(sigma + iu, sv);  // wraps modulo 2^64 like usize
          if (old + sv < old) atomicOr(flags + kFlagOverflow, 1u);
          if (atomicSub(cnt + iu, 1u) == 1u) {
            round[iu] = k + 1;
            atomicOr(mnext + u, 1u << lane);
            atomicMax(flags + kFlagMaxRound, k + 1);
            any = true;
          }
        }
      }
    }
  }
  if (__any_sync(0xffffffffu, any) && lane == 0) work[k + 1] = 1u;
}

// Phase 3, round r (descending): delta_v = sum over DAG successors w of
// (sigma_v / sigma_w)(1 + delta_w); the score of v gains delta_v for v != s.
// A node's chunks add their partial sums atomically.
__global__ void __launch_bounds__(256) k_wb_delta(const uint32_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                  const double* __restrict__ w, const uint32_t* __restrict__ tnode,
                                                  const uint32_t* __restrict__ tbeg, uint32_t ntasks,
                                                  const unsigned long long* __restrict__ dist,
                                                  const unsigned long long* __restrict__ sigma,
                                                  double* __restrict__ delta, const uint32_t* __restrict__ round,
                                                  const uint32_t* __restrict__ src, uint32_t ns,
                                                  double* __restrict__ bc, uint32_t r) {
  const int lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  const uint32_t my_src = (uint32_t)lane < ns ? src[lane] : 0xFFFFFFFFu;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntasks; t += nw) {
    const uint32_t v = tnode[t];
    const size_t iv = (size_t)v * kWb + lane;
    const bool on = round[iv] == r;
    if (!__any_sync(0xffffffffu, on)) continue;
    const double dv = on ? __longlong_as_double((long long)dist[iv]) : 0.0;
    const double sv = on ? __ull2double_rn(sigma[iv]) : 0.0;
    double acc = 0.0;
    const uint32_t b = tbeg[t], e = min(b + kWbChunk, off[v + 1]);
    for (uint32_t j = b; j < e; ++j) {
      const uint32_t u = __ldg(col + j);
      const double wt = wt_of(w, j);
      if (on) {
        const unsigned long long nd = (unsigned long long)__double_as_longlong(__dadd_rn(dv, wt));
        const size_t iu = (size_t)u * kWb + lane;
        if (nd == dist[iu]) {
          const double c = __dmul_rn(__ddiv_rn(sv, __ull2double_rn(sigma[iu])), __dadd_rn(1.0, delta[iu]));
          acc = __dadd_rn(acc, c);
        }
      }
    }
    if (on && acc != 0.0) atomicAdd(delta + iv, acc);
    double add = (on && v != my_src) ? acc : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) add += __shfl_xor_sync(0xffffffffu, add, o);
    if (lane == 0 && add != 0.0) atomicAdd(bc + v, add);
  }
}

__global__ void k_wb_add(double* __restrict__ a, const double* __restrict__ b, uint32_t V) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
    a[v] += b[v];
}

unsigned wb_grid(uint64_t warps) {
  const uint64_t g = (warps * 32 + 255) / 256;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, (uint64_t)sm_count() * 8));
}

// Grid of a round kernel: the CTAs of 256 threads resident at once
// (occupancy x SMs), at most one per 8 warps of work, so the grid-stride loop
// runs in one wave.
template <typename K>
unsigned wb_grid_of(K kernel, uint64_t warps) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
  const uint64_t g = (warps * 32 + 255) / 256;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, (uint64_t)sm_count() * (uint64_t)per_sm));
}

// Runs launch(k) for k = 0, 1, ... in chains of kWbChain until round k has no
// work (work[k] == 0).  Both sweeps have work in at most V + 1 rounds when the
// weights are positive; `work` holds V + 3 + 2 kWbChain flags.
template <class F>
int run_rounds(uint32_t* work, uint32_t V, cudaStream_t s, F launch, uint32_t* rounds_out) {
  uint32_t k = 0;
  for (;;) {
    if ((uint64_t)k > (uint64_t)V + 1) return fail(ZOGCU_ERR_INTERNAL, "weighted betweenness: round limit");
    for (int i = 0; i < kWbChain; ++i) launch(k + (uint32_t)i);
    ZOGCU_CUDA(cudaGetLastError());
    k += kWbChain;
    uint32_t more = 0;
    ZOGCU_CUDA(cudaMemcpyAsync(&more, work + k, 4, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    if (!more) break;
  }
  if (rounds_out) *rounds_out = k;
  return ZOGCU_OK;
}

int run_weighted(Graph* g, const std::vector<uint32_t>& sources, double* out, bool dev_out, zogcu_stats* stats,
                 cudaStream_t s) {
  const uint32_t V = g->V;
  const uint64_t E = g->E;
  if (!g->offsets32) return fail(ZOGCU_ERR_TOO_LARGE, "weighted betweenness needs fewer than 2^32 arcs");
  const uint32_t* off = g->out_off32.as<uint32_t>();
  const uint32_t* col = g->out_col.as<uint32_t>();
  const double* w = g->weighted ? g->out_w.as<double>() : nullptr;
  const size_t n = (size_t)std::max<uint32_t>(V, 1) * kWb;
  const size_t Vs = std::max<uint32_t>(V, 1);
  // work items: (node, first arc) per kWbChunk arcs of every node's out-row
  DevBuf btn, btb;
  std::vector<uint32_t> h_off((size_t)V + 1), tn, tb;
  if (V) ZOGCU_CUDA(cudaMemcpyAsync(h_off.data(), off, ((size_t)V + 1) * 4, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  for (uint32_t v = 0; v < V; ++v)
    for (uint32_t j = h_off[v]; j < h_off[v + 1]; j += kWbChunk) {
      tn.push_back(v);
      tb.push_back(j);
    }
  const uint32_t ntasks = (uint32_t)tn.size();
  ZOGCU_TRY(btn.alloc(std::max<size_t>(tn.size(), 1) * 4, s));
  ZOGCU_TRY(btb.alloc(std::max<size_t>(tb.size(), 1) * 4, s));
  if (ntasks) {
    ZOGCU_CUDA(cudaMemcpyAsync(btn.ptr, tn.data(), tn.size() * 4, cudaMemcpyHostToDevice, s));
    ZOGCU_CUDA(cudaMemcpyAsync(btb.ptr, tb.data(), tb.size() * 4, cudaMemcpyHostToDevice, s));
  }
  const uint32_t* tnode = btn.as<uint32_t>();
  const uint32_t* tbeg = btb.as<uint32_t>();
  const size_t work_n = (size_t)V + 3 + 2 * kWbChain;
  if (w && E) {
    DevBuf chk;
    ZOGCU_TRY(chk.alloc(kFlags * 4, s));
    ZOGCU_CUDA(cudaMemsetAsync(chk.ptr, 0, kFlags * 4, s));
    k_wb_check_weights<<<wb_grid(E / 32 + 1), 256, 0, s>>>(w, E, chk.as<uint32_t>());
    ZOGCU_CUDA(cudaGetLastError());
    uint32_t bad = 0;
    ZOGCU_CUDA(cudaMemcpyAsync(&bad, chk.as<uint32_t>() + kFlagBadWeight, 4, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    if (bad) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "weighted betweenness needs positive finite weights");
  }
  const uint64_t nwork = std::max<uint32_t>(ntasks, V);
  const unsigned g_relax = wb_grid_of(k_wb_relax, nwork), g_count = wb_grid_of(k_wb_dagcount, nwork);
  const unsigned g_sigma = wb_grid_of(k_wb_sigma, nwork), g_delta = wb_grid_of(k_wb_delta, nwork);

  // Batches are dealt to lanes (batch i to lane i mod lanes), each with its
  // own stream, state and score vector and driven by its own host thread:
  // while one lane's thread waits on its round flags, the other lanes' rounds
  // keep the GPU busy.  The lanes' scores are added to the first lane's in
  // lane order at the end, so the result does not depend on timing.  Lanes:
  // up to kWbMaxLanes, as many as a quarter of the device memory holds
  // (ZOGCU_BC_STREAMS=<k> sets the count).  Declaration order makes every exit
  // free the lanes' state first, then drain and destroy their streams, and
  // only then free the score vectors (on stream s).
  const size_t nbatches = (sources.size() + kWb - 1) / kWb;
  const size_t lane_bytes = n * (8 * 3 + 4 * 2) + Vs * 4 * 3 + work_n * 4 + Vs * 8;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) total_b = 0;
  int nlanes = (int)std::min<size_t>(std::max<size_t>(nbatches, 1), kWbMaxLanes);
  if (total_b) nlanes = (int)std::max<size_t>(1, std::min<size_t>(nlanes, total_b / 4 / std::max<size_t>(lane_bytes, 1)));
  if (const char* env = std::getenv("ZOGCU_BC_STREAMS")) {
    const int k = std::atoi(env);
    if (k >= 1) nlanes = std::min(k, kWbMaxLanes);
  }
  DevBuf bcv[kWbMaxLanes];
  StreamGuard lsg[kWbMaxLanes];
  cudaStream_t ls[kWbMaxLanes] = {};
  EventGuardWb start_ev, lane_done[kWbMaxLanes];
  for (int l = 0; l < nlanes; ++l) {
    ZOGCU_TRY(bcv[l].alloc(Vs * 8, s));
    ZOGCU_CUDA(cudaMemsetAsync(bcv[l].ptr, 0, Vs * 8, s));
  }
  ZOGCU_TRY(start_ev.init());
  ZOGCU_CUDA(cudaEventRecord(start_ev.e, s));
  for (int l = 0; l < nlanes; ++l) {
    ZOGCU_TRY(lsg[l].init(nullptr));
    ls[l] = lsg[l].s;
    ZOGCU_CUDA(cudaStreamWaitEvent(ls[l], start_ev.e, 0));  // after the score vectors and work items
  }
  struct Lane {
    DevBuf bdist, bsigma, bdelta, bround, bcnt, bm0, bm1, bm2, bwork, bflags, bsrc;
    uint64_t launches = 0;
    uint32_t deepest = 0;
    int status = ZOGCU_OK;
    std::string error;
  } L[kWbMaxLanes];
  for (int l = 0; l < nlanes; ++l) {
    Lane& A = L[l];
    const cudaStream_t st = ls[l];
    ZOGCU_TRY(A.bdist.alloc(n * 8, st));
    ZOGCU_TRY(A.bsigma.alloc(n * 8, st));
    ZOGCU_TRY(A.bdelta.alloc(n * 8, st));
    ZOGCU_TRY(A.bround.alloc(n * 4, st));
    ZOGCU_TRY(A.bcnt.alloc(n * 4, st));
    ZOGCU_TRY(A.bm0.alloc(Vs * 4, st));
    ZOGCU_TRY(A.bm1.alloc(Vs * 4, st));
    ZOGCU_TRY(A.bm2.alloc(Vs * 4, st));
    ZOGCU_TRY(A.bwork.alloc(work_n * 4, st));
    ZOGCU_TRY(A.bflags.alloc(kFlags * 4, st));
    ZOGCU_TRY(A.bsrc.alloc(kWb * 4, st));
    ZOGCU_CUDA(cudaMemsetAsync(A.bflags.ptr, 0, kFlags * 4, st));
  }
  EventTimer tm;
  ZOGCU_TRY(tm.start(s));
  const uint32_t one = 1;
  // one batch of up to kWb sources on lane l (run by lane l's thread)
  auto run_batch = [&](int l, size_t bi) -> int {
    Lane& A = L[l];
    const cudaStream_t st = ls[l];
    unsigned long long* dist = A.bdist.as<unsigned long long>();
    unsigned long long* sigma = A.bsigma.as<unsigned long long>();
    double* delta = A.bdelta.as<double>();
    uint32_t* round = A.bround.as<uint32_t>();
    uint32_t* cnt = A.bcnt.as<uint32_t>();
    uint32_t* masks[3] = {A.bm0.as<uint32_t>(), A.bm1.as<uint32_t>(), A.bm2.as<uint32_t>()};
    uint32_t* work = A.bwork.as<uint32_t>();
    uint32_t* flags = A.bflags.as<uint32_t>();
    const uint32_t* src = A.bsrc.as<uint32_t>();
    double* bcl = bcv[l].as<double>();
    const size_t b0 = bi * kWb;
    const uint32_t ns = (uint32_t)std::min<size_t>(kWb, sources.size() - b0);
    ZOGCU_CUDA(cudaMemcpyAsync(A.bsrc.ptr, sources.data() + b0, ns * 4, cudaMemcpyHostToDevice, st));
    k_wb_init<<<wb_grid(V), 256, 0, st>>>(V, dist, sigma, delta, round, cnt, masks[0], masks[1]);
    ZOGCU_CUDA(cudaMemsetAsync(masks[2], 0, Vs * 4, st));
    k_wb_seed<<<1, kWb, 0, st>>>(src, ns, dist, sigma, round, masks[0]);
    ZOGCU_CUDA(cudaGetLastError());
    ZOGCU_CUDA(cudaMemsetAsync(flags + kFlagMaxRound, 0, 4, st));
    A.launches += 2;
    // phase 1: distances
    ZOGCU_CUDA(cudaMemsetAsync(work, 0, work_n * 4, st));
    ZOGCU_CUDA(cudaMemcpyAsync(work, &one, 4, cudaMemcpyHostToDevice, st));
    uint32_t r1 = 0;
    ZOGCU_TRY(run_rounds(work, V, st, [&](uint32_t k) {
      k_wb_relax<<<g_relax, 256, 0, st>>>(off, col, w, tnode, tbeg, ntasks, dist, masks[k % 3], masks[(k + 1) % 3],
                                        masks[(k + 2) % 3], V, work, k);
    }, &r1));
    A.launches += r1;
    // phase 2: DAG in-counts, then sigma in topological rounds from the sources
    k_wb_dagcount<<<g_count, 256, 0, st>>>(off, col, w, tnode, tbeg, ntasks, dist, cnt, flags);
    for (int i = 0; i < 3; ++i) ZOGCU_CUDA(cudaMemsetAsync(masks[i], 0, Vs * 4, st));
    k_wb_seed<<<1, kWb, 0, st>>>(src, ns, dist, sigma, round, masks[0]);
    ZOGCU_CUDA(cudaGetLastError());
    ZOGCU_CUDA(cudaMemsetAsync(work, 0, work_n * 4, st));
    ZOGCU_CUDA(cudaMemcpyAsync(work, &one, 4, cudaMemcpyHostToDevice, st));
    uint32_t r2 = 0;
    ZOGCU_TRY(run_rounds(work, V, st, [&](uint32_t k) {
      k_wb_sigma<<<g_sigma, 256, 0, st>>>(off, col, w, tnode, tbeg, ntasks, dist, sigma, cnt, round, masks[k % 3],
                                        masks[(k + 1) % 3], masks[(k + 2) % 3], V, work, flags, k);
    }, &r2));
    A.launches += r2 + 2;
    uint32_t hf[kFlags];
    ZOGCU_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
    ZOGCU_CUDA(cudaStreamSynchronize(st));
    if (hf[kFlagZeroArc])
      return fail(ZOGCU_ERR_INVALID_ARGUMENT,
                  "weighted betweenness: a shortest path holds an arc of effective length zero (fl(d + w) == d)");
    // phase 3: dependencies, rounds in reverse
    const uint32_t maxr = hf[kFlagMaxRound];
    A.deepest = std::max(A.deepest, maxr);
    for (int64_t r = maxr; r >= 0; --r)
      k_wb_delta<<<g_delta, 256, 0, st>>>(off, col, w, tnode, tbeg, ntasks, dist, sigma, delta, round, src, ns, bcl,
                                       (uint32_t)r);
    ZOGCU_CUDA(cudaGetLastError());
    A.launches += (uint64_t)maxr + 1;
    return ZOGCU_OK;
  };
  {
    int device = 0;
    ZOGCU_CUDA(cudaGetDevice(&device));
    std::atomic<bool> stop{false};  // a lane failed: the others stop after their current batch
    auto lane_run = [&](int l) {
      if (cudaSetDevice(device) != cudaSuccess) {
        L[l].status = ZOGCU_ERR_CUDA;
        L[l].error = "weighted betweenness: lane thread could not select the device";
        stop = true;
        return;
      }
      for (size_t bi = (size_t)l; bi < nbatches && !stop; bi += (size_t)nlanes) {
        const int rc = run_batch(l, bi);
        if (rc != ZOGCU_OK) {
          L[l].status = rc;
          L[l].error = zogcu_last_error();  // the message is kept per thread
          stop = true;
          return;
        }
      }
    };
    std::vector<std::thread> th;
    for (int l = 1; l < nlanes; ++l) th.emplace_back(lane_run, l);
    lane_run(0);
    for (auto& t : th) t.join();
  }
  for (int l = 0; l < nlanes; ++l)
    if (L[l].status != ZOGCU_OK) return fail(L[l].status, L[l].error);
  uint64_t launches = 0;
  uint32_t deepest = 0;
  for (int l = 0; l < nlanes; ++l) {
    launches += L[l].launches;
    deepest = std::max(deepest, L[l].deepest);
  }
  // the lanes' scores into the first lane's, in lane order, on stream s
  for (int l = 0; l < nlanes; ++l) {
    ZOGCU_TRY(lane_done[l].init());
    ZOGCU_CUDA(cudaEventRecord(lane_done[l].e, ls[l]));
    ZOGCU_CUDA(cudaStreamWaitEvent(s, lane_done[l].e, 0));
  }
  for (int l = 1; l < nlanes; ++l) {
    k_wb_add<<<wb_grid(Vs / 32 + 1), 256, 0, s>>>(bcv[0].as<double>(), bcv[l].as<double>(), V);
    ZOGCU_CUDA(cudaGetLastError());
    ++launches;
  }
  ZOGCU_TRY(tm.stop(s));
  uint32_t ovf[kWbMaxLanes] = {};
  for (int l = 0; l < nlanes; ++l)
    ZOGCU_CUDA(cudaMemcpyAsync(&ovf[l], L[l].bflags.as<uint32_t>() + kFlagOverflow, 4, cudaMemcpyDeviceToHost, s));
  if (V)
    ZOGCU_CUDA(cudaMemcpyAsync(out, bcv[0].ptr, (size_t)V * 8,
                               dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  if (stats) {
    stats->sources = sources.size();
    stats->elapsed_ms = tm.ms();
    stats->max_depth = deepest;
    uint32_t any = 0;
    for (int l = 0; l < nlanes; ++l) any |= ovf[l];
    stats->sigma_overflow = any ? 1u : 0u;
    stats->launches = launches;
  }
  return ZOGCU_OK;
}

}  // namespace
}  // namespace zogcu

extern "C" {

int zogcu_betweenness_weighted(zogcu_graph* G, const zogcu_bc_opts* opts, double* out_scores, zogcu_stats* stats) {
  using namespace zogcu;
  if (!G) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graph is null");
  if (!out_scores && G->g.V) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out_scores is null");
  if (opts && opts->struct_size != sizeof(zogcu_bc_opts))
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "zogcu_bc_opts.struct_size mismatch");
  Graph* g = &G->g;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  ZOGCU_CUDA(cudaSetDevice(g->device));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(opts ? opts->stream : nullptr));
  // sources: the subset given, or every live node ascending (centrality.zig:589)
  std::vector<uint32_t> src;
  if (opts && opts->sources) {
    src.assign(opts->sources, opts->sources + opts->num_sources);
    for (uint32_t x : src)
      if (x >= g->V) return fail(ZOGCU_ERR_NODE_NOT_FOUND, "source is not a node of the graph");
  } else {
    std::vector<uint32_t> deg(g->V);
    if (g->V) ZOGCU_CUDA(cudaMemcpy(deg.data(), g->out_deg.ptr, (size_t)g->V * 4, cudaMemcpyDeviceToHost));
    for (uint32_t v = 0; v < g->V; ++v)
      if (deg[v] != kDeletedDegree) src.push_back(v);
  }
  return run_weighted(g, src, out_scores, opts && opts->device_pointers, stats, sg.s);
}

int zogcu_graph_export_weights(const zogcu_graph* G, double* out_weights) {
  using namespace zogcu;
  if (!G || (!out_weights && G->g.E)) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  const Graph* g = &G->g;
  if (!g->E) return ZOGCU_OK;
  ZOGCU_CUDA(cudaSetDevice(g->device));
  if (g->weighted) {
    ZOGCU_CUDA(cudaMemcpy(out_weights, g->out_w.ptr, (size_t)g->E * 8, cudaMemcpyDeviceToHost));
  } else {
    for (uint64_t j = 0; j < g->E; ++j) out_weights[j] = 1.0;
  }
  return ZOGCU_OK;
}

}  // extern "C"
