// pagerank.cu -- PageRank power iteration on the device-resident in-CSR.
//
// Reference: priv/zog/src/centrality.zig:858-965 (ArrayGraph branch).  Per
// iteration the reference computes, over live nodes in ascending order,
//     sink     = sum_{deg(u)=0} x[u] / n                        (:926-931)
//     x'[v]    = (1-d)/n + d * (sink + sum_{u in in(v)} x[u]/deg(u))   (:933-944)
//     l1       = sum |x'[v] - x[v]|                                (:947-950)
// swaps, and stops once l1 < tol (:953-957).
//
// B200 design (one fused pass per iteration, warp-granular work):
//   * a PageRank view of the graph built on the first call: nodes renumbered
//     by out-degree (descending), so the contributions gathered most often --
//     c[u] = x[u]/deg(u), the reference's per-term quotient bit for bit -- form
//     a contiguous prefix; each row keeps the reference's ascending-source
//     order.  Random 8-byte gathers are limited by the L1 tag stage (about one
//     128-byte line per SM clock); a prefix of c (the "hub") is copied into
//     shared memory at the start of every iteration and gathered from there;
//   * degree-binned schedule, one warp per work item:
//       A  a block of consecutive rows, each of in-degree <= NNZ, with <= NNZ
//          arcs and <= kWarpRows rows in total: lane l loads arcs l, l+32,
//          ... (coalesced lines), gathers staged in the warp's shared-memory
//          slice with conflict-free stores, rows of in-degree <=
//          kShortLen summed by one lane each in the reference's order, longer
//          ones by the warp;
//       B  one row with NNZ < in-degree <= kLongChunk, reduced by a warp;
//       C  one kLongChunk-arc chunk of a longer row; the last warp to finish a
//          row (arrival counter) adds the chunk partials in chunk order and
//          runs the row's epilogue;
//     each warp runs a software pipeline over its items (descriptors two
//     ahead, arc ranges one ahead), so an item costs two dependent round
//     trips, and warps never wait on each other inside the pass;
//   * the kernel is a template over (CTA size, arcs per item, hub size); the
//     first PageRank solve on a graph times each configuration on its own
//     early iterations and keeps the fastest (ZOGCU_PR_CONFIG forces one),
//     also for later graphs of the same size on the device.  The fastest at
//     scale 24 is the pipelined kernel (pr_iter_kernel_pipe: the next row
//     block's gathers in flight with cp.async while the current one is
//     summed) with one 768-thread CTA per SM sharing a 64 KB hub: the hub's
//     gathers skip the L1 tag stage, and hub plus staging still fit the
//     164 KB shared-memory carveout that leaves L1 for the other gathers;
//   * the work-item lists are built on the device (segmented greedy pass);
//   * arc indices stream with an L2 evict-first policy, bypassing L1; gathered
//     contributions use an L2 evict-last policy;
//   * the epilogue writes x', c' = x'/deg and accumulates |x'-x| and the
//     dangling mass of x' (the next iteration's sink): lane -> warp -> CTA
//     partials, then a deterministic last-CTA reduction over fixed slots;
//   * convergence is decided on the device: the last CTA publishes l1 and a
//     converged flag, later launches of the chain exit at once, and the host
//     enqueues the chain with no round trip (a CUDA-graph while loop ended by
//     the kernel for chains of kLoopMinIters or more iterations);
//   * the precision form's FP32 phase runs propagation-blocked on large
//     graphs (pb_emit_kernel / pb_accum_kernel, below): messages streamed
//     into per-partition pieces and summed as exact integers in shared
//     memory instead of gathered.
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace zogcu {

constexpr int kShortLen = 32;            // in-degree summed by a single lane

// Kernel configurations the autotuner chooses from.
struct PrConfig {
  int threads;      // CTA size
  int nnz;          // arcs per row-block work item
  int hub_bytes;    // shared-memory hub per CTA
  int pipelined;    // 1: row-block gathers issued one item ahead (cp.async)
};
constexpr PrConfig kPrConfigs[] = {
    {1024, 128, 192 * 1024, 0},  // 0: one CTA per SM, biggest hub
    {1024, 256, 160 * 1024, 0},  // 1: one CTA per SM, bigger items
    {512, 256, 64 * 1024, 0},    // 2: two CTAs per SM
    {256, 256, 0, 0},            // 3: four CTAs per SM, no hub
    {256, 128, 0, 0},            // 4: four CTAs per SM, no hub, small items
    {256, 128, 0, 1},            // 5: four CTAs per SM, pipelined gathers
    {256, 256, 0, 1},            // 6: three CTAs per SM, pipelined gathers, bigger items
    {256, 256, 16 * 1024, 1},    // 7: as 6 with a 16 KB hub (a 40 KB hub measured 1.9x slower)
    {256, 256, 20 * 1024, 1},    // 8: as 6 with a 20 KB hub (the largest whose three CTAs fit a 164 KB carveout)
    {768, 256, 56 * 1024, 1},    // 9: one CTA of 24 warps per SM sharing a 56 KB hub
    {768, 256, 64 * 1024, 1},    // 10: as 9 with a 64 KB hub
};
constexpr int kNumPrConfigs = sizeof(kPrConfigs) / sizeof(kPrConfigs[0]);
constexpr int kDefaultPrConfig = 0;

struct PrState {
  unsigned long long iter;  // iterations completed
  double sink;              // sum over dangling live nodes of x_cur / n
  double l1;                // L1 step of the last iteration
  int converged;
  unsigned int done_ctas;   // arrival counter of the running launch
  unsigned int pad[2];
};

template <typename OffT, typename CT>
struct PrArgs {
  const OffT* off;
  const uint32_t* col;
  const uint32_t* deg;
  const PrTask* tasks;
  const uint32_t* long_first;
  uint32_t ntasks;
  uint32_t nlong;
  uint32_t hub;          // contributions [0, hub) are read from shared memory
  double* x0;
  double* x1;
  CT* c0;
  CT* c1;
  double* cta_part;      // [2 * gridDim.x]
  double* chunk_part;    // [ntasks]
  unsigned int* long_cnt;// [ntasks], indexed by a long row's first chunk task
  double* long_part;     // [2 * ntasks], same indexing
  PrState* st;
  const double* teleport;  // personalised teleport p (ranked order) or null
  double damping;
  double n_f;
  double tol;
  double stall;          // > 0: also stop once l1 > stall * previous l1
  unsigned long long max_iter;
  double ka, kb;         // katz: alpha, beta; alpha centrality: alpha
  double* x2;            // eigenvector: third rotating buffer
  uint32_t nv;           // node slots V (bound of every source index)
  unsigned long long cond;  // conditional handle of the CUDA-graph while loop running the chain
  int use_cond;             // 1: launched inside that loop; clear the condition when the chain ends
};

// Epilogue modes of the iteration kernel (all share the schedule and the
// gather path; the non-PageRank modes gather x itself).
enum : int { kModePageRank = 0, kModeKatz = 1, kModeAlpha = 2, kModeEigen = 3 };

// ---- cache-policy loads ------------------------------------------------------
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint4 ld_arcs(const uint4* a, uint64_t pol) {
  uint4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
      : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_arc(const uint32_t* a, uint64_t pol) {
  uint32_t v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_contrib(const double* a, uint64_t pol) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_contrib(const float* a, uint64_t pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
  return (double)v;
}

// Asynchronous gather of one contribution into shared memory (cp.async, 8 or
// 4 bytes, the plain sm_80 form); the copy lands without passing through
// registers, so a warp can keep a whole work item's gathers in flight while
// it sums the previous one.
__device__ __forceinline__ void cp_gather(double* dst, const double* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_gather(float* dst, const float* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <typename CT>
__device__ __forceinline__ double gather(uint32_t p, const CT* __restrict__ hub, uint32_t nhub,
                                         const CT* __restrict__ c, uint64_t pol) {
  return p < nhub ? (double)hub[p] : ld_contrib(c + p, pol);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Epilogue of one row: the reference's update (centrality.zig:943) evaluated
// with explicit round-to-nearest operations (no FMA contraction), then the
// residual / dangling bookkeeping and the next contribution c' = x'/deg.
// `deg`, `xo` and `tp` (teleport, when personalised) were loaded earlier.
template <typename CT>
__device__ __forceinline__ void pr_row_epilogue(uint32_t v, double rank_sum, uint32_t deg, double xo, double tp,
                                                bool personalised, double damping, double n_f,
                                                double* __restrict__ xnxt, CT* __restrict__ cnxt, double tele_u,
                                                double sink, double& l1, double& dsum) {
  if (deg == kDeletedDegree) return;
  const double tele = personalised ? __dmul_rn(1.0 - damping, tp) : tele_u;
  const double xn = __dadd_rn(tele, __dmul_rn(damping, __dadd_rn(sink, rank_sum)));
  l1 += fabs(xn - xo);
  xnxt[v] = xn;
  if (deg == 0) {
    dsum += __ddiv_rn(xn, n_f);
  } else {
    cnxt[v] = (CT)__ddiv_rn(xn, (double)deg);
  }
}

// Sum of c[col[e]] over e in [e0, e1) by one warp (lane partials, then a fixed
// shuffle tree).  Index vectors for the next step are loaded before the
// gathers of the current one, so two round trips overlap.
template <typename OffT, typename CT>
__device__ __forceinline__ double warp_range_sum(const uint32_t* __restrict__ col, const CT* __restrict__ c,
                                                 const CT* __restrict__ hub, uint32_t nhub, OffT e0, OffT e1,
                                                 int lane, uint64_t pol_arc, uint64_t pol_c) {
  const OffT base = e0 & ~(OffT)3;
  const uint32_t nvec = (uint32_t)((e1 - base + 3) >> 2);
  const uint4* cv = reinterpret_cast<const uint4*>(col + base);
  double s = 0.0;
  uint32_t j = lane;
  uint4 q0 = make_uint4(0, 0, 0, 0), q1 = make_uint4(0, 0, 0, 0);
  if (j < nvec) q0 = ld_arcs(cv + j, pol_arc);
  if (j + 32 < nvec) q1 = ld_arcs(cv + j + 32, pol_arc);
  for (; j < nvec; j += 64) {
    uint4 n0 = make_uint4(0, 0, 0, 0), n1 = make_uint4(0, 0, 0, 0);
    if (j + 64 < nvec) n0 = ld_arcs(cv + j + 64, pol_arc);
    if (j + 96 < nvec) n1 = ld_arcs(cv + j + 96, pol_arc);
    const bool two = j + 32 < nvec;
    const OffT ea = base + 4 * (OffT)j, eb = ea + 128;
    double v[8];
    v[0] = (ea >= e0 && ea < e1) ? gather(q0.x, hub, nhub, c, pol_c) : 0.0;
    v[1] = (ea + 1 >= e0 && ea + 1 < e1) ? gather(q0.y, hub, nhub, c, pol_c) : 0.0;
    v[2] = (ea + 2 >= e0 && ea + 2 < e1) ? gather(q0.z, hub, nhub, c, pol_c) : 0.0;
    v[3] = (ea + 3 >= e0 && ea + 3 < e1) ? gather(q0.w, hub, nhub, c, pol_c) : 0.0;
    v[4] = (two && eb < e1) ? gather(q1.x, hub, nhub, c, pol_c) : 0.0;
    v[5] = (two && eb + 1 < e1) ? gather(q1.y, hub, nhub, c, pol_c) : 0.0;
    v[6] = (two && eb + 2 < e1) ? gather(q1.z, hub, nhub, c, pol_c) : 0.0;
    v[7] = (two && eb + 3 < e1) ? gather(q1.w, hub, nhub, c, pol_c) : 0.0;
    s += ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]));
    q0 = n0;
    q1 = n1;
  }
  return warp_sum(s);
}

// Deterministic CTA sum of two doubles; result valid in thread 0.
__device__ __forceinline__ void cta_sum2(double& a, double& b, double* s_red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if (lane == 0) {
    s_red[2 * warp] = a;
    s_red[2 * warp + 1] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ra = 0.0, rb = 0.0;
    for (int w = 0; w < nw; ++w) {
      ra += s_red[2 * w];
      rb += s_red[2 * w + 1];
    }
    a = ra;
    b = rb;
  }
}

// Last-CTA reduction of the per-CTA and per-long-row partial slots, in a fixed
// order, then publication of the iteration's result.
__device__ void final_reduce(PrState* st, const double* cta_part, uint32_t ncta, const double* long_part,
                             const uint32_t* long_first, uint32_t nlong, unsigned long long next_iter, double tol,
                             double stall, bool set_l1, double* s_red, unsigned long long max_iter = 0,
                             unsigned long long cond = 0, int use_cond = 0) {
  double a = 0.0, b = 0.0;
  for (uint32_t i = threadIdx.x; i < ncta; i += blockDim.x) {
    a += __ldcg(cta_part + 2 * i);
    b += __ldcg(cta_part + 2 * i + 1);
  }
  for (uint32_t i = threadIdx.x; i < nlong; i += blockDim.x) {
    const uint32_t f = long_first[i];
    a += __ldcg(long_part + 2 * (size_t)f);
    b += __ldcg(long_part + 2 * (size_t)f + 1);
  }
  cta_sum2(a, b, s_red);
  if (threadIdx.x == 0) {
    st->sink = b;
    if (stall < 0.0) {  // sum-only publication (eigenvector SpMV: b = sum of squares)
      __threadfence();
      st->done_ctas = 0;
      return;
    }
    if (set_l1) {
      const bool stalled = stall > 0.0 && next_iter > 2 && a > stall * st->l1;
      st->l1 = a;
      st->converged = (a < tol || stalled) ? 1 : 0;
    } else {
      st->l1 = 0.0;
      st->converged = 0;
    }
    st->iter = next_iter;
    // inside a CUDA-graph while loop: the chain is over, run no further body
    if (use_cond && (st->converged || next_iter >= max_iter)) cudaGraphSetConditional(cond, 0u);
    __threadfence();
    st->done_ctas = 0;
  }
}

// Publishes a CTA's partials and runs the final reduction in the last CTA.
__device__ __forceinline__ void cta_publish(PrState* st, double* cta_part, const double* long_part,
                                            const uint32_t* long_first, uint32_t nlong, double l1, double dsum,
                                            unsigned long long next_iter, double tol, double stall, bool set_l1,
                                            double* s_red, int* s_flag, unsigned long long max_iter = 0,
                                            unsigned long long cond = 0, int use_cond = 0) {
  cta_sum2(l1, dsum, s_red);
  if (threadIdx.x == 0) {
    cta_part[2 * blockIdx.x] = l1;
    cta_part[2 * blockIdx.x + 1] = dsum;
    __threadfence();
    const unsigned int t = atomicAdd(&st->done_ctas, 1u);
    *s_flag = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (*s_flag) {
    __threadfence();
    final_reduce(st, cta_part, gridDim.x, long_part, long_first, nlong, next_iter, tol, stall, set_l1, s_red,
                 max_iter, cond, use_cond);
  }
}

// x0 / c0 from the start vector; sink of x0.  `given` = x0 already holds a
// caller's start vector in ranked order (warm start), else the uniform 1/n of
// centrality.zig:912-918.
template <typename OffT, typename CT>
__global__ void __launch_bounds__(256) pr_init_kernel(PrArgs<OffT, CT> A, uint32_t V, int given) {
  __shared__ double s_red[2 * 8];
  __shared__ int s_flag;
  double dsum = 0.0;
  const double init = 1.0 / A.n_f;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t deg = A.deg[v];
    double x = 0.0;
    if (deg != kDeletedDegree) {
      x = given ? A.x0[v] : init;
      if (deg == 0) dsum += __ddiv_rn(x, A.n_f);
      else A.c0[v] = (CT)__ddiv_rn(x, (double)deg);
    }
    A.x0[v] = x;
    A.x1[v] = 0.0;
  }
  cta_publish(A.st, A.cta_part, A.long_part, A.long_first, 0, 0.0, dsum, 0ull, A.tol, 0.0, false, s_red, &s_flag);
}

constexpr int pr_min_blocks(int threads) { return threads >= 1024 ? 1 : (threads >= 512 ? 2 : 4); }

// Row epilogue of the non-PageRank modes (katz: alpha*sum + beta,
// centrality.zig:1215; alpha centrality: alpha*sum, :1287; eigenvector: the raw
// sum, with its square added to the norm accumulator).
template <int MODE>
__device__ __forceinline__ void lin_row_epilogue(uint32_t v, double sum, uint32_t deg, double xo, double ka, double kb,
                                                 double* __restrict__ xnxt, double& l1, double& acc) {
  if (deg == kDeletedDegree) return;
  double xn;
  if constexpr (MODE == kModeKatz) {
    xn = __dadd_rn(__dmul_rn(ka, sum), kb);
  } else if constexpr (MODE == kModeAlpha) {
    xn = __dmul_rn(ka, sum);
  } else {
    xn = sum;
    acc += xn * xn;
  }
  if constexpr (MODE != kModeEigen) l1 += fabs(xn - xo);
  xnxt[v] = xn;
}

template <typename OffT, typename CT, int THREADS, int NNZ, int MODE = kModePageRank>
__global__ void __launch_bounds__(THREADS, pr_min_blocks(THREADS)) pr_iter_kernel(PrArgs<OffT, CT> A) {
  constexpr int WARPS = THREADS / 32;
  constexpr int NG = NNZ / 32;  // 32-arc groups of a row block: lane l holds arcs l, l+32, ...
  extern __shared__ __align__(16) unsigned char s_dyn[];
  __shared__ double s_red[2 * WARPS];
  __shared__ int s_flag;

  const PrState* st = A.st;
  const unsigned long long iter = *(volatile const unsigned long long*)&st->iter;
  const int converged = *(volatile const int*)&st->converged;
  if (converged || iter >= A.max_iter) {
    // the chain is over; inside a CUDA-graph while loop, also stop the loop
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(A.cond, 0u);
    return;
  }
  const double sink = *(volatile const double*)&st->sink;

  const int par = (int)(iter & 1ull);
  const double* __restrict__ xcur;
  double* __restrict__ xnxt;
  const CT* __restrict__ ccur;
  CT* __restrict__ cnxt;
  if constexpr (MODE == kModeEigen) {
    const int k3 = (int)(iter % 3ull);
    xcur = k3 == 0 ? A.x0 : (k3 == 1 ? A.x1 : A.x2);
    xnxt = k3 == 0 ? A.x1 : (k3 == 1 ? A.x2 : A.x0);
    ccur = reinterpret_cast<const CT*>(xcur);
    cnxt = nullptr;
  } else if constexpr (MODE != kModePageRank) {
    xcur = par ? A.x1 : A.x0;
    xnxt = par ? A.x0 : A.x1;
    ccur = reinterpret_cast<const CT*>(xcur);
    cnxt = nullptr;
  } else {
    xcur = par ? A.x1 : A.x0;
    xnxt = par ? A.x0 : A.x1;
    ccur = par ? A.c1 : A.c0;
    cnxt = par ? A.c0 : A.c1;
  }
  const double tele_u = (1.0 - A.damping) / A.n_f;
  const bool personalised = A.teleport != nullptr;
  const double damping = A.damping, n_f = A.n_f;
  const double ka = A.ka, kb = A.kb;
  auto epilogue = [&](uint32_t v, double s, uint32_t dg, double xo, double tp, double& el1, double& eacc) {
    if constexpr (MODE == kModePageRank)
      pr_row_epilogue(v, s, dg, xo, tp, personalised, damping, n_f, xnxt, cnxt, tele_u, sink, el1, eacc);
    else
      lin_row_epilogue<MODE>(v, s, dg, xo, ka, kb, xnxt, el1, eacc);
  };

  // ---- dynamic shared memory: [hub | per-warp staging] ----------------------
  const uint32_t nhub = A.hub;
  const size_t hub_bytes = ((size_t)nhub * sizeof(CT) + 15) & ~(size_t)15;
  CT* hub = reinterpret_cast<CT*>(s_dyn);
  double* staging = reinterpret_cast<double*>(s_dyn + hub_bytes);
  if (nhub) {
    const uint4* src = reinterpret_cast<const uint4*>(ccur);
    uint4* dst = reinterpret_cast<uint4*>(hub);
    const uint32_t n16 = (uint32_t)(((size_t)nhub * sizeof(CT)) >> 4);
    for (uint32_t i = threadIdx.x; i < n16; i += THREADS) dst[i] = __ldcg(src + i);
    __syncthreads();
  }

  const uint64_t pol_arc = policy_evict_first();
  const uint64_t pol_c = policy_evict_last();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* sv = staging + (size_t)warp * NNZ;
  double l1 = 0.0, dsum = 0.0;

  // Software pipeline over this warp's work items: descriptors are loaded two
  // items ahead and their arc ranges one item ahead, so a block needs two
  // dependent round trips (index vectors with row data, then gathers).
  const uint32_t nwarps = gridDim.x * WARPS;
  const PrTask none{0, 0};
  auto range_of = [&](const PrTask& tk, OffT& lo, OffT& hi) {
    const uint32_t kind = tk.b >> 30;
    const uint32_t end = (kind == kTaskBlock) ? (tk.b & 0x3FFFFFFFu) : tk.a + 1;
    lo = __ldg(A.off + tk.a);
    hi = __ldg(A.off + end);
  };
  uint32_t ti = blockIdx.x * WARPS + warp;
  PrTask t = ti < A.ntasks ? A.tasks[ti] : none;
  PrTask t1 = ti + nwarps < A.ntasks ? A.tasks[ti + nwarps] : none;
  OffT ra = 0, rb = 0;
  if (ti < A.ntasks) range_of(t, ra, rb);
  while (ti < A.ntasks) {
    const uint32_t tn = ti + nwarps;
    const PrTask t2 = tn + nwarps < A.ntasks ? A.tasks[tn + nwarps] : none;  // two ahead
    OffT na = 0, nb = 0;
    if (tn < A.ntasks) range_of(t1, na, nb);  // one ahead
    const uint32_t kind = t.b >> 30;
    if (kind == kTaskBlock) {
      // ---- rows [r0, r1): <= NNZ arcs, <= kWarpRows rows ------------------
      const uint32_t r0 = t.a, nrows = (t.b & 0x3FFFFFFFu) - t.a;
      const OffT e0 = ra, e1 = rb;
      const uint32_t na = (uint32_t)(e1 - e0);  // <= NNZ
      // round trip 1: arc indices (lane l takes arcs l, l+32, ...: each load
      // is one coalesced 128-byte line, and the staging stores below are
      // conflict-free), row bounds, row data for the epilogue
      uint32_t q[NG];
#pragma unroll
      for (int k = 0; k < NG; ++k)
        q[k] = ((uint32_t)lane + 32 * k < na) ? ld_arc(A.col + e0 + lane + 32 * k, pol_arc) : 0u;
      uint32_t b0 = 0, n0 = 0, b1 = 0, n1 = 0, d0 = kDeletedDegree, d1 = kDeletedDegree;
      double xo0 = 0.0, xo1 = 0.0, tp0 = 0.0, tp1 = 0.0;
      if ((uint32_t)lane < nrows) {
        const uint32_t r = r0 + lane;
        b0 = (uint32_t)(__ldg(A.off + r) - e0);
        n0 = (uint32_t)(__ldg(A.off + r + 1) - e0);
        d0 = __ldg(A.deg + r);
        xo0 = __ldg(xcur + r);
        if (personalised) tp0 = __ldg(A.teleport + r);
      }
      if ((uint32_t)lane + 32 < nrows) {
        const uint32_t r = r0 + lane + 32;
        b1 = (uint32_t)(__ldg(A.off + r) - e0);
        n1 = (uint32_t)(__ldg(A.off + r + 1) - e0);
        d1 = __ldg(A.deg + r);
        xo1 = __ldg(xcur + r);
        if (personalised) tp1 = __ldg(A.teleport + r);
      }
      // round trip 2: gathers into this warp's staging slice, arc order
#pragma unroll
      for (int k = 0; k < NG; ++k)
        if ((uint32_t)lane + 32 * k < na) sv[lane + 32 * k] = gather(q[k], hub, nhub, ccur, pol_c);
      __syncwarp();
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const uint32_t i = lane + 32 * half;
        const bool valid = i < nrows;
        const uint32_t b = half ? b1 : b0, en = half ? n1 : n0;
        const uint32_t dg = half ? d1 : d0;
        const double xo = half ? xo1 : xo0, tp = half ? tp1 : tp0;
        const bool is_short = valid && (en - b) <= (uint32_t)kShortLen;
        if (is_short) {
          double s = 0.0;
          for (uint32_t k = b; k < en; ++k) s += sv[k];  // ascending source order
          epilogue(r0 + i, s, dg, xo, tp, l1, dsum);
        }
        unsigned med = __ballot_sync(0xffffffffu, valid && !is_short);
        while (med) {
          const int k = __ffs(med) - 1;
          med &= med - 1;
          const uint32_t bk = __shfl_sync(0xffffffffu, b, k), ek = __shfl_sync(0xffffffffu, en, k);
          double s = 0.0;
          for (uint32_t j = bk + lane; j < ek; j += 32) s += sv[j];
          s = warp_sum(s);
          if (lane == k) epilogue(r0 + i, s, dg, xo, tp, l1, dsum);
        }
      }
      __syncwarp();
    } else {
      // ---- one heavy row (B) or one chunk of a long row (C) -----------------
      const uint32_t row = t.a;
      uint32_t dg = 0;
      double xo = 0.0, tp = 0.0;
      if (lane == 0) {
        dg = __ldg(A.deg + row);
        xo = __ldg(xcur + row);
        if (personalised) tp = __ldg(A.teleport + row);
      }
      if (kind == kTaskRow) {
        const double s = warp_range_sum(A.col, ccur, hub, nhub, ra, rb, lane, pol_arc, pol_c);
        if (lane == 0) epilogue(row, s, dg, xo, tp, l1, dsum);
      } else {
        const uint32_t c = t.b & 0xFFFFu;
        const uint32_t nch = (uint32_t)((rb - ra + kLongChunk - 1) / kLongChunk);
        const OffT e0 = ra + (OffT)c * kLongChunk;
        const OffT e1 = min(e0 + (OffT)kLongChunk, rb);
        const double s = warp_range_sum(A.col, ccur, hub, nhub, e0, e1, lane, pol_arc, pol_c);
        const uint32_t first = ti - c;
        unsigned int last = 0;
        if (lane == 0) {
          A.chunk_part[ti] = s;
          __threadfence();
          last = (atomicAdd(A.long_cnt + first, 1u) == nch - 1) ? 1u : 0u;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last && lane == 0) {
          __threadfence();
          double tot = 0.0;
          for (uint32_t k = 0; k < nch; ++k) tot += __ldcg(A.chunk_part + (first + k));
          double rl1 = 0.0, rds = 0.0;
          epilogue(row, tot, dg, xo, tp, rl1, rds);
          A.long_part[2 * (size_t)first] = rl1;
          A.long_part[2 * (size_t)first + 1] = rds;
          A.long_cnt[first] = 0;
        }
      }
    }
    t = t1;
    t1 = t2;
    ra = na;
    rb = nb;
    ti = tn;
  }
  cta_publish(A.st, A.cta_part, A.long_part, A.long_first, A.nlong, l1, dsum, iter + 1, A.tol,
              MODE == kModeEigen ? -1.0 : A.stall, true, s_red, &s_flag, A.max_iter, A.cond, A.use_cond);
}

constexpr int pr_pipe_min_blocks(int threads, int nnz) { return threads > 256 ? 1 : (nnz >= 256 ? 3 : 4); }

// The same iteration with the row-block gathers software-pipelined: while a
// warp sums work item i from one staging buffer, the gathers of item i+1 are
// already in flight into the other (cp.async), and the arc indices of item
// i+2 are loading into registers.  A row block thus costs about one memory
// round trip of waiting instead of two.  Each row is summed exactly as in
// pr_iter_kernel (same staging layout, same order); rows of kinds B and C are
// summed synchronously, as there.
template <typename OffT, typename CT, int THREADS, int NNZ, int MODE = kModePageRank, bool HUB = false>
__global__ void __launch_bounds__(THREADS, pr_pipe_min_blocks(THREADS, NNZ)) pr_iter_kernel_pipe(PrArgs<OffT, CT> A) {
  constexpr int WARPS = THREADS / 32;
  constexpr int NG = NNZ / 32;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  __shared__ double s_red[2 * WARPS];
  __shared__ int s_flag;

  const PrState* st = A.st;
  const unsigned long long iter = *(volatile const unsigned long long*)&st->iter;
  const int converged = *(volatile const int*)&st->converged;
  if (converged || iter >= A.max_iter) {
    // the chain is over; inside a CUDA-graph while loop, also stop the loop
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(A.cond, 0u);
    return;
  }
  const double sink = *(volatile const double*)&st->sink;

  const int par = (int)(iter & 1ull);
  const double* __restrict__ xcur;
  double* __restrict__ xnxt;
  const CT* __restrict__ ccur;
  CT* __restrict__ cnxt;
  if constexpr (MODE == kModeEigen) {
    const int k3 = (int)(iter % 3ull);
    xcur = k3 == 0 ? A.x0 : (k3 == 1 ? A.x1 : A.x2);
    xnxt = k3 == 0 ? A.x1 : (k3 == 1 ? A.x2 : A.x0);
    ccur = reinterpret_cast<const CT*>(xcur);
    cnxt = nullptr;
  } else if constexpr (MODE != kModePageRank) {
    xcur = par ? A.x1 : A.x0;
    xnxt = par ? A.x0 : A.x1;
    ccur = reinterpret_cast<const CT*>(xcur);
    cnxt = nullptr;
  } else {
    xcur = par ? A.x1 : A.x0;
    xnxt = par ? A.x0 : A.x1;
    ccur = par ? A.c1 : A.c0;
    cnxt = par ? A.c0 : A.c1;
  }
  const double tele_u = (1.0 - A.damping) / A.n_f;
  const bool personalised = A.teleport != nullptr;
  const double damping = A.damping, n_f = A.n_f;
  const double ka = A.ka, kb = A.kb;
  auto epilogue = [&](uint32_t v, double s, uint32_t dg, double xo, double tp, double& el1, double& eacc) {
    if constexpr (MODE == kModePageRank)
      pr_row_epilogue(v, s, dg, xo, tp, personalised, damping, n_f, xnxt, cnxt, tele_u, sink, el1, eacc);
    else
      lin_row_epilogue<MODE>(v, s, dg, xo, ka, kb, xnxt, el1, eacc);
  };

  // ---- dynamic shared memory: [hub | per-warp staging] ----------------------
  const uint32_t nhub = HUB ? A.hub : 0u;
  const size_t hub_bytes = ((size_t)nhub * sizeof(CT) + 15) & ~(size_t)15;
  CT* const hub = reinterpret_cast<CT*>(s_dyn);
  if constexpr (HUB) {
    if (nhub) {
      const uint4* src = reinterpret_cast<const uint4*>(ccur);
      uint4* dst = reinterpret_cast<uint4*>(hub);
      const uint32_t n16 = (uint32_t)(((size_t)nhub * sizeof(CT)) >> 4);
      for (uint32_t i = threadIdx.x; i < n16; i += THREADS) dst[i] = __ldcg(src + i);
      __syncthreads();
    }
  }
  const uint64_t pol_arc = policy_evict_first();
  const uint64_t pol_c = policy_evict_last();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  CT* const stage = reinterpret_cast<CT*>(s_dyn + hub_bytes) + (size_t)warp * 2 * NNZ;  // two buffers of NNZ
  double l1 = 0.0, dsum = 0.0;

  const uint32_t nwarps = gridDim.x * WARPS;
  const uint32_t ntasks = A.ntasks;
  const PrTask none{0, 0};
  auto task_at = [&](uint32_t i) { return i < ntasks ? A.tasks[i] : none; };
  auto range_of = [&](const PrTask& tk, OffT& lo, OffT& hi) {
    const uint32_t kind = tk.b >> 30;
    const uint32_t end = (kind == kTaskBlock) ? (tk.b & 0x3FFFFFFFu) : tk.a + 1;
    lo = __ldg(A.off + tk.a);
    hi = __ldg(A.off + end);
  };
  // Self-checks: a row block longer than NNZ arcs or a source outside [0, V)
  // sets bit 0 of st->pad[0] (the host reports an internal error) and the
  // access is skipped.
  unsigned int* const err = const_cast<unsigned int*>(&A.st->pad[0]);
  auto block_len = [&](bool blk, OffT lo, OffT hi) -> uint32_t {
    if (!blk) return 0u;
    const uint64_t n = (uint64_t)(hi - lo);
    if (n > (uint64_t)NNZ) {
      if (lane == 0) atomicOr(err, 1u);
      return 0u;
    }
    return (uint32_t)n;
  };
  // arc indices of a row block (lane l: arcs l, l+32, ...); zeros otherwise
  auto load_idx = [&](bool blk, OffT lo, OffT hi, uint32_t (&q)[NG]) {
    const uint32_t na = block_len(blk, lo, hi);
#pragma unroll
    for (int k = 0; k < NG; ++k)
      q[k] = ((uint32_t)lane + 32 * k < na) ? ld_arc(A.col + lo + lane + 32 * k, pol_arc) : 0u;
  };
  auto issue = [&](bool blk, OffT lo, OffT hi, const uint32_t (&q)[NG], CT* dst) {
    const uint32_t na = block_len(blk, lo, hi);
#pragma unroll
    for (int k = 0; k < NG; ++k) {
      if ((uint32_t)lane + 32 * k < na) {
        if (HUB && q[k] < nhub) dst[lane + 32 * k] = hub[q[k]];  // the hub's contributions, from shared memory
        else if (q[k] < A.nv) cp_gather(dst + lane + 32 * k, ccur + q[k]);
        else atomicOr(err, 1u);
      }
    }
    cp_commit();
  };

  uint32_t ti = blockIdx.x * WARPS + warp;
  PrTask t0 = task_at(ti), t1 = task_at(ti + nwarps), t2 = task_at(ti + 2 * nwarps);
  OffT a0 = 0, b0 = 0, a1 = 0, b1 = 0;
  if (ti < ntasks) range_of(t0, a0, b0);
  if (ti + nwarps < ntasks) range_of(t1, a1, b1);
  uint32_t q1[NG];
  {
    uint32_t q0[NG];
    const bool blk0 = ti < ntasks && (t0.b >> 30) == kTaskBlock;
    load_idx(blk0, a0, b0, q0);
    issue(blk0, a0, b0, q0, stage);
  }
  load_idx(ti + nwarps < ntasks && (t1.b >> 30) == kTaskBlock, a1, b1, q1);
  int cur = 0;
  while (ti < ntasks) {
    const uint32_t tn = ti + nwarps;
    const PrTask t3 = task_at(tn + 2 * nwarps);
    OffT a2 = 0, b2 = 0;
    if (tn + nwarps < ntasks) range_of(t2, a2, b2);
    const uint32_t kind = t0.b >> 30;
    // row data of the current block (used after its gathers land)
    const uint32_t r0 = t0.a;
    const uint32_t nrows = kind == kTaskBlock ? (t0.b & 0x3FFFFFFFu) - t0.a : 0u;
    uint32_t rb0 = 0, rn0 = 0, rb1 = 0, rn1 = 0, d0 = kDeletedDegree, d1 = kDeletedDegree;
    double xo0 = 0.0, xo1 = 0.0, tp0 = 0.0, tp1 = 0.0;
    if ((uint32_t)lane < nrows) {
      const uint32_t r = r0 + lane;
      rb0 = (uint32_t)(__ldg(A.off + r) - a0);
      rn0 = (uint32_t)(__ldg(A.off + r + 1) - a0);
      d0 = __ldg(A.deg + r);
      xo0 = __ldg(xcur + r);
      if (personalised) tp0 = __ldg(A.teleport + r);
    }
    if ((uint32_t)lane + 32 < nrows) {
      const uint32_t r = r0 + lane + 32;
      rb1 = (uint32_t)(__ldg(A.off + r) - a0);
      rn1 = (uint32_t)(__ldg(A.off + r + 1) - a0);
      d1 = __ldg(A.deg + r);
      xo1 = __ldg(xcur + r);
      if (personalised) tp1 = __ldg(A.teleport + r);
    }
    // gathers of item i+1 (indices already in registers), then indices of i+2
    issue(tn < ntasks && (t1.b >> 30) == kTaskBlock, a1, b1, q1, stage + (cur ^ 1) * NNZ);
    uint32_t q2[NG];
    load_idx(tn + nwarps < ntasks && (t2.b >> 30) == kTaskBlock, a2, b2, q2);
    if (kind == kTaskBlock) {
      cp_wait<1>();  // this item's gathers (all but the group just issued)
      __syncwarp();
      const CT* sv = stage + cur * NNZ;
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const uint32_t i = lane + 32 * half;
        const bool valid = i < nrows;
        const uint32_t b = half ? rb1 : rb0, en = half ? rn1 : rn0;
        const uint32_t dg = half ? d1 : d0;
        const double xo = half ? xo1 : xo0, tp = half ? tp1 : tp0;
        const bool is_short = valid && (en - b) <= (uint32_t)kShortLen;
        if (is_short) {
          double sum = 0.0;
          for (uint32_t k = b; k < en; ++k) sum += (double)sv[k];  // ascending source order
          epilogue(r0 + i, sum, dg, xo, tp, l1, dsum);
        }
        unsigned med = __ballot_sync(0xffffffffu, valid && !is_short);
        while (med) {
          const int k = __ffs(med) - 1;
          med &= med - 1;
          const uint32_t bk = __shfl_sync(0xffffffffu, b, k), ek = __shfl_sync(0xffffffffu, en, k);
          double sum = 0.0;
          for (uint32_t j = bk + lane; j < ek; j += 32) sum += (double)sv[j];
          sum = warp_sum(sum);
          if (lane == k) epilogue(r0 + i, sum, dg, xo, tp, l1, dsum);
        }
      }
      __syncwarp();  // the buffer is refilled two items later
    } else {
      // ---- one heavy row (B) or one chunk of a long row (C) -----------------
      const uint32_t row = t0.a;
      uint32_t dg = 0;
      double xo = 0.0, tp = 0.0;
      if (lane == 0) {
        dg = __ldg(A.deg + row);
        xo = __ldg(xcur + row);
        if (personalised) tp = __ldg(A.teleport + row);
      }
      if (kind == kTaskRow) {
        const double sum = warp_range_sum<OffT, CT>(A.col, ccur, hub, nhub, a0, b0, lane, pol_arc, pol_c);
        if (lane == 0) epilogue(row, sum, dg, xo, tp, l1, dsum);
      } else {
        const uint32_t c = t0.b & 0xFFFFu;
        const uint32_t nch = (uint32_t)((b0 - a0 + kLongChunk - 1) / kLongChunk);
        const OffT e0 = a0 + (OffT)c * kLongChunk;
        const OffT e1 = min(e0 + (OffT)kLongChunk, b0);
        const double sum = warp_range_sum<OffT, CT>(A.col, ccur, hub, nhub, e0, e1, lane, pol_arc, pol_c);
        const uint32_t first = ti - c;
        unsigned int last = 0;
        if (lane == 0) {
          A.chunk_part[ti] = sum;
          __threadfence();
          last = (atomicAdd(A.long_cnt + first, 1u) == nch - 1) ? 1u : 0u;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last && lane == 0) {
          __threadfence();
          double tot = 0.0;
          for (uint32_t k = 0; k < nch; ++k) tot += __ldcg(A.chunk_part + (first + k));
          double rl1 = 0.0, rds = 0.0;
          epilogue(row, tot, dg, xo, tp, rl1, rds);
          A.long_part[2 * (size_t)first] = rl1;
          A.long_part[2 * (size_t)first + 1] = rds;
          A.long_cnt[first] = 0;
        }
      }
    }
    t0 = t1;
    t1 = t2;
    t2 = t3;
    a0 = a1;
    b0 = b1;
    a1 = a2;
    b1 = b2;
#pragma unroll
    for (int k = 0; k < NG; ++k) q1[k] = q2[k];
    cur ^= 1;
    ti = tn;
  }
  cp_wait<0>();
  cta_publish(A.st, A.cta_part, A.long_part, A.long_first, A.nlong, l1, dsum, iter + 1, A.tol,
              MODE == kModeEigen ? -1.0 : A.stall, true, s_red, &s_flag, A.max_iter, A.cond, A.use_cond);
}

// ---------------------------------------------------------------------------
// PageRank view: degree ranking, re-laid in-CSR, schedules
// ---------------------------------------------------------------------------
__global__ void k_rank_keys(const uint32_t* __restrict__ deg, uint32_t V, uint32_t* __restrict__ key,
                            uint32_t* __restrict__ ids) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t d = deg[v];
    key[v] = (d == kDeletedDegree) ? 0xFFFFFFFFu : 0xFFFFFFFEu - d;  // descending degree, deleted last
    ids[v] = (uint32_t)v;
  }
}

__global__ void k_rank_invert(const uint32_t* __restrict__ perm, uint32_t V, uint32_t* __restrict__ rank,
                              const uint32_t* __restrict__ deg, uint32_t* __restrict__ pdeg,
                              const uint64_t* __restrict__ in_off, unsigned long long* __restrict__ pcnt) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < V; p += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = perm[p];
    rank[v] = (uint32_t)p;
    pdeg[p] = deg[v];
    pcnt[p] = in_off[v + 1] - in_off[v];
  }
}

// Row p of the ranked in-CSR = row perm[p] of the in-CSR with every source
// replaced by its rank; the order inside the row is kept.
// Rows of at most kLongRow arcs: a warp takes 32 consecutive ranked rows,
// each lane loads one row's source start, length and output start (so the
// perm -> in_off lookups of 32 rows overlap), and a warp scan numbers the
// group's arcs.  The warp then copies them 32 at a time across row
// boundaries: the lane for arc t finds its row as the last lane whose scan
// offset is <= t (five shuffles), and four such rounds issue their loads
// together.  Longer rows count as empty here; k_rank_rows_long copies them
// with one CTA per row, because ranking by out-degree gathers the rows of
// largest in-degree into the first groups, where one warp would copy them
// all in turn.
constexpr uint32_t kLongRow = 1024;

__global__ void k_rank_rows(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ rank, uint32_t V,
                            const uint64_t* __restrict__ in_off, const uint32_t* __restrict__ in_col,
                            const uint64_t* __restrict__ poff, uint32_t* __restrict__ pcol,
                            uint32_t* __restrict__ long_rows, unsigned int* __restrict__ n_long) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t p0 = ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5) * 32; p0 < V; p0 += nw * 32) {
    const uint64_t p = p0 + lane;
    unsigned long long src = 0ull, dst = 0ull;
    uint32_t len = 0;
    if (p < V) {
      const uint32_t v = perm[p];
      src = in_off[v];
      const uint64_t n = in_off[v + 1] - src;
      dst = poff[p];
      if (n > kLongRow) long_rows[atomicAdd(n_long, 1u)] = (uint32_t)p;
      else len = (uint32_t)n;
    }
    uint32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t pre = incl - len;  // empty, long and past-V rows add nothing
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);  // <= 32 * kLongRow
    for (uint32_t base = 0; base < total; base += 4 * 32) {
      unsigned long long k[4], q[4];
      uint32_t c[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t t = base + u * 32 + lane;
        int j = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1)
          if (__shfl_sync(0xffffffffu, pre, j + step) <= t) j += step;
        const uint32_t off = t - __shfl_sync(0xffffffffu, pre, j);
        k[u] = __shfl_sync(0xffffffffu, src, j) + off;
        q[u] = __shfl_sync(0xffffffffu, dst, j) + off;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) c[u] = (base + u * 32 + lane < total) ? in_col[k[u]] : 0u;
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (base + u * 32 + lane < total) pcol[q[u]] = rank[c[u]];
    }
  }
}

// The rows longer than kLongRow listed by k_rank_rows, one CTA per row.
__global__ void k_rank_rows_long(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ rank,
                                 const uint64_t* __restrict__ in_off, const uint32_t* __restrict__ in_col,
                                 const uint64_t* __restrict__ poff, const uint32_t* __restrict__ long_rows,
                                 const unsigned int* __restrict__ n_long, uint32_t* __restrict__ pcol) {
  const unsigned int n = *n_long;
  for (unsigned int i = blockIdx.x; i < n; i += gridDim.x) {
    const uint32_t p = long_rows[i];
    const uint32_t v = perm[p];
    const uint64_t s = in_off[v], len = in_off[v + 1] - s, d = poff[p];
#pragma unroll 4
    for (uint64_t k = threadIdx.x; k < len; k += blockDim.x) pcol[d + k] = rank[in_col[s + k]];
  }
}

__global__ void k_permute_in(const double* __restrict__ src, const uint32_t* __restrict__ perm, uint32_t V,
                             double* __restrict__ dst) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < V; p += (uint64_t)gridDim.x * blockDim.x)
    dst[p] = src[perm[p]];
}

__global__ void k_permute_out(const double* __restrict__ src, const uint32_t* __restrict__ rank, uint32_t V,
                              double* __restrict__ dst) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
    dst[v] = src[rank[v]];
}

__global__ void k_off_narrow(const uint64_t* __restrict__ a, uint32_t* __restrict__ b, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    b[i] = (uint32_t)a[i];
}

static unsigned grid_1d(uint64_t n) {
  uint64_t g = (n + 255) / 256;
  const uint64_t cap = (uint64_t)sm_count() * 16;
  if (g > cap) g = cap;
  return (unsigned)std::max<uint64_t>(g, 1);
}

// Ranking and re-laid in-CSR (once per graph; caller holds g->mu).
static int build_ranked_view(Graph* g, cudaStream_t s) {
  PrSchedule& P = g->pr;
  const uint32_t V = g->V;
  PhaseTrace tr("ranked_view", s);
  ZOGCU_TRY(P.rank.alloc((size_t)V * 4));
  ZOGCU_TRY(P.perm.alloc((size_t)V * 4));
  ZOGCU_TRY(P.deg.alloc((size_t)V * 4));
  {
    DevBuf key, key2, ids, tmp;
    ZOGCU_TRY(key.alloc((size_t)V * 4, s));
    ZOGCU_TRY(key2.alloc((size_t)V * 4, s));
    ZOGCU_TRY(ids.alloc((size_t)V * 4, s));
    k_rank_keys<<<grid_1d(V), 256, 0, s>>>(g->out_deg.as<uint32_t>(), V, key.as<uint32_t>(), ids.as<uint32_t>());
    ZOGCU_CUDA(cudaGetLastError());
    size_t tb = 0;
    ZOGCU_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.as<uint32_t>(), key2.as<uint32_t>(),
                                               ids.as<uint32_t>(), P.perm.as<uint32_t>(), (int64_t)V, 0, 32, s));
    ZOGCU_TRY(tmp.alloc(tb, s));
    ZOGCU_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, tb, key.as<uint32_t>(), key2.as<uint32_t>(),
                                               ids.as<uint32_t>(), P.perm.as<uint32_t>(), (int64_t)V, 0, 32, s));
  }
  tr.mark("ranking sort");
  DevBuf cnt, poff64;
  ZOGCU_TRY(cnt.alloc(((size_t)V + 1) * 8, s));
  ZOGCU_TRY(poff64.alloc(((size_t)V + 1) * 8, s));
  ZOGCU_CUDA(cudaMemsetAsync(cnt.ptr, 0, ((size_t)V + 1) * 8, s));
  k_rank_invert<<<grid_1d(V), 256, 0, s>>>(P.perm.as<uint32_t>(), V, P.rank.as<uint32_t>(),
                                           g->out_deg.as<uint32_t>(), P.deg.as<uint32_t>(),
                                           g->in_off64.as<uint64_t>(), cnt.as<unsigned long long>());
  ZOGCU_CUDA(cudaGetLastError());
  {
    size_t tb = 0;
    ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<unsigned long long>(),
                                             poff64.as<unsigned long long>(), (int64_t)V + 1, s));
    DevBuf tmp;
    ZOGCU_TRY(tmp.alloc(tb, s));
    ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, cnt.as<unsigned long long>(),
                                             poff64.as<unsigned long long>(), (int64_t)V + 1, s));
  }
  ZOGCU_TRY(P.col.alloc((g->E + 4) * 4));
  tr.mark("ranks, row offsets, column allocation");
  // k_rank_rows writes every arc; only the 4 padding entries need zeros
  ZOGCU_CUDA(cudaMemsetAsync(P.col.as<uint32_t>() + g->E, 0, 4 * 4, s));
  {
    // at most E / kLongRow rows are long
    DevBuf lrows, nl;
    ZOGCU_TRY(lrows.alloc((g->E / kLongRow + 1) * 4, s));
    ZOGCU_TRY(nl.alloc(4, s));
    ZOGCU_CUDA(cudaMemsetAsync(nl.ptr, 0, 4, s));
    k_rank_rows<<<grid_1d(V), 256, 0, s>>>(P.perm.as<uint32_t>(), P.rank.as<uint32_t>(), V,
                                            g->in_off64.as<uint64_t>(), g->in_col.as<uint32_t>(),
                                            poff64.as<uint64_t>(), P.col.as<uint32_t>(), lrows.as<uint32_t>(),
                                            nl.as<unsigned int>());
    ZOGCU_CUDA(cudaGetLastError());
    k_rank_rows_long<<<sm_count() * 4, 512, 0, s>>>(P.perm.as<uint32_t>(), P.rank.as<uint32_t>(),
                                                    g->in_off64.as<uint64_t>(), g->in_col.as<uint32_t>(),
                                                    poff64.as<uint64_t>(), lrows.as<uint32_t>(),
                                                    nl.as<unsigned int>(), P.col.as<uint32_t>());
    ZOGCU_CUDA(cudaGetLastError());
  }
  tr.mark("ranked rows");
  if (g->offsets32) {
    ZOGCU_TRY(P.off.alloc(((size_t)V + 1) * 4));
    k_off_narrow<<<grid_1d(V + 1), 256, 0, s>>>(poff64.as<uint64_t>(), P.off.as<uint32_t>(), (uint64_t)V + 1);
    ZOGCU_CUDA(cudaGetLastError());
  } else {
    ZOGCU_TRY(P.off.alloc(((size_t)V + 1) * 8));
    ZOGCU_CUDA(cudaMemcpyAsync(P.off.ptr, poff64.ptr, ((size_t)V + 1) * 8, cudaMemcpyDeviceToDevice, s));
  }
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  return ZOGCU_OK;
}

// Work items for row blocks of at most `nnz` arcs, built on the device.  The
// ranked rows are cut into segments of kTaskSegRows rows, and one warp walks
// each segment with the greedy rule: a row longer than nnz becomes one row
// item (<= kLongChunk arcs) or its run of chunk items; otherwise the block
// starting at row r ends at the largest e <= r + kWarpRows with
// off[e] - off[r] <= nnz (offsets never decrease, so the 64 candidates form
// a prefix the warp finds with two ballots).  Blocks never cross a segment
// boundary, so the segments are independent: a counting pass, a scan over
// the segments, and a writing pass that repeats the walk.  A cut costs a work
// item (one extra item per 4,096 rows at most); longer segments leave too few
// warps to hide the walk's dependent loads.
// Which rows share a block does not change any row's sum: a row's summation
// order depends only on its own arcs.
constexpr uint32_t kTaskSegRows = 4096;

constexpr uint32_t kTaskWin = 1024 + 72;  // offsets a warp stages: a window of rows plus one block's reach
constexpr int kTaskWarps = 4;              // warps (segments in flight) per CTA

template <typename OffT>
__global__ void __launch_bounds__(32 * kTaskWarps) k_task_segments(
    const OffT* __restrict__ off, uint32_t V, uint32_t nnz, uint32_t nseg, unsigned long long* __restrict__ seg_tasks,
    unsigned long long* __restrict__ seg_long, PrTask* __restrict__ tasks, uint32_t* __restrict__ long_first,
    int write, unsigned int* __restrict__ err) {
  // Each warp stages its segment's offsets in shared memory, a window at a
  // time with coalesced loads, so the walk's dependent steps read shared
  // memory instead of waiting on global loads.
  __shared__ OffT s_win[kTaskWarps][kTaskWin];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  OffT* const win = s_win[wib];
  const uint32_t nw = gridDim.x * kTaskWarps;
  for (uint32_t sg = blockIdx.x * kTaskWarps + wib; sg < nseg; sg += nw) {
    uint32_t r = sg * kTaskSegRows;  // V < 2^30, so no overflow
    const uint32_t rend = min(V, r + kTaskSegRows);
    unsigned long long nt = write ? seg_tasks[sg] : 0ull, nl = write ? seg_long[sg] : 0ull;
    uint32_t base = 0, have = 0;  // win[i] = off[base + i] for i < have
    while (r < rend) {  // r is the same in every lane
      // a step reads offsets r .. min(r + kWarpRows, rend) <= V
      if (min(r + (uint32_t)kWarpRows, rend) >= base + have) {
        base = r;
        have = min(kTaskWin, V + 1 - r);
        __syncwarp();
        for (uint32_t i = lane; i < have; i += 32) win[i] = __ldg(off + base + i);
        __syncwarp();
      }
      const OffT o0 = win[r - base];
      const uint64_t len = (uint64_t)(win[r + 1 - base] - o0);
      if (len > nnz) {
        if (len <= (uint64_t)kLongChunk) {
          if (write && lane == 0) tasks[nt] = PrTask{r, (kTaskRow << 30) | (r + 1)};
          ++nt;
        } else {
          uint64_t nch = (len + kLongChunk - 1) / kLongChunk;
          if (nch > 0xFFFFull) {
            if (lane == 0) atomicOr(err, 1u);
            nch = 0;
          }
          if (write) {
            if (lane == 0) long_first[nl] = (uint32_t)nt;
            for (uint32_t c = lane; c < (uint32_t)nch; c += 32) tasks[nt + c] = PrTask{r, (kTaskChunk << 30) | c};
          }
          ++nl;
          nt += nch;
        }
        ++r;
        continue;
      }
      const uint32_t lim = min(r + (uint32_t)kWarpRows, rend);
      const uint32_t c1 = r + 1 + lane;
      const bool ok1 = c1 <= lim && (uint64_t)(win[c1 - base] - o0) <= nnz;
      const unsigned m1 = __ballot_sync(0xffffffffu, ok1);
      uint32_t cnt = __popc(m1);
      if (m1 == 0xffffffffu) {
        const uint32_t c2 = r + 33 + lane;
        const bool ok2 = c2 <= lim && (uint64_t)(win[c2 - base] - o0) <= nnz;
        cnt += __popc(__ballot_sync(0xffffffffu, ok2));
      }
      if (write && lane == 0) tasks[nt] = PrTask{r, (kTaskBlock << 30) | (r + cnt)};
      ++nt;
      r += cnt;
    }
    if (!write && lane == 0) {
      seg_tasks[sg] = nt;
      seg_long[sg] = nl;
    }
  }
}

template <typename OffT>
static int build_task_list_t(Graph* g, int nnz, PrTaskList& L, cudaStream_t s) {
  const uint32_t V = g->V;
  const uint32_t nseg = (V + kTaskSegRows - 1) / kTaskSegRows;
  PhaseTrace tr(nnz == 128 ? "work items (128 arcs)" : "work items (256 arcs)", s);
  DevBuf cnt, offs, tmp;
  // [tasks per segment | trailing 0 | long rows per segment | trailing 0] and
  // their exclusive scans; the word after the scans is the error flag
  ZOGCU_TRY(cnt.alloc(2 * ((size_t)nseg + 1) * 8, s));
  ZOGCU_TRY(offs.alloc(2 * ((size_t)nseg + 1) * 8 + 8, s));
  ZOGCU_CUDA(cudaMemsetAsync(cnt.ptr, 0, cnt.bytes, s));
  ZOGCU_CUDA(cudaMemsetAsync(offs.ptr, 0, offs.bytes, s));
  unsigned long long* ct = cnt.as<unsigned long long>();
  unsigned long long* cl = ct + nseg + 1;
  unsigned long long* ot = offs.as<unsigned long long>();
  unsigned long long* ol = ot + nseg + 1;
  unsigned int* err = reinterpret_cast<unsigned int*>(ol + nseg + 1);
  const OffT* off = g->pr.off.as<OffT>();
  const unsigned grid = (unsigned)std::max<uint32_t>((nseg + kTaskWarps - 1) / kTaskWarps, 1);
  if (nseg) {
    k_task_segments<OffT><<<grid, 32 * kTaskWarps, 0, s>>>(off, V, (uint32_t)nnz, nseg, ct, cl, nullptr, nullptr, 0,
                                                           err);
    ZOGCU_CUDA(cudaGetLastError());
  }
  tr.mark("counting pass");
  size_t tb = 0;
  ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, ct, ot, (int64_t)nseg + 1, s));
  ZOGCU_TRY(tmp.alloc(tb, s));
  ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, ct, ot, (int64_t)nseg + 1, s));
  ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, cl, ol, (int64_t)nseg + 1, s));
  unsigned long long h[3] = {0, 0, 0};
  ZOGCU_CUDA(cudaMemcpyAsync(&h[0], ot + nseg, 8, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaMemcpyAsync(&h[1], ol + nseg, 8, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaMemcpyAsync(&h[2], err, 4, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  tr.mark("scan and totals");
  if (h[2]) return fail(ZOGCU_ERR_TOO_LARGE, "row in-degree too large for the chunk schedule");
  if (h[0] >= 0xFFFFFFFFull) return fail(ZOGCU_ERR_TOO_LARGE, "too many PageRank work items");
  L.num_tasks = (uint32_t)h[0];
  L.num_long = (uint32_t)h[1];
  ZOGCU_TRY(L.tasks.alloc(std::max<size_t>(L.num_tasks, 1) * sizeof(PrTask)));
  ZOGCU_TRY(L.long_first.alloc(std::max<size_t>(L.num_long, 1) * 4));
  tr.mark("allocation");
  if (nseg) {
    k_task_segments<OffT><<<grid, 32 * kTaskWarps, 0, s>>>(off, V, (uint32_t)nnz, nseg, ot, ol, L.tasks.as<PrTask>(),
                                               L.long_first.as<uint32_t>(), 1, err);
    ZOGCU_CUDA(cudaGetLastError());
  }
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  tr.mark("writing pass");
  L.built = true;
  return ZOGCU_OK;
}

static int build_task_list(Graph* g, int nnz, PrTaskList& L, cudaStream_t s) {
  return g->offsets32 ? build_task_list_t<uint32_t>(g, nnz, L, s) : build_task_list_t<uint64_t>(g, nnz, L, s);
}

static int list_index(int nnz) { return nnz == 128 ? 0 : 1; }

int ensure_pr_schedule(Graph* g, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g->mu);
  PrSchedule& P = g->pr;
  if (P.built) return ZOGCU_OK;
  if (g->V >= (1u << 30)) return fail(ZOGCU_ERR_TOO_LARGE, "PageRank schedule supports fewer than 2^30 nodes");
  ZOGCU_TRY(build_ranked_view(g, s));
  P.built = true;
  return ZOGCU_OK;
}

int ensure_task_list(Graph* g, int nnz, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g->mu);
  PrTaskList& L = g->pr.lists[list_index(nnz)];
  if (L.built) return ZOGCU_OK;
  return build_task_list(g, nnz, L, s);
}

// ---------------------------------------------------------------------------
// Launching a configuration
// ---------------------------------------------------------------------------
template <typename OffT, typename CT>
struct PrLauncher {
  using Fn = void (*)(PrArgs<OffT, CT>);
  static Fn fn(int cfg) {
    switch (cfg) {
      case 0: return pr_iter_kernel<OffT, CT, 1024, 128>;
      case 1: return pr_iter_kernel<OffT, CT, 1024, 256>;
      case 2: return pr_iter_kernel<OffT, CT, 512, 256>;
      case 3: return pr_iter_kernel<OffT, CT, 256, 256>;
      case 4: return pr_iter_kernel<OffT, CT, 256, 128>;
      case 5: return pr_iter_kernel_pipe<OffT, CT, 256, 128>;
      case 6: return pr_iter_kernel_pipe<OffT, CT, 256, 256>;
      case 9:
      case 10: return pr_iter_kernel_pipe<OffT, CT, 768, 256, kModePageRank, true>;
      case 7:
      default: return pr_iter_kernel_pipe<OffT, CT, 256, 256, kModePageRank, true>;
    }
  }
  static size_t staging_bytes(int cfg) {
    return (size_t)(kPrConfigs[cfg].threads / 32) * kPrConfigs[cfg].nnz * 8 * (kPrConfigs[cfg].pipelined ? 2 : 1);
  }
  // hub entries and dynamic shared memory of configuration `cfg` for V nodes
  static uint32_t hub_entries(int cfg, uint32_t V) {
    const uint32_t cap = (uint32_t)(kPrConfigs[cfg].hub_bytes / sizeof(CT));
    return std::min<uint32_t>(cap, V & ~3u);
  }
  // Grid of configuration `cfg` on the current device (resident CTAs per SM x
  // SMs).  The first call per device sets the kernel's dynamic shared-memory
  // limit; concurrent first calls do the same idempotent work.
  static int grid(int cfg, size_t dyn) {
    constexpr int kMaxDevices = 64;
    static std::atomic<int> cache[kMaxDevices][kNumPrConfigs];
    (void)dyn;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    const int known = cache[dev][cfg].load(std::memory_order_acquire);
    if (known > 0) return known;
    Fn f = fn(cfg);
    const size_t maxdyn = (size_t)kPrConfigs[cfg].hub_bytes + staging_bytes(cfg);
    // configurations can share a kernel (hub sizes differ): its limit must
    // admit the largest of them, whichever was set up last
    size_t limit = maxdyn;
    for (int c2 = 0; c2 < kNumPrConfigs; ++c2)
      if (fn(c2) == f) limit = std::max(limit, (size_t)kPrConfigs[c2].hub_bytes + staging_bytes(c2));
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)limit) != cudaSuccess) return 0;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, kPrConfigs[cfg].threads, maxdyn) != cudaSuccess)
      return 0;
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0) return 0;
    const int g = std::max(per_sm, 1) * nsm;
    cache[dev][cfg].store(g, std::memory_order_release);
    return g;
  }
};

// Per-call workspace, sized for the largest schedule a call may launch.
struct PrWork {
  DevBuf x0, x1, c0, c1, part, chunk, lcnt, lpart, stb, tele, tmp;
};

// Runs kernel `fn` as the body of a CUDA-graph while loop on stream s.  The
// body repeats until a launch clears the loop's condition, which the kernel
// does when the chain has converged or reached max_iter (the last CTA of the
// final iteration, or the first CTA of a launch that finds the chain over).
// So no launches are spent after convergence, and the host enqueues one graph
// launch instead of max_iter kernel launches.  The loop ends by construction:
// every body launch either completes one more iteration, at most max_iter in
// all, or clears the condition.
template <typename OffT, typename CT>
static int pr_launch_loop(void (*fn)(PrArgs<OffT, CT>), PrArgs<OffT, CT> A, int grid, int threads, size_t dyn,
                          cudaStream_t s) {
  cudaGraph_t graph = nullptr;
  ZOGCU_CUDA(cudaGraphCreate(&graph, 0));
  struct GraphGuard {
    cudaGraph_t g;
    ~GraphGuard() { cudaGraphDestroy(g); }
  } guard{graph};
  cudaGraphConditionalHandle h;
  ZOGCU_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1u, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  ZOGCU_CUDA(cudaGraphAddNode(&cnode, graph, nullptr, 0, &cp));
  A.cond = h;
  A.use_cond = 1;
  void* args[] = {&A};
  cudaKernelNodeParams kp = {};
  kp.func = reinterpret_cast<void*>(fn);
  kp.gridDim = dim3((unsigned)grid);
  kp.blockDim = dim3((unsigned)threads);
  kp.sharedMemBytes = (unsigned)dyn;
  kp.kernelParams = args;
  cudaGraphNode_t knode;
  ZOGCU_CUDA(cudaGraphAddKernelNode(&knode, cp.conditional.phGraph_out[0], nullptr, 0, &kp));
  cudaGraphExec_t exec = nullptr;
  ZOGCU_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  const cudaError_t e = cudaGraphLaunch(exec, s);
  cudaGraphExecDestroy(exec);  // an executable graph in flight is freed when it completes
  ZOGCU_CUDA(e);
  return ZOGCU_OK;
}

// Chains of at least this many iterations run as a CUDA-graph while loop.
// Building and instantiating the graph costs about 0.19 ms per call; a
// launch that returns at once after convergence costs about 5 us, so the loop
// pays off once some 40 launches would otherwise be spent after convergence.
constexpr uint64_t kLoopMinIters = 48;

// ZOGCU_PR_GRAPH_LOOP=0 launches every chain as plain kernel launches (same
// iterations, same results), e.g. for a profiler that cannot see kernels
// inside a conditional graph node.
static bool graph_loop_allowed() {
  const char* e = std::getenv("ZOGCU_PR_GRAPH_LOOP");
  return !(e && e[0] == '0');
}

// Launches up to `count` iterations of configuration `cfg`; `init` starts a
// new chain (state cleared, start vector written).  A.max_iter bounds the
// whole chain, so a chain may be launched in pieces of different
// configurations.  A piece of kLoopMinIters or more iterations runs as a
// CUDA-graph while loop; then *loop_from is set to `from_iter` (the chain's
// iteration count when the piece starts), and the caller adds the iterations
// the loop actually ran to *launches once it has read the chain's state.
template <typename OffT, typename CT>
static int pr_launch_chain(Graph* g, int cfg, PrArgs<OffT, CT> A, uint32_t V, int given, uint64_t max_iter,
                           uint64_t count, bool init, cudaStream_t s, uint64_t* launches,
                           int64_t* loop_from = nullptr, uint64_t from_iter = 0) {
  const PrTaskList& L = g->pr.lists[list_index(kPrConfigs[cfg].nnz)];
  A.tasks = L.tasks.as<PrTask>();
  A.long_first = L.long_first.as<uint32_t>();
  A.ntasks = L.num_tasks;
  A.nlong = L.num_long;
  A.hub = PrLauncher<OffT, CT>::hub_entries(cfg, V);
  A.max_iter = max_iter;
  A.cond = 0;
  A.use_cond = 0;
  const size_t dyn = (((size_t)A.hub * sizeof(CT) + 15) & ~(size_t)15) + PrLauncher<OffT, CT>::staging_bytes(cfg);
  int grid = PrLauncher<OffT, CT>::grid(cfg, dyn);
  if (grid <= 0) return fail(ZOGCU_ERR_CUDA, "PageRank kernel configuration could not be set up");
  const uint32_t warps = kPrConfigs[cfg].threads / 32;
  const uint32_t need = (A.ntasks + warps - 1) / warps;
  if (need > 0 && (uint32_t)grid > need) grid = (int)need;
  if (init) {
    ZOGCU_CUDA(cudaMemsetAsync(A.st, 0, sizeof(PrState), s));
    const unsigned init_grid = std::min(grid_1d(V), 148u * 4);
    pr_init_kernel<OffT, CT><<<init_grid, 256, 0, s>>>(A, V, given);
    ZOGCU_CUDA(cudaGetLastError());
    ++*launches;
  }
  auto fn = PrLauncher<OffT, CT>::fn(cfg);
  if (loop_from && count >= kLoopMinIters && graph_loop_allowed()) {
    ZOGCU_TRY((pr_launch_loop<OffT, CT>(fn, A, grid, kPrConfigs[cfg].threads, dyn, s)));
    *loop_from = (int64_t)from_iter;
    return ZOGCU_OK;
  }
  for (uint64_t k = 0; k < count; ++k) fn<<<grid, kPrConfigs[cfg].threads, dyn, s>>>(A);
  ZOGCU_CUDA(cudaGetLastError());
  *launches += count;
  return ZOGCU_OK;
}

// Configurations the tuner chose, per device and graph signature (node and
// arc counts rounded up to powers of two), so that a later graph of the same
// shape (a resource rebuilt from the same kind of data) starts with it instead
// of spending its first iterations on tuning.  Every configuration computes
// the same iteration; ZOGCU_PR_TUNE_CACHE=0 turns the sharing off.
static std::mutex g_tune_mu;
static std::vector<std::pair<uint64_t, int>> g_tune_cache;

static bool tune_cache_on() {
  const char* e = std::getenv("ZOGCU_PR_TUNE_CACHE");
  return !(e && e[0] == '0');
}
static uint64_t tune_key(const Graph* g) {
  auto lg = [](uint64_t x) {
    int b = 0;
    while (b < 63 && (1ull << b) < x) ++b;
    return (uint64_t)b;
  };
  return ((uint64_t)g->device << 16) | (lg(g->V) << 8) | lg(g->E);
}

// Kernel configuration of a graph: the one already chosen, the one forced by
// ZOGCU_PR_CONFIG, the default for small graphs, the one chosen for an
// earlier graph of the same signature, or -1 (time them).
static int pr_config_of(Graph* g) {
  std::lock_guard<std::mutex> lk(g->mu);
  PrSchedule& P = g->pr;
  if (P.config >= 0) return P.config;
  if (const char* e = std::getenv("ZOGCU_PR_CONFIG")) {
    const int c = std::atoi(e);
    if (c >= 0 && c < kNumPrConfigs) return P.config = c;
  }
  if (g->E < (1ull << 22)) return P.config = kDefaultPrConfig;
  if (tune_cache_on()) {
    std::lock_guard<std::mutex> tl(g_tune_mu);
    for (const auto& kv : g_tune_cache)
      if (kv.first == tune_key(g)) return P.config = kv.second;
  }
  return -1;
}

static void remember_config(const Graph* g, int cfg) {
  std::lock_guard<std::mutex> tl(g_tune_mu);
  const uint64_t k = tune_key(g);
  for (auto& kv : g_tune_cache)
    if (kv.first == k) {
      kv.second = cfg;
      return;
    }
  g_tune_cache.emplace_back(k, cfg);
}

// A chain of up to max_iter iterations.  When the graph has no configuration
// yet, the chain's own first iterations choose it: one iteration with the
// default configuration (caches warm), one timed iteration of each
// configuration, then, for each configuration within kSecondRound of that
// round's best, two iterations back to back of which the second is timed.
// The fastest runs the rest of the chain and is kept for the graph.  Every
// configuration computes the same iteration, so the tuning iterations are
// ordinary iterations of the solve.  Only iterations that ran before
// convergence count: a chain that converges during the second round keeps
// the first round's best among the configurations it timed, so one solve
// settles the choice and later solves repeat bit for bit; nothing is kept
// only when no timed iteration ran before convergence.
template <typename OffT, typename CT>
static int pr_run_chain(Graph* g, int cfg, const PrArgs<OffT, CT>& A, uint32_t V, int given, uint64_t max_iter,
                        cudaStream_t s, uint64_t* launches, int* used_cfg, int64_t* loop_from) {
  constexpr double kSecondRound = 1.15;
  constexpr uint64_t kMaxTuneIters = 1 + 3 * (uint64_t)kNumPrConfigs;
  *loop_from = -1;
  if (cfg >= 0 || max_iter <= kMaxTuneIters) {
    if (cfg < 0) cfg = kDefaultPrConfig;
    *used_cfg = cfg;
    return pr_launch_chain<OffT, CT>(g, cfg, A, V, given, max_iter, max_iter, true, s, launches, loop_from, 0);
  }
  // one-time launch setup of every configuration (attributes, occupancy,
  // module loading) happens here, outside the timed launches
  for (int c = 0; c < kNumPrConfigs; ++c)
    if (PrLauncher<OffT, CT>::grid(c, 0) <= 0) return fail(ZOGCU_ERR_CUDA, "PageRank kernel configuration could not be set up");
  ZOGCU_TRY((pr_launch_chain<OffT, CT>(g, kDefaultPrConfig, A, V, given, max_iter, 1, true, s, launches)));
  EventTimer tm[3 * kNumPrConfigs];
  int order[3 * kNumPrConfigs];
  int n = 0;
  auto timed = [&](int c) -> int {
    order[n] = c;
    ZOGCU_TRY(tm[n].start(s));
    ZOGCU_TRY((pr_launch_chain<OffT, CT>(g, c, A, V, given, max_iter, 1, false, s, launches)));
    ZOGCU_TRY(tm[n].stop(s));
    ++n;
    return ZOGCU_OK;
  };
  PrState hs;
  double best_of[kNumPrConfigs];
  int cnt[kNumPrConfigs];
  // timed launch i ran iteration 1 + i, which did work iff the chain reached 2 + i
  auto collect = [&]() -> int {
    ZOGCU_CUDA(cudaMemcpyAsync(&hs, A.st, sizeof(PrState), cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    for (int c = 0; c < kNumPrConfigs; ++c) cnt[c] = 0;
    for (int i = 0; i < n && hs.iter >= (unsigned long long)(2 + i); ++i) {
      const int c = order[i];
      if (c < 0) continue;  // untimed launch
      const double ms = tm[i].ms();
      best_of[c] = ms;  // the latest timed launch of a configuration counts
      ++cnt[c];
    }
    return ZOGCU_OK;
  };
  // Candidates: every configuration, except that the one-CTA-per-SM hub
  // configurations (1,024 threads, the largest hubs) are only timed when
  // their hub holds the contributions of at least half the arcs.  On large
  // graphs they never won (2.2 against 1.3 ms per iteration at scale 24).
  bool cand[kNumPrConfigs];
  {
    const uint32_t h = PrLauncher<OffT, CT>::hub_entries(0, V);
    std::vector<uint32_t> hd(h);
    if (h) ZOGCU_CUDA(cudaMemcpyAsync(hd.data(), g->pr.deg.ptr, (size_t)h * 4, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    uint64_t covered = 0;
    for (uint32_t d : hd)
      if (d != kDeletedDegree) covered += d;
    const bool big_hub_pays = 2 * covered >= g->E;
    for (int c = 0; c < kNumPrConfigs; ++c)
      cand[c] = big_hub_pays || !(kPrConfigs[c].threads >= 1024 && kPrConfigs[c].hub_bytes > 0);
  }
  // fastest configuration of `set` among those with a timing that counts
  // (-1 when none has one)
  auto fastest_of = [&](const bool* set) {
    int best = -1;
    for (int c = 0; c < kNumPrConfigs; ++c) {
      if (!set[c] || cnt[c] == 0) continue;
      if (best < 0 || best_of[c] < best_of[best]) best = c;
    }
    return best;
  };
  for (int c = 0; c < kNumPrConfigs; ++c)
    if (cand[c]) ZOGCU_TRY(timed(c));
  ZOGCU_TRY(collect());
  int best = fastest_of(cand);
  if (best >= 0) {
    // second round: each close configuration runs twice back to back and
    // only the second launch is timed, the one that starts from the caches
    // the configuration itself leaves (a configuration's first launch after
    // another one ran up to 8 % slow)
    const double cut = kSecondRound * best_of[best];
    bool close[kNumPrConfigs];
    for (int c = 0; c < kNumPrConfigs; ++c) close[c] = cand[c] && cnt[c] > 0 && best_of[c] <= cut;
    const int first_round = n;
    for (int c = kNumPrConfigs - 1; c >= 0; --c) {
      if (!close[c]) continue;
      ZOGCU_TRY((pr_launch_chain<OffT, CT>(g, c, A, V, given, max_iter, 1, false, s, launches)));
      order[n] = -1;  // untimed
      ++n;
      ZOGCU_TRY(timed(c));
    }
    ZOGCU_TRY(collect());
    // the close configurations are ranked by their second-round time alone;
    // if the chain converged before any of those counted, the first round's
    // best is kept
    for (int i = 0; i < first_round; ++i)
      if (order[i] >= 0 && close[order[i]] && cnt[order[i]] > 0) --cnt[order[i]];
    const int second = fastest_of(close);
    if (second >= 0) best = second;
  }
  if (std::getenv("ZOGCU_PR_TUNE_LOG")) {  // diagnostic: the tuning launches in order
    for (int i = 0; i < n; ++i)
      if (order[i] >= 0)
        std::fprintf(stderr, "zogcu pagerank tuning: iteration %d config %d %.4f ms%s\n", 1 + i, order[i],
                     tm[i].ms(), hs.iter < (unsigned long long)(2 + i) ? " (after convergence)" : "");
  }
  if (best >= 0) {
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->pr.config < 0) g->pr.config = best;
    best = g->pr.config;
    remember_config(g, best);
  } else {
    best = kDefaultPrConfig;
  }
  *used_cfg = best;
  if (hs.converged || hs.iter >= max_iter) return ZOGCU_OK;  // the chain ended during tuning
  return pr_launch_chain<OffT, CT>(g, best, A, V, given, max_iter, max_iter - 1 - (uint64_t)n, false, s, launches,
                                   loop_from, hs.iter);
}

// ---------------------------------------------------------------------------
// Propagation-blocked iteration: the FP32 bulk phase of the precision form
// ---------------------------------------------------------------------------
// The gather kernels above spend one L1 tag lookup per arc on a random 4- or
// 8-byte contribution, which caps them near one arc per SM clock whatever the
// contribution's width.  The blocked iteration streams instead:
//   emit:       a CTA stages the FP32 contributions of one source block in
//               shared memory and writes one message per position of the
//               block's pieces (coalesced 16-byte stores);
//   accumulate: a CTA zeroes integer accumulators for one partition's rows in
//               shared memory, streams the partition's pieces from every block
//               (16-byte loads), adds each message scaled by 2^kPbShift, and
//               runs the row epilogue of pr_iter_kernel.
// Integer sums do not depend on the order of the additions, so the result is
// deterministic although many warps add at once.  Shared-memory atomics are
// native for 32-bit integers only (64-bit and floating-point additions
// measured 9-15x slower on this part), so each 64-bit accumulator is two
// 32-bit words: the low word's atomicAdd returns the old value, and an
// addition that wraps it adds its carry to the high word.  A message below
// 2^(32 - kPbShift) = 6e-8 touches the low word only.
// Scale: messages lie in [0, 1] and a row's sum is at most the total mass
// (1), far below 2^(64 - kPbShift); rounding a message to a multiple of
// 2^-kPbShift (error <= 6.9e-18) is below the FP32 rounding of any message
// above 1.2e-10.  Within a piece, the arcs of one row are spread by a
// multiplicative permutation, so that lanes of one warp rarely add to the
// same word (measured 1.02 -> 0.65 ms per accumulate at scale 24).
constexpr uint32_t kPbRows = 24576;          // rows per partition (accumulators in shared memory)
constexpr uint32_t kPbSrcs = 24576;          // sources per block (contributions in shared memory)
constexpr uint64_t kPbCutArcs = 1ull << 20;  // arcs per partition / block before a cut
constexpr uint32_t kPbItem = 1u << 18;        // positions per emit work item (about one per block)
constexpr uint64_t kPbMaxPieces = 1ull << 26;
constexpr int kPbShift = 56;
constexpr int kPbThreads = 1024;
constexpr size_t kPbAccBytes = (size_t)2 * (kPbRows + 1) * 4;
constexpr size_t kPbEmitBytes = (size_t)kPbSrcs * 4;

// Group starts: element i starts a group when i is a multiple of rows_max or
// the running count before it crosses a multiple of arcs_max.
template <typename T>
__global__ void k_pb_cut(const T* __restrict__ cum, uint32_t n, uint32_t rows_max, uint64_t arcs_max,
                         uint32_t* __restrict__ flag) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    bool c = (i % rows_max) == 0;
    if (!c) c = ((uint64_t)cum[i] / arcs_max) != ((uint64_t)cum[i - 1] / arcs_max);
    flag[i] = c ? 1u : 0u;
  }
}

// Group of every element (idx = exclusive scan of flag) and first element of
// every group.
__global__ void k_pb_groups(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ idx, uint32_t n,
                            uint32_t* __restrict__ lo, uint32_t* __restrict__ of) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = idx[i] + flag[i] - 1u;
    of[i] = g;
    if (flag[i]) lo[g] = (uint32_t)i;
  }
}

__global__ void k_pb_sizes(const uint32_t* __restrict__ lo, uint32_t ng, uint32_t n, uint32_t* __restrict__ sz) {
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < ng; g += (uint64_t)gridDim.x * blockDim.x)
    sz[g] = (g + 1 < ng ? lo[g + 1] : n) - lo[g];
}

__global__ void k_pb_outdeg(const uint32_t* __restrict__ deg, uint32_t V, unsigned long long* __restrict__ d) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t x = deg[v];
    d[v] = x == kDeletedDegree ? 0ull : x;
  }
}

// Arcs per piece (key = block * P + partition); one warp per row.
template <typename OffT>
__global__ void k_pb_count(const OffT* __restrict__ off, const uint32_t* __restrict__ col, uint32_t V,
                           const uint32_t* __restrict__ blk_of, const uint32_t* __restrict__ part_of, uint32_t P,
                           uint32_t* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; r < V; r += nw) {
    const uint64_t pr = part_of[r];
    const OffT e = off[r + 1];
    for (OffT k = off[r] + lane; k < e; k += 32) atomicAdd(&cnt[(uint64_t)blk_of[col[k]] * P + pr], 1u);
  }
}

// Padded piece sizes; the extra last element makes the exclusive scan's last
// entry the total.
__global__ void k_pb_pad(const uint32_t* __restrict__ cnt, uint64_t nkeys, unsigned long long* __restrict__ padded) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k <= nkeys; k += (uint64_t)gridDim.x * blockDim.x)
    padded[k] = k < nkeys ? (unsigned long long)((cnt[k] + 3u) & ~3u) : 0ull;
}

// Multiplier of each piece's position permutation j -> (j * m) mod n: a prime
// not dividing n, whose residue is neither 1 nor n - 1 (those keep runs
// together); m = 1 (identity) when n <= 2.  Four primes above 7,900 cannot
// all divide an n below 2^32.
__global__ void k_pb_mult(const uint32_t* __restrict__ cnt, uint64_t nkeys, uint32_t* __restrict__ mult) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nkeys; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t n = cnt[k];
    uint32_t m = 1u;
    if (n > 2u) {
      const uint32_t cand[4] = {7919u, 104729u, 1299709u, 15485863u};
      for (int i = 0; i < 4; ++i) {
        const uint32_t r = cand[i] % n;
        if (n % cand[i] != 0u && r > 1u && r != n - 1u) {
          m = cand[i];
          break;
        }
      }
    }
    mult[k] = m;
  }
}

__global__ void k_fill_u16(uint16_t* __restrict__ a, uint64_t n, uint16_t v) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    a[i] = v;
}

// Places every arc at its piece's next position (permuted); one warp per row.
// The same traversal as k_pb_count, so each piece receives exactly cnt arcs.
template <typename OffT>
__global__ void k_pb_scatter(const OffT* __restrict__ off, const uint32_t* __restrict__ col, uint32_t V,
                             const uint32_t* __restrict__ blk_of, const uint32_t* __restrict__ blk_lo,
                             const uint32_t* __restrict__ part_of, const uint32_t* __restrict__ row_lo, uint32_t P,
                             const uint32_t* __restrict__ start, const uint32_t* __restrict__ cnt,
                             const uint32_t* __restrict__ mult, uint32_t* __restrict__ cursor,
                             uint16_t* __restrict__ sl, uint16_t* __restrict__ dl) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; r < V; r += nw) {
    const uint32_t pr = part_of[r];
    const uint16_t dloc = (uint16_t)(r - row_lo[pr]);
    const OffT e = off[r + 1];
    for (OffT k = off[r] + lane; k < e; k += 32) {
      const uint32_t src = col[k];
      const uint32_t b = blk_of[src];
      const uint64_t key = (uint64_t)b * P + pr;
      const uint32_t j = atomicAdd(&cursor[key], 1u);
      const uint32_t pos = start[key] + (uint32_t)(((uint64_t)j * mult[key]) % cnt[key]);
      sl[pos] = (uint16_t)(src - blk_lo[b]);
      dl[pos] = dloc;
    }
  }
}

// Partition-major piece tables, and the first position of every block (the
// block-major position of piece (b, 0)).
__global__ void k_pb_tables(const unsigned long long* __restrict__ start, const uint32_t* __restrict__ cnt, uint32_t B,
                            uint32_t P, uint32_t* __restrict__ pstart, uint32_t* __restrict__ pcount,
                            unsigned long long* __restrict__ blk_pos) {
  const uint64_t nkeys = (uint64_t)B * P;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k <= nkeys; k += (uint64_t)gridDim.x * blockDim.x) {
    if (k < nkeys) {
      const uint64_t b = k / P, p = k % P;
      pstart[p * B + b] = (uint32_t)start[k];
      pcount[p * B + b] = (cnt[k] + 3u) & ~3u;
    }
    if (k % P == 0) blk_pos[k / P] = start[k];
  }
}

// The four rows of largest in-degree (at least kPbHeavyMin) of every
// partition, as local indices (0xFFFF = none); one warp per partition.
constexpr uint32_t kPbHeavyMin = 64;
template <typename OffT>
__global__ void k_pb_heavy(const OffT* __restrict__ off, const uint32_t* __restrict__ row_lo,
                           const uint32_t* __restrict__ row_n, uint32_t P, uint2* __restrict__ heavy) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t p = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; p < P; p += nw) {
    const uint32_t r0 = row_lo[p], nr = row_n[p];
    uint64_t best[4] = {0, 0, 0, 0};  // (in-degree << 16 | 0xFFFF - local row), largest first
    for (uint32_t r = lane; r < nr; r += 32) {
      const uint64_t d = (uint64_t)(off[r0 + r + 1] - off[r0 + r]);
      uint64_t key = (d << 16) | (0xFFFFu - r);
      for (int k = 0; k < 4; ++k)
        if (key > best[k]) {
          const uint64_t t = best[k];
          best[k] = key;
          key = t;
        }
    }
    uint32_t pick[4];
    for (int k = 0; k < 4; ++k) {  // k-th largest over the warp; its lane drops it
      uint64_t m = best[0];
      for (int o = 16; o > 0; o >>= 1) {
        const uint64_t t = __shfl_xor_sync(0xffffffffu, m, o);
        m = t > m ? t : m;
      }
      const unsigned owner = __ballot_sync(0xffffffffu, best[0] == m && m != 0);
      if (m != 0 && lane == __ffs(owner) - 1) {
        best[0] = best[1];
        best[1] = best[2];
        best[2] = best[3];
        best[3] = 0;
      }
      pick[k] = (m >> 16) >= kPbHeavyMin ? 0xFFFFu - (uint32_t)(m & 0xFFFFu) : 0xFFFFu;
    }
    if (lane == 0) heavy[p] = make_uint2(pick[0] | (pick[1] << 16), pick[2] | (pick[3] << 16));
  }
}

template <typename OffT>
__global__ void k_pb_part_arcs(const OffT* __restrict__ off, const uint32_t* __restrict__ row_lo,
                               const uint32_t* __restrict__ row_n, uint32_t P, unsigned long long* __restrict__ arcs) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < P; p += (uint64_t)gridDim.x * blockDim.x)
    arcs[p] = (unsigned long long)(off[row_lo[p] + row_n[p]] - off[row_lo[p]]);
}

// Cuts n elements into groups (flags, exclusive scan, first elements); returns
// the group count, the group of every element (of) and each group's first
// element (lo) and size (sz).
template <typename T>
static int pb_groups(const T* cum, uint32_t n, uint32_t rows_max, uint64_t arcs_max, DevBuf& of, DevArray& lo,
                     DevArray& sz, uint32_t* ngroups, cudaStream_t s) {
  DevBuf flag, idx, tmp;
  ZOGCU_TRY(flag.alloc((size_t)n * 4, s));
  ZOGCU_TRY(idx.alloc((size_t)n * 4, s));
  ZOGCU_TRY(of.alloc((size_t)n * 4, s));
  k_pb_cut<T><<<grid_1d(n), 256, 0, s>>>(cum, n, rows_max, arcs_max, flag.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  size_t tb = 0;
  ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.as<uint32_t>(), idx.as<uint32_t>(), (int64_t)n, s));
  ZOGCU_TRY(tmp.alloc(tb, s));
  ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, flag.as<uint32_t>(), idx.as<uint32_t>(), (int64_t)n, s));
  uint32_t last[2] = {0, 0};
  ZOGCU_CUDA(cudaMemcpyAsync(&last[0], idx.as<uint32_t>() + (n - 1), 4, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaMemcpyAsync(&last[1], flag.as<uint32_t>() + (n - 1), 4, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  const uint32_t ng = last[0] + last[1];
  ZOGCU_TRY(lo.alloc((size_t)ng * 4));
  ZOGCU_TRY(sz.alloc((size_t)ng * 4));
  k_pb_groups<<<grid_1d(n), 256, 0, s>>>(flag.as<uint32_t>(), idx.as<uint32_t>(), n, lo.as<uint32_t>(),
                                         of.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  k_pb_sizes<<<grid_1d(ng), 256, 0, s>>>(lo.as<uint32_t>(), ng, n, sz.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  *ngroups = ng;
  return ZOGCU_OK;
}

// Builds the blocked layout from the degree-ranked view (caller holds g->mu).
// Leaves state -1 (the gather kernels are used instead) when the graph is too
// large for 32-bit positions or the piece tables would exceed kPbMaxPieces.
template <typename OffT>
static int build_pb_view(Graph* g, cudaStream_t s) {
  PbView& Q = g->pb;
  const PrSchedule& S = g->pr;
  const uint32_t V = g->V;
  const OffT* off = S.off.as<OffT>();
  const uint32_t* col = S.col.as<uint32_t>();
  Q.state = -1;
  if (V == 0 || g->E == 0) return ZOGCU_OK;
  DevBuf part_of, blk_of;
  ZOGCU_TRY(pb_groups<OffT>(off, V, kPbRows, kPbCutArcs, part_of, Q.row_lo, Q.row_n, &Q.P, s));
  {
    DevBuf d, cum, tmp;
    ZOGCU_TRY(d.alloc((size_t)V * 8, s));
    ZOGCU_TRY(cum.alloc((size_t)V * 8, s));
    k_pb_outdeg<<<grid_1d(V), 256, 0, s>>>(S.deg.as<uint32_t>(), V, d.as<unsigned long long>());
    ZOGCU_CUDA(cudaGetLastError());
    size_t tb = 0;
    ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, d.as<unsigned long long>(), cum.as<unsigned long long>(),
                                             (int64_t)V, s));
    ZOGCU_TRY(tmp.alloc(tb, s));
    ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, d.as<unsigned long long>(), cum.as<unsigned long long>(),
                                             (int64_t)V, s));
    ZOGCU_TRY(pb_groups<unsigned long long>(cum.as<unsigned long long>(), V, kPbSrcs, kPbCutArcs, blk_of, Q.blk_lo,
                                            Q.blk_n, &Q.B, s));
  }
  const uint64_t nkeys = (uint64_t)Q.B * Q.P;
  if (nkeys > kPbMaxPieces) return ZOGCU_OK;
  DevBuf cnt, padded, start64, start32, mult, cursor, blk_pos;
  ZOGCU_TRY(cnt.alloc(nkeys * 4, s));
  ZOGCU_CUDA(cudaMemsetAsync(cnt.ptr, 0, nkeys * 4, s));
  k_pb_count<OffT><<<grid_1d((uint64_t)V * 32), 256, 0, s>>>(off, col, V, blk_of.as<uint32_t>(), part_of.as<uint32_t>(),
                                                              Q.P, cnt.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_TRY(padded.alloc((nkeys + 1) * 8, s));
  ZOGCU_TRY(start64.alloc((nkeys + 1) * 8, s));
  k_pb_pad<<<grid_1d(nkeys + 1), 256, 0, s>>>(cnt.as<uint32_t>(), nkeys, padded.as<unsigned long long>());
  ZOGCU_CUDA(cudaGetLastError());
  {
    size_t tb = 0;
    DevBuf tmp;
    ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, padded.as<unsigned long long>(),
                                             start64.as<unsigned long long>(), (int64_t)nkeys + 1, s));
    ZOGCU_TRY(tmp.alloc(tb, s));
    ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, padded.as<unsigned long long>(),
                                             start64.as<unsigned long long>(), (int64_t)nkeys + 1, s));
  }
  unsigned long long npad = 0;
  ZOGCU_CUDA(cudaMemcpyAsync(&npad, start64.as<unsigned long long>() + nkeys, 8, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  if (npad >= (1ull << 32) - 4) return ZOGCU_OK;
  Q.npad = npad;
  ZOGCU_TRY(start32.alloc(nkeys * 4, s));
  k_off_narrow<<<grid_1d(nkeys), 256, 0, s>>>(start64.as<uint64_t>(), start32.as<uint32_t>(), nkeys);
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_TRY(mult.alloc(nkeys * 4, s));
  k_pb_mult<<<grid_1d(nkeys), 256, 0, s>>>(cnt.as<uint32_t>(), nkeys, mult.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_TRY(cursor.alloc(nkeys * 4, s));
  ZOGCU_CUDA(cudaMemsetAsync(cursor.ptr, 0, nkeys * 4, s));
  ZOGCU_TRY(Q.sl.alloc(npad * 2 + 16));
  ZOGCU_TRY(Q.dl.alloc(npad * 2 + 16));
  ZOGCU_CUDA(cudaMemsetAsync(Q.sl.ptr, 0, npad * 2 + 16, s));
  k_fill_u16<<<grid_1d(npad + 8), 256, 0, s>>>(Q.dl.as<uint16_t>(), npad + 8, (uint16_t)kPbRows);
  ZOGCU_CUDA(cudaGetLastError());
  k_pb_scatter<OffT><<<grid_1d((uint64_t)V * 32), 256, 0, s>>>(
      off, col, V, blk_of.as<uint32_t>(), Q.blk_lo.as<uint32_t>(), part_of.as<uint32_t>(), Q.row_lo.as<uint32_t>(),
      Q.P, start32.as<uint32_t>(), cnt.as<uint32_t>(), mult.as<uint32_t>(), cursor.as<uint32_t>(), Q.sl.as<uint16_t>(),
      Q.dl.as<uint16_t>());
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_TRY(Q.pstart.alloc(nkeys * 4));
  ZOGCU_TRY(Q.pcount.alloc(nkeys * 4));
  ZOGCU_TRY(blk_pos.alloc(((size_t)Q.B + 1) * 8, s));
  k_pb_tables<<<grid_1d(nkeys + 1), 256, 0, s>>>(start64.as<unsigned long long>(), cnt.as<uint32_t>(), Q.B, Q.P,
                                                 Q.pstart.as<uint32_t>(), Q.pcount.as<uint32_t>(),
                                                 blk_pos.as<unsigned long long>());
  ZOGCU_CUDA(cudaGetLastError());
  // emit work items (chunks of each block's positions, largest first) and
  // partitions ordered by arcs (largest first), so the longest CTAs start first
  std::vector<unsigned long long> bpos((size_t)Q.B + 1), parcs(Q.P);
  {
    DevBuf pa;
    ZOGCU_TRY(pa.alloc((size_t)Q.P * 8, s));
    k_pb_part_arcs<OffT><<<grid_1d(Q.P), 256, 0, s>>>(off, Q.row_lo.as<uint32_t>(), Q.row_n.as<uint32_t>(), Q.P,
                                                      pa.as<unsigned long long>());
    ZOGCU_CUDA(cudaGetLastError());
    ZOGCU_CUDA(cudaMemcpyAsync(parcs.data(), pa.ptr, (size_t)Q.P * 8, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaMemcpyAsync(bpos.data(), blk_pos.ptr, ((size_t)Q.B + 1) * 8, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
  }
  std::vector<PbItem> items;
  for (uint32_t b = 0; b < Q.B; ++b)
    for (uint64_t a = bpos[b]; a < bpos[b + 1]; a += kPbItem)
      items.push_back(PbItem{b, (uint32_t)a, (uint32_t)std::min<uint64_t>(a + kPbItem, bpos[b + 1]), 0u});
  std::stable_sort(items.begin(), items.end(),
                   [](const PbItem& x, const PbItem& y) { return x.hi - x.lo > y.hi - y.lo; });
  std::vector<uint32_t> order(Q.P);
  for (uint32_t p = 0; p < Q.P; ++p) order[p] = p;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return parcs[x] > parcs[y]; });
  Q.nitems = (uint32_t)items.size();
  ZOGCU_TRY(Q.items.alloc(std::max<size_t>(items.size(), 1) * sizeof(PbItem)));
  ZOGCU_TRY(Q.part_order.alloc((size_t)Q.P * 4));
  ZOGCU_TRY(Q.msg.alloc(npad * 4 + 16));
  ZOGCU_TRY(Q.heavy.alloc((size_t)Q.P * 8));
  k_pb_heavy<OffT><<<grid_1d((uint64_t)Q.P * 32), 256, 0, s>>>(off, Q.row_lo.as<uint32_t>(), Q.row_n.as<uint32_t>(),
                                                               Q.P, Q.heavy.as<uint2>());
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_CUDA(cudaMemcpyAsync(Q.items.ptr, items.data(), items.size() * sizeof(PbItem), cudaMemcpyHostToDevice, s));
  ZOGCU_CUDA(cudaMemcpyAsync(Q.part_order.ptr, order.data(), (size_t)Q.P * 4, cudaMemcpyHostToDevice, s));
  ZOGCU_CUDA(cudaMemsetAsync(Q.msg.ptr, 0, npad * 4 + 16, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  Q.state = 1;
  return ZOGCU_OK;
}

// The blocked layout, built on first use; false when the graph cannot use it.
static int ensure_pb_view(Graph* g, cudaStream_t s, bool* usable) {
  std::lock_guard<std::mutex> lk(g->mu);
  if (g->pb.state == 0) {
    if (g->offsets32) {
      const int rc = build_pb_view<uint32_t>(g, s);
      if (rc != ZOGCU_OK) {
        g->pb.reset();
        return rc;
      }
    } else {
      g->pb.state = -1;
    }
  }
  *usable = g->pb.state == 1;
  return ZOGCU_OK;
}

template <typename OffT>
struct PbArgs {
  PrArgs<OffT, float> A;  // state, vectors, options (FP32 contributions)
  const PbItem* items;
  uint32_t nitems, P, B;
  const uint32_t* blk_lo;
  const uint32_t* blk_n;
  const uint16_t* sl;
  const uint16_t* dl;
  float* msg;
  const uint32_t* pstart;
  const uint32_t* pcount;
  const uint32_t* row_lo;
  const uint32_t* row_n;
  const uint32_t* part_order;
  const uint2* heavy;  // per partition: 4 local rows (16 bits each, 0xFFFF = none)
};

template <typename OffT>
__global__ void __launch_bounds__(kPbThreads) pb_emit_kernel(PbArgs<OffT> Q) {
  extern __shared__ __align__(16) unsigned char s_dyn[];
  float* const sc = reinterpret_cast<float*>(s_dyn);
  const PrState* st = Q.A.st;
  const unsigned long long iter = *(volatile const unsigned long long*)&st->iter;
  if (*(volatile const int*)&st->converged || iter >= Q.A.max_iter) return;
  const float* __restrict__ c = (iter & 1ull) ? Q.A.c1 : Q.A.c0;
  for (uint32_t it = blockIdx.x; it < Q.nitems; it += gridDim.x) {
    const PbItem I = Q.items[it];
    const uint32_t lo = Q.blk_lo[I.b], n = Q.blk_n[I.b];
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sc[i] = c[lo + i];
    __syncthreads();
    // four steps per pass, their source loads issued first (more bytes in
    // flight per thread)
    const uint32_t step = 4 * blockDim.x;
    for (uint32_t p0 = I.lo + 4 * threadIdx.x; p0 < I.hi; p0 += 4 * step) {
      uint2 s4[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t p = p0 + u * step;
        s4[u] = p < I.hi ? __ldcs(reinterpret_cast<const uint2*>(Q.sl + p)) : make_uint2(0u, 0u);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t p = p0 + u * step;
        if (p < I.hi) {
          const float4 v = make_float4(sc[s4[u].x & 0xFFFFu], sc[s4[u].x >> 16], sc[s4[u].y & 0xFFFFu],
                                       sc[s4[u].y >> 16]);
          __stcs(reinterpret_cast<float4*>(Q.msg + p), v);
        }
      }
    }
    __syncthreads();
  }
}

// Adds the fixed-point value f to row d's accumulator (low word lo_w[d],
// high word hi_w[d]); exact, whatever the order of the additions.
__device__ __forceinline__ void pb_add_fixed(uint32_t* lo_w, uint32_t* hi_w, uint32_t d, unsigned long long f) {
  const uint32_t lo = (uint32_t)f;
  uint32_t hi = (uint32_t)(f >> 32);
  if (lo) {
    const uint32_t old = atomicAdd(lo_w + d, lo);
    if (old + lo < old) ++hi;
  }
  if (hi) atomicAdd(hi_w + d, hi);
}

// Adds message m (scaled by 2^kPbShift) to row d.  The partition's four
// heaviest rows (h) are summed in the lane's registers (reg), because their
// messages make up much of some pieces, and lanes of one warp adding to one
// shared-memory word serialise.
__device__ __forceinline__ void pb_add(uint32_t* lo_w, uint32_t* hi_w, uint32_t d, float m, const uint32_t (&h)[4],
                                       unsigned long long (&reg)[4]) {
  const unsigned long long f = __float2ull_rn(m * 0x1p56f);
  if (d == h[0]) reg[0] += f;
  else if (d == h[1]) reg[1] += f;
  else if (d == h[2]) reg[2] += f;
  else if (d == h[3]) reg[3] += f;
  else pb_add_fixed(lo_w, hi_w, d, f);
}

template <typename OffT>
__global__ void __launch_bounds__(kPbThreads, 1) pb_accum_kernel(PbArgs<OffT> Q) {
  static_assert(kPbShift == 56, "pb_add scales by 2^56");
  extern __shared__ __align__(16) unsigned char s_dyn[];
  uint32_t* const lo_w = reinterpret_cast<uint32_t*>(s_dyn);  // [kPbRows + 1], row kPbRows takes the padding
  uint32_t* const hi_w = lo_w + (kPbRows + 1);
  __shared__ double s_red[2 * (kPbThreads / 32)];
  __shared__ int s_flag;
  const PrArgs<OffT, float>& A = Q.A;
  PrState* st = A.st;
  const unsigned long long iter = *(volatile const unsigned long long*)&st->iter;
  if (*(volatile const int*)&st->converged || iter >= A.max_iter) {
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(A.cond, 0u);
    return;
  }
  const double sink = *(volatile const double*)&st->sink;
  const int par = (int)(iter & 1ull);
  const double* __restrict__ xcur = par ? A.x1 : A.x0;
  double* __restrict__ xnxt = par ? A.x0 : A.x1;
  float* __restrict__ cnxt = par ? A.c0 : A.c1;
  const double tele_u = (1.0 - A.damping) / A.n_f;
  const bool personalised = A.teleport != nullptr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t p = Q.part_order[blockIdx.x];
  const uint32_t r0 = Q.row_lo[p], nr = Q.row_n[p];
  __shared__ unsigned int s_next;  // next piece to hand out
  if (threadIdx.x == 0) s_next = kPbThreads / 32;
  for (uint32_t i = threadIdx.x; i < 2 * (kPbRows + 1); i += blockDim.x) lo_w[i] = 0u;
  __syncthreads();
  const uint32_t* __restrict__ ps = Q.pstart + (size_t)p * Q.B;
  const uint32_t* __restrict__ pc = Q.pcount + (size_t)p * Q.B;
  // Each warp streams whole pieces, 128 positions per step; the loads of the
  // next step are issued before the current step's additions.  Lanes past a
  // piece's end add 0 to the spare row.
  constexpr uint32_t kPad2 = kPbRows | (kPbRows << 16);
  const uint2 hv = __ldg(Q.heavy + p);
  const uint32_t h[4] = {hv.x & 0xFFFFu, hv.x >> 16, hv.y & 0xFFFFu, hv.y >> 16};
  unsigned long long reg[4] = {0ull, 0ull, 0ull, 0ull};
  // Warp w starts with piece w and then takes the next piece not yet handed
  // out; the heavy blocks' large pieces come first, so the warps reach the
  // barrier below within about one piece of each other.
  for (uint32_t b = warp; b < Q.B;) {
    const uint32_t s0 = __ldg(ps + b), n = __ldg(pc + b);
    uint2 d4 = make_uint2(kPad2, kPad2);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (4 * lane < n) {
      d4 = __ldcs(reinterpret_cast<const uint2*>(Q.dl + s0 + 4 * lane));
      v = __ldcs(reinterpret_cast<const float4*>(Q.msg + s0 + 4 * lane));
    }
    for (uint32_t j0 = 0; j0 < n; j0 += 128) {
      uint2 dn = make_uint2(kPad2, kPad2);
      float4 vn = make_float4(0.f, 0.f, 0.f, 0.f);
      const uint32_t jn = j0 + 128 + 4 * lane;
      if (jn < n) {
        dn = __ldcs(reinterpret_cast<const uint2*>(Q.dl + s0 + jn));
        vn = __ldcs(reinterpret_cast<const float4*>(Q.msg + s0 + jn));
      }
      pb_add(lo_w, hi_w, d4.x & 0xFFFFu, v.x, h, reg);
      pb_add(lo_w, hi_w, d4.x >> 16, v.y, h, reg);
      pb_add(lo_w, hi_w, d4.y & 0xFFFFu, v.z, h, reg);
      pb_add(lo_w, hi_w, d4.y >> 16, v.w, h, reg);
      d4 = dn;
      v = vn;
    }
    unsigned int nb = 0u;
    if (lane == 0) nb = atomicAdd(&s_next, 1u);
    b = __shfl_sync(0xffffffffu, nb, 0);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    unsigned long long t = reg[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0 && h[k] < kPbRows) pb_add_fixed(lo_w, hi_w, h[k], t);
  }
  __syncthreads();
  double l1 = 0.0, dsum = 0.0;
  for (uint32_t r = threadIdx.x; r < nr; r += blockDim.x) {
    const uint32_t v = r0 + r;
    const double sum = (double)(((unsigned long long)hi_w[r] << 32) | lo_w[r]) * 0x1p-56;
    pr_row_epilogue<float>(v, sum, __ldg(A.deg + v), xcur[v], personalised ? __ldg(A.teleport + v) : 0.0,
                           personalised, A.damping, A.n_f, xnxt, cnxt, tele_u, sink, l1, dsum);
  }
  cta_publish(st, A.cta_part, nullptr, nullptr, 0u, l1, dsum, iter + 1, A.tol, A.stall, true, s_red, &s_flag,
              A.max_iter, A.cond, A.use_cond);
}

// Runs the emit / accumulate pair as the body of a CUDA-graph while loop (the
// accumulate's last CTA clears the condition; see pr_launch_loop).
template <typename OffT>
static int pb_launch_loop(PbArgs<OffT> Q, int egrid, int agrid, cudaStream_t s) {
  cudaGraph_t graph = nullptr;
  ZOGCU_CUDA(cudaGraphCreate(&graph, 0));
  struct GraphGuard {
    cudaGraph_t g;
    ~GraphGuard() { cudaGraphDestroy(g); }
  } guard{graph};
  cudaGraphConditionalHandle h;
  ZOGCU_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1u, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  ZOGCU_CUDA(cudaGraphAddNode(&cnode, graph, nullptr, 0, &cp));
  Q.A.cond = h;
  Q.A.use_cond = 1;
  void* args[] = {&Q};
  cudaKernelNodeParams ke = {};
  ke.func = reinterpret_cast<void*>(pb_emit_kernel<OffT>);
  ke.gridDim = dim3((unsigned)egrid);
  ke.blockDim = dim3((unsigned)kPbThreads);
  ke.sharedMemBytes = (unsigned)kPbEmitBytes;
  ke.kernelParams = args;
  cudaKernelNodeParams ka = ke;
  ka.func = reinterpret_cast<void*>(pb_accum_kernel<OffT>);
  ka.gridDim = dim3((unsigned)agrid);
  ka.sharedMemBytes = (unsigned)kPbAccBytes;
  cudaGraphNode_t en, an;
  ZOGCU_CUDA(cudaGraphAddKernelNode(&en, cp.conditional.phGraph_out[0], nullptr, 0, &ke));
  ZOGCU_CUDA(cudaGraphAddKernelNode(&an, cp.conditional.phGraph_out[0], &en, 1, &ka));
  cudaGraphExec_t exec = nullptr;
  ZOGCU_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  const cudaError_t e = cudaGraphLaunch(exec, s);
  cudaGraphExecDestroy(exec);
  ZOGCU_CUDA(e);
  return ZOGCU_OK;
}

// A blocked chain of up to max_iter iterations (start vector as in
// pr_init_kernel).  Adds the launches it enqueued to *launches; the caller
// adds two per iteration the chain ran (*looped = true) once it has read the
// chain's state.
template <typename OffT>
static int pb_run_chain(const PbArgs<OffT>& Q, uint32_t V, int given, uint64_t max_iter, cudaStream_t s,
                        uint64_t* launches, bool* looped) {
  PbArgs<OffT> R = Q;
  R.A.max_iter = max_iter;
  R.A.cond = 0;
  R.A.use_cond = 0;
  ZOGCU_CUDA(cudaFuncSetAttribute(pb_emit_kernel<OffT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPbEmitBytes));
  ZOGCU_CUDA(cudaFuncSetAttribute(pb_accum_kernel<OffT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPbAccBytes));
  int per_sm = 0;
  ZOGCU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pb_emit_kernel<OffT>, kPbThreads, kPbEmitBytes));
  const int egrid = (int)std::min<uint64_t>(std::max<uint64_t>(R.nitems, 1), (uint64_t)std::max(per_sm, 1) * sm_count());
  const int agrid = (int)R.P;
  ZOGCU_CUDA(cudaMemsetAsync(R.A.st, 0, sizeof(PrState), s));
  const unsigned init_grid = std::min(grid_1d(V), 148u * 4);
  pr_init_kernel<OffT, float><<<init_grid, 256, 0, s>>>(R.A, V, given);
  ZOGCU_CUDA(cudaGetLastError());
  ++*launches;
  *looped = false;
  if (max_iter >= kLoopMinIters && graph_loop_allowed()) {
    ZOGCU_TRY(pb_launch_loop<OffT>(R, egrid, agrid, s));
    *looped = true;
    return ZOGCU_OK;
  }
  for (uint64_t k = 0; k < max_iter; ++k) {
    pb_emit_kernel<OffT><<<egrid, kPbThreads, kPbEmitBytes, s>>>(R);
    pb_accum_kernel<OffT><<<agrid, kPbThreads, kPbAccBytes, s>>>(R);
  }
  ZOGCU_CUDA(cudaGetLastError());
  *launches += 2 * max_iter;
  return ZOGCU_OK;
}

// Whether the precision form's FP32 phase runs blocked: ZOGCU_PR_BLOCKED=0
// never, =1 whenever the layout can be built, otherwise on graphs of at least
// 2^23 nodes and 2^24 arcs.  Below that the FP32 contributions (4 bytes per
// node) sit in L2 and the gather kernels win: on Barabasi-Albert n = 2^22
// (33.5M arcs) a blocked iteration took 0.67 ms against 0.23 ms.
static bool pb_wanted(const Graph* g) {
  if (const char* e = std::getenv("ZOGCU_PR_BLOCKED")) {
    if (e[0] == '0') return false;
    if (e[0] == '1') return true;
  }
  return g->V >= (1u << 23) && g->E >= (1ull << 24);
}

// FP32-phase switch: the FP32 contributions carry relative rounding ~6e-8, so
// the L1 step of the FP32 iterates floors near 1e-7; the FP32 phase stops at
// kMixedSwitchTol or when the step stops shrinking (kMixedStall), and the FP64
// polish continues from its vector to the caller's tolerance.
constexpr double kMixedSwitchTol = 1e-6;
constexpr double kMixedStall = 0.97;

// ZOGCU_PR_MIXED_SWITCH=<tol> moves the FP32 -> FP64 switch (for measuring
// where the precision form's time goes); the result's bound is unchanged,
// since the FP64 polish always runs to the caller's tolerance.
static double mixed_switch_tol() {
  if (const char* e = std::getenv("ZOGCU_PR_MIXED_SWITCH")) {
    const double v = std::atof(e);
    if (v > 0.0 && v < 1.0) return v;
  }
  return kMixedSwitchTol;
}

template <typename OffT>
static int run_pagerank(Graph* g, double damping, uint64_t max_iter, double tol, const zogcu_pr_opts* o, double* out,
                        zogcu_stats* stats, cudaStream_t s, PhaseTrace* tr) {
  const PrSchedule& P = g->pr;
  const uint32_t V = g->V;
  const bool dev_ptrs = o && o->device_pointers;
  const bool mixed = o && o->precision == ZOGCU_PREC_MIXED;
  // the work-item list of the graph's configuration, or both lists when the
  // solve will tune; the workspace is sized for the lists built so far
  int cfg = pr_config_of(g);
  if (cfg >= 0) {
    ZOGCU_TRY(ensure_task_list(g, kPrConfigs[cfg].nnz, s));
  } else {
    ZOGCU_TRY(ensure_task_list(g, 128, s));
    ZOGCU_TRY(ensure_task_list(g, 256, s));
  }
  tr->mark("work-item lists");
  const uint32_t max_tasks = cfg >= 0 ? P.lists[list_index(kPrConfigs[cfg].nnz)].num_tasks
                                      : std::max(P.lists[0].num_tasks, P.lists[1].num_tasks);
  // the graph's cached scratch when no other call holds it (declared before
  // the buffers, so it outlives them)
  WorkLease lease(&g->pr_ws, s);
  PrWork W;
  DevBuf cf0, cf1, pbpart;
  bool blocked32 = false;
  ZOGCU_TRY(lease.get(W.x0, 0, (size_t)V * 8));
  ZOGCU_TRY(lease.get(W.x1, 1, (size_t)V * 8));
  ZOGCU_TRY(lease.get(W.c0, 2, (size_t)V * 8 + 16));
  ZOGCU_TRY(lease.get(W.c1, 3, (size_t)V * 8 + 16));
  ZOGCU_TRY(lease.get(W.part, 4, (size_t)std::max<int>(sm_count() * 8, 148 * 4) * 16));
  ZOGCU_TRY(lease.get(W.chunk, 5, (size_t)std::max<uint32_t>(max_tasks, 1) * 8));
  ZOGCU_TRY(lease.get(W.lcnt, 6, (size_t)std::max<uint32_t>(max_tasks, 1) * 4));
  ZOGCU_TRY(lease.get(W.lpart, 7, (size_t)std::max<uint32_t>(max_tasks, 1) * 16));
  ZOGCU_TRY(lease.get(W.stb, 8, sizeof(PrState)));
  ZOGCU_CUDA(cudaMemsetAsync(W.lcnt.ptr, 0, W.lcnt.bytes, s));
  ZOGCU_CUDA(cudaMemsetAsync(W.c0.ptr, 0, W.c0.bytes, s));
  ZOGCU_CUDA(cudaMemsetAsync(W.c1.ptr, 0, W.c1.bytes, s));
  if (mixed) {
    ZOGCU_TRY(lease.get(cf0, 9, (size_t)V * 4 + 16));
    ZOGCU_TRY(lease.get(cf1, 10, (size_t)V * 4 + 16));
    ZOGCU_CUDA(cudaMemsetAsync(cf0.ptr, 0, cf0.bytes, s));
    ZOGCU_CUDA(cudaMemsetAsync(cf1.ptr, 0, cf1.bytes, s));
  }

  PrArgs<OffT, double> A{};
  A.off = P.off.as<OffT>();
  A.col = P.col.as<uint32_t>();
  A.deg = P.deg.as<uint32_t>();
  A.x0 = W.x0.as<double>();
  A.x1 = W.x1.as<double>();
  A.c0 = W.c0.as<double>();
  A.c1 = W.c1.as<double>();
  A.cta_part = W.part.as<double>();
  A.chunk_part = W.chunk.as<double>();
  A.long_cnt = W.lcnt.as<unsigned int>();
  A.long_part = W.lpart.as<double>();
  A.st = W.stb.as<PrState>();
  A.teleport = nullptr;
  A.damping = damping;
  A.n_f = (double)g->n_live;
  A.tol = tol;
  A.stall = 0.0;
  A.nv = V;

  tr->mark("workspace");

  int given = 0;
  if (o && o->x0) {  // caller order -> ranked order
    ZOGCU_TRY(lease.get(W.tmp, 11, (size_t)V * 8));
    ZOGCU_CUDA(cudaMemcpyAsync(W.tmp.ptr, o->x0, (size_t)V * 8, dev_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    k_permute_in<<<grid_1d(V), 256, 0, s>>>(W.tmp.as<double>(), P.perm.as<uint32_t>(), V, W.x0.as<double>());
    ZOGCU_CUDA(cudaGetLastError());
    given = 1;
  }
  if (o && o->teleport) {
    ZOGCU_TRY(lease.get(W.tele, 12, (size_t)V * 8));
    if (!W.tmp.ptr) ZOGCU_TRY(lease.get(W.tmp, 11, (size_t)V * 8));
    ZOGCU_CUDA(cudaMemcpyAsync(W.tmp.ptr, o->teleport, (size_t)V * 8, dev_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    k_permute_in<<<grid_1d(V), 256, 0, s>>>(W.tmp.as<double>(), P.perm.as<uint32_t>(), V, W.tele.as<double>());
    ZOGCU_CUDA(cudaGetLastError());
    A.teleport = W.tele.as<double>();
  }

  EventTimer tm;
  uint64_t launches = 0, it32 = 0;
  PrState hs;
  ZOGCU_TRY(tm.start(s));
  if (mixed && max_iter > 0) {
    // ---- FP32 phase: x in FP64, contributions in FP32 -----------------------
    PrArgs<OffT, float> Af{};
    std::memcpy(&Af, &A, sizeof(Af));  // same layout; only the contribution pointers differ in type
    Af.c0 = cf0.as<float>();
    Af.c1 = cf1.as<float>();
    Af.tol = std::max(tol, mixed_switch_tol());
    Af.stall = kMixedStall;
    int64_t from32 = -1;
    bool blocked = false, looped = false;
    if (pb_wanted(g)) ZOGCU_TRY(ensure_pb_view(g, s, &blocked));
    if (blocked) {
      // the propagation-blocked iteration (same update, streamed messages)
      const PbView& B = g->pb;
      PbArgs<OffT> Q{};
      Q.A = Af;
      ZOGCU_TRY(lease.get(pbpart, 13, (size_t)std::max<uint32_t>(B.P, 148u * 4u) * 16));
      Q.A.cta_part = pbpart.as<double>();
      Q.items = B.items.as<PbItem>();
      Q.nitems = B.nitems;
      Q.P = B.P;
      Q.B = B.B;
      Q.blk_lo = B.blk_lo.as<uint32_t>();
      Q.blk_n = B.blk_n.as<uint32_t>();
      Q.sl = B.sl.as<uint16_t>();
      Q.dl = B.dl.as<uint16_t>();
      Q.msg = B.msg.as<float>();
      Q.pstart = B.pstart.as<uint32_t>();
      Q.pcount = B.pcount.as<uint32_t>();
      Q.row_lo = B.row_lo.as<uint32_t>();
      Q.row_n = B.row_n.as<uint32_t>();
      Q.part_order = B.part_order.as<uint32_t>();
      Q.heavy = B.heavy.as<uint2>();
      ZOGCU_TRY(pb_run_chain<OffT>(Q, V, given, max_iter, s, &launches, &looped));
    } else {
      ZOGCU_TRY((pr_run_chain<OffT, float>(g, cfg, Af, V, given, max_iter, s, &launches, &cfg, &from32)));
    }
    ZOGCU_CUDA(cudaMemcpyAsync(&hs, W.stb.ptr, sizeof(PrState), cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    if (hs.pad[0]) return fail(ZOGCU_ERR_INTERNAL, "PageRank work item failed a bound check");
    if (from32 >= 0) launches += hs.iter - (uint64_t)from32 + (hs.iter == (uint64_t)from32 ? 1 : 0);
    if (looped) launches += 2 * hs.iter;
    blocked32 = blocked;
    it32 = hs.iter;
    // ---- FP64 polish from the FP32 phase's last vector ----------------------
    if (it32 & 1ull) std::swap(A.x0, A.x1);
    given = 1;
  }
  int64_t from64 = -1;
  ZOGCU_TRY((pr_run_chain<OffT, double>(g, cfg, A, V, given, max_iter - it32, s, &launches, &cfg, &from64)));
  ZOGCU_TRY(tm.stop(s));
  ZOGCU_CUDA(cudaMemcpyAsync(&hs, W.stb.ptr, sizeof(PrState), cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  if (hs.pad[0]) return fail(ZOGCU_ERR_INTERNAL, "PageRank work item failed a bound check");
  // kernel launches of a graph loop: one per iteration it ran (a loop that
  // found the chain already over ran one launch that only ended the loop)
  if (from64 >= 0) launches += hs.iter - (uint64_t)from64 + (hs.iter == (uint64_t)from64 ? 1 : 0);
  tr->mark("solve");
  const double* result = (hs.iter & 1ull) ? A.x1 : A.x0;
  double* unperm = (hs.iter & 1ull) ? A.x0 : A.x1;  // the other buffer is free now
  k_permute_out<<<grid_1d(V), 256, 0, s>>>(result, P.rank.as<uint32_t>(), V, unperm);
  ZOGCU_CUDA(cudaGetLastError());
  ++launches;
  if (dev_ptrs) ZOGCU_CUDA(cudaMemcpyAsync(out, unperm, (size_t)V * 8, cudaMemcpyDeviceToDevice, s));
  else ZOGCU_TRY(copy_host(unperm, out, (size_t)V * 8, false, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  tr->mark("scores to the caller");
  if (stats) {
    stats->iterations = it32 + hs.iter;
    stats->residual = hs.l1;
    stats->elapsed_ms = tm.ms();
    const double per_iter64 = 4.0 * (double)g->E + (double)sizeof(OffT) * ((double)V + 1) + 36.0 * (double)V;
    const double per_iter32 = per_iter64 - 8.0 * (double)V;  // c read and written as 4 bytes
    stats->bytes_moved = per_iter64 * (double)hs.iter + per_iter32 * (double)it32;
    stats->launches = launches;
    stats->polish_iterations = mixed ? hs.iter : 0;
    stats->kernel_config = (uint32_t)cfg;
    stats->reserved = blocked32 ? 1u : 0u;
  }
  return ZOGCU_OK;
}

// ---------------------------------------------------------------------------
// Katz, alpha and eigenvector centrality (centrality.zig:1050-1321): the same
// schedule and gather path as PageRank, gathering x itself.
// ---------------------------------------------------------------------------
__global__ void k_fill_start(const uint32_t* __restrict__ deg, const uint32_t* __restrict__ perm, uint32_t V,
                             int eigen, double start, double* __restrict__ x) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < V; p += (uint64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (deg[p] != kDeletedDegree) v = eigen ? 1.0 + (double)perm[p] / 1000.0 : start;  // :1076-1078
    x[p] = v;
  }
}

// Eigenvector step 2: normalise the raw sums by their L2 norm, measure the
// L2 step against the current vector and the one two steps back, and decide
// (converged = 1 step < tol, 2 zero vector, 3 oscillation) on the device.
__global__ void __launch_bounds__(256) k_eigen_normalise(PrArgs<uint32_t, double> A, const uint32_t* __restrict__ deg,
                                                         uint32_t V) {
  __shared__ double s_red[16];
  __shared__ int s_flag;
  PrState* st = A.st;
  const unsigned long long iter = *(volatile unsigned long long*)&st->iter;
  if (*(volatile int*)&st->converged || iter >= A.max_iter) return;
  const double norm2 = *(volatile double*)&st->sink;
  if (norm2 == 0.0) {  // degenerate: every CTA returns, block 0 records it
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->converged = 2;
      st->iter = iter + 1;
    }
    return;
  }
  const int k3 = (int)(iter % 3ull);
  const double* cur = k3 == 0 ? A.x0 : (k3 == 1 ? A.x1 : A.x2);
  double* nw = k3 == 0 ? A.x1 : (k3 == 1 ? A.x2 : A.x0);
  const double* pp = k3 == 0 ? A.x2 : (k3 == 1 ? A.x0 : A.x1);
  const double norm = sqrt(norm2);
  double d1 = 0.0, d2 = 0.0;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < V; p += (uint64_t)gridDim.x * blockDim.x) {
    if (deg[p] == kDeletedDegree) continue;
    const double xn = nw[p] / norm;
    nw[p] = xn;
    const double a = xn - cur[p];
    d1 += a * a;
    if (iter >= 1) {
      const double b = xn - pp[p];
      d2 += b * b;
    }
  }
  cta_sum2(d1, d2, s_red);
  if (threadIdx.x == 0) {
    A.cta_part[2 * blockIdx.x] = d1;
    A.cta_part[2 * blockIdx.x + 1] = d2;
    __threadfence();
    s_flag = (atomicAdd(&st->done_ctas, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_flag) return;
  __threadfence();
  double D1 = 0.0, D2 = 0.0;
  for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
    D1 += __ldcg(A.cta_part + 2 * i);
    D2 += __ldcg(A.cta_part + 2 * i + 1);
  }
  cta_sum2(D1, D2, s_red);
  if (threadIdx.x == 0) {
    const double step = D1 > 0.0 ? sqrt(D1) : 0.0;
    const double step2 = D2 > 0.0 ? sqrt(D2) : 0.0;
    const bool osc = iter >= 1 && step2 < A.tol;  // :1136-1150
    st->l1 = step;
    st->converged = osc ? 3 : (step < A.tol ? 1 : 0);
    st->iter = iter + 1;
    __threadfence();
    st->done_ctas = 0;
  }
}

// Normalised average of two vectors (the oscillation exit, :1152-1172), in
// two passes: squares into CTA partials, then one CTA folds them and scales.
__global__ void __launch_bounds__(256) k_avg_squares(const double* __restrict__ a, const double* __restrict__ b,
                                                     const uint32_t* __restrict__ deg, uint32_t V,
                                                     double* __restrict__ avg, double* __restrict__ part) {
  __shared__ double s_red[16];
  double s = 0.0, unused = 0.0;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < V; p += (uint64_t)gridDim.x * blockDim.x) {
    const double v = deg[p] == kDeletedDegree ? 0.0 : (a[p] + b[p]) / 2.0;
    avg[p] = v;
    s += v * v;
  }
  cta_sum2(s, unused, s_red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}
__global__ void __launch_bounds__(256) k_avg_scale(double* __restrict__ avg, uint32_t V, const double* __restrict__ part,
                                                   uint32_t nparts) {
  __shared__ double s_red[16];
  __shared__ double s_norm;
  double s = 0.0, unused = 0.0;
  for (uint32_t i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
  cta_sum2(s, unused, s_red);
  if (threadIdx.x == 0) s_norm = s > 0.0 ? sqrt(s) : 1.0;
  __syncthreads();
  const double n = s_norm;
  for (uint64_t p = threadIdx.x; p < V; p += blockDim.x) avg[p] /= n;
}

template <typename OffT, int MODE>
static int run_linear(Graph* g, double ka, double kb, double start, uint64_t max_iter, double tol, double* out,
                      bool dev_out, zogcu_stats* stats, cudaStream_t s) {
  const uint32_t V = g->V;
  ZOGCU_TRY(ensure_pr_schedule(g, s));
  ZOGCU_TRY(ensure_task_list(g, 256, s));
  const PrSchedule& P = g->pr;
  const PrTaskList& L = P.lists[list_index(256)];
  PrWork W;
  DevBuf x2;
  ZOGCU_TRY(W.x0.alloc((size_t)V * 8 + 16, s));
  ZOGCU_TRY(W.x1.alloc((size_t)V * 8 + 16, s));
  ZOGCU_TRY(x2.alloc((size_t)V * 8 + 16, s));
  ZOGCU_TRY(W.part.alloc((size_t)std::max<int>(sm_count() * 8, 148 * 4) * 16, s));
  ZOGCU_TRY(W.chunk.alloc((size_t)std::max<uint32_t>(L.num_tasks, 1) * 8, s));
  ZOGCU_TRY(W.lcnt.alloc((size_t)std::max<uint32_t>(L.num_tasks, 1) * 4, s));
  ZOGCU_TRY(W.lpart.alloc((size_t)std::max<uint32_t>(L.num_tasks, 1) * 16, s));
  ZOGCU_TRY(W.stb.alloc(sizeof(PrState), s));
  ZOGCU_CUDA(cudaMemsetAsync(W.lcnt.ptr, 0, W.lcnt.bytes, s));
  ZOGCU_CUDA(cudaMemsetAsync(W.stb.ptr, 0, sizeof(PrState), s));
  ZOGCU_CUDA(cudaMemsetAsync(W.x1.ptr, 0, W.x1.bytes, s));
  ZOGCU_CUDA(cudaMemsetAsync(x2.ptr, 0, x2.bytes, s));
  k_fill_start<<<grid_1d(V), 256, 0, s>>>(P.deg.as<uint32_t>(), P.perm.as<uint32_t>(), V, MODE == kModeEigen ? 1 : 0,
                                          start, W.x0.as<double>());
  ZOGCU_CUDA(cudaGetLastError());
  PrArgs<OffT, double> A{};
  A.off = P.off.as<OffT>();
  A.col = P.col.as<uint32_t>();
  A.deg = P.deg.as<uint32_t>();
  A.tasks = L.tasks.as<PrTask>();
  A.long_first = L.long_first.as<uint32_t>();
  A.ntasks = L.num_tasks;
  A.nlong = L.num_long;
  A.hub = 0;
  A.x0 = W.x0.as<double>();
  A.x1 = W.x1.as<double>();
  A.x2 = x2.as<double>();
  A.c0 = A.x0;
  A.c1 = A.x1;
  A.cta_part = W.part.as<double>();
  A.chunk_part = W.chunk.as<double>();
  A.long_cnt = W.lcnt.as<unsigned int>();
  A.long_part = W.lpart.as<double>();
  A.st = W.stb.as<PrState>();
  A.n_f = (double)g->n_live;
  A.tol = tol;
  A.max_iter = max_iter;
  A.ka = ka;
  A.kb = kb;
  auto fn = pr_iter_kernel<OffT, double, 256, 256, MODE>;
  constexpr int cfg = 3;
  const size_t dyn = PrLauncher<OffT, double>::staging_bytes(cfg);
  static std::atomic<int> grid{0};  // same value for every B200 device
  if (!grid.load(std::memory_order_acquire)) {
    int per_sm = 0;
    ZOGCU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, dyn));
    grid.store(std::max(per_sm, 1) * sm_count(), std::memory_order_release);
  }
  int gr = grid.load(std::memory_order_acquire);
  const uint32_t need = (A.ntasks + 7) / 8;
  if (need > 0 && (uint32_t)gr > need) gr = (int)need;
  const unsigned gn = std::min(grid_1d(V), 148u * 4);
  EventTimer tm;
  ZOGCU_TRY(tm.start(s));
  uint64_t launches = 1;
  for (uint64_t k = 0; k < max_iter; ++k) {
    fn<<<gr, 256, dyn, s>>>(A);
    ++launches;
    if constexpr (MODE == kModeEigen) {
      if constexpr (sizeof(OffT) == 4) {
        k_eigen_normalise<<<gn, 256, 0, s>>>(A, A.deg, V);
        ++launches;
      }
    }
  }
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_TRY(tm.stop(s));
  PrState hs;
  ZOGCU_CUDA(cudaMemcpyAsync(&hs, W.stb.ptr, sizeof(PrState), cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  double* X[3] = {A.x0, A.x1, A.x2};
  double* result;
  double* spare;
  if (MODE == kModeEigen) {
    result = X[hs.iter % 3];
    spare = X[(hs.iter + 1) % 3];
    if (hs.converged == 2) {  // zero vector: uniform 1/sqrt(n) (:1101-1112)
      k_fill_start<<<grid_1d(V), 256, 0, s>>>(P.deg.as<uint32_t>(), P.perm.as<uint32_t>(), V, 0,
                                              1.0 / std::sqrt((double)g->n_live), spare);
      result = spare;
      spare = X[(hs.iter + 2) % 3];
    } else if (hs.converged == 3) {  // oscillation: normalised average of the last two
      const double* prev = X[(hs.iter + 2) % 3];
      k_avg_squares<<<gn, 256, 0, s>>>(result, prev, P.deg.as<uint32_t>(), V, spare, A.cta_part);
      k_avg_scale<<<1, 256, 0, s>>>(spare, V, A.cta_part, gn);
      launches += 2;
      result = spare;
      spare = const_cast<double*>(prev);
    }
  } else {
    result = (hs.iter & 1ull) ? A.x1 : A.x0;
    spare = x2.as<double>();
  }
  k_permute_out<<<grid_1d(V), 256, 0, s>>>(result, P.rank.as<uint32_t>(), V, spare);
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_CUDA(cudaMemcpyAsync(out, spare, (size_t)V * 8, dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  if (stats) {
    stats->iterations = hs.iter;
    stats->residual = hs.l1;
    stats->elapsed_ms = tm.ms();
    stats->launches = launches + 1;
    stats->kernel_config = cfg;
    stats->reserved = (uint32_t)hs.converged;
  }
  return ZOGCU_OK;
}

// Common entry: argument checks, n <= 1 shortcuts, offset-width dispatch.
template <int MODE>
static int linear_entry(zogcu_graph* G, double ka, double kb, double start, uint64_t max_iter, double tol, double* out,
                        zogcu_stats* stats) {
  if (!G) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graph is null");
  Graph* g = &G->g;
  if (!out && g->V) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out_scores is null");
  ZOGCU_CUDA(cudaSetDevice(g->device));
  if (stats) std::memset(stats, 0, sizeof(*stats));
  const uint32_t V = g->V;
  if (g->n_live == 0 || (MODE == kModeEigen && g->n_live == 1)) {
    // empty graph: every slot 0.0; eigenvector with one node: 1.0 (:1069-1072)
    std::vector<double> h(V, 0.0);
    if (g->n_live == 1) {
      std::vector<uint32_t> deg(V);
      ZOGCU_CUDA(cudaMemcpy(deg.data(), g->out_deg.ptr, (size_t)V * 4, cudaMemcpyDeviceToHost));
      for (uint32_t v = 0; v < V; ++v)
        if (deg[v] != kDeletedDegree) h[v] = 1.0;
    }
    if (V) std::memcpy(out, h.data(), (size_t)V * 8);
    return ZOGCU_OK;
  }
  if (MODE == kModeEigen && g->has_deleted)
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "eigenvector on graphs with deleted nodes is not supported");
  if (MODE == kModeEigen && !g->offsets32)
    return fail(ZOGCU_ERR_TOO_LARGE, "eigenvector needs fewer than 2^32 arcs");
  StreamGuard sg;
  ZOGCU_TRY(sg.init(nullptr));
  if (g->offsets32) return run_linear<uint32_t, MODE>(g, ka, kb, start, max_iter, tol, out, false, stats, sg.s);
  return run_linear<uint64_t, MODE>(g, ka, kb, start, max_iter, tol, out, false, stats, sg.s);
}

}  // namespace zogcu



using namespace zogcu;

extern "C" {

int zogcu_pagerank_ex(zogcu_graph* G, double damping, uint64_t max_iterations, double tolerance,
                      const zogcu_pr_opts* opts, double* out_scores, zogcu_stats* stats) {
  if (!G) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graph is null");
  if (!out_scores && G->g.V) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out_scores is null");
  if (opts && opts->struct_size != sizeof(zogcu_pr_opts))
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "zogcu_pr_opts.struct_size mismatch");
  if (opts && opts->precision != ZOGCU_PREC_FP64 && opts->precision != ZOGCU_PREC_MIXED)
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "unknown precision");
  Graph* g = &G->g;
  ZOGCU_CUDA(cudaSetDevice(g->device));
  if (stats) std::memset(stats, 0, sizeof(*stats));
  const uint32_t V = g->V;
  const bool dev_ptrs = opts && opts->device_pointers;
  // n == 0 / n == 1 short cuts (centrality.zig:875-879); extractScores gives
  // 0.0 for every slot without a score (.Elixir.Zog.ResourceGraph.zig:72-80).
  if (g->n_live <= 1) {
    std::vector<double> h(V, 0.0);
    if (g->n_live == 1) {
      std::vector<uint32_t> deg(V);
      if (V) ZOGCU_CUDA(cudaMemcpy(deg.data(), g->out_deg.ptr, (size_t)V * 4, cudaMemcpyDeviceToHost));
      for (uint32_t v = 0; v < V; ++v)
        if (deg[v] != kDeletedDegree) h[v] = 1.0;
    }
    if (V) ZOGCU_CUDA(cudaMemcpy(out_scores, h.data(), (size_t)V * 8, dev_ptrs ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost));
    return ZOGCU_OK;
  }
  StreamGuard sg;
  ZOGCU_TRY(sg.init(opts ? opts->stream : nullptr));
  PhaseTrace tr("pagerank", sg.s);
  ZOGCU_TRY(ensure_pr_schedule(g, sg.s));
  tr.mark("degree-ranked view");
  if (g->offsets32)
    return run_pagerank<uint32_t>(g, damping, max_iterations, tolerance, opts, out_scores, stats, sg.s, &tr);
  return run_pagerank<uint64_t>(g, damping, max_iterations, tolerance, opts, out_scores, stats, sg.s, &tr);
}

int zogcu_pagerank(zogcu_graph* G, double damping, uint64_t max_iterations, double tolerance, double* out_scores,
                   zogcu_stats* stats) {
  return zogcu_pagerank_ex(G, damping, max_iterations, tolerance, nullptr, out_scores, stats);
}

int zogcu_katz(zogcu_graph* G, double alpha, double beta, uint64_t max_iterations, double tolerance,
               double* out_scores, zogcu_stats* stats) {
  return linear_entry<kModeKatz>(G, alpha, beta, beta, max_iterations, tolerance, out_scores, stats);
}

int zogcu_alpha_centrality(zogcu_graph* G, double alpha, double initial, uint64_t max_iterations, double tolerance,
                           double* out_scores, zogcu_stats* stats) {
  return linear_entry<kModeAlpha>(G, alpha, 0.0, initial, max_iterations, tolerance, out_scores, stats);
}

int zogcu_eigenvector(zogcu_graph* G, uint64_t max_iterations, double tolerance, double* out_scores,
                      zogcu_stats* stats) {
  return linear_entry<kModeEigen>(G, 0.0, 0.0, 0.0, max_iterations, tolerance, out_scores, stats);
}

}  // extern "C"
