// ppr.cu -- personalised PageRank for many seeds at once, as a CSR SpMM.
//
// Per seed s the iteration is the reference's (priv/zog/src/centrality.zig:
// 924-958) with its uniform teleport (1-d)/n replaced by (1-d) e_s (a one-hot
// personalisation vector) while the dangling mass stays uniform:
//     sink_s   = sum_{deg(u)=0} x_s[u] / n
//     x'_s[v]  = (1-d) [v == s] + d (sink_s + sum_{u in in(v)} x_s[u]/deg(u))
//     l1_s     = sum |x'_s - x_s|,  stop seed s once l1_s < tol (after the swap)
// from the uniform start 1/n -- the generalised form the CPU oracle's
// og_pagerank_ext computes for one seed.
//
// B200 design: S seeds (64 per pass; the kernel also builds for 128 and 256) are the columns of node-major matrices
// X, C = X/deg (V x S, FP64), so every arc of the in-CSR gathers one
// contiguous row of S values (2 KB at S = 256: whole lines, streamed) instead
// of S scattered scalars.  The degree-ranked view and warp work items of the
// single-vector kernel are reused (row blocks, single rows, and 4096-arc
// chunks of hub rows; chunk partials are added into a side matrix and the
// last chunk to arrive runs the row's epilogue).  Each lane owns S/32
// consecutive columns, reads them with 32-byte loads that skip L1 allocation,
// and sums a row's arcs in the reference's order.  A
// seed that has converged is frozen (its column is carried over unchanged),
// so every seed returns exactly the vector of its own stopping iteration.
// Per-column L1 steps and dangling masses go lane -> warp -> CTA partials ->
// a last-CTA reduction in a fixed order, which also updates the per-seed
// state.  A whole call is one CUDA graph: per pass, the start-vector kernel,
// a conditional while node whose body is the iteration kernel (the kernel
// clears the loop's condition once every seed of the pass has stopped or
// max_iterations is reached), and the kernel that writes the pass's columns
// out; the passes follow one another and share the matrices.  The host
// launches the graph once and no iteration launch is spent after convergence.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace zogcu {
namespace {

constexpr int kPprThreads = 256;
constexpr uint32_t kNoSeed = 0xFFFFFFFFu;

struct PprState {
  unsigned long long iter;  // iterations launched so far
  int done;                 // every seed has stopped (or max_iter reached)
  int pad;
};

template <int S>
struct PprArgs {
  static_assert(S % 32 == 0 && S <= 256, "columns per pass: 32, 64, 128 or 256");
  const uint32_t* off;     // ranked in-CSR offsets
  const uint32_t* col;     // ranked source ids, ascending original id per row
  const uint32_t* deg;     // out-degree by rank
  const PrTask* tasks;
  uint32_t num_tasks;
  double* X[2];            // V x S, node-major
  double* C[2];
  double* Y;               // chunk partials of hub rows (zero between uses)
  uint32_t* arrive;        // chunk arrivals per row (zero between uses)
  const uint32_t* seed_rank;  // rank of the seed of column s, kNoSeed = unused column
  int* active;             // per column
  unsigned long long* iters;  // per column
  double* l1;              // per column, last step
  double* sink;            // per column, sink of the current iterate
  double* part;            // [grid][S][2] CTA partials
  PprState* st;
  uint32_t* task_next;
  uint32_t* cta_arrive;
  uint32_t V;
  double n_f;
  double damping;
  double tol;
  unsigned long long max_iter;
  unsigned long long cond;  // conditional handle of the pass's while loop
  int use_cond;             // 1: clear the condition when the pass is over
};

// PL consecutive doubles of one contribution row, read with 32-byte loads
// that skip L1 allocation (16-byte loads when PL is 2): the row is streamed,
// never re-read by this warp.
template <int PL>
__device__ __forceinline__ void ld_row(const double* p, double (&v)[PL]) {
  if constexpr (PL == 1) {
    asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v[0]) : "l"(p));
  } else if constexpr (PL % 4 == 0) {
#pragma unroll
    for (int q = 0; q < PL / 4; ++q)
      asm volatile("ld.global.nc.L1::no_allocate.v4.f64 {%0,%1,%2,%3}, [%4];"
                   : "=d"(v[4 * q]), "=d"(v[4 * q + 1]), "=d"(v[4 * q + 2]), "=d"(v[4 * q + 3])
                   : "l"(p + 4 * q));
  } else {
#pragma unroll
    for (int q = 0; q < PL / 2; ++q) {
      const double2 x = __ldg(reinterpret_cast<const double2*>(p) + q);
      v[2 * q] = x.x;
      v[2 * q + 1] = x.y;
    }
  }
}

template <int S>
__device__ __forceinline__ void ppr_row_sum(const PprArgs<S>& A, const double* __restrict__ Cc, uint32_t b, uint32_t e,
                                            int c0, double (&acc)[S / 32]) {
  constexpr int PL = S / 32;
#pragma unroll
  for (int i = 0; i < PL; ++i) acc[i] = 0.0;
  uint32_t j = b;
  for (; j + 2 <= e; j += 2) {
    const uint32_t u0 = __ldg(A.col + j), u1 = __ldg(A.col + j + 1);
    double v0[PL], v1[PL];
    ld_row<PL>(Cc + (size_t)u0 * S + c0, v0);
    ld_row<PL>(Cc + (size_t)u1 * S + c0, v1);
#pragma unroll
    for (int i = 0; i < PL; ++i) {  // arc j, then arc j+1: the reference's order per column
      acc[i] = __dadd_rn(acc[i], v0[i]);
      acc[i] = __dadd_rn(acc[i], v1[i]);
    }
  }
  if (j < e) {
    const uint32_t u = __ldg(A.col + j);
    double v[PL];
    ld_row<PL>(Cc + (size_t)u * S + c0, v);
#pragma unroll
    for (int i = 0; i < PL; ++i) acc[i] = __dadd_rn(acc[i], v[i]);
  }
}

template <int S>
__device__ __forceinline__ void ppr_epilogue(const PprArgs<S>& A, uint32_t r, int c0, const double (&acc)[S / 32],
                                             const double (&sink)[S / 32], uint32_t act_bits,
                                             const uint32_t (&seed)[S / 32], const double* __restrict__ X,
                                             const double* __restrict__ Cc, double* __restrict__ Xn,
                                             double* __restrict__ Cn, double (&l1p)[S / 32],
                                             double (&dgp)[S / 32]) {
  constexpr int PL = S / 32;
  const uint32_t d = __ldg(A.deg + r);
  const size_t base = (size_t)r * S + c0;
  if constexpr (PL == 1) {  // one column per lane
    const double xold = X[base];
    double xn = xold, cn;
    if (act_bits & 1u) {
      const double tele = seed[0] == r ? 1.0 - A.damping : 0.0;
      const double v = __dadd_rn(tele, __dmul_rn(A.damping, __dadd_rn(sink[0], acc[0])));
      l1p[0] += fabs(v - xold);
      xn = v;
      if (d == 0) {
        cn = 0.0;
        dgp[0] += __ddiv_rn(v, A.n_f);
      } else {
        cn = __ddiv_rn(v, (double)d);
      }
    } else {  // a stopped seed: carry its vector over unchanged
      cn = Cc[base];
    }
    Xn[base] = xn;
    Cn[base] = cn;
    return;
  }
#pragma unroll
  for (int q = 0; q < PL / 2; ++q) {
    const double2 xo = *reinterpret_cast<const double2*>(X + base + 2 * q);
    double xn[2], cn[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = 2 * q + h;
      const double xold = h ? xo.y : xo.x;
      if (act_bits >> i & 1u) {
        const double tele = seed[i] == r ? 1.0 - A.damping : 0.0;
        const double v = __dadd_rn(tele, __dmul_rn(A.damping, __dadd_rn(sink[i], acc[i])));
        l1p[i] += fabs(v - xold);
        xn[h] = v;
        if (d == 0) {
          cn[h] = 0.0;
          dgp[i] += __ddiv_rn(v, A.n_f);
        } else {
          cn[h] = __ddiv_rn(v, (double)d);
        }
      } else {  // a stopped seed: carry its vector over unchanged
        xn[h] = xold;
        cn[h] = Cc[base + i];
      }
    }
    *reinterpret_cast<double2*>(Xn + base + 2 * q) = make_double2(xn[0], xn[1]);
    *reinterpret_cast<double2*>(Cn + base + 2 * q) = make_double2(cn[0], cn[1]);
  }
}

template <int S>
__global__ void __launch_bounds__(kPprThreads) k_ppr_iter(PprArgs<S> A) {
  constexpr int PL = S / 32;
  constexpr int NW = kPprThreads / 32;
  __shared__ double s_part[NW][S][2];
  __shared__ int s_last;
  const unsigned long long it = *(volatile unsigned long long*)&A.st->iter;
  if (*(volatile int*)&A.st->done || it >= A.max_iter) {
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(A.cond, 0u);
    return;
  }
  const int par = (int)(it & 1ull);
  const double* __restrict__ X = A.X[par];
  const double* __restrict__ Cc = A.C[par];
  double* __restrict__ Xn = A.X[par ^ 1];
  double* __restrict__ Cn = A.C[par ^ 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c0 = lane * PL;
  double sink[PL], l1p[PL], dgp[PL];
  uint32_t seed[PL];
  uint32_t act_bits = 0;
#pragma unroll
  for (int i = 0; i < PL; ++i) {
    sink[i] = A.sink[c0 + i];
    seed[i] = A.seed_rank[c0 + i];
    act_bits |= (A.active[c0 + i] ? 1u : 0u) << i;
    l1p[i] = 0.0;
    dgp[i] = 0.0;
  }
  // work items from a shared counter, one per atomic: items differ in cost,
  // and both a fixed split (478 ms for 256 seeds at scale 22) and four items
  // per atomic (481 ms) left warps idle at the end of the iteration (429 ms)
  for (;;) {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(A.task_next, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= A.num_tasks) break;
    const PrTask T = A.tasks[t];
    const uint32_t kind = T.b >> 30;
    double acc[PL];
    if (kind == kTaskChunk) {
      const uint32_t r = T.a, ch = T.b & 0xFFFFu;
      const uint32_t rb = __ldg(A.off + r), re = __ldg(A.off + r + 1);
      const uint32_t b = rb + ch * (uint32_t)kLongChunk, e = min(re, b + (uint32_t)kLongChunk);
      ppr_row_sum<S>(A, Cc, b, e, c0, acc);
      double* y = A.Y + (size_t)r * S + c0;
#pragma unroll
      for (int i = 0; i < PL; ++i) atomicAdd(y + i, acc[i]);
      __threadfence();
      __syncwarp();
      uint32_t last = 0;
      const uint32_t nch = (re - rb + kLongChunk - 1) / kLongChunk;
      if (lane == 0) last = atomicAdd(A.arrive + r, 1u) == nch - 1 ? 1u : 0u;
      last = __shfl_sync(0xffffffffu, last, 0);
      if (!last) continue;
      __threadfence();
#pragma unroll
      for (int i = 0; i < PL; ++i) {
        acc[i] = __ldcg(y + i);
        y[i] = 0.0;
      }
      if (lane == 0) A.arrive[r] = 0;
      ppr_epilogue<S>(A, r, c0, acc, sink, act_bits, seed, X, Cc, Xn, Cn, l1p, dgp);
    } else {
      const uint32_t r0 = T.a, r1 = kind == kTaskRow ? T.a + 1 : (T.b & 0x3FFFFFFFu);
      for (uint32_t r = r0; r < r1; ++r) {
        ppr_row_sum<S>(A, Cc, __ldg(A.off + r), __ldg(A.off + r + 1), c0, acc);
        ppr_epilogue<S>(A, r, c0, acc, sink, act_bits, seed, X, Cc, Xn, Cn, l1p, dgp);
      }
    }
  }
  // CTA partials per column, warps added in a fixed order
#pragma unroll
  for (int i = 0; i < PL; ++i) {
    s_part[warp][c0 + i][0] = l1p[i];
    s_part[warp][c0 + i][1] = dgp[i];
  }
  __syncthreads();
  for (int c = threadIdx.x; c < S; c += kPprThreads) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < NW; ++w) {
      a += s_part[w][c][0];
      b += s_part[w][c][1];
    }
    A.part[((size_t)blockIdx.x * S + c) * 2] = a;
    A.part[((size_t)blockIdx.x * S + c) * 2 + 1] = b;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(A.cta_arrive, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // last CTA: per-column totals over the CTAs in block order, per-seed state
  int any = 0;
  for (int c = threadIdx.x; c < S; c += kPprThreads) {
    double a = 0.0, b = 0.0;
    for (unsigned k = 0; k < gridDim.x; ++k) {
      a += __ldcg(A.part + ((size_t)k * S + c) * 2);
      b += __ldcg(A.part + ((size_t)k * S + c) * 2 + 1);
    }
    if (A.active[c]) {
      A.iters[c] += 1;
      A.l1[c] = a;
      A.sink[c] = b;
      if (a < A.tol) A.active[c] = 0;  // centrality.zig:957, after the swap
      else any = 1;
    }
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    const int done = (!any || it + 1 >= A.max_iter) ? 1 : 0;
    A.st->iter = it + 1;
    A.st->done = done;
    *A.task_next = 0;
    *A.cta_arrive = 0;
    if (done && A.use_cond) cudaGraphSetConditional(A.cond, 0u);
  }
}

// X = 1/n, C = X/deg for every column (V x S), seed columns in ranked order.
template <int S>
__global__ void k_ppr_init(const uint32_t* __restrict__ deg, uint32_t V, double x0, double* __restrict__ X,
                           double* __restrict__ C) {
  const uint64_t total = (uint64_t)V * S;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t d = deg[i / S];
    X[i] = x0;
    C[i] = d == 0 ? 0.0 : __ddiv_rn(x0, (double)d);
  }
}

// out[s * V + node] = X[rank(node) * S + s] for the first `ns` columns, X
// the pass's last iterate (X0 or X1 by the parity of its iteration count)
template <int S>
__global__ void k_ppr_out(const double* __restrict__ X0, const double* __restrict__ X1,
                          const PprState* __restrict__ st, const uint32_t* __restrict__ rank, uint32_t V, uint32_t ns,
                          double* __restrict__ out) {
  const double* __restrict__ X = (st->iter & 1ull) ? X1 : X0;
  const uint64_t total = (uint64_t)V * ns;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = (uint32_t)(i / V), v = (uint32_t)(i % V);
    out[i] = X[(size_t)rank[v] * S + s];
  }
}

unsigned grid_for(uint64_t n) {
  const uint64_t g = (n + 255) / 256;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, (uint64_t)sm_count() * 16));
}

// What every pass of a call needs from the host: the rank of every node, and
// the sink of the uniform start -- x/n summed over the dangling nodes in
// ascending order, as the reference's first sink (centrality.zig:926-931).
struct PprHost {
  std::vector<uint32_t> rank;
  double sink0 = 0.0;
  int load(const Graph* g, cudaStream_t s) {
    const uint32_t V = g->V;
    rank.resize(V);
    std::vector<uint32_t> deg(V);
    ZOGCU_CUDA(cudaMemcpyAsync(rank.data(), g->pr.rank.ptr, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaMemcpyAsync(deg.data(), g->out_deg.ptr, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    const double n_f = (double)V;
    const double x0 = 1.0 / n_f;
    for (uint32_t v = 0; v < V; ++v)
      if (deg[v] == 0) sink0 += x0 / n_f;
    return ZOGCU_OK;
  }
};

// The matrices every pass of a call shares (V x width columns, node-major):
// passes run one after another inside the call's graph.  Y and the arrival
// counters are zero between uses (the kernel restores them).
struct PprShared {
  DevBuf X0, X1, C0, C1, Y, arrive;
  int alloc(uint32_t V, uint32_t width, cudaStream_t s) {
    const size_t mat = (size_t)V * width * 8;
    ZOGCU_TRY(X0.alloc(mat, s));
    ZOGCU_TRY(X1.alloc(mat, s));
    ZOGCU_TRY(C0.alloc(mat, s));
    ZOGCU_TRY(C1.alloc(mat, s));
    ZOGCU_TRY(Y.alloc(mat, s));
    ZOGCU_TRY(arrive.alloc((size_t)V * 4, s));
    ZOGCU_CUDA(cudaMemsetAsync(Y.ptr, 0, mat, s));
    ZOGCU_CUDA(cudaMemsetAsync(arrive.ptr, 0, (size_t)V * 4, s));
    return ZOGCU_OK;
  }
};

// One pass's own state (per-column seeds, flags, counts, partials), set up
// before the graph is launched.
struct PprPass {
  uint32_t first = 0, ns = 0;
  int S = 64;
  unsigned grid = 1;
  DevBuf seed_rank, active, iters, l1, sink, part, st, ctr;
  double* dst = nullptr;
};

template <int S>
int ppr_pass_setup(const PprHost& H, const uint32_t* seeds, PprPass& P, cudaStream_t s) {
  // per-column state: seeds as ranks (padding columns never start)
  std::vector<uint32_t> h_seed(S, kNoSeed);
  std::vector<int> h_active(S, 0);
  for (uint32_t i = 0; i < P.ns; ++i) {
    h_seed[i] = H.rank[seeds[P.first + i]];
    h_active[i] = 1;
  }
  std::vector<double> h_sink(S, H.sink0);
  ZOGCU_TRY(P.seed_rank.alloc(S * 4, s));
  ZOGCU_TRY(P.active.alloc(S * 4, s));
  ZOGCU_TRY(P.iters.alloc(S * 8, s));
  ZOGCU_TRY(P.l1.alloc(S * 8, s));
  ZOGCU_TRY(P.sink.alloc(S * 8, s));
  ZOGCU_CUDA(cudaMemcpyAsync(P.seed_rank.ptr, h_seed.data(), S * 4, cudaMemcpyHostToDevice, s));
  ZOGCU_CUDA(cudaMemcpyAsync(P.active.ptr, h_active.data(), S * 4, cudaMemcpyHostToDevice, s));
  ZOGCU_CUDA(cudaMemcpyAsync(P.sink.ptr, h_sink.data(), S * 8, cudaMemcpyHostToDevice, s));
  ZOGCU_CUDA(cudaMemsetAsync(P.iters.ptr, 0, S * 8, s));
  ZOGCU_CUDA(cudaMemsetAsync(P.l1.ptr, 0, S * 8, s));
  int per_sm = 0;
  ZOGCU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ppr_iter<S>, kPprThreads, 0));
  P.grid = (unsigned)std::max(1, per_sm) * (unsigned)sm_count();
  ZOGCU_TRY(P.part.alloc((size_t)P.grid * S * 16, s));
  ZOGCU_TRY(P.st.alloc(sizeof(PprState), s));
  ZOGCU_TRY(P.ctr.alloc(16, s));
  ZOGCU_CUDA(cudaMemsetAsync(P.st.ptr, 0, sizeof(PprState), s));
  ZOGCU_CUDA(cudaMemsetAsync(P.ctr.ptr, 0, 16, s));
  // the sync copies above come from pageable vectors that go out of scope
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  return ZOGCU_OK;
}

int add_kernel_node(cudaGraph_t graph, cudaGraphNode_t* node, const cudaGraphNode_t* dep, void* fn, unsigned grid,
                    unsigned threads, void** args) {
  cudaKernelNodeParams kp = {};
  kp.func = fn;
  kp.gridDim = dim3(grid);
  kp.blockDim = dim3(threads);
  kp.sharedMemBytes = 0;
  kp.kernelParams = args;
  ZOGCU_CUDA(cudaGraphAddKernelNode(node, graph, dep, dep ? 1 : 0, &kp));
  return ZOGCU_OK;
}

// Adds one pass to the call's graph after *tail: start vector, the while loop
// of iterations, the columns out; *tail becomes the pass's last node.
template <int S>
int ppr_pass_nodes(cudaGraph_t graph, cudaGraphNode_t* tail, Graph* g, PprShared& M, PprPass& P, double damping,
                   uint64_t max_iter, double tol) {
  const PrSchedule& Ps = g->pr;
  const PrTaskList& L = g->pr.lists[1];  // row blocks of up to 256 arcs
  const uint32_t V = g->V;
  const double n_f = (double)V;
  double x0 = 1.0 / n_f;
  const uint32_t* deg = Ps.deg.as<uint32_t>();
  double* X0 = M.X0.as<double>();
  double* C0 = M.C0.as<double>();
  uint32_t Vv = V;
  void* init_args[] = {(void*)&deg, &Vv, &x0, &X0, &C0};
  cudaGraphNode_t n_init;
  ZOGCU_TRY(add_kernel_node(graph, &n_init, *tail ? tail : nullptr, reinterpret_cast<void*>(k_ppr_init<S>),
                            grid_for((uint64_t)V * S), 256, init_args));
  PprArgs<S> A{};
  A.off = Ps.off.as<uint32_t>();
  A.col = Ps.col.as<uint32_t>();
  A.deg = deg;
  A.tasks = L.tasks.as<PrTask>();
  A.num_tasks = L.num_tasks;
  A.X[0] = X0;
  A.X[1] = M.X1.as<double>();
  A.C[0] = C0;
  A.C[1] = M.C1.as<double>();
  A.Y = M.Y.as<double>();
  A.arrive = M.arrive.as<uint32_t>();
  A.seed_rank = P.seed_rank.as<uint32_t>();
  A.active = P.active.as<int>();
  A.iters = P.iters.as<unsigned long long>();
  A.l1 = P.l1.as<double>();
  A.sink = P.sink.as<double>();
  A.part = P.part.as<double>();
  A.st = P.st.as<PprState>();
  A.task_next = P.ctr.as<uint32_t>();
  A.cta_arrive = P.ctr.as<uint32_t>() + 1;
  A.V = V;
  A.n_f = n_f;
  A.damping = damping;
  A.tol = tol;
  A.max_iter = max_iter;
  // the loop's condition starts at 1 on every launch; a pass with no
  // iterations to run is over before its first body launch, which clears it
  cudaGraphConditionalHandle h;
  ZOGCU_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1u, cudaGraphCondAssignDefault));
  A.cond = h;
  A.use_cond = 1;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t n_loop;
  ZOGCU_CUDA(cudaGraphAddNode(&n_loop, graph, &n_init, 1, &cp));
  void* iter_args[] = {&A};
  cudaGraphNode_t n_body;
  ZOGCU_TRY(add_kernel_node(cp.conditional.phGraph_out[0], &n_body, nullptr, reinterpret_cast<void*>(k_ppr_iter<S>),
                            P.grid, kPprThreads, iter_args));
  const double* X1c = A.X[1];
  const double* X0c = X0;
  const PprState* stc = A.st;
  const uint32_t* rank = Ps.rank.as<uint32_t>();
  uint32_t ns = P.ns;
  double* dst = P.dst;
  void* out_args[] = {(void*)&X0c, (void*)&X1c, (void*)&stc, (void*)&rank, &Vv, &ns, &dst};
  cudaGraphNode_t n_out;
  ZOGCU_TRY(add_kernel_node(graph, &n_out, &n_loop, reinterpret_cast<void*>(k_ppr_out<S>),
                            grid_for((uint64_t)V * P.ns), 256, out_args));
  *tail = n_out;
  return ZOGCU_OK;
}

}  // namespace
}  // namespace zogcu

extern "C" int zogcu_ppr(zogcu_graph* G, const uint32_t* seeds, uint32_t num_seeds, double damping,
                         uint64_t max_iterations, double tolerance, const zogcu_pr_opts* opts, double* out_scores,
                         uint64_t* iterations, zogcu_stats* stats) {
  using namespace zogcu;
  if (!G) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graph is null");
  if (num_seeds && (!seeds || !out_scores)) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  if (opts && opts->struct_size != sizeof(zogcu_pr_opts))
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "zogcu_pr_opts.struct_size mismatch");
  if (opts && (opts->precision != ZOGCU_PREC_FP64 || opts->x0 || opts->teleport))
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "personalised PageRank takes FP64, the uniform start and one-hot seeds");
  Graph* g = &G->g;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (g->has_deleted) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "personalised PageRank needs a graph without deleted nodes");
  if (!g->offsets32) return fail(ZOGCU_ERR_TOO_LARGE, "personalised PageRank needs fewer than 2^32 arcs");
  for (uint32_t i = 0; i < num_seeds; ++i)
    if (seeds[i] >= g->V) return fail(ZOGCU_ERR_NODE_NOT_FOUND, "seed is not a node of the graph");
  if (num_seeds == 0 || g->V == 0) return ZOGCU_OK;
  ZOGCU_CUDA(cudaSetDevice(g->device));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(opts ? opts->stream : nullptr));
  const cudaStream_t s = sg.s;
  ZOGCU_TRY(ensure_pr_schedule(g, s));
  ZOGCU_TRY(ensure_task_list(g, 256, s));
  const bool dev_out = opts && opts->device_pointers;
  const uint32_t V = g->V;
  // Pass width: on graphs of 2^19 nodes and more, passes of 64 seeds -- the
  // 64-column kernel (62 registers) runs twice the warps per SM of the
  // 256-column one (128 registers), which outweighs streaming the arc indices
  // once per pass (256 seeds: 422 against 570 ms at scale 22, 98 against
  // 114 ms at scale 20); on smaller graphs one pass of 256 (47 against 58 ms
  // at scale 18).
  PprHost H;
  ZOGCU_TRY(H.load(g, s));
  uint32_t width = V < (1u << 19) ? 256u : 64u;  // ZOGCU_PPR_PASS=32/64/128/256 overrides
  if (const char* e = std::getenv("ZOGCU_PPR_PASS")) {
    const int w = std::atoi(e);
    if (w == 32 || w == 64 || w == 128 || w == 256) width = (uint32_t)w;
  }
  const uint32_t npass = (num_seeds + width - 1) / width;
  std::vector<PprPass> passes(npass);
  int max_S = 32;
  for (uint32_t p = 0; p < npass; ++p) {
    PprPass& P = passes[p];
    P.first = p * width;
    P.ns = std::min<uint32_t>(num_seeds - P.first, width);
    P.S = P.ns > 128 ? 256 : P.ns > 64 ? 128 : (P.ns > 32 || width > 32) ? 64 : 32;
    max_S = std::max(max_S, P.S);
  }
  PprShared M;
  ZOGCU_TRY(M.alloc(V, (uint32_t)max_S, s));
  DevBuf res;
  if (!dev_out) ZOGCU_TRY(res.alloc((size_t)V * num_seeds * 8, s));
  for (PprPass& P : passes) {
    P.dst = (dev_out ? out_scores : res.as<double>()) + (size_t)P.first * V;
    if (P.S == 256) ZOGCU_TRY(ppr_pass_setup<256>(H, seeds, P, s));
    else if (P.S == 128) ZOGCU_TRY(ppr_pass_setup<128>(H, seeds, P, s));
    else if (P.S == 64) ZOGCU_TRY(ppr_pass_setup<64>(H, seeds, P, s));
    else ZOGCU_TRY(ppr_pass_setup<32>(H, seeds, P, s));
  }
  // the call's graph: every pass after the previous one
  cudaGraph_t graph = nullptr;
  ZOGCU_CUDA(cudaGraphCreate(&graph, 0));
  struct GraphGuard {
    cudaGraph_t gr;
    ~GraphGuard() { cudaGraphDestroy(gr); }
  } guard{graph};
  cudaGraphNode_t tail = nullptr;  // the previous pass's last node (none before the first)
  for (PprPass& P : passes) {
    if (P.S == 256) ZOGCU_TRY(ppr_pass_nodes<256>(graph, &tail, g, M, P, damping, max_iterations, tolerance));
    else if (P.S == 128) ZOGCU_TRY(ppr_pass_nodes<128>(graph, &tail, g, M, P, damping, max_iterations, tolerance));
    else if (P.S == 64) ZOGCU_TRY(ppr_pass_nodes<64>(graph, &tail, g, M, P, damping, max_iterations, tolerance));
    else ZOGCU_TRY(ppr_pass_nodes<32>(graph, &tail, g, M, P, damping, max_iterations, tolerance));
  }
  cudaGraphExec_t exec = nullptr;
  ZOGCU_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  EventTimer tm;
  ZOGCU_TRY(tm.start(s));
  const cudaError_t le = cudaGraphLaunch(exec, s);
  cudaGraphExecDestroy(exec);  // an executable graph in flight is freed when it completes
  ZOGCU_CUDA(le);
  ZOGCU_TRY(tm.stop(s));
  if (!dev_out) ZOGCU_CUDA(cudaMemcpyAsync(out_scores, res.ptr, (size_t)V * num_seeds * 8, cudaMemcpyDeviceToHost, s));
  // per-pass iteration counts and per-seed iterations
  uint64_t kernel_runs = 0, max_it = 0;
  for (PprPass& P : passes) {
    PprState hs{};
    std::vector<unsigned long long> h_it(P.ns);
    ZOGCU_CUDA(cudaMemcpyAsync(&hs, P.st.ptr, sizeof(hs), cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaMemcpyAsync(h_it.data(), P.iters.ptr, (size_t)P.ns * 8, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    for (uint32_t i = 0; i < P.ns; ++i) {
      if (iterations) iterations[P.first + i] = h_it[i];
      max_it = std::max<uint64_t>(max_it, h_it[i]);
    }
    // the loop's body ran once per iteration (the last one clears the loop's
    // condition; with max_iterations 0, one run finds the pass over), plus
    // the start and out kernels
    kernel_runs += std::max<uint64_t>(hs.iter, 1) + 2;
    if (stats) {
      // per iteration: arc indices and offsets once, every column of C
      // gathered once per arc, X read and X', C' written
      const double per_iter = 4.0 * (double)g->E + 4.0 * ((double)V + 1) + 8.0 * P.S * (double)g->E +
                              24.0 * P.S * (double)V;
      stats->bytes_moved += per_iter * (double)hs.iter;
    }
  }
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  if (stats) {
    stats->iterations = max_it;
    stats->elapsed_ms = tm.ms();
    stats->launches = kernel_runs;
    stats->reserved = 1;  // host-side launches: the call's one graph
  }
  return ZOGCU_OK;
}
