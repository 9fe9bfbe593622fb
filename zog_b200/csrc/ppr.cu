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
// state; the host enqueues max_iterations launches and launches after the
// last active seed has stopped return at once.
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
  static_assert(S % 64 == 0 && S <= 256, "columns per pass: 64, 128 or 256");
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
};

// PL consecutive doubles of one contribution row, read with 32-byte loads
// that skip L1 allocation (16-byte loads when PL is 2): the row is streamed,
// never re-read by this warp.
template <int PL>
__device__ __forceinline__ void ld_row(const double* p, double (&v)[PL]) {
  if constexpr (PL % 4 == 0) {
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
  if (*(volatile int*)&A.st->done) return;
  const unsigned long long it = *(volatile unsigned long long*)&A.st->iter;
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
    A.st->iter = it + 1;
    A.st->done = (!any || it + 1 >= A.max_iter) ? 1 : 0;
    *A.task_next = 0;
    *A.cta_arrive = 0;
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

// out[s * V + node] = X[rank(node) * S + s] for the first `ns` columns
template <int S>
__global__ void k_ppr_out(const double* __restrict__ X, const uint32_t* __restrict__ rank, uint32_t V, uint32_t ns,
                          double* __restrict__ out) {
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

// One pass over up to S seeds.
template <int S>
int ppr_pass(Graph* g, const PprHost& H, const uint32_t* seeds, uint32_t ns, double damping, uint64_t max_iter,
             double tol, double* out, bool dev_out, uint64_t* iters_out, zogcu_stats* stats, cudaStream_t s) {
  const PrSchedule& P = g->pr;
  const PrTaskList& L = g->pr.lists[1];  // row blocks of up to 256 arcs
  const uint32_t V = g->V;
  const size_t mat = (size_t)V * S * 8;
  DevBuf X0, X1, C0, C1, Y, arrive, seed_rank, active, iters, l1, sink, part, st, ctr, host_seeds, res;
  ZOGCU_TRY(X0.alloc(mat, s));
  ZOGCU_TRY(X1.alloc(mat, s));
  ZOGCU_TRY(C0.alloc(mat, s));
  ZOGCU_TRY(C1.alloc(mat, s));
  ZOGCU_TRY(Y.alloc(mat, s));
  ZOGCU_TRY(arrive.alloc((size_t)V * 4, s));
  ZOGCU_CUDA(cudaMemsetAsync(Y.ptr, 0, mat, s));
  ZOGCU_CUDA(cudaMemsetAsync(arrive.ptr, 0, (size_t)V * 4, s));
  // per-column state: seeds as ranks (padding columns never start)
  std::vector<uint32_t> h_seed(S, kNoSeed);
  std::vector<int> h_active(S, 0);
  for (uint32_t i = 0; i < ns; ++i) {
    h_seed[i] = H.rank[seeds[i]];
    h_active[i] = 1;
  }
  const double n_f = (double)V;
  const double x0 = 1.0 / n_f;
  std::vector<double> h_sink(S, H.sink0);
  ZOGCU_TRY(seed_rank.alloc(S * 4, s));
  ZOGCU_TRY(active.alloc(S * 4, s));
  ZOGCU_TRY(iters.alloc(S * 8, s));
  ZOGCU_TRY(l1.alloc(S * 8, s));
  ZOGCU_TRY(sink.alloc(S * 8, s));
  ZOGCU_CUDA(cudaMemcpyAsync(seed_rank.ptr, h_seed.data(), S * 4, cudaMemcpyHostToDevice, s));
  ZOGCU_CUDA(cudaMemcpyAsync(active.ptr, h_active.data(), S * 4, cudaMemcpyHostToDevice, s));
  ZOGCU_CUDA(cudaMemcpyAsync(sink.ptr, h_sink.data(), S * 8, cudaMemcpyHostToDevice, s));
  ZOGCU_CUDA(cudaMemsetAsync(iters.ptr, 0, S * 8, s));
  ZOGCU_CUDA(cudaMemsetAsync(l1.ptr, 0, S * 8, s));
  int per_sm = 0;
  ZOGCU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ppr_iter<S>, kPprThreads, 0));
  const unsigned grid = (unsigned)std::max(1, per_sm) * (unsigned)sm_count();
  ZOGCU_TRY(part.alloc((size_t)grid * S * 16, s));
  ZOGCU_TRY(st.alloc(sizeof(PprState), s));
  ZOGCU_TRY(ctr.alloc(16, s));
  ZOGCU_CUDA(cudaMemsetAsync(st.ptr, 0, sizeof(PprState), s));
  ZOGCU_CUDA(cudaMemsetAsync(ctr.ptr, 0, 16, s));
  k_ppr_init<S><<<grid_for((uint64_t)V * S), 256, 0, s>>>(P.deg.as<uint32_t>(), V, x0, X0.as<double>(), C0.as<double>());
  ZOGCU_CUDA(cudaGetLastError());
  PprArgs<S> A{};
  A.off = P.off.as<uint32_t>();
  A.col = P.col.as<uint32_t>();
  A.deg = P.deg.as<uint32_t>();
  A.tasks = L.tasks.as<PrTask>();
  A.num_tasks = L.num_tasks;
  A.X[0] = X0.as<double>();
  A.X[1] = X1.as<double>();
  A.C[0] = C0.as<double>();
  A.C[1] = C1.as<double>();
  A.Y = Y.as<double>();
  A.arrive = arrive.as<uint32_t>();
  A.seed_rank = seed_rank.as<uint32_t>();
  A.active = active.as<int>();
  A.iters = iters.as<unsigned long long>();
  A.l1 = l1.as<double>();
  A.sink = sink.as<double>();
  A.part = part.as<double>();
  A.st = st.as<PprState>();
  A.task_next = ctr.as<uint32_t>();
  A.cta_arrive = ctr.as<uint32_t>() + 1;
  A.V = V;
  A.n_f = n_f;
  A.damping = damping;
  A.tol = tol;
  A.max_iter = max_iter;
  if (max_iter == 0) {
    int one = 1;
    ZOGCU_CUDA(cudaMemcpyAsync(&st.as<PprState>()->done, &one, 4, cudaMemcpyHostToDevice, s));
  }
  EventTimer tm;
  ZOGCU_TRY(tm.start(s));
  for (uint64_t k = 0; k < max_iter; ++k) k_ppr_iter<S><<<grid, kPprThreads, 0, s>>>(A);
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_TRY(tm.stop(s));
  PprState hs{};
  ZOGCU_CUDA(cudaMemcpyAsync(&hs, st.ptr, sizeof(hs), cudaMemcpyDeviceToHost, s));
  std::vector<unsigned long long> h_it(S);
  ZOGCU_CUDA(cudaMemcpyAsync(h_it.data(), iters.ptr, S * 8, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  const double* Xr = (hs.iter & 1ull) ? X1.as<double>() : X0.as<double>();
  double* dst = out;
  if (!dev_out) {
    ZOGCU_TRY(res.alloc((size_t)V * ns * 8, s));
    dst = res.as<double>();
  }
  k_ppr_out<S><<<grid_for((uint64_t)V * ns), 256, 0, s>>>(Xr, P.rank.as<uint32_t>(), V, ns, dst);
  ZOGCU_CUDA(cudaGetLastError());
  if (!dev_out) ZOGCU_CUDA(cudaMemcpyAsync(out, dst, (size_t)V * ns * 8, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  uint64_t max_it = 0;
  for (uint32_t i = 0; i < ns; ++i) {
    if (iters_out) iters_out[i] = h_it[i];
    max_it = std::max<uint64_t>(max_it, h_it[i]);
  }
  if (stats) {
    stats->iterations = std::max<uint64_t>(stats->iterations, max_it);
    stats->elapsed_ms += tm.ms();
    // per launch: arc indices and offsets once, every column of C gathered
    // once per arc, X read and X', C' written
    const double per_iter = 4.0 * (double)g->E + 4.0 * ((double)V + 1) + 8.0 * S * (double)g->E +
                            24.0 * S * (double)V;
    stats->bytes_moved += per_iter * (double)hs.iter;
    stats->launches += hs.iter + 2;
  }
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
  ZOGCU_TRY(ensure_pr_schedule(g, sg.s));
  ZOGCU_TRY(ensure_task_list(g, 256, sg.s));
  const bool dev_out = opts && opts->device_pointers;
  const size_t V = g->V;
  // Pass width: on graphs of 2^19 nodes and more, passes of 64 seeds -- the
  // 64-column kernel (62 registers) runs twice the warps per SM of the
  // 256-column one (128 registers), which outweighs streaming the arc indices
  // once per pass (256 seeds: 422 against 570 ms at scale 22, 98 against
  // 114 ms at scale 20); on smaller graphs one pass of 256 (47 against 58 ms
  // at scale 18).
  PprHost H;
  ZOGCU_TRY(H.load(g, sg.s));
  uint32_t width = V < (1u << 19) ? 256u : 64u;  // ZOGCU_PPR_PASS=64/128/256 overrides
  if (const char* e = std::getenv("ZOGCU_PPR_PASS")) {
    const int w = std::atoi(e);
    if (w == 64 || w == 128 || w == 256) width = (uint32_t)w;
  }
  for (uint32_t s0 = 0; s0 < num_seeds;) {
    const uint32_t ns = std::min<uint32_t>(num_seeds - s0, width);
    double* o = out_scores + (size_t)s0 * V;
    uint64_t* it = iterations ? iterations + s0 : nullptr;
    if (ns > 128)
      ZOGCU_TRY(ppr_pass<256>(g, H, seeds + s0, ns, damping, max_iterations, tolerance, o, dev_out, it, stats, sg.s));
    else if (ns > 64)
      ZOGCU_TRY(ppr_pass<128>(g, H, seeds + s0, ns, damping, max_iterations, tolerance, o, dev_out, it, stats, sg.s));
    else
      ZOGCU_TRY(ppr_pass<64>(g, H, seeds + s0, ns, damping, max_iterations, tolerance, o, dev_out, it, stats, sg.s));
    s0 += ns;
  }
  return ZOGCU_OK;
}
