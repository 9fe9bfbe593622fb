// pagerank.cu -- PageRank power iteration on the device-resident in-CSR.
//
// Reference: priv/zog/src/centrality.zig:858-965 (ArrayGraph branch).  Per
// iteration the reference computes, over live nodes in ascending order,
//     sink     = sum_{deg(u)=0} x[u] / n                        (:926-931)
//     x'[v]    = (1-d)/n + d * (sink + sum_{u in in(v)} x[u]/deg(u))   (:933-944)
//     l1       = sum |x'[v] - x[v]|                                (:947-950)
// swaps, and stops once l1 < tol (:953-957).
//
// B200 design (one fused, persistent pass per iteration):
//   * pull SpMV over the in-CSR with a precomputed contribution vector
//     c[u] = x[u]/deg(u) (the reference's per-term quotient, bit for bit);
//   * degree-binned schedule built once per graph: rows are packed into blocks
//     of <= kBlockNnz arcs and <= kRowCap rows; inside a block, rows of
//     in-degree <= kShortLen are summed by one thread each (sequentially, in
//     the reference's ascending-source order), longer rows by a warp, and rows
//     longer than kBlockNnz are split into CTA-sized chunks whose partials the
//     last-arriving CTA combines;
//   * arc indices stream in as 16-byte vectors (ld.global.cs, evict-first) and
//     the gathered c values are staged in shared memory;
//   * the epilogue writes x', c' = x'/deg, and accumulates |x'-x| and the
//     dangling mass of x' (the next iteration's sink) -- warp shuffle, CTA
//     reduction, then a deterministic last-CTA reduction over fixed slots;
//   * the convergence test runs on the device: the last CTA publishes l1 and a
//     converged flag, and later launches of the same chain exit at once, so the
//     host enqueues max_iterations launches without a round trip.
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace zogcu {

constexpr int kPrThreads = 256;
constexpr int kBlockNnz = 2048;   // arcs per block / per long-row chunk
constexpr int kRowCap = 512;      // rows per block
constexpr int kShortLen = 32;     // rows up to this in-degree: one thread each

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
  uint32_t ntasks;
  uint32_t nlong;
  double* x0;
  double* x1;
  CT* c0;
  CT* c1;
  double* cta_part;      // [2 * gridDim.x]
  double* chunk_part;    // [ntasks]
  unsigned int* long_cnt;// [nlong]
  double* long_part;     // [2 * nlong]
  PrState* st;
  const double* teleport;  // personalised teleport p[v] or null (uniform)
  double damping;
  double n_f;
  double tol;
  unsigned long long max_iter;
};

__device__ __forceinline__ uint4 ld_stream_u4(const uint4* p) { return __ldcs(p); }

template <typename CT>
__device__ __forceinline__ double to_d(CT v) { return (double)v; }

// Epilogue of one row: the reference's update (centrality.zig:943) evaluated
// with explicit round-to-nearest operations (no FMA contraction), then the
// residual / dangling bookkeeping and the next contribution c' = x'/deg.
template <typename OffT, typename CT>
__device__ __forceinline__ void pr_row_epilogue(const PrArgs<OffT, CT>& A, uint32_t v, double rank_sum,
                                                const double* __restrict__ xcur, double* __restrict__ xnxt,
                                                CT* __restrict__ cnxt, double tele_u, double sink, double& l1,
                                                double& dsum) {
  const uint32_t deg = __ldg(A.deg + v);
  if (deg == kDeletedDegree) return;
  const double tele = A.teleport ? __dmul_rn(1.0 - A.damping, __ldg(A.teleport + v)) : tele_u;
  const double xn = __dadd_rn(tele, __dmul_rn(A.damping, __dadd_rn(sink, rank_sum)));
  const double xo = __ldg(xcur + v);
  l1 += fabs(xn - xo);
  xnxt[v] = xn;
  if (deg == 0) {
    dsum += __ddiv_rn(xn, A.n_f);
  } else {
    cnxt[v] = (CT)__ddiv_rn(xn, (double)deg);
  }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic CTA sum of two doubles; result valid in thread 0.
__device__ __forceinline__ void cta_sum2(double& a, double& b, double* s_red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
    for (int w = 0; w < kPrThreads / 32; ++w) {
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
                             uint32_t nlong, unsigned long long next_iter, double tol, bool set_l1,
                             double* s_red) {
  double a = 0.0, b = 0.0;
  for (uint32_t i = threadIdx.x; i < ncta; i += kPrThreads) {
    a += __ldcg(cta_part + 2 * i);
    b += __ldcg(cta_part + 2 * i + 1);
  }
  for (uint32_t i = threadIdx.x; i < nlong; i += kPrThreads) {
    a += __ldcg(long_part + 2 * i);
    b += __ldcg(long_part + 2 * i + 1);
  }
  cta_sum2(a, b, s_red);
  if (threadIdx.x == 0) {
    st->sink = b;
    if (set_l1) {
      st->l1 = a;
      st->converged = (a < tol) ? 1 : 0;
    } else {
      st->l1 = 0.0;
      st->converged = 0;
    }
    st->iter = next_iter;
    __threadfence();
    st->done_ctas = 0;
  }
}

// x0 / c0 from the start vector; sink of x0.  `given` = x0 already holds a
// caller's start vector (warm start), else the uniform 1/n of :912-918.
template <typename OffT, typename CT>
__global__ void __launch_bounds__(kPrThreads) pr_init_kernel(PrArgs<OffT, CT> A, uint32_t V, int given) {
  __shared__ double s_red[2 * (kPrThreads / 32)];
  __shared__ int s_last;
  double dsum = 0.0, unused = 0.0;
  const double init = 1.0 / A.n_f;
  for (uint64_t v = blockIdx.x * (uint64_t)kPrThreads + threadIdx.x; v < V; v += (uint64_t)gridDim.x * kPrThreads) {
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
  cta_sum2(unused, dsum, s_red);
  if (threadIdx.x == 0) {
    A.cta_part[2 * blockIdx.x] = 0.0;
    A.cta_part[2 * blockIdx.x + 1] = dsum;
    __threadfence();
    unsigned int t = atomicAdd(&A.st->done_ctas, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    final_reduce(A.st, A.cta_part, gridDim.x, A.long_part, 0, 0ull, A.tol, false, s_red);
  }
}

template <typename OffT, typename CT>
__global__ void __launch_bounds__(kPrThreads, 4) pr_iter_kernel(PrArgs<OffT, CT> A) {
  __shared__ __align__(16) double s_val[kBlockNnz];
  __shared__ uint32_t s_off[kRowCap + 1];
  __shared__ double s_red[2 * (kPrThreads / 32)];
  __shared__ int s_flag;

  const PrState* st = A.st;
  const unsigned long long iter = *(volatile const unsigned long long*)&st->iter;
  const int converged = *(volatile const int*)&st->converged;
  if (converged || iter >= A.max_iter) return;
  const double sink = *(volatile const double*)&st->sink;

  const int par = (int)(iter & 1ull);
  const double* __restrict__ xcur = par ? A.x1 : A.x0;
  double* __restrict__ xnxt = par ? A.x0 : A.x1;
  const CT* __restrict__ ccur = par ? A.c1 : A.c0;
  CT* __restrict__ cnxt = par ? A.c0 : A.c1;
  const double tele_u = (1.0 - A.damping) / A.n_f;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double l1 = 0.0, dsum = 0.0;

  for (uint32_t ti = blockIdx.x; ti < A.ntasks; ti += gridDim.x) {
    const PrTask t = A.tasks[ti];
    if ((t.kind & 0xFFFFu) == 0) {
      // ---- block of rows [r0, r1) --------------------------------------
      const uint32_t r0 = t.a, r1 = t.b, nrows = r1 - r0;
      const OffT e0 = __ldg(A.off + r0), e1 = __ldg(A.off + r1);
      for (uint32_t i = tid; i <= nrows; i += kPrThreads) s_off[i] = (uint32_t)(__ldg(A.off + r0 + i) - e0);
      const OffT base = e0 & ~(OffT)3;
      const uint32_t nvec = (uint32_t)((e1 - base + 3) >> 2);
      const uint4* cv = reinterpret_cast<const uint4*>(A.col + base);
      for (uint32_t j = tid; j < nvec; j += kPrThreads) {
        const uint4 q = ld_stream_u4(cv + j);
        const OffT e = base + 4 * (OffT)j;
        if (e >= e0 && e < e1) s_val[e - e0] = to_d(__ldg(ccur + q.x));
        if (e + 1 >= e0 && e + 1 < e1) s_val[e + 1 - e0] = to_d(__ldg(ccur + q.y));
        if (e + 2 >= e0 && e + 2 < e1) s_val[e + 2 - e0] = to_d(__ldg(ccur + q.z));
        if (e + 3 >= e0 && e + 3 < e1) s_val[e + 3 - e0] = to_d(__ldg(ccur + q.w));
      }
      __syncthreads();
      for (uint32_t wb = (uint32_t)warp * 32; wb < nrows; wb += kPrThreads) {
        const uint32_t i = wb + lane;
        const bool valid = i < nrows;
        uint32_t b = 0, en = 0;
        if (valid) {
          b = s_off[i];
          en = s_off[i + 1];
        }
        const bool is_short = valid && (en - b) <= (uint32_t)kShortLen;
        if (is_short) {
          double s = 0.0;
          for (uint32_t k = b; k < en; ++k) s += s_val[k];  // ascending source order
          pr_row_epilogue(A, r0 + i, s, xcur, xnxt, cnxt, tele_u, sink, l1, dsum);
        }
        unsigned med = __ballot_sync(0xffffffffu, valid && !is_short);
        while (med) {
          const int k = __ffs(med) - 1;
          med &= med - 1;
          const uint32_t bk = __shfl_sync(0xffffffffu, b, k), ek = __shfl_sync(0xffffffffu, en, k);
          double s = 0.0;
          for (uint32_t j = bk + lane; j < ek; j += 32) s += s_val[j];
          s = warp_sum(s);
          if (lane == k) pr_row_epilogue(A, r0 + i, s, xcur, xnxt, cnxt, tele_u, sink, l1, dsum);
        }
      }
      __syncthreads();
    } else {
      // ---- chunk c of nch of long row `row` ------------------------------
      const uint32_t row = t.a, c = t.b, nch = t.kind >> 16, slot = t.slot;
      const OffT rs = __ldg(A.off + row), re = __ldg(A.off + row + 1);
      const OffT e0 = rs + (OffT)c * kBlockNnz;
      const OffT e1 = min(e0 + (OffT)kBlockNnz, re);
      const OffT base = e0 & ~(OffT)3;
      const uint32_t nvec = (uint32_t)((e1 - base + 3) >> 2);
      const uint4* cv = reinterpret_cast<const uint4*>(A.col + base);
      double s = 0.0;
      for (uint32_t j = tid; j < nvec; j += kPrThreads) {
        const uint4 q = ld_stream_u4(cv + j);
        const OffT e = base + 4 * (OffT)j;
        if (e >= e0 && e < e1) s += to_d(__ldg(ccur + q.x));
        if (e + 1 >= e0 && e + 1 < e1) s += to_d(__ldg(ccur + q.y));
        if (e + 2 >= e0 && e + 2 < e1) s += to_d(__ldg(ccur + q.z));
        if (e + 3 >= e0 && e + 3 < e1) s += to_d(__ldg(ccur + q.w));
      }
      double unused = 0.0;
      cta_sum2(unused, s, s_red);
      if (tid == 0) {
        A.chunk_part[ti] = s;
        __threadfence();
        const unsigned int old = atomicAdd(A.long_cnt + slot, 1u);
        s_flag = (old == nch - 1);
      }
      __syncthreads();
      if (s_flag && tid == 0) {
        __threadfence();
        double tot = 0.0;
        for (uint32_t k = 0; k < nch; ++k) tot += __ldcg(A.chunk_part + (ti - c + k));
        double rl1 = 0.0, rds = 0.0;
        pr_row_epilogue(A, row, tot, xcur, xnxt, cnxt, tele_u, sink, rl1, rds);
        A.long_part[2 * slot] = rl1;
        A.long_part[2 * slot + 1] = rds;
        A.long_cnt[slot] = 0;
      }
      __syncthreads();
    }
  }

  // ---- publish this CTA's residual / dangling partials ---------------------
  cta_sum2(l1, dsum, s_red);
  if (tid == 0) {
    A.cta_part[2 * blockIdx.x] = l1;
    A.cta_part[2 * blockIdx.x + 1] = dsum;
    __threadfence();
    const unsigned int t = atomicAdd(&A.st->done_ctas, 1u);
    s_flag = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (s_flag) {
    __threadfence();
    final_reduce(A.st, A.cta_part, gridDim.x, A.long_part, A.nlong, iter + 1, A.tol, true, s_red);
  }
}

// ---------------------------------------------------------------------------
// Schedule: greedy packing of rows into blocks, long rows into chunks.
// ---------------------------------------------------------------------------
int ensure_pr_schedule(Graph* g, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g->mu);
  if (g->pr.built) return ZOGCU_OK;
  const uint32_t V = g->V;
  std::vector<uint64_t> off((size_t)V + 1);
  ZOGCU_CUDA(cudaMemcpyAsync(off.data(), g->in_off64.ptr, ((size_t)V + 1) * 8, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  std::vector<PrTask> tasks;
  tasks.reserve(g->E / kBlockNnz + V / kRowCap + 16);
  uint32_t nlong = 0, maxch = 0;
  uint32_t r = 0;
  while (r < V) {
    uint64_t len = off[r + 1] - off[r];
    if (len > (uint64_t)kBlockNnz) {
      const uint32_t nch = (uint32_t)((len + kBlockNnz - 1) / kBlockNnz);
      if (nch > 0xFFFFu) return fail(ZOGCU_ERR_TOO_LARGE, "row in-degree too large for the chunk schedule");
      for (uint32_t c = 0; c < nch; ++c) tasks.push_back(PrTask{r, c, 1u | (nch << 16), nlong});
      maxch = std::max(maxch, nch);
      ++nlong;
      ++r;
      continue;
    }
    const uint32_t r0 = r;
    uint64_t nnz = 0;
    while (r < V && (r - r0) < (uint32_t)kRowCap) {
      len = off[r + 1] - off[r];
      if (len > (uint64_t)kBlockNnz || nnz + len > (uint64_t)kBlockNnz) break;
      nnz += len;
      ++r;
    }
    tasks.push_back(PrTask{r0, r, 0u, 0u});
  }
  g->pr.num_tasks = (uint32_t)tasks.size();
  g->pr.num_long = nlong;
  g->pr.max_chunks = maxch;
  if (!tasks.empty()) {
    ZOGCU_TRY(g->pr.tasks.alloc(tasks.size() * sizeof(PrTask)));
    ZOGCU_CUDA(cudaMemcpyAsync(g->pr.tasks.ptr, tasks.data(), tasks.size() * sizeof(PrTask),
                               cudaMemcpyHostToDevice, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
  }
  g->pr.built = true;
  return ZOGCU_OK;
}

template <typename OffT, typename CT>
static int pr_grid() {
  static int grid = 0;
  if (grid == 0) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pr_iter_kernel<OffT, CT>, kPrThreads, 0);
    if (per_sm <= 0) per_sm = 1;
    grid = per_sm * sm_count();
  }
  return grid;
}

template <typename OffT>
static int run_pagerank_fp64(Graph* g, const OffT* off, double damping, uint64_t max_iter, double tol,
                             const zogcu_pr_opts* o, double* out, zogcu_stats* stats, cudaStream_t s) {
  const uint32_t V = g->V;
  const uint32_t ntasks = g->pr.num_tasks, nlong = g->pr.num_long;
  int grid = pr_grid<OffT, double>();
  if (ntasks > 0 && (uint32_t)grid > ntasks) grid = (int)ntasks;
  if (grid < 1) grid = 1;
  const bool dev_ptrs = o && o->device_pointers;

  DevBuf x0, x1, c0, c1, part, chunk, lcnt, lpart, stb, tele;
  ZOGCU_TRY(x0.alloc((size_t)V * 8, s));
  ZOGCU_TRY(x1.alloc((size_t)V * 8, s));
  ZOGCU_TRY(c0.alloc((size_t)V * 8, s));
  ZOGCU_TRY(c1.alloc((size_t)V * 8, s));
  ZOGCU_TRY(part.alloc((size_t)grid * 16, s));
  ZOGCU_TRY(chunk.alloc((size_t)std::max<uint32_t>(ntasks, 1) * 8, s));
  ZOGCU_TRY(lcnt.alloc((size_t)std::max<uint32_t>(nlong, 1) * 4, s));
  ZOGCU_TRY(lpart.alloc((size_t)std::max<uint32_t>(nlong, 1) * 16, s));
  ZOGCU_TRY(stb.alloc(sizeof(PrState), s));
  ZOGCU_CUDA(cudaMemsetAsync(lcnt.ptr, 0, lcnt.bytes, s));
  ZOGCU_CUDA(cudaMemsetAsync(lpart.ptr, 0, lpart.bytes, s));
  ZOGCU_CUDA(cudaMemsetAsync(stb.ptr, 0, sizeof(PrState), s));
  ZOGCU_CUDA(cudaMemsetAsync(c0.ptr, 0, c0.bytes, s));
  ZOGCU_CUDA(cudaMemsetAsync(c1.ptr, 0, c1.bytes, s));
  int given = 0;
  if (o && o->x0) {
    ZOGCU_CUDA(cudaMemcpyAsync(x0.ptr, o->x0, (size_t)V * 8, dev_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    given = 1;
  }
  const double* tele_ptr = nullptr;
  if (o && o->teleport) {
    if (dev_ptrs) {
      tele_ptr = o->teleport;
    } else {
      ZOGCU_TRY(tele.alloc((size_t)V * 8, s));
      ZOGCU_CUDA(cudaMemcpyAsync(tele.ptr, o->teleport, (size_t)V * 8, cudaMemcpyHostToDevice, s));
      tele_ptr = tele.as<double>();
    }
  }

  PrArgs<OffT, double> A;
  A.off = off;
  A.col = g->in_col.as<uint32_t>();
  A.deg = g->out_deg.as<uint32_t>();
  A.tasks = g->pr.tasks.as<PrTask>();
  A.ntasks = ntasks;
  A.nlong = nlong;
  A.x0 = x0.as<double>();
  A.x1 = x1.as<double>();
  A.c0 = c0.as<double>();
  A.c1 = c1.as<double>();
  A.cta_part = part.as<double>();
  A.chunk_part = chunk.as<double>();
  A.long_cnt = lcnt.as<unsigned int>();
  A.long_part = lpart.as<double>();
  A.st = stb.as<PrState>();
  A.teleport = tele_ptr;
  A.damping = damping;
  A.n_f = (double)g->n_live;
  A.tol = tol;
  A.max_iter = max_iter;

  EventTimer tm;
  ZOGCU_TRY(tm.start(s));
  pr_init_kernel<OffT, double><<<grid, kPrThreads, 0, s>>>(A, V, given);
  ZOGCU_CUDA(cudaGetLastError());
  uint64_t launches = 1;
  for (uint64_t k = 0; k < max_iter; ++k) {
    pr_iter_kernel<OffT, double><<<grid, kPrThreads, 0, s>>>(A);
    ++launches;
  }
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_TRY(tm.stop(s));
  PrState hs;
  ZOGCU_CUDA(cudaMemcpyAsync(&hs, stb.ptr, sizeof(PrState), cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  const double* result = (hs.iter & 1ull) ? A.x1 : A.x0;
  ZOGCU_CUDA(cudaMemcpyAsync(out, result, (size_t)V * 8, dev_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  if (stats) {
    stats->iterations = hs.iter;
    stats->residual = hs.l1;
    stats->elapsed_ms = tm.ms();
    const double per_iter = 4.0 * (double)g->E + (double)sizeof(OffT) * ((double)V + 1) + 36.0 * (double)V;
    stats->bytes_moved = per_iter * (double)hs.iter;
    stats->launches = launches;
    stats->polish_iterations = 0;
  }
  return ZOGCU_OK;
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
  ZOGCU_TRY(ensure_pr_schedule(g, sg.s));
  if (g->offsets32)
    return run_pagerank_fp64<uint32_t>(g, g->in_off32.as<uint32_t>(), damping, max_iterations, tolerance, opts,
                                       out_scores, stats, sg.s);
  return run_pagerank_fp64<uint64_t>(g, g->in_off64.as<uint64_t>(), damping, max_iterations, tolerance, opts,
                                     out_scores, stats, sg.s);
}

int zogcu_pagerank(zogcu_graph* G, double damping, uint64_t max_iterations, double tolerance, double* out_scores,
                   zogcu_stats* stats) {
  return zogcu_pagerank_ex(G, damping, max_iterations, tolerance, nullptr, out_scores, stats);
}

}  // extern "C"
