// noalloc.cu -- PageRank for callers that cannot allocate device memory.
//
// Some callers of this library can't call cudaMalloc or any allocating
// routine: code that runs inside another runtime's memory budget, a host
// process whose allocator is owned by someone else (a BEAM NIF sharing a GPU
// with a framework that reserves the device pool up front), or a caller that
// must not allocate between two pre-planned phases.  zogcu_pagerank_noalloc
// serves them: the caller owns every input and output buffer, and the
// iteration's scratch (two rank vectors, two contribution vectors, CTA
// partials and the convergence state) lives in one file-scope device array of
// about 8 MiB that stays reserved until the process exits.
//
// Contract:
//   * at most kNoAllocMaxNodes nodes; larger graphs get ZOGCU_ERR_TOO_LARGE;
//   * no cudaMalloc / cudaMallocAsync / cudaFree, no stream or event creation,
//     no allocating library call -- only kernel launches, memsets and copies
//     on the caller's stream (NULL = the legacy default stream);
//   * the first call on a device does the set-up, with that device current:
//     it looks up the array's device address with cudaGetSymbolAddress (cached
//     per device) and loads this file's kernels.  CUDA loads modules lazily
//     by default, so that first call is when the array and the kernels' code
//     take their device memory: make it before another runtime takes the
//     device's memory, and before any stream capture;
//   * the iterations are enqueued in chunks of kNaChunk launches; after each
//     chunk the call reads the chain's state back (a small copy and a stream
//     synchronisation) and stops once the chain has converged or reached
//     max_iterations, so any cap, UINT64_MAX included, costs only the
//     iterations actually run plus at most one partial chunk;
//   * all calls share the one array, and it keeps the last call's contents:
//     the state each call needs zeroed is cleared at its start, and two calls
//     whose work overlaps on the GPU (different streams, or host threads
//     calling at once) race on it -- serialise them.
//
// The iteration is the reference's (priv/zog/src/centrality.zig:924-958) with
// every node live, computed one warp per row over the caller's in-CSR.
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"

namespace zogcu {
namespace {

constexpr uint32_t kNoAllocMaxNodes = 1u << 18;  // 262,144 nodes
constexpr int kNaThreads = 256;
constexpr int kNaMaxCtas = 1184;                 // partial slots (148 SMs x 8)
constexpr size_t kNaStateBytes = 256;
constexpr size_t kNaPartBytes = (size_t)kNaMaxCtas * 16;
constexpr size_t kNaVecBytes = (size_t)kNoAllocMaxNodes * 8;
constexpr size_t kNaScratchBytes = kNaStateBytes + kNaPartBytes + 4 * kNaVecBytes;  // ~8 MiB
constexpr uint64_t kNaChunk = 32;                // iteration launches between state reads

// The scratch array.  In host code its name is only a stand-in: kernels get
// the device address that cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaScratchBytes];

struct NaState {
  unsigned long long iter;
  double sink;
  double l1;
  int converged;
  unsigned int done_ctas;
};

struct NaArgs {
  const uint32_t* off;
  const uint32_t* col;
  const uint32_t* deg;
  uint32_t V;
  double damping, n_f, tol;
  unsigned long long max_iter;
  NaState* st;
  double* part;
  double* x0;
  double* x1;
  double* c0;
  double* c1;
};

__device__ __forceinline__ double na_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic CTA sum of two doubles, then the last CTA folds the per-CTA
// slots in order and publishes the result.
__device__ void na_publish(const NaArgs& A, double l1, double ds, unsigned long long next_iter, bool set_l1) {
  __shared__ double s_red[2 * (kNaThreads / 32)];
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  l1 = na_warp_sum(l1);
  ds = na_warp_sum(ds);
  if (lane == 0) {
    s_red[2 * warp] = l1;
    s_red[2 * warp + 1] = ds;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < kNaThreads / 32; ++w) {
      a += s_red[2 * w];
      b += s_red[2 * w + 1];
    }
    A.part[2 * blockIdx.x] = a;
    A.part[2 * blockIdx.x + 1] = b;
    __threadfence();
    s_last = (atomicAdd(&A.st->done_ctas, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    double a = 0.0, b = 0.0;
    for (uint32_t i = 0; i < gridDim.x; ++i) {
      a += __ldcg(A.part + 2 * i);
      b += __ldcg(A.part + 2 * i + 1);
    }
    A.st->sink = b;
    A.st->l1 = set_l1 ? a : 0.0;
    A.st->converged = (set_l1 && a < A.tol) ? 1 : 0;
    A.st->iter = next_iter;
    __threadfence();
    A.st->done_ctas = 0;
  }
}

__global__ void __launch_bounds__(kNaThreads) na_init_kernel(NaArgs A) {
  double ds = 0.0;
  const double x = 1.0 / A.n_f;  // uniform start (centrality.zig:912-918)
  for (uint32_t v = blockIdx.x * kNaThreads + threadIdx.x; v < A.V; v += gridDim.x * kNaThreads) {
    const uint32_t d = A.deg[v];
    A.x0[v] = x;
    A.x1[v] = 0.0;
    if (d == 0) ds += __ddiv_rn(x, A.n_f);
    else A.c0[v] = __ddiv_rn(x, (double)d);
  }
  na_publish(A, 0.0, ds, 0ull, false);
}

__global__ void __launch_bounds__(kNaThreads) na_iter_kernel(NaArgs A) {
  const unsigned long long iter = *(volatile unsigned long long*)&A.st->iter;
  if (*(volatile int*)&A.st->converged || iter >= A.max_iter) return;
  const double sink = *(volatile double*)&A.st->sink;
  const bool odd = iter & 1ull;
  const double* xc = odd ? A.x1 : A.x0;
  double* xn_out = odd ? A.x0 : A.x1;
  const double* cc = odd ? A.c1 : A.c0;
  double* cn = odd ? A.c0 : A.c1;
  const double tele = (1.0 - A.damping) / A.n_f;
  const int lane = threadIdx.x & 31;
  double l1 = 0.0, ds = 0.0;
  const uint32_t nw = gridDim.x * (kNaThreads / 32);
  for (uint32_t v = blockIdx.x * (kNaThreads / 32) + (threadIdx.x >> 5); v < A.V; v += nw) {
    const uint32_t b = A.off[v], e = A.off[v + 1];
    double s = 0.0;
    for (uint32_t j = b + lane; j < e; j += 32) s += cc[A.col[j]];
    s = na_warp_sum(s);
    if (lane == 0) {
      const double x = __dadd_rn(tele, __dmul_rn(A.damping, __dadd_rn(sink, s)));
      l1 += fabs(x - xc[v]);
      xn_out[v] = x;
      const uint32_t d = A.deg[v];
      if (d == 0) ds += __ddiv_rn(x, A.n_f);
      else cn[v] = __ddiv_rn(x, (double)d);
    }
  }
  na_publish(A, l1, ds, iter + 1, true);
}

// Copies the last iterate (chosen on the device by the iteration count) to
// the caller's output.
__global__ void na_copy_out(NaArgs A, double* out) {
  const bool odd = (*(volatile unsigned long long*)&A.st->iter) & 1ull;
  const double* x = odd ? A.x1 : A.x0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < A.V; v += gridDim.x * blockDim.x) out[v] = x[v];
}

std::mutex g_na_mu;
void* g_na_ptr[64] = {};  // device address of the scratch array, per device

}  // namespace
}  // namespace zogcu

using namespace zogcu;

extern "C" int zogcu_pagerank_noalloc(const uint32_t* d_in_off, const uint32_t* d_in_col,
                                      const uint32_t* d_out_degree, uint32_t num_nodes, uint64_t num_arcs,
                                      double damping, uint64_t max_iterations, double tolerance,
                                      double* d_out_scores, zogcu_stats* stats, void* stream) {
  if (num_nodes > kNoAllocMaxNodes)
    return fail(ZOGCU_ERR_TOO_LARGE, "zogcu_pagerank_noalloc handles at most " + std::to_string(kNoAllocMaxNodes) +
                                         " nodes; got " + std::to_string(num_nodes));
  if (num_arcs >= 0xFFFFFFFFull) return fail(ZOGCU_ERR_TOO_LARGE, "arc count exceeds u32 offsets");
  if (num_nodes && (!d_in_off || !d_out_degree || !d_out_scores))
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null device pointer");
  if (num_arcs && !d_in_col) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null in_col");
  if (stats) std::memset(stats, 0, sizeof(*stats));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (num_nodes == 0) return ZOGCU_OK;
  int dev = 0;
  ZOGCU_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(ZOGCU_ERR_NO_DEVICE, "device ordinal out of range");
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[dev]) {
      // once per device, with that device current: the array's device address,
      // and the kernels loaded now rather than at their first launch
      cudaFuncAttributes fa;
      ZOGCU_CUDA(cudaFuncGetAttributes(&fa, na_init_kernel));
      ZOGCU_CUDA(cudaFuncGetAttributes(&fa, na_iter_kernel));
      ZOGCU_CUDA(cudaFuncGetAttributes(&fa, na_copy_out));
      void* addr = nullptr;
      ZOGCU_CUDA(cudaGetSymbolAddress(&addr, g_noalloc_scratch));
      g_na_ptr[dev] = addr;
    }
    base = g_na_ptr[dev];
  }
  unsigned char* p = static_cast<unsigned char*>(base);
  NaArgs A;
  A.off = d_in_off;
  A.col = d_in_col;
  A.deg = d_out_degree;
  A.V = num_nodes;
  A.damping = damping;
  A.n_f = (double)num_nodes;
  A.tol = tolerance;
  A.max_iter = max_iterations;
  A.st = reinterpret_cast<NaState*>(p);
  A.part = reinterpret_cast<double*>(p + kNaStateBytes);
  A.x0 = reinterpret_cast<double*>(p + kNaStateBytes + kNaPartBytes);
  A.x1 = A.x0 + kNoAllocMaxNodes;
  A.c0 = A.x1 + kNoAllocMaxNodes;
  A.c1 = A.c0 + kNoAllocMaxNodes;

  if (num_nodes == 1) {  // centrality.zig:876-879
    const double one = 1.0;
    ZOGCU_CUDA(cudaMemcpyAsync(d_out_scores, &one, 8, cudaMemcpyHostToDevice, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    return ZOGCU_OK;
  }
  int grid = (int)std::min<uint32_t>((num_nodes + (kNaThreads / 32) - 1) / (kNaThreads / 32), kNaMaxCtas);
  if (grid < 1) grid = 1;
  ZOGCU_CUDA(cudaMemsetAsync(A.st, 0, kNaStateBytes, s));  // iteration state starts at zero
  na_init_kernel<<<grid, kNaThreads, 0, s>>>(A);
  ZOGCU_CUDA(cudaGetLastError());
  uint64_t launches = 1;
  NaState hs;
  std::memset(&hs, 0, sizeof(hs));
  // Chunks of iteration launches; a launch after the chain is over returns at
  // once, and the chain's state read after each chunk ends the loop.
  for (uint64_t queued = 0; queued < max_iterations;) {
    const uint64_t k = std::min<uint64_t>(kNaChunk, max_iterations - queued);
    for (uint64_t i = 0; i < k; ++i) na_iter_kernel<<<grid, kNaThreads, 0, s>>>(A);
    ZOGCU_CUDA(cudaGetLastError());
    queued += k;
    launches += k;
    ZOGCU_CUDA(cudaMemcpyAsync(&hs, A.st, sizeof(NaState), cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    if (hs.converged || hs.iter >= max_iterations) break;
  }
  na_copy_out<<<grid, kNaThreads, 0, s>>>(A, d_out_scores);
  ZOGCU_CUDA(cudaGetLastError());
  ++launches;
  ZOGCU_CUDA(cudaMemcpyAsync(&hs, A.st, sizeof(NaState), cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  if (stats) {
    stats->iterations = hs.iter;
    stats->residual = hs.l1;
    stats->launches = launches;
  }
  return ZOGCU_OK;
}
