// graph.cu -- device-resident graph resource: CSR construction, the seeded
// R-MAT generator, the edge-list reader front end, and the ABI entry points
// that create, inspect and destroy a graph.
//
// The reference keeps an ArrayGraph (per-node singly linked out-edge lists with
// head insertion, priv/zog/src/models/array_graph.zig:88-108) inside a BEAM
// resource and rebuilds in_neighbors / out_degrees on every PageRank call
// (centrality.zig:881-910).  Here the equivalent CSRs are built once on the
// device with two stable radix sorts and stay resident:
//   out-CSR  rows = successors in SuccessorIterator order (reverse insertion)
//   in-CSR   rows = sources ascending, duplicates adjacent -- exactly the
//            in_neighbors lists of centrality.zig:893-899
//   out_deg  successor counts (centrality.zig:901-910)
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <unordered_map>

#include "common.cuh"
#include "runs.h"

namespace zogcu {

// ---------------------------------------------------------------------------
// errors, small RAII helpers
// ---------------------------------------------------------------------------
static thread_local std::string t_last_error;

void set_error(const std::string& msg) { t_last_error = msg; }
int fail(int status, const std::string& msg) {
  t_last_error = msg;
  return status;
}

int DevBuf::alloc(size_t n, cudaStream_t s) {
  release();
  stream = s;
  bytes = n;
  if (n == 0) return ZOGCU_OK;
  cudaError_t e = cudaMallocAsync(&ptr, n, s);
  if (e != cudaSuccess) {
    ptr = nullptr;
    return fail(ZOGCU_ERR_OUT_OF_MEMORY, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
  }
  return ZOGCU_OK;
}
void DevBuf::release() {
  if (ptr && owned) cudaFreeAsync(ptr, stream);
  ptr = nullptr;
  bytes = 0;
  owned = true;
}

// Persistent arrays come from the device's stream-ordered pool as well, so
// creating and destroying graphs reuses reserved memory instead of mapping
// and unmapping pages (about 1 ms per GB each way).  The allocation has
// completed before the array is handed out, so any stream may use it.
int DevArray::alloc(size_t n) {
  release();
  bytes = n;
  if (n == 0) return ZOGCU_OK;
  cudaError_t e = cudaMallocAsync(&ptr, n, cudaStreamPerThread);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
  if (e != cudaSuccess) {
    if (ptr) cudaFreeAsync(ptr, cudaStreamPerThread);
    ptr = nullptr;
    bytes = 0;
    return fail(ZOGCU_ERR_OUT_OF_MEMORY, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
  }
  return ZOGCU_OK;
}
void DevArray::release() {
  if (ptr) {
    // as cudaFree does, wait for work in flight that may still read the array
    cudaDeviceSynchronize();
    cudaFreeAsync(ptr, cudaStreamPerThread);
  }
  ptr = nullptr;
  bytes = 0;
}

int StreamGuard::init(void* user) {
  if (user) {
    s = static_cast<cudaStream_t>(user);
    owned = false;
    return ZOGCU_OK;
  }
  ZOGCU_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  owned = true;
  return ZOGCU_OK;
}
StreamGuard::~StreamGuard() {
  if (owned && s) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
}

int EventTimer::start(cudaStream_t s) {
  if (!a) ZOGCU_CUDA(cudaEventCreate(&a));
  if (!b) ZOGCU_CUDA(cudaEventCreate(&b));
  ZOGCU_CUDA(cudaEventRecord(a, s));
  return ZOGCU_OK;
}
int EventTimer::stop(cudaStream_t s) {
  ZOGCU_CUDA(cudaEventRecord(b, s));
  return ZOGCU_OK;
}
float EventTimer::ms() {
  float t = 0.f;
  if (a && b && cudaEventSynchronize(b) == cudaSuccess) cudaEventElapsedTime(&t, a, b);
  return t;
}
EventTimer::~EventTimer() {
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
}

// ---------------------------------------------------------------------------
// host <-> device copies of caller arrays that may be pageable
// ---------------------------------------------------------------------------
// A NIF hands over slices from the BEAM's allocator: pageable memory.  The
// driver copies pageable memory through its own small staging buffers, one
// copy at a time.  Here a pageable range is cut into kCopyThreads contiguous
// parts, and each part is copied by its own host thread through two
// library-owned pinned chunks of kBounceBytes on its own stream: while the DMA
// engine moves one chunk, the thread fills the other, and the parts' DMAs
// queue back to back on the link.  The pinned chunks, the helper streams and
// one event per chunk are created on a device's first call and kept (one call
// at a time uses them; a concurrent call copies directly).  A call never
// drains the helpers: a chunk is refilled once the event of its last DMA has
// fired, in this call or an earlier one, so calls in a row (the chunked
// upload makes sixteen) keep the link busy.  Pinned caller memory is copied
// directly.
constexpr int kCopyThreads = 16;
constexpr size_t kBounceBytes = 16u << 20;
constexpr int kMaxCopyDevices = 16;

struct BounceSet {
  void* buf[2 * kCopyThreads] = {};
  cudaEvent_t done[2 * kCopyThreads] = {};  // the last DMA through buf[i]
  bool used[2 * kCopyThreads] = {};         // done[i] has been recorded
  cudaStream_t st[kCopyThreads] = {};
  cudaEvent_t tail[kCopyThreads] = {};      // end of a call's work on st[t]
  cudaEvent_t start = nullptr;
  bool ready = false;
};
static std::mutex g_bounce_mu;
static BounceSet g_bounce[kMaxCopyDevices];

static bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the error of an unknown pointer
    return false;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

static int bounce_setup(BounceSet& B) {
  if (B.ready) return ZOGCU_OK;
  for (void*& b : B.buf)
    if (!b) ZOGCU_CUDA(cudaHostAlloc(&b, kBounceBytes, cudaHostAllocPortable));
  for (cudaEvent_t& e : B.done)
    if (!e) ZOGCU_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (cudaEvent_t& e : B.tail)
    if (!e) ZOGCU_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (cudaStream_t& t : B.st)
    if (!t) ZOGCU_CUDA(cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
  if (!B.start) ZOGCU_CUDA(cudaEventCreateWithFlags(&B.start, cudaEventDisableTiming));
  B.ready = true;
  return ZOGCU_OK;
}

// Copies `bytes` between host memory `host` and device memory `dev` (h2d:
// host -> device) ordered after the work already on stream s; the copy is
// ordered before later work on s (s waits for the helper streams).
int copy_host(void* dev, void* host, size_t bytes, bool h2d, cudaStream_t s) {
  if (bytes == 0) return ZOGCU_OK;
  const cudaMemcpyKind kind = h2d ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  int device = 0;
  ZOGCU_CUDA(cudaGetDevice(&device));
  std::unique_lock<std::mutex> lk(g_bounce_mu, std::try_to_lock);
  if (bytes < 2 * kBounceBytes || device >= kMaxCopyDevices || is_pinned(host) || !lk.owns_lock()) {
    ZOGCU_CUDA(h2d ? cudaMemcpyAsync(dev, host, bytes, kind, s) : cudaMemcpyAsync(host, dev, bytes, kind, s));
    return ZOGCU_OK;
  }
  BounceSet& B = g_bounce[device];
  ZOGCU_TRY(bounce_setup(B));
  ZOGCU_CUDA(cudaEventRecord(B.start, s));
  for (int t = 0; t < kCopyThreads; ++t) ZOGCU_CUDA(cudaStreamWaitEvent(B.st[t], B.start, 0));
  std::atomic<int> err{0};
  {
    std::vector<std::thread> th;
    const size_t part = (bytes / kCopyThreads + 15) & ~(size_t)15;
    for (int t = 0; t < kCopyThreads; ++t) {
      const size_t lo = std::min(bytes, part * t), hi = std::min(bytes, part * (t + 1));
      auto copy_part = [&, t, lo, hi] {
        char* hb = static_cast<char*>(host);
        char* db = static_cast<char*>(dev);
        int k = 0;
        for (size_t o = lo; o < hi; o += kBounceBytes, ++k) {
          const size_t n = std::min(kBounceBytes, hi - o);
          const int i = 2 * t + (k & 1);
          // the chunk is free once its last DMA (this call's or an earlier one's) finished
          if (B.used[i] && cudaEventSynchronize(B.done[i]) != cudaSuccess) { err = 1; return; }
          if (h2d) {
            std::memcpy(B.buf[i], hb + o, n);
            if (cudaMemcpyAsync(db + o, B.buf[i], n, kind, B.st[t]) != cudaSuccess ||
                cudaEventRecord(B.done[i], B.st[t]) != cudaSuccess) { err = 1; return; }
            B.used[i] = true;
          } else {
            if (cudaMemcpyAsync(B.buf[i], db + o, n, kind, B.st[t]) != cudaSuccess ||
                cudaEventRecord(B.done[i], B.st[t]) != cudaSuccess ||
                cudaEventSynchronize(B.done[i]) != cudaSuccess) { err = 1; return; }
            B.used[i] = true;
            std::memcpy(hb + o, B.buf[i], n);
          }
        }
      };
      try {
        th.emplace_back(copy_part);
      } catch (...) {  // no thread to be had: this part on the calling thread
        copy_part();
      }
    }
    for (auto& x : th) x.join();
  }
  // later work on s follows every helper's copies, without a host wait
  for (int t = 0; t < kCopyThreads; ++t) {
    ZOGCU_CUDA(cudaEventRecord(B.tail[t], B.st[t]));
    ZOGCU_CUDA(cudaStreamWaitEvent(s, B.tail[t], 0));
  }
  if (err) return fail(ZOGCU_ERR_CUDA, "pipelined host copy failed");
  return ZOGCU_OK;
}

// SM count of the first device queried (every device of a B200 node has the
// same count); concurrent first calls store the same value.
static std::atomic<int> g_sm_count{0};
int sm_count() {
  int n = g_sm_count.load(std::memory_order_relaxed);
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    g_sm_count.store(n, std::memory_order_relaxed);
  }
  return n;
}

int ensure_device(int* dev) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(ZOGCU_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  ZOGCU_CUDA(cudaGetDevice(dev));
  int major = 0;
  ZOGCU_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, *dev));
  if (major != 10)
    return fail(ZOGCU_ERR_NO_DEVICE, "libzogcu is built for sm_100a (B200); device has compute capability major " +
                                         std::to_string(major));
  // Keep freed stream-ordered memory in the pool instead of returning it to
  // the driver at every synchronisation (per-process setting).
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, *dev) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  return ZOGCU_OK;
}

static int bits_for(uint64_t v) {  // bits needed for values in [0, v)
  int b = 1;
  while (b < 64 && (1ull << b) < v) ++b;
  return b;
}

// ---------------------------------------------------------------------------
// CSR construction kernels
// ---------------------------------------------------------------------------
__global__ void k_reverse_copy(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst,
                               uint32_t* __restrict__ ksrc, uint32_t* __restrict__ vdst, uint64_t E,
                               int reverse) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t j = reverse ? (E - 1 - i) : i;
    ksrc[i] = src[j];
    vdst[i] = dst[j];
  }
}

__global__ void k_reverse_copy_u64(const unsigned long long* __restrict__ w, unsigned long long* __restrict__ out,
                                   uint64_t E, int reverse) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = w[reverse ? (E - 1 - i) : i];
}

// flags[0]: an endpoint is >= V; flags[1]: the sources are not in
// non-decreasing order (the sorted-input fast path of the CSR build is off)
__global__ void k_validate(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint64_t E,
                           uint32_t V, unsigned int* flags) {
  bool bad = false, unsorted = false;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t ai = a[i];
    bad |= ai >= V || b[i] >= V;
    unsorted |= i + 1 < E && a[i + 1] < ai;
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flags, 1u);
  if (__any_sync(0xffffffffu, unsorted) && (threadIdx.x & 31) == 0) atomicOr(flags + 1, 1u);
}

// One chunk's destination counts -> prefixes: cnt[d] becomes the arcs into d
// in earlier chunks (total[d] before this chunk), and total[d] adds the count.
__global__ void k_running_prefix(uint32_t* __restrict__ cnt, unsigned long long* __restrict__ total, uint64_t n) {
  for (uint64_t d = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; d < n; d += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t x = cnt[d];
    const unsigned long long t = total[d];
    cnt[d] = (uint32_t)t;
    total[d] = t + x;
  }
}

// In-CSR from per-chunk sorted runs: the j-th pair of chunk c's run with
// destination d goes to in_off[d] + (arcs into d in earlier chunks) + j.  Each
// row thus lists its chunks in chunk order, and each chunk's arcs in arc
// order.  A CTA takes a slice of kMergeSlice positions of in_col, finds the
// rows at its two ends, and copies from each chunk the contiguous part of the
// run that lands in the slice: all chunks' writes to the slice come from one
// CTA close together (they merge in L2), and hub rows are shared out by
// position, so every CTA copies the same number of arcs.
constexpr uint64_t kMergeSlice = 4096;

// a run entry: read once, so it neither stays in L1 nor displaces the slices'
// partly written in_col lines in L2
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* a, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
  return v;
}

// the row holding in_col position pos < E: the last r with in_off[r] <= pos
__device__ __forceinline__ uint32_t row_of(const uint64_t* __restrict__ in_off, uint32_t V, uint64_t pos) {
  uint32_t lo = 0, hi = V;  // in_off[lo] <= pos < in_off[hi] = E
  while (hi - lo > 1) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (__ldg(in_off + mid) <= pos) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void k_merge_runs(ChunkRuns R, uint32_t V, const uint64_t* __restrict__ in_off,
                             uint32_t* __restrict__ in_col) {
  const uint64_t stride = (uint64_t)V + 1, E = R.bound[R.chunks];
  const uint64_t nslices = (E + kMergeSlice - 1) / kMergeSlice;
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  __shared__ uint32_t s_rows[2];
  for (uint64_t sl = blockIdx.x; sl < nslices; sl += gridDim.x) {
    const uint64_t p0 = sl * kMergeSlice, p1 = min(E, p0 + kMergeSlice);
    __syncthreads();  // s_rows of the previous slice are no longer read
    if (threadIdx.x == 0) s_rows[0] = row_of(in_off, V, p0);
    if (threadIdx.x == 32) s_rows[1] = row_of(in_off, V, p1 - 1);
    __syncthreads();
    const uint32_t ra = s_rows[0], rb = s_rows[1];
    for (int c = 0; c < R.chunks; ++c) {
      const uint32_t* __restrict__ st = R.start + c * stride;
      const uint32_t* __restrict__ pre = R.pre + c * stride;
      const uint64_t base = R.bound[c];
      // chunk c's arcs of rows ra..rb whose positions fall in [p0, p1)
      const uint64_t oa = __ldg(in_off + ra) + __ldg(pre + ra), ob = __ldg(in_off + rb) + __ldg(pre + rb);
      const uint32_t na = __ldg(st + ra + 1) - __ldg(st + ra), nb = __ldg(st + rb + 1) - __ldg(st + rb);
      const uint64_t ua = p0 > oa ? p0 - oa : 0, ub = p1 > ob ? p1 - ob : 0;
      const uint32_t ja = ua < na ? (uint32_t)ua : na, jb = ub < nb ? (uint32_t)ub : nb;
      const uint32_t q0 = __ldg(st + ra) + ja, q1 = __ldg(st + rb) + jb;
      for (uint32_t q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
        const uint32_t d = ld_stream(R.dst + base + q, pol);
        const uint32_t v = ld_stream(R.src + base + q, pol);
        in_col[__ldg(in_off + d) + __ldg(pre + d) + (q - __ldg(st + d))] = v;
      }
    }
  }
}

// Sorted-input out-CSR: input arc j of source r = src[j] goes to position
// off[r] + off[r+1] - 1 - j when each row is reversed (ArrayGraph successor
// order is the reverse of insertion order), or stays at j otherwise.
__global__ void k_scatter_sorted(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst,
                                 const unsigned long long* __restrict__ w, const uint64_t* __restrict__ off,
                                 uint64_t E, int reverse, uint32_t* __restrict__ out_col,
                                 unsigned long long* __restrict__ out_w) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < E;
       j += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t p = j;
    if (reverse) {
      const uint32_t r = src[j];
      p = off[r] + off[r + 1] - 1 - j;
    }
    out_col[p] = dst[j];
    if (w) out_w[p] = w[j];
  }
}

// Per-row arc counts of SORTED keys: each warp reads 32 consecutive keys, and
// the first lane of every run of equal keys adds the run's length (a run that
// spans warps is added in parts), one atomic per run instead of per arc.
// cnt[k] += the number of keys equal to k, for keys below `limit` (runs of
// equal keys add once; larger keys, which validation rejects later, are skipped)
template <class C>
__global__ void k_histogram_sorted(const uint32_t* __restrict__ keys, uint64_t E, C* cnt, uint32_t limit) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t base = ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < E; base += nw * 32) {
    const uint64_t i = base + lane;
    const bool valid = i < E;
    const uint32_t k = valid ? keys[i] : 0u;
    const uint32_t kp = __shfl_up_sync(0xffffffffu, k, 1);
    const bool head = valid && (lane == 0 || k != kp);
    const unsigned hb = __ballot_sync(0xffffffffu, head);
    const uint32_t nvalid = (E - base < 32) ? (uint32_t)(E - base) : 32u;
    if (head && k < limit) {
      const unsigned above = lane < 31 ? (hb >> (lane + 1)) : 0u;
      const uint32_t next = above ? (uint32_t)(lane + __ffs(above)) : nvalid;
      atomicAdd(&cnt[k], (C)(next - lane));
    }
  }
}

__global__ void k_degrees(const uint64_t* __restrict__ off, const uint8_t* __restrict__ live, uint32_t V,
                          uint32_t* __restrict__ deg) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t d = (uint32_t)(off[v + 1] - off[v]);
    deg[v] = (live && !live[v]) ? kDeletedDegree : d;
  }
}

__global__ void k_off32(const uint64_t* __restrict__ a, uint32_t* __restrict__ b, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    b[i] = (uint32_t)a[i];
}

static unsigned grid_for(uint64_t n, unsigned block = 256) {
  uint64_t g = (n + block - 1) / block;
  uint64_t cap = (uint64_t)sm_count() * 32;
  if (g > cap) g = cap;
  if (g == 0) g = 1;
  return (unsigned)g;
}

// offsets (u64, V+1) from a per-row count histogram (u64, V)
static int counts_to_offsets(unsigned long long* d_cnt, uint64_t* d_off, uint32_t V, cudaStream_t s) {
  // exclusive scan over V+1 entries (the histogram has a trailing zero slot)
  size_t tmp = 0;
  ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_cnt, (unsigned long long*)d_off,
                                           (int64_t)V + 1, s));
  DevBuf t;
  ZOGCU_TRY(t.alloc(tmp, s));
  ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(t.ptr, tmp, d_cnt, (unsigned long long*)d_off,
                                           (int64_t)V + 1, s));
  return ZOGCU_OK;
}

int build_graph_from_device_edges(Graph* g, uint32_t V, const uint32_t* d_src, const uint32_t* d_dst,
                                  uint64_t E, bool reverse_within_source, const uint8_t* h_node_deleted,
                                  cudaStream_t s, const double* d_w, int src_sorted, ChunkRuns* runs) {
  ZOGCU_TRY(ensure_device(&g->device));
  g->V = V;
  g->E = E;
  g->offsets32 = E < 0xFFFFFFF0ull;
  g->has_deleted = false;
  uint64_t live = V;
  if (h_node_deleted) {
    live = 0;
    for (uint32_t v = 0; v < V; ++v) {
      if (h_node_deleted[v]) g->has_deleted = true;
      else ++live;
    }
  }
  g->n_live = live;

  const size_t colBytes = (E + 4) * sizeof(uint32_t);
  ZOGCU_TRY(g->in_col.alloc(colBytes));
  ZOGCU_TRY(g->out_col.alloc(colBytes));
  ZOGCU_TRY(g->in_off64.alloc((size_t)(V + 1) * 8));
  ZOGCU_TRY(g->out_off64.alloc((size_t)(V + 1) * 8));
  ZOGCU_TRY(g->out_deg.alloc((size_t)std::max<uint32_t>(V, 1) * 4));
  // the 4 padding entries after the arcs (16-byte loads read them) are zero
  ZOGCU_CUDA(cudaMemsetAsync(g->in_col.as<uint32_t>() + E, 0, 4 * sizeof(uint32_t), s));
  ZOGCU_CUDA(cudaMemsetAsync(g->out_col.as<uint32_t>() + E, 0, 4 * sizeof(uint32_t), s));
  if (g->has_deleted) {
    ZOGCU_TRY(g->live.alloc(V));
    std::vector<uint8_t> lv(V);
    for (uint32_t v = 0; v < V; ++v) lv[v] = h_node_deleted[v] ? 0 : 1;
    ZOGCU_CUDA(cudaMemcpyAsync(g->live.ptr, lv.data(), V, cudaMemcpyHostToDevice, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
  }

  DevBuf cnt;
  ZOGCU_TRY(cnt.alloc((size_t)(V + 1) * 8, s));
  PhaseTrace tr("csr_build", s);
  if (E > 0) {
    const int bits = bits_for(V);
    bool sorted = src_sorted > 0;
    if (src_sorted < 0) {  // find out: one pass over the sources
      DevBuf fl;
      ZOGCU_TRY(fl.alloc(8, s));
      ZOGCU_CUDA(cudaMemsetAsync(fl.ptr, 0, 8, s));
      k_validate<<<grid_for(E), 256, 0, s>>>(d_src, d_src, E, 0xFFFFFFFFu, fl.as<unsigned int>());
      ZOGCU_CUDA(cudaGetLastError());
      unsigned int h[2] = {0, 0};
      ZOGCU_CUDA(cudaMemcpyAsync(h, fl.ptr, 8, cudaMemcpyDeviceToHost, s));
      ZOGCU_CUDA(cudaStreamSynchronize(s));
      sorted = h[1] == 0;
    }
    DevBuf ks, vs, ks2, t;
    size_t tmp = 0;
    const bool merge_runs = sorted && runs && runs->chunks > 0 && !d_w;
    if (!merge_runs) ZOGCU_TRY(ks.alloc(E * 4, s));
    const uint32_t* keys_out;  // the source of every out-CSR arc (rows ascending)
    if (sorted) {
      // Sources already non-decreasing: the out offsets come straight from
      // them, and one scatter places each row (reversed for insertion order).
      if (merge_runs) {  // counted chunk by chunk during the upload
        ZOGCU_TRY(counts_to_offsets(runs->out_cnt, g->out_off64.as<uint64_t>(), V, s));
      } else {
        ZOGCU_CUDA(cudaMemsetAsync(cnt.ptr, 0, (size_t)(V + 1) * 8, s));
        k_histogram_sorted<<<grid_for(E), 256, 0, s>>>(d_src, E, cnt.as<unsigned long long>(), V);
        ZOGCU_CUDA(cudaGetLastError());
        ZOGCU_TRY(counts_to_offsets(cnt.as<unsigned long long>(), g->out_off64.as<uint64_t>(), V, s));
      }
      if (d_w) {
        ZOGCU_TRY(g->out_w.alloc(E * 8));
        g->weighted = true;
      }
      k_scatter_sorted<<<grid_for(E), 256, 0, s>>>(d_src, d_dst, reinterpret_cast<const unsigned long long*>(d_w),
                                                   g->out_off64.as<uint64_t>(), E, reverse_within_source ? 1 : 0,
                                                   g->out_col.as<uint32_t>(), g->out_w.as<unsigned long long>());
      ZOGCU_CUDA(cudaGetLastError());
      keys_out = d_src;  // rows are contiguous, so the sources stay in place
    } else {
      ZOGCU_TRY(vs.alloc(E * 4, s));
      ZOGCU_TRY(ks2.alloc(E * 4, s));
      k_reverse_copy<<<grid_for(E), 256, 0, s>>>(d_src, d_dst, ks.as<uint32_t>(), vs.as<uint32_t>(), E,
                                                 reverse_within_source ? 1 : 0);
      ZOGCU_CUDA(cudaGetLastError());
      // (1) stable sort by source: rows in successor order -> out-CSR
      ZOGCU_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ks.as<uint32_t>(), ks2.as<uint32_t>(),
                                                 vs.as<uint32_t>(), g->out_col.as<uint32_t>(), (int64_t)E,
                                                 0, bits, s));
      ZOGCU_TRY(t.alloc(tmp, s));
      ZOGCU_CUDA(cub::DeviceRadixSort::SortPairs(t.ptr, tmp, ks.as<uint32_t>(), ks2.as<uint32_t>(),
                                                 vs.as<uint32_t>(), g->out_col.as<uint32_t>(), (int64_t)E,
                                                 0, bits, s));
      if (d_w) {
        // the same stable sort of the same keys carries the weights along
        DevBuf wr, kd;
        ZOGCU_TRY(wr.alloc(E * 8, s));
        ZOGCU_TRY(kd.alloc(E * 4, s));
        ZOGCU_TRY(g->out_w.alloc(E * 8));
        k_reverse_copy_u64<<<grid_for(E), 256, 0, s>>>(reinterpret_cast<const unsigned long long*>(d_w),
                                                       wr.as<unsigned long long>(), E, reverse_within_source ? 1 : 0);
        ZOGCU_CUDA(cudaGetLastError());
        size_t tmpw = 0;
        ZOGCU_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpw, ks.as<uint32_t>(), kd.as<uint32_t>(),
                                                   wr.as<unsigned long long>(), g->out_w.as<unsigned long long>(),
                                                   (int64_t)E, 0, bits, s));
        DevBuf tw;
        ZOGCU_TRY(tw.alloc(tmpw, s));
        ZOGCU_CUDA(cub::DeviceRadixSort::SortPairs(tw.ptr, tmpw, ks.as<uint32_t>(), kd.as<uint32_t>(),
                                                   wr.as<unsigned long long>(), g->out_w.as<unsigned long long>(),
                                                   (int64_t)E, 0, bits, s));
        g->weighted = true;
      }
      // out offsets
      ZOGCU_CUDA(cudaMemsetAsync(cnt.ptr, 0, (size_t)(V + 1) * 8, s));
      k_histogram_sorted<<<grid_for(E), 256, 0, s>>>(ks2.as<uint32_t>(), E, cnt.as<unsigned long long>(), V);
      ZOGCU_CUDA(cudaGetLastError());
      ZOGCU_TRY(counts_to_offsets(cnt.as<unsigned long long>(), g->out_off64.as<uint64_t>(), V, s));
      keys_out = ks2.as<uint32_t>();
    }
    tr.mark(sorted ? "out-CSR (sorted sources)" : "out-CSR (radix sort)");
    if (merge_runs) {
      // (2') sources non-decreasing: each chunk's run lists a row's sources
      // ascending, and the chunks follow one another in source order, so the
      // in-CSR is every row's chunk segments placed in chunk order
      ZOGCU_TRY(counts_to_offsets(runs->total, g->in_off64.as<uint64_t>(), V, s));
      tr.mark("in offsets from the chunk counts");
      k_merge_runs<<<grid_for((E + kMergeSlice - 1) / kMergeSlice * 256), 256, 0, s>>>(
          *runs, V, g->in_off64.as<uint64_t>(), g->in_col.as<uint32_t>());
      ZOGCU_CUDA(cudaGetLastError());
      tr.mark("in-CSR merge of the chunk runs");
    } else {
      // (2) stable sort of (dst, src) pairs by dst: sources stay ascending
      size_t tmp2 = 0;
      ZOGCU_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp2, g->out_col.as<uint32_t>(), ks.as<uint32_t>(),
                                                 keys_out, g->in_col.as<uint32_t>(), (int64_t)E, 0, bits, s));
      if (tmp2 > tmp) {
        ZOGCU_TRY(t.alloc(tmp2, s));
        tmp = tmp2;
      }
      ZOGCU_CUDA(cub::DeviceRadixSort::SortPairs(t.ptr, tmp, g->out_col.as<uint32_t>(), ks.as<uint32_t>(),
                                                 keys_out, g->in_col.as<uint32_t>(), (int64_t)E, 0, bits, s));
      tr.mark("in-CSR radix sort");
      ZOGCU_CUDA(cudaMemsetAsync(cnt.ptr, 0, (size_t)(V + 1) * 8, s));
      k_histogram_sorted<<<grid_for(E), 256, 0, s>>>(ks.as<uint32_t>(), E, cnt.as<unsigned long long>(), V);
      ZOGCU_CUDA(cudaGetLastError());
      ZOGCU_TRY(counts_to_offsets(cnt.as<unsigned long long>(), g->in_off64.as<uint64_t>(), V, s));
    }
  } else {
    ZOGCU_CUDA(cudaMemsetAsync(g->in_off64.ptr, 0, (size_t)(V + 1) * 8, s));
    ZOGCU_CUDA(cudaMemsetAsync(g->out_off64.ptr, 0, (size_t)(V + 1) * 8, s));
  }
  if (V > 0) {
    k_degrees<<<grid_for(V), 256, 0, s>>>(g->out_off64.as<uint64_t>(), g->live.as<uint8_t>(), V,
                                          g->out_deg.as<uint32_t>());
    ZOGCU_CUDA(cudaGetLastError());
  }
  if (g->offsets32) {
    ZOGCU_TRY(g->in_off32.alloc((size_t)(V + 1) * 4));
    ZOGCU_TRY(g->out_off32.alloc((size_t)(V + 1) * 4));
    k_off32<<<grid_for(V + 1), 256, 0, s>>>(g->in_off64.as<uint64_t>(), g->in_off32.as<uint32_t>(), V + 1);
    k_off32<<<grid_for(V + 1), 256, 0, s>>>(g->out_off64.as<uint64_t>(), g->out_off32.as<uint32_t>(), V + 1);
    ZOGCU_CUDA(cudaGetLastError());
  }
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  tr.mark("in offsets, degrees, 32-bit offsets");
  return ZOGCU_OK;
}

// ---------------------------------------------------------------------------
// Seeded R-MAT generator (the same definition as the CPU oracle's):
//   key     = splitmix64(seed)
//   r(i,k)  = splitmix64(key ^ (i << 6 | k))   for level k of edge i
//   u       = r >> 11 compared with the integer thresholds floor(p * 2^53)
//   quadrant 0:(0,0) 1:(0,1) 2:(1,0) 3:(1,1) appended MSB first to (src, dst)
// SplitMix64: the public-domain mixer of Steele, Lea and Flood (2014).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Packs (src, dst) as src << scale | dst; undirected edges are canonicalised to
// (lo, hi).  Every self-loop maps to the all-ones key of 2*scale bits, which is
// itself the self-loop (V-1, V-1): after sort + unique it is the last key and
// is cut.
__global__ void k_rmat(uint64_t key, uint64_t M, int scale, uint64_t ta, uint64_t tab, uint64_t tabc,
                       int directed, uint64_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < M;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s = 0, d = 0;
    for (int k = 0; k < scale; ++k) {
      uint64_t u = splitmix64(key ^ ((i << 6) | (uint64_t)k)) >> 11;
      uint32_t q = u < ta ? 0u : (u < tab ? 1u : (u < tabc ? 2u : 3u));
      s = (s << 1) | (q >> 1);
      d = (d << 1) | (q & 1u);
    }
    if (!directed && s > d) {
      uint32_t t = s; s = d; d = t;
    }
    out[i] = (s == d) ? ((1ull << (2 * scale)) - 1) : (((uint64_t)s << scale) | d);
  }
}

__global__ void k_unpack(const uint64_t* __restrict__ keys, uint64_t m, int scale, int directed,
                         uint32_t* __restrict__ src, uint32_t* __restrict__ dst) {
  const uint64_t mask = (1ull << scale) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s = (uint32_t)(keys[i] >> scale), d = (uint32_t)(keys[i] & mask);
    if (directed) {
      src[i] = s; dst[i] = d;
    } else {
      src[2 * i] = s; dst[2 * i] = d;
      src[2 * i + 1] = d; dst[2 * i + 1] = s;
    }
  }
}

// raw endpoints of edges [i0, i0+m) -- lets tests compare with the CPU generator
__global__ void k_rmat_raw(uint64_t key, uint64_t i0, uint64_t m, int scale, uint64_t ta, uint64_t tab,
                           uint64_t tabc, uint32_t* src, uint32_t* dst) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < m;
       j += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = i0 + j;
    uint32_t s = 0, d = 0;
    for (int k = 0; k < scale; ++k) {
      uint64_t u = splitmix64(key ^ ((i << 6) | (uint64_t)k)) >> 11;
      uint32_t q = u < ta ? 0u : (u < tab ? 1u : (u < tabc ? 2u : 3u));
      s = (s << 1) | (q >> 1);
      d = (d << 1) | (q & 1u);
    }
    src[j] = s;
    dst[j] = d;
  }
}

static void rmat_thresholds(double a, double b, double c, uint64_t* ta, uint64_t* tab, uint64_t* tabc) {
  const double two53 = 9007199254740992.0;
  *ta = (uint64_t)std::floor(a * two53);
  *tab = (uint64_t)std::floor((a + b) * two53);
  *tabc = (uint64_t)std::floor((a + b + c) * two53);
}

struct EventGuard {
  cudaEvent_t e = nullptr;
  int init() {
    ZOGCU_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return ZOGCU_OK;
  }
  ~EventGuard() {
    if (e) cudaEventDestroy(e);
  }
};

// ---------------------------------------------------------------------------
// Sorted sources cross PCIe run-length encoded
// ---------------------------------------------------------------------------
// When a chunk's sources are non-decreasing (an ArrayGraph's arcs, most edge
// lists, the generators' output), the chunk is fixed by its source range
// [s0, s1] and the position where each of those sources' runs starts:
// s1 - s0 + 2 offsets, about 4 bytes per node instead of 4 bytes per arc.
// Host threads check the chunk and write the offsets in one pass over it, and
// the device expands them back into the chunk's source array.  A chunk that
// is not sorted, holds a source >= V, or whose offsets would take more than
// half its bytes is copied as it is.  ZOGCU_UPLOAD_RUNS=0 copies every chunk
// as it is.
constexpr double kLinkBytesPerSecond = 50e9;  // pinned host-to-device copies on PCIe Gen5 x16

struct RunCodes {
  uint32_t* host = nullptr;  // pinned; kept per device, grown on demand
  size_t cap = 0;            // entries
  cudaEvent_t done = nullptr;  // after the last copy out of `host`
  bool used = false;           // done has been recorded
};
static std::mutex g_runs_mu;
static RunCodes g_runs[kMaxCopyDevices];

static bool upload_runs_on() {
  const char* e = std::getenv("ZOGCU_UPLOAD_RUNS");
  return !(e && e[0] == '0');
}

// Inverse of encode_runs: out[off[j] .. off[j+1]) = s0 + j for j < runs, one
// warp per run (lanes write consecutive positions).
__global__ void k_expand_runs(const uint32_t* __restrict__ off, uint32_t runs, uint32_t s0, uint64_t n,
                              uint32_t* __restrict__ out) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t j = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; j < runs; j += nw) {
    const uint32_t a = off[j], b = min((uint64_t)off[j + 1], n);
    for (uint32_t i = a + lane; i < b; i += 32) out[i] = s0 + (uint32_t)j;
  }
}

// Arc lists from host memory of at least this many arcs are copied in
// kUploadChunks chunks, each sorted by destination while the next ones are
// still being copied.
constexpr uint64_t kChunkedMinArcs = 1ull << 22;
constexpr int kUploadChunks = 8;
static_assert(kUploadChunks <= kMaxUploadChunks, "chunk bound array");

// Copies the host arc arrays to d_from / d_to chunk by chunk on stream `up`
// and, on stream s as each chunk lands, sorts its (destination, source) pairs
// stably by destination and counts and scans its destinations (ChunkRuns).
// On return s is ordered after every copy.
static int upload_chunked(const uint32_t* from, const uint32_t* to, uint64_t E, uint32_t V, uint32_t* d_from,
                          uint32_t* d_to, cudaStream_t s, cudaStream_t up, ChunkRuns& R, DevBuf& dst, DevBuf& src,
                          DevBuf& cnt, DevBuf& start, DevBuf& total, DevBuf& out_cnt, DevBuf& flags) {
  const uint64_t stride = (uint64_t)V + 1;
  // The device sorts a chunk about nine times faster than PCIe delivers it,
  // so only the last chunk's work is exposed: it gets 1/64 of the arcs, and
  // the other chunks split the rest evenly.
  R.chunks = kUploadChunks;
  const uint64_t head = E - E / 64;
  for (int c = 0; c < kUploadChunks; ++c) R.bound[c] = head * (uint64_t)c / (kUploadChunks - 1);
  R.bound[kUploadChunks] = E;
  uint64_t longest = 0;
  for (int c = 0; c < kUploadChunks; ++c) longest = std::max(longest, R.bound[c + 1] - R.bound[c]);
  ZOGCU_TRY(dst.alloc(E * 4, s));
  ZOGCU_TRY(src.alloc(E * 4, s));
  ZOGCU_TRY(cnt.alloc(stride * kUploadChunks * 4, s));
  ZOGCU_TRY(start.alloc(stride * kUploadChunks * 4, s));
  ZOGCU_TRY(total.alloc(stride * 8, s));
  ZOGCU_TRY(out_cnt.alloc(stride * 8, s));
  ZOGCU_TRY(flags.alloc(8, s));
  ZOGCU_CUDA(cudaMemsetAsync(cnt.ptr, 0, stride * kUploadChunks * 4, s));
  ZOGCU_CUDA(cudaMemsetAsync(total.ptr, 0, stride * 8, s));
  ZOGCU_CUDA(cudaMemsetAsync(out_cnt.ptr, 0, stride * 8, s));
  ZOGCU_CUDA(cudaMemsetAsync(flags.ptr, 0, 8, s));
  const int bits = bits_for(V);
  size_t sort_bytes = 0, scan_bytes = 0;
  ZOGCU_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, d_to, dst.as<uint32_t>(), d_from,
                                             src.as<uint32_t>(), (int64_t)longest, 0, bits, s));
  ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, cnt.as<uint32_t>(), start.as<uint32_t>(),
                                           (int64_t)stride, s));
  DevBuf tmp;
  ZOGCU_TRY(tmp.alloc(std::max(sort_bytes, scan_bytes), s));
  // run-length encoded sources: the pinned offsets buffer of this device
  // (one call at a time; a concurrent call copies the sources as they are)
  int device = 0;
  ZOGCU_CUDA(cudaGetDevice(&device));
  std::unique_lock<std::mutex> rl(g_runs_mu, std::defer_lock);
  RunCodes* rc = nullptr;
  DevBuf d_runs;
  const size_t runs_cap = (size_t)V + 3 * kUploadChunks;
  if (upload_runs_on() && device < kMaxCopyDevices && rl.try_lock()) {
    RunCodes& r = g_runs[device];
    // an earlier call's copies out of the buffer have finished
    if (r.used && cudaEventSynchronize(r.done) != cudaSuccess) return fail(ZOGCU_ERR_CUDA, "run offsets copy failed");
    r.used = false;
    if (!r.done) ZOGCU_CUDA(cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming));
    if (r.cap < runs_cap) {
      if (r.host) cudaFreeHost(r.host);
      r.host = nullptr;
      r.cap = 0;
      if (cudaHostAlloc(reinterpret_cast<void**>(&r.host), runs_cap * 4, cudaHostAllocPortable) == cudaSuccess)
        r.cap = runs_cap;
      else
        cudaGetLastError();
    }
    if (r.cap >= runs_cap) {
      ZOGCU_TRY(d_runs.alloc(runs_cap * 4, s));
      rc = &r;
    }
  }
  // the copies start once the device arrays, allocated in stream order on s, exist
  EventGuard ready;
  ZOGCU_TRY(ready.init());
  ZOGCU_CUDA(cudaEventRecord(ready.e, s));
  ZOGCU_CUDA(cudaStreamWaitEvent(up, ready.e, 0));
  EventGuard landed[kUploadChunks];
  size_t runs_at = 0;
  const bool trace = std::getenv("ZOGCU_TRACE") != nullptr;
  bool code_more = true;  // later chunks may still be sent as run offsets
  for (int c = 0; c < kUploadChunks; ++c) {
    const uint64_t lo = R.bound[c], n = R.bound[c + 1] - lo;
    ZOGCU_TRY(landed[c].init());
    // the sources: their run offsets when sorted and at most half the bytes,
    // else as they are.  The check reads the chunk's sources on host threads
    // while the destinations are copied (for pageable memory, by the copy's
    // own host threads at the same time).
    bool coded = false;
    uint32_t s0 = 0, nruns = 0;
    uint64_t entries = 0;
    if (rc && code_more && n) {
      s0 = from[lo];
      const uint32_t s1 = from[lo + n - 1];
      entries = s1 >= s0 ? (uint64_t)(s1 - s0) + 2 : 0;
      if (!(entries && 2 * entries <= n && runs_at + entries <= rc->cap)) entries = 0;
    }
    {
      bool enc = false;
      double scan_ms = 0.0;
      const auto t0 = std::chrono::steady_clock::now();
      std::thread scanner;
      auto check = [&] {
        enc = encode_runs(from + lo, n, c > 0 ? (int64_t)from[lo - 1] : -1, V, rc->host + runs_at);
        scan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      };
      if (entries) {
        try {
          scanner = std::thread(check);
        } catch (...) {  // no thread to be had: check before the copy instead
          check();
        }
      }
      const int crc = copy_host(d_to + lo, const_cast<uint32_t*>(to + lo), n * 4, true, up);
      const double copy_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      if (scanner.joinable()) scanner.join();
      // The check pays while it ends before the sources sent as they are
      // would have: both arrays' time on the link for pinned memory, twice
      // the destinations' host copy for pageable memory.  When host threads
      // are short (a busy host), the later chunks go as they are.
      if (entries && scan_ms > std::max(2.0 * copy_ms, 1e3 * (double)(8 * n) / kLinkBytesPerSecond))
        code_more = false;
      if (trace)
        std::fprintf(stderr, "zogcu trace: upload chunk %d: %llu arcs, source check %.3f ms (%s), destination copy call %.3f ms\n",
                     c, (unsigned long long)n, scan_ms, enc ? "run offsets" : (entries ? "not sorted" : "sent as is"),
                     copy_ms);
      ZOGCU_TRY(crc);
      if (enc) {
        nruns = (uint32_t)(entries - 1);
        ZOGCU_CUDA(cudaMemcpyAsync(d_runs.as<uint32_t>() + runs_at, rc->host + runs_at, entries * 4,
                                   cudaMemcpyHostToDevice, up));
        ZOGCU_CUDA(cudaEventRecord(rc->done, up));
        rc->used = true;
        coded = true;
      }
    }
    if (!coded) ZOGCU_TRY(copy_host(d_from + lo, const_cast<uint32_t*>(from + lo), n * 4, true, up));
    ZOGCU_CUDA(cudaEventRecord(landed[c].e, up));
    ZOGCU_CUDA(cudaStreamWaitEvent(s, landed[c].e, 0));
    if (coded) {
      k_expand_runs<<<sm_count() * 8, 256, 0, s>>>(d_runs.as<uint32_t>() + runs_at, nruns, s0, n, d_from + lo);
      ZOGCU_CUDA(cudaGetLastError());
      runs_at += (size_t)nruns + 1;
    }
    // endpoints < V and sources non-decreasing, the pair across the previous
    // chunk's end included; arcs per source (used when they are sorted)
    const uint64_t back = c > 0 ? 1 : 0;
    k_validate<<<grid_for(n + back), 256, 0, s>>>(d_from + lo - back, d_to + lo - back, n + back, V,
                                                 flags.as<unsigned int>());
    k_histogram_sorted<<<grid_for(n), 256, 0, s>>>(d_from + lo, n, out_cnt.as<unsigned long long>(), V);
    ZOGCU_CUDA(cudaGetLastError());
    size_t b = sort_bytes;
    ZOGCU_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, b, d_to + lo, dst.as<uint32_t>() + lo, d_from + lo,
                                               src.as<uint32_t>() + lo, (int64_t)n, 0, bits, s));
    uint32_t* cc = cnt.as<uint32_t>() + c * stride;
    k_histogram_sorted<<<grid_for(n), 256, 0, s>>>(dst.as<uint32_t>() + lo, n, cc, V);
    ZOGCU_CUDA(cudaGetLastError());
    b = scan_bytes;
    ZOGCU_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, b, cc, start.as<uint32_t>() + c * stride, (int64_t)stride, s));
    k_running_prefix<<<grid_for(stride), 256, 0, s>>>(cc, total.as<unsigned long long>(), stride);
    ZOGCU_CUDA(cudaGetLastError());
  }
  R.dst = dst.as<uint32_t>();
  R.src = src.as<uint32_t>();
  R.pre = cnt.as<uint32_t>();
  R.start = start.as<uint32_t>();
  R.total = total.as<unsigned long long>();
  R.out_cnt = out_cnt.as<unsigned long long>();
  R.flags = flags.as<unsigned int>();
  return ZOGCU_OK;
}

// Validates device edge arrays (addEdge's hasNode check, array_graph.zig:88-89)
// and builds the graph on stream s.
static int create_from_device_edges_on(uint32_t node_count, const uint32_t* d_from, const uint32_t* d_to,
                                       uint64_t num_edges, cudaStream_t s, zogcu_graph** out,
                                       const double* d_w = nullptr, ChunkRuns* runs = nullptr) {
  int sorted = 0;
  if (num_edges) {
    DevBuf fl;
    const unsigned int* flags = runs ? runs->flags : nullptr;  // already checked chunk by chunk
    if (!flags) {
      ZOGCU_TRY(fl.alloc(8, s));
      ZOGCU_CUDA(cudaMemsetAsync(fl.ptr, 0, 8, s));
      k_validate<<<grid_for(num_edges), 256, 0, s>>>(d_from, d_to, num_edges, node_count, fl.as<unsigned int>());
      ZOGCU_CUDA(cudaGetLastError());
      flags = fl.as<unsigned int>();
    }
    unsigned int h[2] = {0, 0};
    ZOGCU_CUDA(cudaMemcpyAsync(h, flags, 8, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    if (h[0]) return fail(ZOGCU_ERR_NODE_NOT_FOUND, "edge endpoint >= node_count");
    sorted = h[1] == 0 ? 1 : 0;
  }
  std::unique_ptr<zogcu_graph> G(new (std::nothrow) zogcu_graph());
  if (!G) return fail(ZOGCU_ERR_OUT_OF_MEMORY, "host allocation failed");
  ZOGCU_TRY(build_graph_from_device_edges(&G->g, node_count, d_from, d_to, num_edges, true, nullptr, s, d_w,
                                          sorted, runs));
  *out = G.release();
  return ZOGCU_OK;
}

}  // namespace zogcu

using namespace zogcu;

// ---------------------------------------------------------------------------
// ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* zogcu_status_string(int status) {
  switch (status) {
    case ZOGCU_OK: return "ok";
    case ZOGCU_ERR_INVALID_ARGUMENT: return "invalid argument";
    case ZOGCU_ERR_NODE_NOT_FOUND: return "node not found";
    case ZOGCU_ERR_OUT_OF_MEMORY: return "out of memory";
    case ZOGCU_ERR_CUDA: return "CUDA error";
    case ZOGCU_ERR_NO_DEVICE: return "no usable device";
    case ZOGCU_ERR_TIMEOUT: return "device wait timed out";
    case ZOGCU_ERR_IO: return "I/O error";
    case ZOGCU_ERR_TOO_LARGE: return "too large";
    case ZOGCU_ERR_INTERNAL: return "internal error";
    default: return "unknown status";
  }
}

const char* zogcu_last_error(void) { return t_last_error.c_str(); }
int zogcu_abi_version(void) { return ZOGCU_ABI_VERSION; }
void zogcu_free(void* p) { std::free(p); }

int zogcu_release_cached_memory(void) {
  int dev;
  ZOGCU_TRY(ensure_device(&dev));
  ZOGCU_CUDA(cudaDeviceSynchronize());
  cudaMemPool_t pool;
  ZOGCU_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  ZOGCU_CUDA(cudaMemPoolTrimTo(pool, 0));
  return ZOGCU_OK;
}

int zogcu_graph_create_from_device_edges(uint32_t node_count, const uint32_t* d_from, const uint32_t* d_to,
                                         uint64_t num_edges, void* stream, zogcu_graph** out) {
  if (!out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  if (num_edges && (!d_from || !d_to)) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "edge arrays are null");
  if (num_edges >= 0xFFFFFFFFull) return fail(ZOGCU_ERR_TOO_LARGE, "edge count exceeds u32 edge indices");
  int dev;
  ZOGCU_TRY(ensure_device(&dev));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(stream));
  return create_from_device_edges_on(node_count, d_from, d_to, num_edges, sg.s, out);
}

int zogcu_graph_create_from_edges(uint32_t node_count, const uint32_t* from, const uint32_t* to,
                                  const double* weight, uint64_t num_edges, zogcu_graph** out) {
  // PageRank and unweighted Brandes ignore the weights (centrality.zig:936-941);
  // weighted betweenness reads them (centrality.zig:528-682)
  if (!out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  if (num_edges && (!from || !to)) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "edge arrays are null");
  if (num_edges >= 0xFFFFFFFFull) return fail(ZOGCU_ERR_TOO_LARGE, "edge count exceeds u32 edge indices");
  int dev;
  ZOGCU_TRY(ensure_device(&dev));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(nullptr));
  PhaseTrace tr("graph_create_from_edges", sg.s);
  DevBuf df, dt;
  ZOGCU_TRY(df.alloc(num_edges * 4, sg.s));
  ZOGCU_TRY(dt.alloc(num_edges * 4, sg.s));
  DevBuf dw, rdst, rsrc, rcnt, rstart, rtotal, routc, rflags;
  ChunkRuns runs;
  if (num_edges >= kChunkedMinArcs && !weight) {
    // Chunks of both arrays cross PCIe on a second stream; each chunk's stable
    // sort by destination runs while the next ones are copied.  When the
    // sources turn out non-decreasing, the in-CSR is then one merge of the runs.
    StreamGuard up;
    ZOGCU_TRY(up.init(nullptr));
    ZOGCU_TRY(upload_chunked(from, to, num_edges, node_count, df.as<uint32_t>(), dt.as<uint32_t>(), sg.s, up.s,
                             runs, rdst, rsrc, rcnt, rstart, rtotal, routc, rflags));
    tr.mark("arcs to the device, chunks sorted meanwhile");
  } else if (num_edges) {
    ZOGCU_TRY(copy_host(df.ptr, const_cast<uint32_t*>(from), num_edges * 4, true, sg.s));
    ZOGCU_TRY(copy_host(dt.ptr, const_cast<uint32_t*>(to), num_edges * 4, true, sg.s));
    if (weight) {
      ZOGCU_TRY(dw.alloc(num_edges * 8, sg.s));
      ZOGCU_TRY(copy_host(dw.ptr, const_cast<double*>(weight), num_edges * 8, true, sg.s));
    }
    tr.mark("arcs to the device");
  }
  const int rc = create_from_device_edges_on(node_count, df.as<uint32_t>(), dt.as<uint32_t>(), num_edges, sg.s, out,
                                             weight ? dw.as<double>() : nullptr, runs.chunks ? &runs : nullptr);
  tr.mark("validation and CSR build");
  return rc;
}

static int create_from_arraygraph(uint32_t V, const uint32_t* first_edge, const uint8_t* node_deleted,
                                  uint64_t edge_capacity, const uint32_t* to, const uint32_t* next_edge,
                                  const uint8_t* edge_deleted, const double* data, zogcu_graph** out) {
  if (!out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  if (V && !first_edge) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "first_edge is null");
  if (edge_capacity && (!to || !next_edge)) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "edge slices are null");
  // Walk every live node's list like SuccessorIterator.next (array_graph.zig:164-180).
  std::vector<uint32_t> src, dst;
  std::vector<double> wts;
  src.reserve(edge_capacity);
  dst.reserve(edge_capacity);
  if (data) wts.reserve(edge_capacity);
  for (uint32_t v = 0; v < V; ++v) {
    if (node_deleted && node_deleted[v]) continue;
    uint32_t idx = first_edge[v];
    uint64_t steps = 0;
    while (idx != 0xFFFFFFFFu) {
      if (idx >= edge_capacity || ++steps > edge_capacity)
        return fail(ZOGCU_ERR_INVALID_ARGUMENT, "corrupt edge list at node " + std::to_string(v));
      uint32_t nxt = next_edge[idx];
      if (!(edge_deleted && edge_deleted[idx])) {
        uint32_t d = to[idx];
        if (d >= V) return fail(ZOGCU_ERR_NODE_NOT_FOUND, "edge target >= node capacity");
        if (!(node_deleted && node_deleted[d])) {
          src.push_back(v);
          dst.push_back(d);
          if (data) wts.push_back(data[idx]);
        }
      }
      idx = nxt;
    }
  }
  int dev;
  ZOGCU_TRY(ensure_device(&dev));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(nullptr));
  uint64_t E = src.size();
  DevBuf df, dt, dw;
  ZOGCU_TRY(df.alloc(E * 4, sg.s));
  ZOGCU_TRY(dt.alloc(E * 4, sg.s));
  if (E) {
    ZOGCU_CUDA(cudaMemcpyAsync(df.ptr, src.data(), E * 4, cudaMemcpyHostToDevice, sg.s));
    ZOGCU_CUDA(cudaMemcpyAsync(dt.ptr, dst.data(), E * 4, cudaMemcpyHostToDevice, sg.s));
    if (data) {
      ZOGCU_TRY(dw.alloc(E * 8, sg.s));
      ZOGCU_CUDA(cudaMemcpyAsync(dw.ptr, wts.data(), E * 8, cudaMemcpyHostToDevice, sg.s));
    }
  }
  std::unique_ptr<zogcu_graph> G(new (std::nothrow) zogcu_graph());
  if (!G) return fail(ZOGCU_ERR_OUT_OF_MEMORY, "host allocation failed");
  ZOGCU_TRY(build_graph_from_device_edges(&G->g, V, df.as<uint32_t>(), dt.as<uint32_t>(), E,
                                          /*already successor order*/ false, node_deleted, sg.s,
                                          data && E ? dw.as<double>() : nullptr));
  if (data) G->g.weighted = true;
  *out = G.release();
  return ZOGCU_OK;
}

int zogcu_graph_create_from_arraygraph(uint32_t V, const uint32_t* first_edge, const uint8_t* node_deleted,
                                       uint64_t edge_capacity, const uint32_t* to, const uint32_t* next_edge,
                                       const uint8_t* edge_deleted, zogcu_graph** out) {
  return create_from_arraygraph(V, first_edge, node_deleted, edge_capacity, to, next_edge, edge_deleted, nullptr,
                                out);
}

int zogcu_graph_create_from_arraygraph_weighted(uint32_t V, const uint32_t* first_edge, const uint8_t* node_deleted,
                                                uint64_t edge_capacity, const uint32_t* to,
                                                const uint32_t* next_edge, const uint8_t* edge_deleted,
                                                const double* data, zogcu_graph** out) {
  if (edge_capacity && !data) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "data is null");
  return create_from_arraygraph(V, first_edge, node_deleted, edge_capacity, to, next_edge, edge_deleted, data, out);
}

int zogcu_graph_generate_rmat(int scale, int edge_factor, uint64_t seed, double a, double b, double c,
                              int directed, zogcu_graph** out) {
  if (!out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  if (scale < 1 || scale > 31 || edge_factor < 1 || edge_factor > 64)
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "scale must be in [1,31], edge_factor in [1,64]");
  if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0))
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "R-MAT probabilities must be >= 0 with a+b+c <= 1");
  const uint64_t M = (uint64_t)edge_factor << scale;
  if (!directed && 2 * M >= 0xFFFFFFFFull) return fail(ZOGCU_ERR_TOO_LARGE, "too many arcs");
  int dev;
  ZOGCU_TRY(ensure_device(&dev));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(nullptr));
  uint64_t ta, tab, tabc;
  rmat_thresholds(a, b, c, &ta, &tab, &tabc);
  DevBuf k1, k2, nsel;
  ZOGCU_TRY(k1.alloc(M * 8, sg.s));
  ZOGCU_TRY(k2.alloc(M * 8, sg.s));
  ZOGCU_TRY(nsel.alloc(8, sg.s));
  k_rmat<<<grid_for(M), 256, 0, sg.s>>>(splitmix64(seed), M, scale, ta, tab, tabc, directed,
                                        k1.as<uint64_t>());
  ZOGCU_CUDA(cudaGetLastError());
  size_t tmp = 0;
  ZOGCU_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, k1.as<uint64_t>(), k2.as<uint64_t>(), (int64_t)M, 0,
                                            2 * scale, sg.s));
  DevBuf t;
  ZOGCU_TRY(t.alloc(tmp, sg.s));
  ZOGCU_CUDA(cub::DeviceRadixSort::SortKeys(t.ptr, tmp, k1.as<uint64_t>(), k2.as<uint64_t>(), (int64_t)M, 0,
                                            2 * scale, sg.s));
  size_t tmp2 = 0;
  ZOGCU_CUDA(cub::DeviceSelect::Unique(nullptr, tmp2, k2.as<uint64_t>(), k1.as<uint64_t>(),
                                       nsel.as<unsigned long long>(), (int64_t)M, sg.s));
  if (tmp2 > tmp) ZOGCU_TRY(t.alloc(tmp2, sg.s));
  tmp2 = std::max(tmp, tmp2);
  ZOGCU_CUDA(cub::DeviceSelect::Unique(t.ptr, tmp2, k2.as<uint64_t>(), k1.as<uint64_t>(),
                                       nsel.as<unsigned long long>(), (int64_t)M, sg.s));
  unsigned long long m = 0;
  ZOGCU_CUDA(cudaMemcpyAsync(&m, nsel.ptr, 8, cudaMemcpyDeviceToHost, sg.s));
  ZOGCU_CUDA(cudaStreamSynchronize(sg.s));
  // drop the self-loop sentinel (largest key) if present
  if (m > 0) {
    uint64_t last = 0;
    ZOGCU_CUDA(cudaMemcpy(&last, k1.as<uint64_t>() + (m - 1), 8, cudaMemcpyDeviceToHost));
    if (last == (1ull << (2 * scale)) - 1) m -= 1;
  }
  t.release();
  k2.release();
  const uint64_t E = directed ? m : 2 * m;
  DevBuf es, ed;
  ZOGCU_TRY(es.alloc(std::max<uint64_t>(E, 1) * 4, sg.s));
  ZOGCU_TRY(ed.alloc(std::max<uint64_t>(E, 1) * 4, sg.s));
  if (m) {
    k_unpack<<<grid_for(m), 256, 0, sg.s>>>(k1.as<uint64_t>(), m, scale, directed, es.as<uint32_t>(),
                                            ed.as<uint32_t>());
    ZOGCU_CUDA(cudaGetLastError());
  }
  k1.release();
  std::unique_ptr<zogcu_graph> G(new (std::nothrow) zogcu_graph());
  if (!G) return fail(ZOGCU_ERR_OUT_OF_MEMORY, "host allocation failed");
  ZOGCU_TRY(build_graph_from_device_edges(&G->g, 1u << scale, es.as<uint32_t>(), ed.as<uint32_t>(), E, true,
                                          nullptr, sg.s));
  *out = G.release();
  return ZOGCU_OK;
}

// Raw R-MAT endpoints into device arrays (test hook for generator parity).
int zogcu_rmat_raw_device(int scale, uint64_t seed, double a, double b, double c, uint64_t i0, uint64_t m,
                          uint32_t* d_src, uint32_t* d_dst) {
  if (!d_src || !d_dst || scale < 1 || scale > 31) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "bad arguments");
  int dev;
  ZOGCU_TRY(ensure_device(&dev));
  uint64_t ta, tab, tabc;
  rmat_thresholds(a, b, c, &ta, &tab, &tabc);
  k_rmat_raw<<<grid_for(m), 256>>>(splitmix64(seed), i0, m, scale, ta, tab, tabc, d_src, d_dst);
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_CUDA(cudaDeviceSynchronize());
  return ZOGCU_OK;
}

int zogcu_graph_destroy(zogcu_graph* g) {
  if (!g) return ZOGCU_OK;
  cudaSetDevice(g->g.device);
  delete g;
  return ZOGCU_OK;
}

int zogcu_graph_info(const zogcu_graph* g, uint32_t* V, uint64_t* E, uint64_t* live) {
  if (!g) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graph is null");
  if (V) *V = g->g.V;
  if (E) *E = g->g.E;
  if (live) *live = g->g.n_live;
  return ZOGCU_OK;
}

int zogcu_graph_export_csr(const zogcu_graph* G, uint64_t* in_off, uint32_t* in_col, uint64_t* out_off,
                           uint32_t* out_col, uint32_t* out_degree) {
  if (!G) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graph is null");
  const Graph& g = G->g;
  ZOGCU_CUDA(cudaSetDevice(g.device));
  if (in_off) ZOGCU_CUDA(cudaMemcpy(in_off, g.in_off64.ptr, (size_t)(g.V + 1) * 8, cudaMemcpyDeviceToHost));
  if (out_off) ZOGCU_CUDA(cudaMemcpy(out_off, g.out_off64.ptr, (size_t)(g.V + 1) * 8, cudaMemcpyDeviceToHost));
  if (in_col && g.E) ZOGCU_CUDA(cudaMemcpy(in_col, g.in_col.ptr, g.E * 4, cudaMemcpyDeviceToHost));
  if (out_col && g.E) ZOGCU_CUDA(cudaMemcpy(out_col, g.out_col.ptr, g.E * 4, cudaMemcpyDeviceToHost));
  if (out_degree && g.V) ZOGCU_CUDA(cudaMemcpy(out_degree, g.out_deg.ptr, (size_t)g.V * 4, cudaMemcpyDeviceToHost));
  return ZOGCU_OK;
}

}  // extern "C"
