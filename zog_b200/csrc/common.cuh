// common.cuh -- internal types and helpers of libzogcu (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "zogcu.h"

namespace zogcu {

// Marks a deleted node slot in the out-degree array.  Deleted nodes have no
// stored arcs, so the value never reaches a gather; PageRank uses it to skip
// the slot (the reference only iterates live nodes, utils.zig:42-48).
constexpr uint32_t kDeletedDegree = 0xFFFFFFFFu;
constexpr uint32_t kUnreached = 0xFFFFFFFFu;

// Last error message of the calling thread (zogcu_last_error).
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);

#define ZOGCU_CUDA(call)                                                        \
  do {                                                                          \
    cudaError_t _e = (call);                                                    \
    if (_e != cudaSuccess) {                                                    \
      return ::zogcu::fail(_e == cudaErrorMemoryAllocation ? ZOGCU_ERR_OUT_OF_MEMORY \
                                                           : ZOGCU_ERR_CUDA,    \
                           std::string(#call) + ": " + cudaGetErrorString(_e)); \
    }                                                                           \
  } while (0)

#define ZOGCU_TRY(call)                 \
  do {                                  \
    int _s = (call);                    \
    if (_s != ZOGCU_OK) return _s;      \
  } while (0)

// Stream-ordered device buffer (cudaMallocAsync on the owning stream), or a
// view of memory owned elsewhere (borrow: release() then frees nothing).
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  bool owned = true;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes), stream(o.stream), owned(o.owned) { o.ptr = nullptr; }
  ~DevBuf() { release(); }
  int alloc(size_t n, cudaStream_t s);
  void borrow(void* p, size_t n) {
    release();
    ptr = p;
    bytes = n;
    owned = false;
  }
  void release();
  template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Persistent device allocation owned by a graph (from the stream-ordered pool;
// release waits for the device like cudaFree).
struct DevArray {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevArray() = default;
  DevArray(const DevArray&) = delete;
  DevArray& operator=(const DevArray&) = delete;
  ~DevArray() { release(); }
  int alloc(size_t n);
  void release();
  template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Scratch kept by a graph or a model between calls, so that repeated calls
// allocate nothing.  Alternating calls with differently sized per-call
// allocations (a warm-start inference, then a PageRank solve) made the
// stream-ordered pool stall the host for up to 0.2 s per call.  A call that
// takes the cache (try_lock) holds it until its work on the GPU has finished;
// a concurrent call finds it taken and allocates its own buffers as before.
struct WorkCache {
  static constexpr int kSlots = 16;
  std::mutex mu;
  DevArray slot[kSlots];
};

// One call's hold on a WorkCache.  get() hands out slot i (grown to n bytes
// when needed) when the cache was free, else a buffer of its own on stream s.
// The destructor waits for stream s before letting the next call in.
struct WorkLease {
  WorkCache* cache = nullptr;
  cudaStream_t s = nullptr;
  bool held = false;
  WorkLease(WorkCache* c, cudaStream_t st) : cache(c), s(st) { held = c && c->mu.try_lock(); }
  WorkLease(const WorkLease&) = delete;
  WorkLease& operator=(const WorkLease&) = delete;
  ~WorkLease() {
    if (held) {
      cudaStreamSynchronize(s);
      cache->mu.unlock();
    }
  }
  int get(DevBuf& b, int i, size_t n) {
    if (!held) return b.alloc(n, s);
    DevArray& a = cache->slot[i];
    if (a.bytes < n) {
      const int rc = a.alloc(n);
      if (rc != ZOGCU_OK) return rc;
    }
    b.borrow(a.ptr, n);
    return ZOGCU_OK;
  }
};

// PageRank work-item schedule (shared by the single-vector kernel and the
// personalised SpMM): row blocks hold at most kWarpRows rows, long rows are
// cut into chunks of kLongChunk arcs.
constexpr int kWarpRows = 64;
constexpr int kLongChunk = 4096;
enum : uint32_t { kTaskBlock = 0, kTaskRow = 1, kTaskChunk = 2 };

// One PageRank work item (8 bytes): kind = b >> 30.
//   kind 0: rows [a, b & 0x3FFFFFFF) of the degree-ranked in-CSR
//   kind 1: the single row a
//   kind 2: chunk (b & 0xFFFF) of the long row a
struct PrTask {
  uint32_t a;
  uint32_t b;
};

// PageRank view of a graph, built on the first PageRank call: nodes renumbered
// by out-degree (descending; deleted slots last), so the most gathered
// contributions form a contiguous prefix that fits in shared memory, with the
// in-CSR re-laid in that order (each row keeps the reference's ascending
// source order), plus one schedule of warp work items per work-item size.
struct PrTaskList {
  bool built = false;
  uint32_t num_tasks = 0;
  uint32_t num_long = 0;      // rows split into chunks
  DevArray tasks;             // PrTask[num_tasks]
  DevArray long_first;        // uint32_t[num_long]: first chunk task of each long row
};

// Propagation-blocked layout of the PageRank view (pagerank.cu), built on the
// first precision-form solve of a large graph.  Rows are cut into partitions
// (at most kPbRows rows, about 2^20 in-arcs each) and sources into blocks (at
// most kPbSrcs sources, about 2^20 out-arcs each); the arcs of block b into
// partition p form one piece.  Pieces are stored block by block, each padded
// to a multiple of 4 positions; a position holds the arc's source relative to
// its block (sl) and its row relative to its partition (dl; padding points at
// a spare row).
struct PbItem {
  uint32_t b, lo, hi, pad;  // positions [lo, hi) of block b
};
struct PbView {
  int state = 0;              // 0 not built, 1 built, -1 not usable for this graph
  uint32_t P = 0, B = 0, nitems = 0;
  uint64_t npad = 0;
  DevArray row_lo, row_n, part_order;   // uint32_t[P]; part_order: partitions by arcs, largest first
  DevArray blk_lo, blk_n;               // uint32_t[B]
  DevArray pstart, pcount;              // uint32_t[P * B], partition-major
  DevArray sl, dl;                      // uint16_t[npad]
  DevArray items;                       // PbItem[nitems]: emit work, largest first
  DevArray msg;                         // float[npad]: one contribution per position
  DevArray heavy;                       // uint16_t[P][4]: each partition's heaviest rows (local)
  void reset() {
    for (DevArray* a : {&row_lo, &row_n, &part_order, &blk_lo, &blk_n, &pstart, &pcount, &sl, &dl, &items, &msg, &heavy})
      a->release();
    state = 0;
    P = B = nitems = 0;
    npad = 0;
  }
};

struct PrSchedule {
  bool built = false;
  DevArray rank;              // uint32_t[V]: rank of node v
  DevArray perm;              // uint32_t[V]: node of rank p
  DevArray off;               // uint32_t[V+1] (or uint64_t when E >= 2^32)
  DevArray col;               // uint32_t[E+4]: ranks of the sources
  DevArray deg;               // uint32_t[V]: out-degree of rank p
  PrTaskList lists[2];        // work items of 128 and of 256 arcs
  int config = -1;            // kernel configuration chosen by the autotuner
};

// Device-resident graph (one per NIF resource).
struct Graph {
  int device = 0;
  uint32_t V = 0;             // node capacity
  uint64_t E = 0;             // stored arcs (live edges between live nodes)
  uint64_t n_live = 0;        // live nodes
  bool has_deleted = false;
  bool offsets32 = false;     // E < 2^32: 32-bit offset copies exist
  DevArray in_off64, out_off64;   // uint64_t[V+1]
  DevArray in_off32, out_off32;   // uint32_t[V+1] (when offsets32)
  DevArray in_col, out_col;       // uint32_t[E + 4] (padded for 16-byte loads)
  DevArray out_deg;               // uint32_t[V], kDeletedDegree for deleted slots
  bool weighted = false;          // arc weights were given (else every weight is 1.0)
  DevArray out_w;                 // double[E]: weight of each out-CSR arc (when weighted)
  DevArray live;                  // uint8_t[V] (when has_deleted)
  std::mutex mu;                  // guards lazy schedule builds
  PrSchedule pr;                  // PageRank schedule (built on first call)
  WorkCache pr_ws;                // PageRank solve scratch, reused by later calls
  PbView pb;                      // propagation-blocked layout (precision form)
  // Brandes: vertices whose in- / out-degree exceeds the heavy threshold,
  // by degree descending (built on the first betweenness call)
  bool bc_built = false;
  uint32_t n_heavy_in = 0, n_heavy_out = 0;
  DevArray heavy_in, heavy_out;
  // Brandes lanes' workspaces and instantiated CUDA graphs, kept for later
  // calls on this graph (brandes.cu; released with the graph)
  std::shared_ptr<void> bc_cache;
};

int ensure_device(int* dev);

// Builds a Graph from device edge arrays (src,dst) in ArrayGraph insertion
// order (reverse_within_source = true) or already in successor order (false).
// All endpoints must be < V and refer to live nodes.
// d_w (may be null) holds one weight per edge in the same order as d_src / d_dst.
// The arcs sorted stably by destination chunk by chunk, made while later
// chunks were still being copied to the device (zogcu_graph_create_from_edges).
// Chunk c holds arcs [bound[c], bound[c+1]); dst and src hold each chunk's
// (destination, source) pairs in that order; pre[c * (V + 1) + d] counts the
// arcs into d in chunks before c, start[c * (V + 1) + d] is where d's segment
// begins in chunk c's run, and total[d] counts the arcs into d (V + 1 slots,
// the last zero).
constexpr int kMaxUploadChunks = 8;
struct ChunkRuns {
  int chunks = 0;
  uint64_t bound[kMaxUploadChunks + 1] = {};
  const uint32_t* dst = nullptr;
  const uint32_t* src = nullptr;
  const uint32_t* pre = nullptr;
  const uint32_t* start = nullptr;
  unsigned long long* total = nullptr;
  unsigned long long* out_cnt = nullptr;  // arcs per source (V + 1 slots)
  unsigned int* flags = nullptr;          // [0] an endpoint >= V, [1] sources not non-decreasing
};

// src_sorted: 1 = d_src is non-decreasing (the out-CSR is then placed by one
// scatter instead of a sort), 0 = it is not, -1 = unknown (checked here).
// runs (may be null; used only when d_src is non-decreasing): per-chunk
// sorted runs of the same arcs, so the in-CSR is one merge scatter instead of
// a second sort (each row's chunks in chunk order list its sources ascending).
int build_graph_from_device_edges(Graph* g, uint32_t V, const uint32_t* d_src,
                                  const uint32_t* d_dst, uint64_t E, bool reverse_within_source,
                                  const uint8_t* h_node_deleted, cudaStream_t stream,
                                  const double* d_w = nullptr, int src_sorted = -1,
                                  ChunkRuns* runs = nullptr);

// PageRank schedule (pagerank.cu): the degree-ranked view, and the work-item
// list of row blocks of at most nnz (128 or 256) arcs.
int ensure_pr_schedule(Graph* g, cudaStream_t stream);
int ensure_task_list(Graph* g, int nnz, cudaStream_t stream);

// Host <-> device copy of a caller array that may be pageable (pipelined
// through pinned chunks on helper threads when it is), ordered on stream s.
int copy_host(void* dev, void* host, size_t bytes, bool h2d, cudaStream_t s);

// Small helper: number of SMs of the current device.
int sm_count();

// RAII private stream.
struct StreamGuard {
  cudaStream_t s = nullptr;
  bool owned = false;
  int init(void* user);
  ~StreamGuard();
};

// Phase timing of one call, for diagnostics: with ZOGCU_TRACE set in the
// environment, mark() synchronises the stream and prints the wall time since
// the previous mark to stderr.  Off by default; it changes no result.
struct PhaseTrace {
  const char* what;
  cudaStream_t s;
  bool on;
  std::chrono::steady_clock::time_point t;
  PhaseTrace(const char* w, cudaStream_t st) : what(w), s(st), on(std::getenv("ZOGCU_TRACE") != nullptr) {
    if (on) {
      cudaStreamSynchronize(s);
      t = std::chrono::steady_clock::now();
    }
  }
  void mark(const char* phase) {
    if (!on) return;
    cudaStreamSynchronize(s);
    const auto n = std::chrono::steady_clock::now();
    std::fprintf(stderr, "zogcu trace: %s: %s %.3f ms\n", what, phase,
                 std::chrono::duration<double, std::milli>(n - t).count());
    t = n;
  }
};

// Event timer on one stream.
struct EventTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  int start(cudaStream_t s);
  int stop(cudaStream_t s);
  float ms();
  ~EventTimer();
};

}  // namespace zogcu

struct zogcu_graph {
  zogcu::Graph g;
};
