// brandes.cu -- exact unweighted betweenness (Brandes) with many sources in
// flight per launch.
//
// Reference: priv/zog/src/centrality.zig:687-798 (ArrayGraph branch).  For
// every live source s (ascending) the reference runs a BFS that fills
// dist[] and the path counts sigma[] (`sigma[w] += sigma[v]` for every arc
// v->w with dist[w] == dist[v]+1, duplicates counted, :745-767), then walks the
// BFS order backwards accumulating delta[u] += sigma[u]/sigma[v] * (1+delta[v])
// over predecessors and adds delta[v] to the score of every v != s (:769-787).
//
// B200 design: a batch of 64 sources advances level by level in lock-step.
// Per vertex the batch keeps 64-bit masks -- visited, and the frontier of
// every level (kept for the backward sweep) -- and, per (vertex, source) pair,
// dist (u32), sigma (u64) and q = (1+delta)/sigma (f64) in vertex-major rows
// of 64, so one warp owns one vertex and each lane owns sources lane and
// lane+32.
//   forward (pull): a vertex w with unvisited sources scans its in-neighbours
//     32 at a time (one coalesced index load, one frontier-mask gather per
//     lane), keeps only neighbours whose mask meets w's unvisited mask, and the
//     lanes add the matching sigma[v][b], four neighbour rows in flight at a
//     time -- no atomics, deterministic, exact integer sums that wrap modulo
//     2^64 like the reference's usize;
//   backward (pull over successors): at level l a vertex v with sources at
//     depth l (its level-l mask) gathers q[w][b] of successors w whose level-l+1
//     mask has bit b, so delta[v][b] = sigma[v][b] * sum q[w][b] -- the
//     reference's sum of sigma_v/sigma_w * (1+delta_w), reassociated -- and
//     the warp adds sum_b delta[v][b] to BC[v] (only v's warp touches BC[v]);
//   level loop on the device: forward launches are enqueued in chunks and a
//     launch returns at once when the previous level discovered nothing, so
//     the host synchronises once per chunk of levels, not once per level.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace zogcu {

constexpr int kBcBatch = 64;
constexpr int kBcThreads = 256;
constexpr int kLevelChunk = 8;     // forward levels enqueued between host checks
constexpr int kMaxStoredLevels = 64;  // frontier masks kept for the backward sweep
constexpr int kOverflowFlag = kMaxStoredLevels + 8;
constexpr int kHeavyDegree = 512;  // vertices above this degree get whole CTAs
constexpr int kHeavyChunk = 1024;  // arcs of a heavy vertex per CTA work item

// One CTA work item of a heavy vertex: arcs [chunk * kHeavyChunk, ...) of
// vertex v, which has nch items starting at index `first` of the list.
struct BcHeavy {
  uint32_t v;
  uint32_t first;
  uint32_t chunk;
  uint32_t nch;
};

// Level state of one batch when its levels run as CUDA-graph while loops: the
// forward level, the depth found (the first level that discovered nothing),
// the backward level still to sweep, and the deepest depth of the lane's
// batches so far (kept across batches).
struct BcLoop {
  uint32_t level;
  uint32_t depth;
  uint32_t blevel;
  uint32_t max_depth;
  uint32_t push;                  // direction of the current forward level: 1 push, 0 pull
  uint32_t active;                // the current batch holds sources (0: an empty slot of the graph)
  uint32_t batch;                 // the lane's current batch: sources [64 * batch, 64 * batch + 64)
  uint32_t nlanes;                // lanes of the call (the cursor's stride)
  unsigned long long next_arcs;   // out-arcs of the next frontier, summed during the level
  unsigned long long full;        // mask of the batch's sources
  unsigned long long ns;          // sources of the call
};

__device__ __forceinline__ unsigned long long shfl_u64(unsigned long long v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}

// One neighbour of the inner loops: its id and the mask of the batch's sources
// for which it matters (0 = none).
struct Nb {
  uint32_t v;
  unsigned long long m;
};

// Neighbours whose rows are gathered together (loads in flight per lane:
// 2 x kPop).  Eight measured +6 % at scale 16 and -5 % at scale 18: the forward
// kernel then needs 80 registers and loses a quarter of its warps.
constexpr int kPop = 4;

// Pops up to kPop set lanes of `bal` and broadcasts their (v, m) pairs.
__device__ __forceinline__ void pop_n(unsigned& bal, uint32_t v, unsigned long long m, Nb (&out)[kPop]) {
#pragma unroll
  for (int i = 0; i < kPop; ++i) {
    const int k = bal ? __ffs(bal) - 1 : 0;
    const bool any = bal != 0;
    bal &= bal - 1;
    out[i].v = __shfl_sync(0xffffffffu, v, k);
    const unsigned long long mk = shfl_u64(m, k);
    out[i].m = any ? mk : 0ull;
  }
}

// Work of one vertex's adjacency slice for the forward step: neighbours
// [j0, e) in steps of `stride`, 32 at a time; lanes accumulate sigma of their
// two sources over neighbours in the frontier for those sources.
template <typename OffT>
__device__ __forceinline__ void fwd_scan(const uint32_t* __restrict__ col, const unsigned long long* __restrict__ front_cur,
                                         const unsigned long long* __restrict__ sigma, unsigned long long cand, OffT j0,
                                         OffT e, OffT stride, int lane, unsigned long long& acc0,
                                         unsigned long long& acc1, bool& got0, bool& got1, bool& ovf) {
  for (; j0 < e; j0 += stride) {
    const OffT j = j0 + lane;
    uint32_t v = 0;
    unsigned long long m = 0;
    if (j < e) {
      v = __ldg(col + j);
      m = __ldg(front_cur + v) & cand;
    }
    unsigned bal = __ballot_sync(0xffffffffu, m != 0);
    while (bal) {
      Nb nb[kPop];
      pop_n(bal, v, m, nb);
      unsigned long long s0[kPop], s1[kPop];
#pragma unroll
      for (int i = 0; i < kPop; ++i) {
        const uint64_t row = (uint64_t)nb[i].v * kBcBatch;
        s0[i] = ((nb[i].m >> lane) & 1ull) ? sigma[row + lane] : 0ull;
        s1[i] = ((nb[i].m >> (lane + 32)) & 1ull) ? sigma[row + lane + 32] : 0ull;
      }
#pragma unroll
      for (int i = 0; i < kPop; ++i) {
        got0 |= ((nb[i].m >> lane) & 1ull) != 0;
        got1 |= ((nb[i].m >> (lane + 32)) & 1ull) != 0;
        unsigned long long n = acc0 + s0[i];
        ovf |= n < acc0;
        acc0 = n;
        n = acc1 + s1[i];
        ovf |= n < acc1;
        acc1 = n;
      }
    }
  }
}

// Publishes the level-(l+1) result of vertex w (one warp).
__device__ __forceinline__ void fwd_commit(uint64_t w, unsigned long long vis, unsigned long long newmask,
                                           unsigned long long acc0, unsigned long long acc1, uint32_t level, int lane,
                                           unsigned long long* __restrict__ front_nxt,
                                           unsigned long long* __restrict__ visited,
                                           unsigned long long* __restrict__ sigma, uint32_t* __restrict__ dist,
                                           bool& any_new) {
  if ((newmask >> lane) & 1ull) {
    sigma[w * kBcBatch + lane] = acc0;
    dist[w * kBcBatch + lane] = level + 1;
  }
  if ((newmask >> (lane + 32)) & 1ull) {
    sigma[w * kBcBatch + lane + 32] = acc1;
    dist[w * kBcBatch + lane + 32] = level + 1;
  }
  if (lane == 0) {
    front_nxt[w] = newmask;
    if (newmask) {
      visited[w] = vis | newmask;
      any_new = true;
    }
  }
}

// Forward step of level `level`: the CTA first takes the heavy vertices (a
// whole CTA per vertex, its 8 warps splitting the adjacency, partial sums
// added in shared memory), then blocks of 8 light vertices (a warp each).
template <typename OffT>
__global__ void __launch_bounds__(kBcThreads) bc_forward_kernel(
    uint32_t V, const OffT* __restrict__ off, const uint32_t* __restrict__ col,
    const unsigned long long* __restrict__ front_cur, unsigned long long* __restrict__ front_nxt,
    unsigned long long* __restrict__ visited, unsigned long long* __restrict__ sigma, uint32_t* __restrict__ dist,
    unsigned long long full, uint32_t level, unsigned int* __restrict__ flags, const BcHeavy* __restrict__ heavy,
    uint32_t nheavy, unsigned long long* __restrict__ hpart, unsigned long long* __restrict__ hgot,
    unsigned int* __restrict__ harrive, const BcLoop* __restrict__ loop, unsigned long long* __restrict__ masks,
    const OffT* __restrict__ out_off) {
  // flags[l % kMaxStoredLevels] = 1 when level l discovered a vertex;
  // flags[kOverflowFlag] = some path count wrapped.  With `loop` (the level
  // loop runs on the device) the level and its frontier masks come from the
  // batch's loop state and the mask ring `masks`.
  if (loop) {
    if (!*(volatile const uint32_t*)&loop->active) return;  // an empty batch slot
    if (*(volatile const uint32_t*)&loop->push) return;     // a push level (bc_push_kernel)
    level = *(volatile const uint32_t*)&loop->level;
    full = *(volatile const unsigned long long*)&loop->full;
    front_cur = masks + (size_t)(level % (kMaxStoredLevels + 1)) * V;
    front_nxt = masks + (size_t)((level + 1) % (kMaxStoredLevels + 1)) * V;
  }
  if (level > 0 && *(volatile unsigned int*)(flags + (level - 1) % kMaxStoredLevels) == 0u) return;
  // out-arcs of the vertices this CTA adds to the next frontier (device loop
  // only: the next level's direction is chosen from their sum)
  unsigned long long nxt_arcs = 0;
  constexpr int W = kBcThreads / 32;
  __shared__ unsigned long long s_acc[W][kBcBatch];
  __shared__ unsigned long long s_got[W];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool any_ovf = false, any_new = false;
  const uint64_t ntasks = (uint64_t)nheavy + ((uint64_t)V + W - 1) / W;
  for (uint64_t t = blockIdx.x; t < ntasks; t += gridDim.x) {
    if (t < nheavy) {
      const BcHeavy ht = heavy[t];
      const uint64_t w = ht.v;
      const unsigned long long vis = visited[w];
      const unsigned long long cand = full & ~vis;
      unsigned long long acc0 = 0, acc1 = 0;
      bool got0 = false, got1 = false;
      if (cand) {
        const OffT b = __ldg(off + w) + (OffT)ht.chunk * (OffT)kHeavyChunk;
        const OffT e = min(b + (OffT)kHeavyChunk, __ldg(off + w + 1));
        fwd_scan<OffT>(col, front_cur, sigma, cand, b + (OffT)(32 * warp), e, (OffT)(32 * W), lane, acc0, acc1, got0,
                       got1, any_ovf);
      }
      s_acc[warp][lane] = acc0;
      s_acc[warp][lane + 32] = acc1;
      const unsigned long long gm = (unsigned long long)__ballot_sync(0xffffffffu, got0) |
                                    ((unsigned long long)__ballot_sync(0xffffffffu, got1) << 32);
      if (lane == 0) s_got[warp] = gm;
      __syncthreads();
      if (warp == 0) {
        unsigned long long t0 = 0, t1 = 0, newmask = 0;
        for (int k = 0; k < W; ++k) {
          unsigned long long n = t0 + s_acc[k][lane];
          any_ovf |= n < t0;
          t0 = n;
          n = t1 + s_acc[k][lane + 32];
          any_ovf |= n < t1;
          t1 = n;
          newmask |= s_got[k];
        }
        if (ht.nch == 1) {
          fwd_commit(w, vis, newmask, t0, t1, level, lane, front_nxt, visited, sigma, dist, any_new);
          if (loop && lane == 0 && newmask) nxt_arcs += (unsigned long long)(__ldg(out_off + w + 1) - __ldg(out_off + w));
        } else {
          // chunk partials; the last chunk to arrive adds them in chunk order
          // (exact integer sums) and commits the vertex
          hpart[(size_t)t * kBcBatch + lane] = t0;
          hpart[(size_t)t * kBcBatch + lane + 32] = t1;
          if (lane == 0) hgot[t] = newmask;
          __threadfence();
          __syncwarp();
          unsigned last = 0;
          if (lane == 0) last = atomicAdd(harrive + ht.first, 1u) == ht.nch - 1 ? 1u : 0u;
          last = __shfl_sync(0xffffffffu, last, 0);
          if (last) {
            __threadfence();
            unsigned long long u0 = 0, u1 = 0, nm = 0;
            for (uint32_t k = 0; k < ht.nch; ++k) {
              const size_t r = (size_t)(ht.first + k) * kBcBatch;
              unsigned long long n = u0 + __ldcg(hpart + r + lane);
              any_ovf |= n < u0;
              u0 = n;
              n = u1 + __ldcg(hpart + r + lane + 32);
              any_ovf |= n < u1;
              u1 = n;
              nm |= __ldcg(hgot + ht.first + k);
            }
            fwd_commit(w, vis, nm, u0, u1, level, lane, front_nxt, visited, sigma, dist, any_new);
            if (loop && lane == 0 && nm) nxt_arcs += (unsigned long long)(__ldg(out_off + w + 1) - __ldg(out_off + w));
            if (lane == 0) harrive[ht.first] = 0u;
          }
        }
      }
      __syncthreads();
    } else {
      const uint64_t w = (t - nheavy) * W + warp;
      if (w < V) {
        const OffT b = __ldg(off + w), e = __ldg(off + w + 1);
        if ((uint64_t)(e - b) <= (uint64_t)kHeavyDegree) {  // heavy vertices were done above
          const unsigned long long vis = visited[w];
          const unsigned long long cand = full & ~vis;
          unsigned long long acc0 = 0, acc1 = 0;
          bool got0 = false, got1 = false;
          if (cand) fwd_scan<OffT>(col, front_cur, sigma, cand, b, e, (OffT)32, lane, acc0, acc1, got0, got1, any_ovf);
          const unsigned long long newmask = (unsigned long long)__ballot_sync(0xffffffffu, got0) |
                                             ((unsigned long long)__ballot_sync(0xffffffffu, got1) << 32);
          fwd_commit(w, vis, newmask, acc0, acc1, level, lane, front_nxt, visited, sigma, dist, any_new);
          if (loop && lane == 0 && newmask) nxt_arcs += (unsigned long long)(__ldg(out_off + w + 1) - __ldg(out_off + w));
        }
      }
    }
  }
  if (__any_sync(0xffffffffu, any_new) && lane == 0) flags[level % kMaxStoredLevels] = 1u;
  if (__any_sync(0xffffffffu, any_ovf) && lane == 0) flags[kOverflowFlag] = 1u;
  if (loop) {
    __shared__ unsigned long long s_arcs;
    if (threadIdx.x == 0) s_arcs = 0;
    __syncthreads();
    if (nxt_arcs) atomicAdd(&s_arcs, nxt_arcs);
    __syncthreads();
    if (threadIdx.x == 0 && s_arcs) atomicAdd(const_cast<unsigned long long*>(&loop->next_arcs), s_arcs);
  }
}

// Level-l mask of v recomputed from dist (deep BFS, masks not stored).
__device__ __forceinline__ unsigned long long dist_mask(const uint32_t* __restrict__ dist, uint64_t v, uint32_t level,
                                                        int lane) {
  const bool a0 = dist[v * kBcBatch + lane] == level;
  const bool a1 = dist[v * kBcBatch + lane + 32] == level;
  return (unsigned long long)__ballot_sync(0xffffffffu, a0) | ((unsigned long long)__ballot_sync(0xffffffffu, a1) << 32);
}

// Sum of q[w][b] over successors w in [j0, e) (stride `stride`) whose
// level-(l+1) mask has bit b.
template <typename OffT>
__device__ __forceinline__ void bwd_scan(const uint32_t* __restrict__ col, const unsigned long long* __restrict__ mask_next,
                                         const double* __restrict__ q, unsigned long long act, OffT j0, OffT e,
                                         OffT stride, int lane, double& acc0, double& acc1) {
  for (; j0 < e; j0 += stride) {
    const OffT j = j0 + lane;
    uint32_t w = 0;
    unsigned long long g = 0;
    if (j < e) {
      w = __ldg(col + j);
      g = __ldg(mask_next + w) & act;
    }
    unsigned bal = __ballot_sync(0xffffffffu, g != 0);
    while (bal) {
      Nb nb[kPop];
      pop_n(bal, w, g, nb);
      double t0[kPop], t1[kPop];
#pragma unroll
      for (int i = 0; i < kPop; ++i) {
        const uint64_t row = (uint64_t)nb[i].v * kBcBatch;
        t0[i] = ((nb[i].m >> lane) & 1ull) ? q[row + lane] : 0.0;
        t1[i] = ((nb[i].m >> (lane + 32)) & 1ull) ? q[row + lane + 32] : 0.0;
      }
#pragma unroll
      for (int i = 0; i < kPop; ++i) {
        acc0 += t0[i];
        acc1 += t1[i];
      }
    }
  }
}

// delta, q and the BC contribution of vertex v at this level (one warp).
__device__ __forceinline__ void bwd_commit(uint64_t v, unsigned long long act, double acc0, double acc1, int lane,
                                           const unsigned long long* __restrict__ sigma, double* __restrict__ q,
                                           double* __restrict__ bc) {
  double dsum = 0.0;
  if ((act >> lane) & 1ull) {
    const double sv = (double)sigma[v * kBcBatch + lane];
    const double d = __dmul_rn(sv, acc0);
    q[v * kBcBatch + lane] = __ddiv_rn(1.0 + d, sv);
    dsum += d;
  }
  if ((act >> (lane + 32)) & 1ull) {
    const double sv = (double)sigma[v * kBcBatch + lane + 32];
    const double d = __dmul_rn(sv, acc1);
    q[v * kBcBatch + lane + 32] = __ddiv_rn(1.0 + d, sv);
    dsum += d;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
  if (lane == 0) bc[v] += dsum;
}

// Backward step of level `level`.  mask_l / mask_next: stored masks of levels
// l and l+1; when null, level l is derived from dist and written to mask_out
// for the next (shallower) launch, which reads it as its mask_next.
template <typename OffT>
__global__ void __launch_bounds__(kBcThreads) bc_backward_kernel(
    uint32_t V, const OffT* __restrict__ off, const uint32_t* __restrict__ col,
    const unsigned long long* __restrict__ mask_l, const unsigned long long* __restrict__ mask_next,
    unsigned long long* __restrict__ mask_out, const uint32_t* __restrict__ dist,
    const unsigned long long* __restrict__ sigma, double* __restrict__ q, double* __restrict__ bc, uint32_t level,
    int last_level, const BcHeavy* __restrict__ heavy, uint32_t nheavy, double* __restrict__ hpart,
    unsigned int* __restrict__ harrive, const BcLoop* __restrict__ loop, unsigned long long* __restrict__ masks,
    unsigned long long* __restrict__ mbuf_a, unsigned long long* __restrict__ mbuf_b) {
  if (loop) {
    // the level, and where its masks come from, from the batch's loop state:
    // stored frontiers when the BFS was shallower than the ring, else masks
    // derived from dist that alternate between two buffers (level depth - k
    // reads buffer k % 2 and writes the other)
    level = *(volatile const uint32_t*)&loop->blevel;
    if (level == 0) return;
    const uint32_t depth = *(volatile const uint32_t*)&loop->depth;
    last_level = level == depth ? 1 : 0;
    if (depth < (uint32_t)kMaxStoredLevels) {
      mask_l = masks + (size_t)(level % (kMaxStoredLevels + 1)) * V;
      mask_next = masks + (size_t)((level + 1) % (kMaxStoredLevels + 1)) * V;
      mask_out = nullptr;
    } else {
      const bool odd = ((depth - level) & 1u) != 0;
      mask_l = nullptr;
      mask_next = odd ? mbuf_b : mbuf_a;
      mask_out = odd ? mbuf_a : mbuf_b;
    }
  }
  constexpr int W = kBcThreads / 32;
  __shared__ double s_acc[W][kBcBatch];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t ntasks = (uint64_t)nheavy + ((uint64_t)V + W - 1) / W;
  for (uint64_t t = blockIdx.x; t < ntasks; t += gridDim.x) {
    if (t < nheavy) {
      const BcHeavy ht = heavy[t];
      const uint64_t v = ht.v;
      const unsigned long long act = mask_l ? __ldg(mask_l + v) : dist_mask(dist, v, level, lane);
      if (mask_out && ht.chunk == 0 && warp == 0 && lane == 0) mask_out[v] = act;
      if (!act) continue;                        // every chunk of v sees the same mask
      if (last_level && ht.chunk != 0) continue;  // no successors to scan: chunk 0 commits alone
      double acc0 = 0.0, acc1 = 0.0;
      if (!last_level) {
        const OffT b = __ldg(off + v) + (OffT)ht.chunk * (OffT)kHeavyChunk;
        const OffT e = min(b + (OffT)kHeavyChunk, __ldg(off + v + 1));
        bwd_scan<OffT>(col, mask_next, q, act, b + (OffT)(32 * warp), e, (OffT)(32 * W), lane, acc0, acc1);
      }
      s_acc[warp][lane] = acc0;
      s_acc[warp][lane + 32] = acc1;
      __syncthreads();
      if (warp == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int k = 0; k < W; ++k) {  // fixed order: deterministic
          t0 += s_acc[k][lane];
          t1 += s_acc[k][lane + 32];
        }
        if (ht.nch == 1 || last_level) {
          bwd_commit(v, act, t0, t1, lane, sigma, q, bc);
        } else {
          // chunk partials; the last chunk to arrive adds them in chunk order
          hpart[(size_t)t * kBcBatch + lane] = t0;
          hpart[(size_t)t * kBcBatch + lane + 32] = t1;
          __threadfence();
          __syncwarp();
          unsigned last = 0;
          if (lane == 0) last = atomicAdd(harrive + ht.first, 1u) == ht.nch - 1 ? 1u : 0u;
          last = __shfl_sync(0xffffffffu, last, 0);
          if (last) {
            __threadfence();
            double u0 = 0.0, u1 = 0.0;
            for (uint32_t k = 0; k < ht.nch; ++k) {
              const size_t r = (size_t)(ht.first + k) * kBcBatch;
              u0 += __ldcg(hpart + r + lane);
              u1 += __ldcg(hpart + r + lane + 32);
            }
            bwd_commit(v, act, u0, u1, lane, sigma, q, bc);
            if (lane == 0) harrive[ht.first] = 0u;
          }
        }
      }
      __syncthreads();
    } else {
      const uint64_t v = (t - nheavy) * W + warp;
      if (v < V) {
        const OffT b = __ldg(off + v), e = __ldg(off + v + 1);
        if ((uint64_t)(e - b) <= (uint64_t)kHeavyDegree) {
          const unsigned long long act = mask_l ? __ldg(mask_l + v) : dist_mask(dist, v, level, lane);
          if (mask_out && lane == 0) mask_out[v] = act;
          if (act) {
            double acc0 = 0.0, acc1 = 0.0;
            if (!last_level) bwd_scan<OffT>(col, mask_next, q, act, b, e, (OffT)32, lane, acc0, acc1);
            bwd_commit(v, act, acc0, acc1, lane, sigma, q, bc);
          }
        }
      }
    }
  }
}

__global__ void bc_seed_kernel(const uint32_t* __restrict__ sources, int nb, unsigned long long* visited,
                               unsigned long long* front, unsigned long long* sigma, uint32_t* dist) {
  const int b = threadIdx.x;
  if (b < nb) {
    const uint64_t s = sources[b];
    atomicOr(visited + s, 1ull << b);
    atomicOr(front + s, 1ull << b);
    sigma[s * kBcBatch + b] = 1ull;
    dist[s * kBcBatch + b] = 0u;
  }
}

// Grid of a Brandes kernel: the CTAs that are resident at once (occupancy x
// SMs), at most one per task, so the grid-stride task loop runs in a single
// wave and no CTA waits for a slot while others idle at the end of a level.
template <typename K>
static int bc_grid(K kernel, uint32_t V) {
  const uint64_t tasks = ((uint64_t)V + (kBcThreads / 32) - 1) / (kBcThreads / 32);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBcThreads, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  uint64_t blocks = (uint64_t)sm_count() * (uint64_t)per_sm;
  if (blocks > tasks) blocks = tasks;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

// Work items of the vertices of in- (forward) and out-degree (backward) above
// kHeavyDegree, by degree descending so the biggest start first: each vertex
// gets one item per kHeavyChunk arcs, consecutive in the list.
static int ensure_heavy_lists(Graph* g, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g->mu);
  if (g->bc_built) return ZOGCU_OK;
  const uint32_t V = g->V;
  for (int dir = 0; dir < 2; ++dir) {
    std::vector<uint64_t> off((size_t)V + 1);
    const DevArray& o = dir == 0 ? g->in_off64 : g->out_off64;
    ZOGCU_CUDA(cudaMemcpyAsync(off.data(), o.ptr, ((size_t)V + 1) * 8, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    std::vector<std::pair<uint64_t, uint32_t>> hv;
    for (uint32_t v = 0; v < V; ++v) {
      const uint64_t d = off[v + 1] - off[v];
      if (d > (uint64_t)kHeavyDegree) hv.emplace_back(d, v);
    }
    std::sort(hv.begin(), hv.end(), [](const auto& a, const auto& b) { return a.first != b.first ? a.first > b.first : a.second < b.second; });
    std::vector<BcHeavy> items;
    for (const auto& h : hv) {
      const uint64_t nch = (h.first + kHeavyChunk - 1) / kHeavyChunk;
      if (items.size() + nch >= 0xFFFFFFFFull) return fail(ZOGCU_ERR_TOO_LARGE, "too many heavy-vertex work items");
      const uint32_t first = (uint32_t)items.size();
      for (uint64_t c = 0; c < nch; ++c) items.push_back(BcHeavy{h.second, first, (uint32_t)c, (uint32_t)nch});
    }
    DevArray& dst = dir == 0 ? g->heavy_in : g->heavy_out;
    ZOGCU_TRY(dst.alloc(std::max<size_t>(items.size(), 1) * sizeof(BcHeavy)));
    if (!items.empty())
      ZOGCU_CUDA(cudaMemcpyAsync(dst.ptr, items.data(), items.size() * sizeof(BcHeavy), cudaMemcpyHostToDevice, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    (dir == 0 ? g->n_heavy_in : g->n_heavy_out) = (uint32_t)items.size();
  }
  g->bc_built = true;
  return ZOGCU_OK;
}

constexpr int kFlagWords = kMaxStoredLevels + 16;

struct BcWork {
  // masks: kMaxStoredLevels + 1 frontier arrays (level l at masks + l*V); when
  // the BFS is deeper, levels wrap around and the backward sweep derives its
  // masks from dist instead.
  // hpart / hgot / harrive: chunk partials, chunk masks and per-vertex arrival
  // counters of the heavy work items (counters are zero between launches)
  DevBuf visited, masks, mbuf_a, mbuf_b, sigma, dist, q, flags, src, hpart, hgot, harrive;
  int alloc(const Graph* g, uint64_t ns, cudaStream_t s, bool need_q) {
    const uint32_t V = g->V;
    const size_t Vs = std::max<uint32_t>(V, 1);
    const size_t nh = std::max<uint32_t>(std::max(g->n_heavy_in, g->n_heavy_out), 1);
    ZOGCU_TRY(hpart.alloc(nh * kBcBatch * 8, s));
    ZOGCU_TRY(hgot.alloc(nh * 8, s));
    ZOGCU_TRY(harrive.alloc(nh * 4, s));
    ZOGCU_CUDA(cudaMemsetAsync(harrive.ptr, 0, nh * 4, s));
    ZOGCU_TRY(visited.alloc(Vs * 8, s));
    ZOGCU_TRY(masks.alloc(Vs * 8 * (kMaxStoredLevels + 1), s));
    ZOGCU_TRY(sigma.alloc(Vs * 8 * kBcBatch, s));
    ZOGCU_TRY(dist.alloc(Vs * 4 * kBcBatch, s));
    if (need_q) {
      ZOGCU_TRY(q.alloc(Vs * 8 * kBcBatch, s));
      ZOGCU_TRY(mbuf_a.alloc(Vs * 8, s));
      ZOGCU_TRY(mbuf_b.alloc(Vs * 8, s));
    }
    ZOGCU_TRY(flags.alloc(kFlagWords * 4, s));
    ZOGCU_TRY(src.alloc(std::max<uint64_t>(ns, 1) * 4, s));
    return ZOGCU_OK;
  }
  unsigned long long* level(uint32_t l, uint32_t V) const {
    return masks.as<unsigned long long>() + (size_t)(l % (kMaxStoredLevels + 1)) * std::max<uint32_t>(V, 1);
  }
};

// Forward phase of one batch; returns the deepest level reached in *depth.
// Levels are enqueued kLevelChunk at a time (never across a multiple of
// kMaxStoredLevels, where the per-level flag words are reused) and the host
// reads the flags once per chunk.
template <typename OffT>
static int bc_forward_batch(const Graph* g, const OffT* in_off, BcWork& W, uint64_t first, int nb,
                            cudaStream_t s, uint32_t* depth, bool* overflow, uint64_t* launches,
                            unsigned int* h_flags) {
  const uint32_t V = g->V;
  const int grid = bc_grid(bc_forward_kernel<OffT>, V);
  const unsigned long long full = nb == 64 ? ~0ull : ((1ull << nb) - 1);
  ZOGCU_CUDA(cudaMemsetAsync(W.visited.ptr, 0, (size_t)V * 8, s));
  ZOGCU_CUDA(cudaMemsetAsync(W.level(0, V), 0, (size_t)V * 8, s));
  ZOGCU_CUDA(cudaMemsetAsync(W.dist.ptr, 0xFF, (size_t)V * 4 * kBcBatch, s));
  ZOGCU_CUDA(cudaMemsetAsync(W.flags.ptr, 0, kFlagWords * 4, s));
  bc_seed_kernel<<<1, 64, 0, s>>>(W.src.as<uint32_t>() + first, nb, W.visited.as<unsigned long long>(),
                                  W.level(0, V), W.sigma.as<unsigned long long>(), W.dist.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  *launches += 1;
  uint32_t level = 0;
  for (;;) {
    const uint32_t lo = level;
    // flag words of levels lo-64 .. lo-2 are all set; clear them for reuse
    // (the word of level lo-1, which level lo checks, stays set)
    if (lo > 0 && lo % kMaxStoredLevels == 0)
      ZOGCU_CUDA(cudaMemsetAsync(W.flags.ptr, 0, (kMaxStoredLevels - 1) * 4, s));
    const uint32_t hi = std::min<uint32_t>(lo + kLevelChunk, (lo / kMaxStoredLevels + 1) * kMaxStoredLevels);
    for (uint32_t l = lo; l < hi; ++l) {
      bc_forward_kernel<OffT><<<grid, kBcThreads, 0, s>>>(V, in_off, g->in_col.as<uint32_t>(), W.level(l, V),
                                                          W.level(l + 1, V), W.visited.as<unsigned long long>(),
                                                          W.sigma.as<unsigned long long>(), W.dist.as<uint32_t>(),
                                                          full, l, W.flags.as<unsigned int>(),
                                                          g->heavy_in.as<BcHeavy>(), g->n_heavy_in,
                                                          W.hpart.as<unsigned long long>(),
                                                          W.hgot.as<unsigned long long>(), W.harrive.as<unsigned int>(),
                                                          nullptr, nullptr, nullptr);
      ZOGCU_CUDA(cudaGetLastError());
      *launches += 1;
    }
    level = hi;
    ZOGCU_CUDA(cudaMemcpyAsync(h_flags, W.flags.ptr, kFlagWords * 4, cudaMemcpyDeviceToHost, s));
    ZOGCU_CUDA(cudaStreamSynchronize(s));
    if (h_flags[kOverflowFlag]) *overflow = true;
    for (uint32_t l = lo; l < hi; ++l) {
      if (!h_flags[l % kMaxStoredLevels]) {  // level l found nothing: depth l
        *depth = l;
        return ZOGCU_OK;
      }
    }
  }
}


// ---- push levels (direction-optimising forward) ------------------------------
// When the frontier's out-arcs are few against the graph's arcs (level 0, whose
// frontier is the batch's sources, and the sparse levels that follow or end a
// BFS), the level pushes instead of pulling: every frontier vertex v (mask
// m_v) walks its out-arcs, and for each successor w the sources b of m_v not
// yet visited at w get sigma[w][b] += sigma[v][b] (64-bit integer atomics:
// exact, so the order of the additions does not matter and the sums equal the
// pull kernel's, wrap included) and w's next-frontier mask the bits
// (atomicOr).  visited and dist of the new vertices are written afterwards by
// bc_push_finalize, so every push of the level reads the visited masks of the
// level's start.  Each CTA first stages its window of frontier vertices in
// shared memory (compacted from the frontier masks); light vertices are
// walked by one warp each, vertices of more than kPushCtaDegree out-arcs by
// the whole CTA.
constexpr int kPushCtaDegree = 256;

__device__ __forceinline__ unsigned long long* ring_slot(unsigned long long* masks, uint32_t level, uint32_t V) {
  return masks + (size_t)(level % (kMaxStoredLevels + 1)) * V;
}

__device__ __forceinline__ void push_arc(uint32_t v, unsigned long long m, uint32_t w,
                                         const unsigned long long* __restrict__ visited,
                                         unsigned long long* __restrict__ nxt, unsigned long long* __restrict__ sigma,
                                         bool& any_new, bool& ovf) {
  const unsigned long long nb = m & ~visited[w];
  if (!nb) return;
  atomicOr(nxt + w, nb);
  any_new = true;
  for (unsigned long long bb = nb; bb; bb &= bb - 1) {
    const int b = __ffsll((long long)bb) - 1;
    const unsigned long long add = sigma[(uint64_t)v * kBcBatch + b];
    const unsigned long long old = atomicAdd(sigma + (uint64_t)w * kBcBatch + b, add);
    ovf |= old + add < old;
  }
}

template <typename OffT>
__global__ void __launch_bounds__(kBcThreads) bc_push_kernel(uint32_t V, const OffT* __restrict__ out_off,
                                                             const uint32_t* __restrict__ out_col,
                                                             const unsigned long long* __restrict__ visited,
                                                             unsigned long long* __restrict__ sigma,
                                                             unsigned int* __restrict__ flags, const BcLoop* __restrict__ loop,
                                                             unsigned long long* __restrict__ masks) {
  if (!*(volatile const uint32_t*)&loop->active || !*(volatile const uint32_t*)&loop->push) return;
  const uint32_t level = *(volatile const uint32_t*)&loop->level;
  const unsigned long long* __restrict__ cur = ring_slot(masks, level, V);
  unsigned long long* __restrict__ nxt = ring_slot(masks, level + 1, V);
  constexpr int W = kBcThreads / 32;
  __shared__ uint32_t s_v[kBcThreads];
  __shared__ unsigned long long s_m[kBcThreads];
  __shared__ int s_n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool any_new = false, ovf = false;
  for (uint64_t base = (uint64_t)blockIdx.x * kBcThreads; base < V; base += (uint64_t)gridDim.x * kBcThreads) {
    // stage the window's frontier vertices in shared memory
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    const uint64_t vv = base + threadIdx.x;
    const unsigned long long m = vv < V ? cur[vv] : 0ull;
    if (m) {
      const int k = atomicAdd(&s_n, 1);
      s_v[k] = (uint32_t)vv;
      s_m[k] = m;
    }
    __syncthreads();
    const int n = s_n;
    // light vertices: one warp each
    for (int i = warp; i < n; i += W) {
      const uint32_t v = s_v[i];
      const OffT b = __ldg(out_off + v), e = __ldg(out_off + v + 1);
      if ((uint64_t)(e - b) > (uint64_t)kPushCtaDegree) continue;
      for (OffT j = b + lane; j < e; j += 32) push_arc(v, s_m[i], __ldg(out_col + j), visited, nxt, sigma, any_new, ovf);
    }
    // heavy vertices: the whole CTA
    for (int i = 0; i < n; ++i) {
      const uint32_t v = s_v[i];
      const OffT b = __ldg(out_off + v), e = __ldg(out_off + v + 1);
      if ((uint64_t)(e - b) <= (uint64_t)kPushCtaDegree) continue;
      for (OffT j = b + threadIdx.x; j < e; j += kBcThreads)
        push_arc(v, s_m[i], __ldg(out_col + j), visited, nxt, sigma, any_new, ovf);
    }
    __syncthreads();
  }
  if (__any_sync(0xffffffffu, any_new) && lane == 0) flags[level % kMaxStoredLevels] = 1u;
  if (__any_sync(0xffffffffu, ovf) && lane == 0) flags[kOverflowFlag] = 1u;
}

// After a push level: the new vertices' visited bits and dist, and the
// out-arcs of the next frontier.  One warp per 32 vertices.
template <typename OffT>
__global__ void __launch_bounds__(kBcThreads) bc_push_finalize(uint32_t V, const OffT* __restrict__ out_off,
                                                               unsigned long long* __restrict__ visited,
                                                               uint32_t* __restrict__ dist, BcLoop* __restrict__ loop,
                                                               unsigned long long* __restrict__ masks) {
  if (!*(volatile const uint32_t*)&loop->active || !*(volatile const uint32_t*)&loop->push) return;
  const uint32_t level = *(volatile const uint32_t*)&loop->level;
  const unsigned long long* __restrict__ nxt = ring_slot(masks, level + 1, V);
  const int lane = threadIdx.x & 31;
  unsigned long long arcs = 0;
  const uint64_t nw = (uint64_t)gridDim.x * (kBcThreads / 32);
  for (uint64_t g32 = ((uint64_t)blockIdx.x * kBcThreads + threadIdx.x) >> 5; g32 * 32 < V; g32 += nw) {
    const uint64_t w = g32 * 32 + lane;
    const unsigned long long nm = w < V ? nxt[w] : 0ull;
    if (nm) {
      visited[w] |= nm;
      arcs += (unsigned long long)(__ldg(out_off + w + 1) - __ldg(out_off + w));
    }
    for (unsigned bal = __ballot_sync(0xffffffffu, nm != 0); bal; bal &= bal - 1) {
      const int k = __ffs(bal) - 1;
      const unsigned long long mk = __shfl_sync(0xffffffffu, nm, k);
      const uint64_t wk = g32 * 32 + k;
      if ((mk >> lane) & 1ull) dist[wk * kBcBatch + lane] = level + 1;
      if ((mk >> (lane + 32)) & 1ull) dist[wk * kBcBatch + lane + 32] = level + 1;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) arcs += __shfl_xor_sync(0xffffffffu, arcs, o);
  if (lane == 0 && arcs) atomicAdd(&loop->next_arcs, arcs);
}

// Before a push level: its next-frontier masks start at zero (a pull level
// writes every vertex's mask itself).
__global__ void bc_level_prep(uint32_t V, const BcLoop* __restrict__ loop, unsigned long long* __restrict__ masks) {
  if (!*(volatile const uint32_t*)&loop->active || !*(volatile const uint32_t*)&loop->push) return;
  const uint32_t level = *(volatile const uint32_t*)&loop->level;
  unsigned long long* nxt = ring_slot(masks, level + 1, V);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V; i += (uint64_t)gridDim.x * blockDim.x)
    nxt[i] = 0ull;
}

// Resets one batch's state: visited and level-0 masks zero, dist all
// unreached, the level flags zero (the overflow word is kept), loop state zero.
__global__ void bc_batch_reset(uint32_t V, unsigned long long* __restrict__ visited,
                               unsigned long long* __restrict__ mask0, uint32_t* __restrict__ dist,
                               unsigned long long* __restrict__ sigma, unsigned int* __restrict__ flags,
                               BcLoop* __restrict__ loop, uint32_t push0) {
  // the lane's batch comes from its cursor; a slot past the call's sources
  // is empty and every kernel of it returns at once
  const uint64_t first = (uint64_t)*(volatile const uint32_t*)&loop->batch * kBcBatch;
  const uint64_t ns = *(volatile const unsigned long long*)&loop->ns;
  if (first >= ns) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      loop->active = 0u;
      loop->level = loop->depth = loop->blevel = 0u;
      loop->push = 0u;
    }
    return;
  }
  const uint64_t n = (uint64_t)V * kBcBatch;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    dist[i] = kUnreached;
    sigma[i] = 0ull;  // push levels add into sigma
    if (i < V) {
      visited[i] = 0ull;
      mask0[i] = 0ull;
    }
  }
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i < kMaxStoredLevels; i += blockDim.x) flags[i] = 0u;
    if (threadIdx.x == 0) {
      const uint64_t nb = ns - first < (uint64_t)kBcBatch ? ns - first : (uint64_t)kBcBatch;
      loop->active = 1u;
      loop->full = nb == 64 ? ~0ull : ((1ull << nb) - 1ull);
      loop->level = 0u;
      loop->depth = 0u;
      loop->blevel = 0u;
      loop->push = push0;  // level 0: the frontier is the batch's sources
      loop->next_arcs = 0ull;
    }
  }
}

// The batch's sources into the level-0 frontier (sigma 1, dist 0).
__global__ void bc_seed_loop(const uint32_t* __restrict__ sources, const BcLoop* __restrict__ loop,
                             unsigned long long* visited, unsigned long long* front, unsigned long long* sigma,
                             uint32_t* dist) {
  if (!*(volatile const uint32_t*)&loop->active) return;
  const uint64_t first = (uint64_t)loop->batch * kBcBatch;
  const uint64_t b = threadIdx.x;
  if (first + b < loop->ns && b < (uint64_t)kBcBatch) {
    const uint64_t s = sources[first + b];
    atomicOr(visited + s, 1ull << b);
    atomicOr(front + s, 1ull << b);
    sigma[s * kBcBatch + b] = 1ull;
    dist[s * kBcBatch + b] = 0u;
  }
}

// After forward level l: if it discovered nothing the BFS depth is l -- the
// backward sweep starts there and the forward loop ends; otherwise the next
// level follows (and the flag words of the previous 63 levels are cleared when
// the ring of flag words wraps, as the host loop did).  One thread.
__global__ void bc_fwd_advance(BcLoop* __restrict__ loop, unsigned int* __restrict__ flags,
                               uint32_t* __restrict__ depths, unsigned long long cond, unsigned long long arcs,
                               uint32_t push_ratio) {
  if (threadIdx.x != 0) return;
  if (!loop->active) {  // an empty slot: no levels
    cudaGraphSetConditional(cond, 0u);
    return;
  }
  const uint32_t l = loop->level;
  // the next level pushes when its frontier's out-arcs, times push_ratio,
  // stay below the graph's arcs (push_ratio 0: every level pulls)
  const unsigned long long na = loop->next_arcs;
  loop->next_arcs = 0ull;
  loop->push = (push_ratio && na * push_ratio < arcs) ? 1u : 0u;
  if (flags[l % kMaxStoredLevels] == 0u) {
    loop->depth = l;
    loop->blevel = l;
    if (l > loop->max_depth) loop->max_depth = l;
    depths[loop->batch] = l;
    cudaGraphSetConditional(cond, 0u);
    return;
  }
  const uint32_t nl = l + 1;
  if (nl % kMaxStoredLevels == 0)
    for (int i = 0; i < kMaxStoredLevels - 1; ++i) flags[i] = 0u;
  loop->level = nl;
}

// After backward level l: the next shallower level, or, once level 1 is done
// (a batch of depth 0 or an empty slot has none), the end of the loop and the
// lane's cursor moved to its next batch.  One thread.
__global__ void bc_bwd_advance(BcLoop* __restrict__ loop, unsigned long long cond) {
  if (threadIdx.x != 0) return;
  const uint32_t b = loop->blevel;
  if (b <= 1u) {
    loop->blevel = 0u;
    loop->batch += loop->nlanes;
    cudaGraphSetConditional(cond, 0u);
  } else {
    loop->blevel = b - 1u;
  }
}

// d_bc[v] = sum over the lanes of their scores, in lane order.
__global__ void k_bc_sum_lanes(double* __restrict__ out, const double* __restrict__ lanes, int nlanes, uint32_t V) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int w = 0; w < nlanes; ++w) t += lanes[(size_t)w * V + v];
    out[v] = t;
  }
}

// Batches of kBcBatch sources are dealt to lanes (batch b to lane b % lanes;
// up to kBcLanes, as many as a quarter of the device memory holds), each with
// its own workspace and score vector.  The batches run as CUDA graphs: every
// lane is a chain of K batch slots -- reset, seed, a while loop of forward
// levels (each level's kernels followed by a one-thread kernel that ends the
// loop when the level discovered nothing and otherwise chooses the next
// level's direction), a while loop of backward levels from that depth up to
// level 1 -- and the lanes' chains are independent branches, so one lane's
// levels fill the SMs another's finishing level frees.  A slot takes its batch
// from the lane's cursor in device memory (lane w starts at batch w and steps
// by the lane count), so one instantiated graph serves any number of sources:
// the call launches it until every batch has run, and a slot past the last
// batch returns at once.  The workspaces and the instantiated graphs stay with
// the graph resource for later calls (a concurrent call on the same graph
// builds its own).  No host synchronisation happens between batches or levels.
// The lanes' score vectors are added in lane order at the end, so the result
// is deterministic.  ZOGCU_BC_STREAMS=<k> sets the lane count.
constexpr int kBcMaxLanes = 8;
constexpr int kBcLanes = 8;
constexpr int kBcSlots = 8;  // batch slots per lane in one graph
constexpr uint32_t kBcPushRatio = 16;

struct BcExec {
  int lanes = 0, slots = 0;
  uint32_t push_ratio = 0;
  cudaGraphExec_t exec = nullptr;
};

struct BcCache {
  std::mutex mu;
  int lanes = 0;          // lanes whose workspaces exist
  uint64_t src_cap = 0;   // sources the source array holds
  uint64_t batch_cap = 0; // batches the depth array holds
  DevArray visited[kBcMaxLanes], masks[kBcMaxLanes], mbuf_a[kBcMaxLanes], mbuf_b[kBcMaxLanes], sigma[kBcMaxLanes],
      dist[kBcMaxLanes], q[kBcMaxLanes], flags[kBcMaxLanes], hpart[kBcMaxLanes], hgot[kBcMaxLanes],
      harrive[kBcMaxLanes];
  DevArray scores, loops, src, depths;
  std::vector<BcExec> execs;
  void drop_execs() {
    for (auto& e : execs)
      if (e.exec) cudaGraphExecDestroy(e.exec);
    execs.clear();
  }
  ~BcCache() { drop_execs(); }
};

// Lane workspaces for `lanes` lanes of graph g, a source array of at least ns
// and a depth array of at least nb batches; any reallocation drops the
// instantiated graphs (they hold the old addresses).
static int bc_cache_size(const Graph* g, BcCache& C, int lanes, uint64_t ns, uint64_t nb, cudaStream_t s) {
  const size_t Vs = std::max<uint32_t>(g->V, 1);
  const size_t nh = std::max<uint32_t>(std::max(g->n_heavy_in, g->n_heavy_out), 1);
  if (lanes > C.lanes) {
    C.drop_execs();
    for (int w = C.lanes; w < lanes; ++w) {
      ZOGCU_TRY(C.hpart[w].alloc(nh * kBcBatch * 8));
      ZOGCU_TRY(C.hgot[w].alloc(nh * 8));
      ZOGCU_TRY(C.harrive[w].alloc(nh * 4));
      ZOGCU_CUDA(cudaMemsetAsync(C.harrive[w].ptr, 0, nh * 4, s));
      ZOGCU_TRY(C.visited[w].alloc(Vs * 8));
      ZOGCU_TRY(C.masks[w].alloc(Vs * 8 * (kMaxStoredLevels + 1)));
      ZOGCU_TRY(C.sigma[w].alloc(Vs * 8 * kBcBatch));
      ZOGCU_TRY(C.dist[w].alloc(Vs * 4 * kBcBatch));
      ZOGCU_TRY(C.q[w].alloc(Vs * 8 * kBcBatch));
      ZOGCU_TRY(C.mbuf_a[w].alloc(Vs * 8));
      ZOGCU_TRY(C.mbuf_b[w].alloc(Vs * 8));
      ZOGCU_TRY(C.flags[w].alloc(kFlagWords * 4));
    }
    ZOGCU_TRY(C.scores.alloc((size_t)lanes * Vs * 8));
    ZOGCU_TRY(C.loops.alloc(sizeof(BcLoop) * kBcMaxLanes));
    C.lanes = lanes;
  }
  if (ns > C.src_cap) {
    C.drop_execs();
    const uint64_t cap = std::max<uint64_t>((ns + 4095) / 4096 * 4096, 4096);
    ZOGCU_TRY(C.src.alloc(cap * 4));
    C.src_cap = cap;
  }
  if (nb > C.batch_cap) {
    C.drop_execs();
    const uint64_t cap = std::max<uint64_t>((nb + 1023) / 1024 * 1024, 1024);
    ZOGCU_TRY(C.depths.alloc(cap * 4));
    C.batch_cap = cap;
  }
  return ZOGCU_OK;
}

static int bc_kernel_node(cudaGraph_t graph, cudaGraphNode_t* node, const cudaGraphNode_t* deps, size_t ndeps,
                          const void* fn, unsigned grid, unsigned threads, void** args) {
  cudaKernelNodeParams kp = {};
  kp.func = const_cast<void*>(fn);
  kp.gridDim = dim3(grid);
  kp.blockDim = dim3(threads);
  kp.kernelParams = args;
  ZOGCU_CUDA(cudaGraphAddKernelNode(node, graph, deps, ndeps, &kp));
  return ZOGCU_OK;
}

// A conditional while node after `deps`; its body graph is returned in *body.
static int bc_while_node(cudaGraph_t graph, cudaGraphNode_t* node, const cudaGraphNode_t* deps, size_t ndeps,
                         cudaGraphConditionalHandle* h, cudaGraph_t* body) {
  ZOGCU_CUDA(cudaGraphConditionalHandleCreate(h, graph, 1u, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = *h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  ZOGCU_CUDA(cudaGraphAddNode(node, graph, deps, ndeps, &cp));
  *body = cp.conditional.phGraph_out[0];
  return ZOGCU_OK;
}

// The graph of `lanes` chains of `slots` batch slots over the cache's arrays.
template <typename OffT>
static int bc_build_exec(const Graph* g, const OffT* in_off, const OffT* out_off, BcCache& C, int lanes, int slots,
                         uint32_t push_ratio, cudaGraphExec_t* out) {
  uint32_t V = g->V;
  const unsigned fgrid = (unsigned)bc_grid(bc_forward_kernel<OffT>, V);
  const unsigned bgrid = (unsigned)bc_grid(bc_backward_kernel<OffT>, V);
  const unsigned pgrid = (unsigned)bc_grid(bc_push_kernel<OffT>, V);
  const unsigned rgrid = std::max<unsigned>(1u, std::min<unsigned>((unsigned)(((uint64_t)V * kBcBatch + 255) / 256),
                                                                   (unsigned)sm_count() * 8));
  const unsigned zgrid = std::max<unsigned>(1u, std::min<unsigned>((unsigned)(((uint64_t)V + 255) / 256),
                                                                   (unsigned)sm_count() * 8));
  uint32_t push0 = push_ratio ? 1u : 0u;
  cudaGraph_t graph = nullptr;
  ZOGCU_CUDA(cudaGraphCreate(&graph, 0));
  struct GraphGuard {
    cudaGraph_t gr;
    ~GraphGuard() { cudaGraphDestroy(gr); }
  } guard{graph};
  for (int w = 0; w < lanes; ++w) {
    BcLoop* loop = C.loops.as<BcLoop>() + w;
    const BcLoop* cloop = loop;
    unsigned long long* visited = C.visited[w].as<unsigned long long>();
    unsigned long long* masks = C.masks[w].as<unsigned long long>();
    unsigned long long* mask0 = masks;  // level 0's slot of the ring
    unsigned long long* sigma = C.sigma[w].as<unsigned long long>();
    uint32_t* dist = C.dist[w].as<uint32_t>();
    unsigned int* flags = C.flags[w].as<unsigned int>();
    const uint32_t* src = C.src.as<uint32_t>();
    uint32_t* depths = C.depths.as<uint32_t>();
    double* scores = C.scores.as<double>() + (size_t)w * std::max<uint32_t>(V, 1);
    cudaGraphNode_t tail = nullptr;
    for (int k = 0; k < slots; ++k) {
      const cudaGraphNode_t* dep = tail ? &tail : nullptr;
      const size_t ndep = tail ? 1 : 0;
      cudaGraphNode_t n_reset, n_seed;
      void* reset_args[] = {&V, &visited, &mask0, &dist, &sigma, &flags, &loop, &push0};
      ZOGCU_TRY(bc_kernel_node(graph, &n_reset, dep, ndep, (const void*)bc_batch_reset, rgrid, 256, reset_args));
      void* seed_args[] = {(void*)&src, (void*)&cloop, &visited, &mask0, &sigma, &dist};
      ZOGCU_TRY(bc_kernel_node(graph, &n_seed, &n_reset, 1, (const void*)bc_seed_loop, 1, 64, seed_args));
      // forward levels: prep (zero the next masks of a push level) -> pull ->
      // push -> finalize -> advance
      cudaGraphNode_t n_fwd;
      cudaGraphConditionalHandle hf;
      cudaGraph_t fbody;
      ZOGCU_TRY(bc_while_node(graph, &n_fwd, &n_seed, 1, &hf, &fbody));
      {
        const uint32_t* col = g->in_col.as<uint32_t>();
        const unsigned long long* fcur = nullptr;
        unsigned long long* fnxt = nullptr;
        uint32_t level0 = 0;
        unsigned long long full = 0;
        const BcHeavy* heavy = g->heavy_in.as<BcHeavy>();
        uint32_t nheavy = g->n_heavy_in;
        unsigned long long* hpart = C.hpart[w].as<unsigned long long>();
        unsigned long long* hgot = C.hgot[w].as<unsigned long long>();
        unsigned int* harrive = C.harrive[w].as<unsigned int>();
        void* fargs[] = {&V, (void*)&in_off, (void*)&col, (void*)&fcur, &fnxt, &visited, &sigma, &dist, &full,
                         &level0, &flags, (void*)&heavy, &nheavy, &hpart, &hgot, &harrive, (void*)&cloop, &masks,
                         (void*)&out_off};
        const uint32_t* ocol = g->out_col.as<uint32_t>();
        const unsigned long long* cvisited = visited;
        void* pargs[] = {&V, (void*)&out_off, (void*)&ocol, (void*)&cvisited, &sigma, &flags, (void*)&cloop, &masks};
        void* prep_args[] = {&V, (void*)&cloop, &masks};
        void* fin_args[] = {&V, (void*)&out_off, &visited, &dist, &loop, &masks};
        cudaGraphNode_t k0, k1, k2, k3, k4;
        ZOGCU_TRY(bc_kernel_node(fbody, &k0, nullptr, 0, (const void*)bc_level_prep, zgrid, 256, prep_args));
        ZOGCU_TRY(bc_kernel_node(fbody, &k1, &k0, 1, (const void*)bc_forward_kernel<OffT>, fgrid, kBcThreads, fargs));
        ZOGCU_TRY(bc_kernel_node(fbody, &k2, &k1, 1, (const void*)bc_push_kernel<OffT>, pgrid, kBcThreads, pargs));
        ZOGCU_TRY(bc_kernel_node(fbody, &k3, &k2, 1, (const void*)bc_push_finalize<OffT>, zgrid, kBcThreads, fin_args));
        unsigned long long cond = hf;
        unsigned long long arcs = g->E;
        uint32_t ratio = push_ratio;
        void* aargs[] = {&loop, &flags, &depths, &cond, &arcs, &ratio};
        ZOGCU_TRY(bc_kernel_node(fbody, &k4, &k3, 1, (const void*)bc_fwd_advance, 1, 32, aargs));
      }
      // backward levels, depth .. 1
      cudaGraphNode_t n_bwd;
      cudaGraphConditionalHandle hb;
      cudaGraph_t bbody;
      ZOGCU_TRY(bc_while_node(graph, &n_bwd, &n_fwd, 1, &hb, &bbody));
      {
        const uint32_t* col = g->out_col.as<uint32_t>();
        const unsigned long long* ml = nullptr;
        const unsigned long long* mn = nullptr;
        unsigned long long* mo = nullptr;
        double* q = C.q[w].as<double>();
        uint32_t level0 = 0;
        int last0 = 0;
        const BcHeavy* heavy = g->heavy_out.as<BcHeavy>();
        uint32_t nheavy = g->n_heavy_out;
        double* hpart = reinterpret_cast<double*>(C.hpart[w].ptr);
        unsigned int* harrive = C.harrive[w].as<unsigned int>();
        unsigned long long* ma = C.mbuf_a[w].as<unsigned long long>();
        unsigned long long* mb = C.mbuf_b[w].as<unsigned long long>();
        const uint32_t* cdist = dist;
        const unsigned long long* csigma = sigma;
        void* bargs[] = {&V, (void*)&out_off, (void*)&col, (void*)&ml, (void*)&mn, &mo, (void*)&cdist,
                         (void*)&csigma, &q, &scores, &level0, &last0, (void*)&heavy, &nheavy, &hpart, &harrive,
                         (void*)&cloop, &masks, &ma, &mb};
        cudaGraphNode_t k1, k2;
        ZOGCU_TRY(bc_kernel_node(bbody, &k1, nullptr, 0, (const void*)bc_backward_kernel<OffT>, bgrid, kBcThreads, bargs));
        unsigned long long cond = hb;
        void* aargs[] = {&loop, &cond};
        ZOGCU_TRY(bc_kernel_node(bbody, &k2, &k1, 1, (const void*)bc_bwd_advance, 1, 32, aargs));
      }
      tail = n_bwd;
    }
  }
  ZOGCU_CUDA(cudaGraphInstantiate(out, graph, 0));
  return ZOGCU_OK;
}

template <typename OffT>
static int run_betweenness(Graph* g, const OffT* in_off, const OffT* out_off, const std::vector<uint32_t>& sources,
                           double* d_bc, cudaStream_t s, zogcu_stats* stats) {
  const uint32_t V = g->V;
  const size_t Vs = std::max<uint32_t>(V, 1);
  const uint64_t ns = sources.size();
  PhaseTrace tr("betweenness", s);
  ZOGCU_TRY(ensure_heavy_lists(g, s));
  const uint64_t nbatches = (ns + kBcBatch - 1) / kBcBatch;
  if (nbatches == 0) {
    if (stats) stats->sources = 0;
    return ZOGCU_OK;
  }
  int lanes_max = kBcLanes;
  if (const char* env = std::getenv("ZOGCU_BC_STREAMS")) lanes_max = std::max(1, std::min(kBcMaxLanes, std::atoi(env)));
  {
    // a lane's workspace is about V * 1.8 KB (dist, sigma, q, the mask ring):
    // keep all lanes within a quarter of the device memory (the free figure
    // would not count what the stream-ordered pool keeps in reserve)
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
      const uint64_t per_lane = (uint64_t)Vs * (4 + 8 + 8) * kBcBatch + (uint64_t)Vs * 8 * (kMaxStoredLevels + 4);
      const uint64_t fit = per_lane ? (uint64_t)(total_b / 4) / per_lane : (uint64_t)lanes_max;
      lanes_max = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)lanes_max, fit));
    }
  }
  const int lanes = (int)std::min<uint64_t>((uint64_t)lanes_max, nbatches);
  const int slots = (int)std::min<uint64_t>(kBcSlots, (nbatches + lanes - 1) / lanes);
  uint32_t push_ratio = kBcPushRatio;
  if (const char* env = std::getenv("ZOGCU_BC_PUSH_RATIO")) push_ratio = (uint32_t)std::max(0, std::atoi(env));
  // the graph's cache, or a call-local one when another call holds it
  if (!g->bc_cache) {
    std::lock_guard<std::mutex> lk(g->mu);
    if (!g->bc_cache) g->bc_cache = std::make_shared<BcCache>();
  }
  std::shared_ptr<BcCache> shared = std::static_pointer_cast<BcCache>(g->bc_cache);
  std::unique_lock<std::mutex> held(shared->mu, std::try_to_lock);
  std::unique_ptr<BcCache> local;
  BcCache* C = shared.get();
  if (!held.owns_lock()) {
    local.reset(new BcCache());
    C = local.get();
  }
  ZOGCU_TRY(bc_cache_size(g, *C, lanes_max, ns, nbatches, s));
  // the call's state: sources, zero scores and overflow words, lane cursors
  ZOGCU_CUDA(cudaMemcpyAsync(C->src.ptr, sources.data(), ns * 4, cudaMemcpyHostToDevice, s));
  ZOGCU_CUDA(cudaMemsetAsync(C->scores.ptr, 0, (size_t)lanes * Vs * 8, s));
  for (int w = 0; w < lanes; ++w) ZOGCU_CUDA(cudaMemsetAsync(C->flags[w].ptr, 0, kFlagWords * 4, s));
  std::vector<BcLoop> h_loops(lanes);
  for (int w = 0; w < lanes; ++w) {
    std::memset(&h_loops[w], 0, sizeof(BcLoop));
    h_loops[w].batch = (uint32_t)w;
    h_loops[w].nlanes = (uint32_t)lanes;
    h_loops[w].ns = ns;
  }
  ZOGCU_CUDA(cudaMemcpyAsync(C->loops.ptr, h_loops.data(), sizeof(BcLoop) * lanes, cudaMemcpyHostToDevice, s));
  // the sources and loop copies read host vectors that end with this call
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  tr.mark("workspaces");
  cudaGraphExec_t exec = nullptr;
  for (const auto& e : C->execs)
    if (e.lanes == lanes && e.slots == slots && e.push_ratio == push_ratio) exec = e.exec;
  if (!exec) {
    ZOGCU_TRY(bc_build_exec<OffT>(g, in_off, out_off, *C, lanes, slots, push_ratio, &exec));
    C->execs.push_back(BcExec{lanes, slots, push_ratio, exec});
    tr.mark("graph built and instantiated");
  }
  // one launch runs lanes x slots batches; the cursors carry on between launches
  const uint64_t per_launch = (uint64_t)lanes * slots;
  uint64_t host_launches = 0;
  for (uint64_t done = 0; done < nbatches; done += per_launch) {
    ZOGCU_CUDA(cudaGraphLaunch(exec, s));
    ++host_launches;
  }
  k_bc_sum_lanes<<<std::max<unsigned>(1u, std::min<unsigned>((V + 255) / 256, 148u * 8)), 256, 0, s>>>(
      d_bc, C->scores.as<double>(), lanes, V);
  ZOGCU_CUDA(cudaGetLastError());
  tr.mark("graphs ran");
  // depths, overflow flags and the kernels the graphs ran
  std::vector<uint32_t> h_depth(nbatches);
  ZOGCU_CUDA(cudaMemcpyAsync(h_depth.data(), C->depths.ptr, nbatches * 4, cudaMemcpyDeviceToHost, s));
  std::vector<unsigned int> h_ovf(lanes);
  for (int w = 0; w < lanes; ++w)
    ZOGCU_CUDA(cudaMemcpyAsync(&h_ovf[w], C->flags[w].as<unsigned int>() + kOverflowFlag, 4, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  bool overflow = false;
  for (int w = 0; w < lanes; ++w) overflow |= h_ovf[w] != 0u;
  uint32_t max_depth = 0;
  uint64_t launches = 1;  // the lanes' sum
  for (uint64_t bi = 0; bi < nbatches; ++bi) {
    const uint32_t d = h_depth[bi];
    max_depth = std::max(max_depth, d);
    // reset, seed, (prep, pull, push, finalize, advance) x (depth + 1) forward,
    // (level, advance) x max(depth, 1) backward
    launches += 2 + 5 * ((uint64_t)d + 1) + 2 * std::max<uint64_t>(d, 1);
  }
  // the empty slots of the last launch: reset, seed, one forward and one backward pass
  launches += (host_launches * per_launch - nbatches) * (2 + 5 + 2);
  if (stats) {
    stats->sources = ns;
    stats->max_depth = max_depth;
    stats->sigma_overflow = overflow ? 1u : 0u;
    stats->launches = launches;
    stats->reserved = (uint32_t)host_launches;  // graph launches of the call
  }
  return ZOGCU_OK;
}

static std::vector<uint32_t> live_sources(Graph* g) {
  std::vector<uint32_t> src;
  if (!g->has_deleted) {
    src.resize(g->V);
    for (uint32_t v = 0; v < g->V; ++v) src[v] = v;
    return src;
  }
  std::vector<uint32_t> deg(g->V);
  cudaMemcpy(deg.data(), g->out_deg.ptr, (size_t)g->V * 4, cudaMemcpyDeviceToHost);
  for (uint32_t v = 0; v < g->V; ++v)
    if (deg[v] != kDeletedDegree) src.push_back(v);
  return src;
}

}  // namespace zogcu

using namespace zogcu;

extern "C" {

int zogcu_betweenness_unweighted_ex(zogcu_graph* G, const zogcu_bc_opts* opts, double* out_scores,
                                    zogcu_stats* stats) {
  if (!G) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graph is null");
  if (opts && opts->struct_size != sizeof(zogcu_bc_opts))
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "zogcu_bc_opts.struct_size mismatch");
  Graph* g = &G->g;
  const uint32_t V = g->V;
  if (!out_scores && V) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out_scores is null");
  ZOGCU_CUDA(cudaSetDevice(g->device));
  if (stats) std::memset(stats, 0, sizeof(*stats));
  std::vector<uint32_t> sources;
  if (opts && opts->sources) {
    sources.assign(opts->sources, opts->sources + opts->num_sources);
    for (uint32_t s : sources)
      if (s >= V) return fail(ZOGCU_ERR_NODE_NOT_FOUND, "source id >= node capacity");
  } else {
    sources = live_sources(g);
  }
  const bool dev_out = opts && opts->device_pointers;
  StreamGuard sg;
  ZOGCU_TRY(sg.init(opts ? opts->stream : nullptr));
  DevBuf bc;
  ZOGCU_TRY(bc.alloc((size_t)std::max<uint32_t>(V, 1) * 8, sg.s));
  ZOGCU_CUDA(cudaMemsetAsync(bc.ptr, 0, (size_t)std::max<uint32_t>(V, 1) * 8, sg.s));
  EventTimer tm;
  ZOGCU_TRY(tm.start(sg.s));
  if (V) {
    if (g->offsets32)
      ZOGCU_TRY(run_betweenness<uint32_t>(g, g->in_off32.as<uint32_t>(), g->out_off32.as<uint32_t>(), sources,
                                          bc.as<double>(), sg.s, stats));
    else
      ZOGCU_TRY(run_betweenness<uint64_t>(g, g->in_off64.as<uint64_t>(), g->out_off64.as<uint64_t>(), sources,
                                          bc.as<double>(), sg.s, stats));
  }
  ZOGCU_TRY(tm.stop(sg.s));
  if (V)
    ZOGCU_CUDA(cudaMemcpyAsync(out_scores, bc.ptr, (size_t)V * 8,
                               dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, sg.s));
  ZOGCU_CUDA(cudaStreamSynchronize(sg.s));
  if (stats) stats->elapsed_ms = tm.ms();
  return ZOGCU_OK;
}

int zogcu_betweenness_unweighted(zogcu_graph* G, double* out_scores, zogcu_stats* stats) {
  return zogcu_betweenness_unweighted_ex(G, nullptr, out_scores, stats);
}

int zogcu_bfs_sigma(zogcu_graph* G, const uint32_t* sources, uint64_t num_sources, uint32_t* dist_out,
                    uint64_t* sigma_out, uint32_t* overflow) {
  if (!G) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "graph is null");
  if (num_sources && !sources) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "sources is null");
  Graph* g = &G->g;
  const uint32_t V = g->V;
  for (uint64_t i = 0; i < num_sources; ++i)
    if (sources[i] >= V) return fail(ZOGCU_ERR_NODE_NOT_FOUND, "source id >= node capacity");
  ZOGCU_CUDA(cudaSetDevice(g->device));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(nullptr));
  ZOGCU_TRY(ensure_heavy_lists(g, sg.s));
  BcWork W;
  ZOGCU_TRY(W.alloc(g, num_sources, sg.s, false));
  if (num_sources) ZOGCU_CUDA(cudaMemcpyAsync(W.src.ptr, sources, num_sources * 4, cudaMemcpyHostToDevice, sg.s));
  unsigned int* h_flags = nullptr;
  ZOGCU_CUDA(cudaMallocHost(&h_flags, kFlagWords * 4));
  std::vector<uint32_t> hd((size_t)V * kBcBatch);
  std::vector<unsigned long long> hs((size_t)V * kBcBatch);
  bool ovf = false;
  uint64_t launches = 0;
  int rc = ZOGCU_OK;
  for (uint64_t first = 0; first < num_sources && rc == ZOGCU_OK; first += kBcBatch) {
    const int nb = (int)std::min<uint64_t>(kBcBatch, num_sources - first);
    uint32_t depth = 0;
    rc = g->offsets32 ? bc_forward_batch<uint32_t>(g, g->in_off32.as<uint32_t>(), W, first, nb, sg.s, &depth, &ovf,
                                                   &launches, h_flags)
                      : bc_forward_batch<uint64_t>(g, g->in_off64.as<uint64_t>(), W, first, nb, sg.s, &depth, &ovf,
                                                   &launches, h_flags);
    if (rc != ZOGCU_OK) break;
    if (cudaMemcpy(hd.data(), W.dist.ptr, hd.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hs.data(), W.sigma.ptr, hs.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = fail(ZOGCU_ERR_CUDA, "copy of BFS state failed");
      break;
    }
    for (int b = 0; b < nb; ++b) {
      for (uint32_t v = 0; v < V; ++v) {
        const uint32_t d = hd[(size_t)v * kBcBatch + b];
        if (dist_out) dist_out[(first + b) * V + v] = d;
        if (sigma_out) sigma_out[(first + b) * V + v] = (d == kUnreached) ? 0ull : hs[(size_t)v * kBcBatch + b];
      }
    }
  }
  cudaFreeHost(h_flags);
  if (overflow) *overflow = ovf ? 1u : 0u;
  return rc;
}

}  // extern "C"
