// gnn.cu -- the learned PageRank warm start: a small message-passing network
// whose prediction is only the start vector of the power iteration, which
// then runs to the same residual (so the plain method alone decides the result).
//
// Model (hidden width 64, messages 8 wide; FP32 master weights, BF16 weights
// and BF16 operands in the dense layers, FP32 accumulation everywhere):
//   features  F(v) = [log(1+indeg), log(1+outdeg), outdeg == 0, 1/n]   (FP32)
//   inv(u)    = 1/outdeg(u), 0 for dangling and deleted nodes           (FP32)
//   layer 0   M_0(u) = F(u) inv(u);  A_0(v) = sum_{u in in(v)} M_0(u)
//             H_0 = bf16(relu(bf16(F) Ws_0 + bf16(A_0) Wn_0 + b_0))
//   layer l   M_l(u) = bf16(inv(u) (H_{l-1}(u) U_l));  A_l = sum over in(v)
//             H_l = bf16(relu(H_{l-1} Ws_l + bf16(A_l) Wn_l + b_l)),  l = 1, 2
//   head      y(v) = H_2(v) . w_o + b_o   (a prediction of log(n * pr(v)))
//   start     x0(v) = exp(y(v)) / sum_u exp(y(u))  (positive, sums to 1)
// Each layer's aggregate is the PageRank propagation operator applied to a
// message; the message of layers 1 and 2 is a learned 8-wide projection U_l
// of the hidden state (agg(H) Wn of a full-width layer in the rank-8 form
// agg(H U) Wn), so every arc gathers 16 bytes instead of a 128-byte row, and
// the aggregates that go through HBM are 32 bytes per node.
//
// Kernels (all hand-written):
//   * k_gnn_agg16: the forward aggregate (inference and training) -- arcs cut
//     into 128-arc chunks dealt to warps in a fixed interleaving, each chunk's
//     16-byte messages gathered into shared memory (index loads marked
//     evict-first, message loads evict-last, the next chunk's gathers issued
//     before this chunk's sums) and summed one row per lane;
//   * k_gnn_spmm: the arc-chunked SpMM of the transpose (training);
//   * k_gnn_infer: inference's dense layers with each warp's 16-node hidden
//     tile kept in registers between the two products of a layer (mma.sync);
//   * k_gnn_infer_tc: the same layers on tcgen05 with the accumulators in
//     TMEM, 128-node tiles (opt-in: ZOGCU_GNN_TC=1);
//   * k_gnn_dense0 / k_gnn_dense_mid: training's dense layers on the tensor cores
//     (mma.m16n8k16, BF16 in, FP32 accumulate) fused with their epilogues --
//     bias, ReLU, the BF16 hidden state, the next layer's message (a second
//     product with U) or the head.  A warp owns 16-node tiles; the hidden
//     tile arrives by a TMA tensor load (128-byte swizzle) and the aggregate
//     tile by a bulk copy, both double-buffered on mbarriers, and the new
//     hidden tile leaves by a TMA tensor store from a swizzled staging tile;
//   * training: the data- and weight-gradient kernels of the dense layers and
//     of the message projection, the head, the softmax (FP64), the KL and
//     log-MSE losses, and Adam.  The gradients are checked against a CPU
//     oracle that torch autograd pins.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_bf16.h>

#include "common.cuh"

namespace zogcu {
namespace {

constexpr int kH = 64;     // hidden width
constexpr int kF = 4;      // input features
constexpr int kR = 8;      // message width of layers 1 and 2
constexpr int kLayers = 3;
constexpr uint32_t kGnnMagic = 0x5A4F474E;  // "ZOGN"
constexpr uint32_t kGnnVersion = 2;

// Flat parameter layout: layer 0 [Ws (4 x 64) | Wn (4 x 64) | b (64)];
// layers 1, 2 [U (64 x 8) | Ws (64 x 64) | Wn (8 x 64) | b (64)]; then
// [w_o (64) | b_o].  Row-major (input index first) throughout.
constexpr int layer_in(int l) { return l == 0 ? kF : kH; }
constexpr int layer_msg(int l) { return l == 0 ? kF : kR; }
constexpr int layer_u(int l) { return l == 0 ? 0 : layer_in(l) * layer_msg(l); }
constexpr int layer_size(int l) { return layer_u(l) + layer_in(l) * kH + layer_msg(l) * kH + kH; }
constexpr int layer_offset(int l) { return l == 0 ? 0 : layer_offset(l - 1) + layer_size(l - 1); }
constexpr int ws_offset(int l) { return layer_offset(l) + layer_u(l); }
constexpr int wn_offset(int l) { return ws_offset(l) + layer_in(l) * kH; }
constexpr int bias_offset(int l) { return wn_offset(l) + layer_msg(l) * kH; }
constexpr int kHeadOffset = layer_offset(kLayers);
constexpr int kNumParams = kHeadOffset + kH + 1;
static_assert(kNumParams == 11009, "parameter layout");

constexpr int kTile = 16;                       // nodes per warp tile
constexpr int kDenseWarps = 4;                  // warps per dense CTA
constexpr int kWarpSmem = 8192;                 // per-warp staging area
constexpr uint64_t kWaitLimitNs = 1000000000ull;  // bounded mbarrier waits: 1 s

// ---- features, inverse out-degrees and the layer-0 message ---------------------
__global__ void k_gnn_features(const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ out_deg, uint32_t V,
                               float inv_n, float* __restrict__ F, float* __restrict__ inv_deg,
                               float* __restrict__ M0) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t od = out_deg[v];
    const bool deleted = od == kDeletedDegree;
    const float id = (float)(in_off[v + 1] - in_off[v]);
    const float f0 = deleted ? 0.f : log1pf(id);
    const float f1 = deleted ? 0.f : log1pf((float)od);
    const float f2 = (!deleted && od == 0) ? 1.f : 0.f;
    const float f3 = deleted ? 0.f : inv_n;
    const float iv = (deleted || od == 0) ? 0.f : 1.f / (float)od;
    *reinterpret_cast<float4*>(F + (size_t)v * kF) = make_float4(f0, f1, f2, f3);
    *reinterpret_cast<float4*>(M0 + (size_t)v * kF) = make_float4(f0 * iv, f1 * iv, f2 * iv, f3 * iv);
    inv_deg[v] = iv;
  }
}

// ---- BF16 helpers --------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo in the low half
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t v) { return __uint_as_float(v & 0xFFFF0000u); }
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float to_f32(float x) { return x; }
__device__ __forceinline__ float to_f32(__nv_bfloat16 x) { return __bfloat162float(x); }

// ---- SpMM: Z(v) = sum over row v of X(u)  [* inv(v) when transposed] -----------
// Forward: in-CSR, the messages already carry 1/outdeg of their source.
// Transpose (training): out-CSR, the row sum scaled by inv(v) -- the gradient
// of a message through its 1/outdeg factor.
//
// Work split: the arcs are cut into chunks of kChunk arcs dealt to warps in a
// fixed interleaving (so a hub row is shared by many warps); the first row of
// every chunk is precomputed (k_chunk_rows).  A row that crosses a chunk boundary is added with atomics,
// a row inside one chunk is stored directly.  Each arc's row (D values of T)
// is read 16 bytes per lane by LPA = D*sizeof(T)/16 lanes, and a chunk runs in
// one of two modes:
//   * rows mode (the chunk holds several rows, none long): each group of LPA
//     lanes owns one row and walks its arcs, 32/LPA rows in flight per warp,
//     four independent gathers in flight per group;
//   * arcs mode (one or two rows, or a long segment): the whole warp walks
//     each row's arcs 32/LPA at a time (indices loaded once, coalesced, and
//     broadcast by shuffles), then folds the groups.
// Sums are FP32.  The caller zeroes Z first (rows that hold no arc of any
// chunk are never visited).
constexpr uint32_t kChunk = 128;

__global__ void k_chunk_rows(const uint32_t* __restrict__ off, uint32_t V, uint32_t E, uint32_t chunk,
                             uint32_t* __restrict__ first_row) {
  const uint32_t nchunks = (uint32_t)(((uint64_t)E + chunk - 1) / chunk);
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x) {
    const uint32_t cs = c * chunk;
    uint32_t lo = 0, hi = V;  // the last r < V with off[r] <= cs (off[V] = E > cs)
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (off[mid] <= cs) lo = mid;
      else hi = mid;
    }
    first_row[c] = lo;
  }
}

template <class T, int PER>
__device__ __forceinline__ void add_row(float (&acc)[PER], const uint4 x) {
  if (sizeof(T) == 4) {
    acc[0] += __uint_as_float(x.x);
    acc[1] += __uint_as_float(x.y);
    acc[2] += __uint_as_float(x.z);
    acc[3] += __uint_as_float(x.w);
  } else {
    acc[0] += bf16_lo(x.x);
    acc[1] += bf16_hi(x.x);
    acc[2 % PER] += bf16_lo(x.y);
    acc[3 % PER] += bf16_hi(x.y);
    acc[4 % PER] += bf16_lo(x.z);
    acc[5 % PER] += bf16_hi(x.z);
    acc[6 % PER] += bf16_lo(x.w);
    acc[7 % PER] += bf16_hi(x.w);
  }
}

// adds one row's PER values held by one lane (whole rows are stored: Z starts at zero)
template <int D, int PER>
__device__ __forceinline__ void put_row(float* __restrict__ Z, uint32_t r, int sub, float (&acc)[PER], bool whole) {
  float* z = Z + (size_t)r * D + sub * PER;
  if (whole) {
#pragma unroll
    for (int i = 0; i < PER; i += 4) *reinterpret_cast<float4*>(z + i) = make_float4(acc[i], acc[i + 1], acc[i + 2], acc[i + 3]);
  } else {
    // 16-byte vector reductions (one L2 atomic per four values, z is 16-byte aligned)
#pragma unroll
    for (int i = 0; i < PER; i += 4)
      asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(z + i), "f"(acc[i]), "f"(acc[i + 1]),
                   "f"(acc[i + 2]), "f"(acc[i + 3])
                   : "memory");
  }
}

template <class T, int D>
__global__ void __launch_bounds__(256) k_gnn_spmm(const uint32_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                  const float* __restrict__ inv_deg, const T* __restrict__ X,
                                                  uint32_t V, uint32_t E, int transpose, float* __restrict__ Z,
                                                  uint32_t* __restrict__ next_chunk,
                                                  const uint32_t* __restrict__ first_row) {
  constexpr int PER = 16 / (int)sizeof(T);  // values per lane
  constexpr int LPA = D / PER;              // lanes per arc
  constexpr int APW = 32 / LPA;             // arcs per warp step = rows per warp in rows mode
  static_assert(LPA >= 1 && LPA <= 32 && 32 % LPA == 0, "row width");
  const int lane = threadIdx.x & 31, sub = lane % LPA, grp = lane / LPA;
  const uint4* __restrict__ X16 = reinterpret_cast<const uint4*>(X);
  const uint32_t nchunks = (uint32_t)(((uint64_t)E + kChunk - 1) / kChunk);
  const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nchunks; c += nwarps) {
    const uint32_t cs = c * kChunk, ce = min(cs + kChunk, E);
    for (uint32_t r0 = __ldg(first_row + c); r0 < V;) {
      // rows r0 .. r0+31: lane i holds the start and end of row r0 + i
      const uint32_t ri = r0 + lane;
      const uint32_t rb = ri < V ? __ldg(off + ri) : E;
      const uint32_t re = ri < V ? __ldg(off + ri + 1) : E;
      const bool in = rb < ce;  // row r0 + i starts inside the chunk (lane 0 always)
      const uint32_t mask = __ballot_sync(0xffffffffu, in);
      const int nrows = __popc(mask);
      const uint32_t seg = in ? min(re, ce) - max(rb, cs) : 0u;
      uint32_t longest = seg;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) longest = max(longest, __shfl_xor_sync(0xffffffffu, longest, o));
      if (nrows > 2 && longest <= 48) {
        // rows mode: group grp owns rows r0 + grp, r0 + grp + APW, ...
        // (the groups leave this loop at different times: no shuffles inside)
        for (int q = grp; q < nrows; q += APW) {
          const uint32_t qb = __ldg(off + r0 + q), qe = __ldg(off + r0 + q + 1);
          const uint32_t b = max(qb, cs), e = min(qe, ce);
          float acc[PER];
#pragma unroll
          for (int i = 0; i < PER; ++i) acc[i] = 0.f;
          uint32_t j = b;
          for (; j + 4 <= e; j += 4) {
            uint32_t u[4];
            uint4 x[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) u[k] = __ldg(col + j + k);
#pragma unroll
            for (int k = 0; k < 4; ++k) x[k] = __ldg(X16 + (size_t)u[k] * LPA + sub);
#pragma unroll
            for (int k = 0; k < 4; ++k) add_row<T, PER>(acc, x[k]);
          }
          for (; j < e; ++j) add_row<T, PER>(acc, __ldg(X16 + (size_t)__ldg(col + j) * LPA + sub));
          const uint32_t r = r0 + q;
          if (transpose) {
            const float sc = __ldg(inv_deg + r);
#pragma unroll
            for (int i = 0; i < PER; ++i) acc[i] *= sc;
          }
          put_row<D, PER>(Z, r, sub, acc, qb >= cs && qe <= ce);
        }
        // rows are sync-free in this mode; reconverge before the next ballot
        __syncwarp();
      } else {
        // arcs mode: the warp walks each row in turn
        for (int q = 0; q < nrows; ++q) {
          const uint32_t qb = __shfl_sync(0xffffffffu, rb, q), qe = __shfl_sync(0xffffffffu, re, q);
          const uint32_t b = max(qb, cs), e = min(qe, ce);
          float acc[PER];
#pragma unroll
          for (int i = 0; i < PER; ++i) acc[i] = 0.f;
          for (uint32_t j0 = b; j0 < e; j0 += 32) {
            const uint32_t n = min(32u, e - j0);
            const uint32_t u_l = (uint32_t)lane < n ? __ldg(col + j0 + lane) : 0u;
#pragma unroll 4
            for (uint32_t k = 0; k < n; k += APW) {
              const uint32_t idx = k + grp;
              const uint32_t u = __shfl_sync(0xffffffffu, u_l, idx & 31);
              if (idx < n) add_row<T, PER>(acc, __ldg(X16 + (size_t)u * LPA + sub));
            }
          }
#pragma unroll
          for (int o = LPA; o < 32; o <<= 1)
#pragma unroll
            for (int i = 0; i < PER; ++i) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
          const uint32_t r = r0 + q;
          if (lane < LPA) {
            if (transpose) {
              const float sc = __ldg(inv_deg + r);
#pragma unroll
              for (int i = 0; i < PER; ++i) acc[i] *= sc;
            }
            put_row<D, PER>(Z, r, sub, acc, qb >= cs && qe <= ce);
          }
        }
      }
      if (nrows < 32) break;  // the chunk ended inside these rows
      r0 += 32;
    }
  }
}

// ---- forward aggregate with the messages staged in shared memory ---------------
// Z(v) = sum over the in-arcs u -> v of X(u), every message X(u) 16 bytes (8
// BF16 or 4 FP32 values).  Warps take kAggChunk-arc chunks in a fixed
// interleaving (chunk c goes to warp c mod warps), and a chunk is done in two
// phases.  First every lane loads the
// messages of four of the chunk's arcs (coalesced index loads, 16-byte
// message loads) and writes them to the warp's staging tile in shared memory;
// the next chunk's loads are issued into registers before the current chunk
// is summed, so they are in flight meanwhile.  Then each lane sums one row's
// staged messages in arc order (a row with more than 32 arcs in the chunk is
// summed by the whole warp).  A row inside one chunk is stored; a row that
// crosses a chunk boundary is added with atomics.  The arc indices stream with
// an L2 evict-first policy and skip L1; the messages, which other arcs gather
// again, are loaded with an evict-last policy.  Sums are FP32; Z starts at zero.
constexpr int kAggWarps = 8;
constexpr uint32_t kAggChunk = 128;  // arcs per aggregation chunk: four messages per lane

__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// an arc index: streamed once, so it neither stays in L1 nor displaces messages in L2
__device__ __forceinline__ uint32_t ld_index(const uint32_t* a, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
  return v;
}
// a message: gathered again by other arcs, kept in L2 ahead of the streams
__device__ __forceinline__ uint4 ld_message(const uint4* a, uint64_t pol) {
  uint4 v;
  asm volatile("ld.global.nc.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(a), "l"(pol));
  return v;
}

template <class T, int D>
__global__ void __launch_bounds__(kAggWarps * 32) k_gnn_agg16(const uint32_t* __restrict__ off,
                                                              const uint32_t* __restrict__ col,
                                                              const T* __restrict__ X, uint32_t V, uint32_t E,
                                                              float* __restrict__ Z, uint32_t* __restrict__ next_chunk,
                                                              const uint32_t* __restrict__ first_row) {
  constexpr int PER = 16 / (int)sizeof(T);
  constexpr int K = (int)kAggChunk / 32;  // messages per lane and chunk
  static_assert(PER == D, "one 16-byte message per arc");
  __shared__ __align__(16) uint4 s_stage[kAggWarps][kAggChunk];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint4* __restrict__ X16 = reinterpret_cast<const uint4*>(X);
  const uint64_t pol_idx = l2_evict_first(), pol_msg = l2_evict_last();
  const uint32_t nchunks = (uint32_t)(((uint64_t)E + kAggChunk - 1) / kAggChunk);
  uint4* st = s_stage[warp];
  // chunks are dealt to warps statically (c, c + warps, ...): they all hold
  // kAggChunk arcs, and a shared counter would serialise millions of atomics
  const uint32_t nwarps = gridDim.x * kAggWarps;
  uint32_t next = blockIdx.x * kAggWarps + warp;
  auto take = [&]() {
    const uint32_t c = next;
    next += nwarps;
    return c;
  };
  // the messages of chunk c into registers (issued; used one chunk later)
  auto gather = [&](uint32_t c, uint4 (&v)[K]) {
    const uint32_t cs = c * kAggChunk, ce = min(cs + kAggChunk, E);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const uint32_t j = cs + lane + 32 * k;
      v[k] = j < ce ? ld_message(X16 + ld_index(col + j, pol_idx), pol_msg) : make_uint4(0u, 0u, 0u, 0u);
    }
  };
  // the arc range of row r0 + lane (rows past the end read as empty at E)
  auto row_range = [&](uint32_t r0, uint32_t& rb, uint32_t& re) {
    const uint32_t ri = r0 + lane;
    rb = ri < V ? __ldg(off + ri) : E;
    re = ri < V ? __ldg(off + ri + 1) : E;
  };
  // Chunk c's messages, first row and first 32 row ranges are loaded one
  // chunk ahead, and the first row of the chunk after that two ahead, so a
  // chunk starts summing without waiting on a dependent load chain.
  uint4 v[K];
  uint32_t c = take(), r0c = 0, rbc = E, rec = E;
  if (c < nchunks) {
    gather(c, v);
    r0c = __ldg(first_row + c);
    row_range(r0c, rbc, rec);
  }
  uint32_t cn = take();
  uint32_t r0n = cn < nchunks ? __ldg(first_row + cn) : 0u;
  while (c < nchunks) {
#pragma unroll
    for (int k = 0; k < K; ++k) st[lane + 32 * k] = v[k];
    __syncwarp();
    // in flight while chunk c is summed
    uint32_t rbn = E, ren = E;
    if (cn < nchunks) {
      gather(cn, v);
      row_range(r0n, rbn, ren);
    }
    const uint32_t cnn = take();
    const uint32_t r0nn = cnn < nchunks ? __ldg(first_row + cnn) : 0u;
    const uint32_t cs = c * kAggChunk, ce = min(cs + kAggChunk, E);
    uint32_t rb = rbc, re = rec;
    for (uint32_t r0 = r0c; r0 < V;) {
      const uint32_t ri = r0 + lane;
      const bool in = rb < ce;  // row r0 + lane starts inside the chunk (lane 0 always)
      const int nrows = __popc(__ballot_sync(0xffffffffu, in));
      const uint32_t b0 = max(rb, cs), e0 = in ? min(re, ce) : b0;
      const bool whole = rb >= cs && re <= ce;
      const bool longseg = in && e0 - b0 > 32u;
      if (in && !longseg) {
        float acc[PER];
#pragma unroll
        for (int i = 0; i < PER; ++i) acc[i] = 0.f;
        for (uint32_t j = b0; j < e0; ++j) add_row<T, PER>(acc, st[j - cs]);
        put_row<D, PER>(Z, ri, 0, acc, whole);
      }
      // rows with more than 32 of their arcs in this chunk: the whole warp
      for (unsigned lb = __ballot_sync(0xffffffffu, longseg); lb; lb &= lb - 1) {
        const int q = __ffs(lb) - 1;
        const uint32_t qb = __shfl_sync(0xffffffffu, b0, q), qe = __shfl_sync(0xffffffffu, e0, q);
        const bool qw = __shfl_sync(0xffffffffu, whole ? 1 : 0, q) != 0;
        float acc[PER];
#pragma unroll
        for (int i = 0; i < PER; ++i) acc[i] = 0.f;
        for (uint32_t j = qb + lane; j < qe; j += 32) add_row<T, PER>(acc, st[j - cs]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
          for (int i = 0; i < PER; ++i) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
        if (lane == 0) put_row<D, PER>(Z, r0 + q, 0, acc, qw);
      }
      if (nrows < 32) break;  // the chunk ended inside these rows
      r0 += 32;
      row_range(r0, rb, re);
    }
    __syncwarp();  // every lane is done with the staging tile before it is refilled
    c = cn;
    r0c = r0n;
    rbc = rbn;
    rec = ren;
    cn = cnn;
    r0n = r0nn;
  }
}

// ---- the same aggregate with the gathers copied straight to shared memory ----
// cp.async.cg (16 bytes, through L2 only) puts each message in the warp's
// staging tile with no register round trip and no separate shared-memory
// store; three tiles per warp keep two chunks' gathers in flight while a third
// chunk is summed.  Chunking, row ranges and row sums are k_gnn_agg16's; the
// results differ only where both differ from run to run, in the order of the
// atomic adds of rows spanning three or more chunks.
constexpr int kAggStages = 3;

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
               "l"(gsrc)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <class T, int D>
__global__ void __launch_bounds__(kAggWarps * 32) k_gnn_agg16_async(const uint32_t* __restrict__ off,
                                                                    const uint32_t* __restrict__ col,
                                                                    const T* __restrict__ X, uint32_t V, uint32_t E,
                                                                    float* __restrict__ Z,
                                                                    const uint32_t* __restrict__ first_row) {
  constexpr int PER = 16 / (int)sizeof(T);
  constexpr int K = (int)kAggChunk / 32;  // messages per lane and chunk
  static_assert(PER == D, "one 16-byte message per arc");
  __shared__ __align__(16) uint4 s_stage[kAggWarps][kAggStages][kAggChunk];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint4* __restrict__ X16 = reinterpret_cast<const uint4*>(X);
  const uint64_t pol_idx = l2_evict_first();
  const uint32_t nchunks = (uint32_t)(((uint64_t)E + kAggChunk - 1) / kAggChunk);
  const uint32_t nwarps = gridDim.x * kAggWarps;
  uint32_t next = blockIdx.x * kAggWarps + warp;
  auto take = [&]() {
    const uint32_t c = next;
    next += nwarps;
    return c;
  };
  // chunk c's messages into stage tile b (copies issued, completed later)
  auto issue = [&](uint32_t c, int b) {
    const uint32_t cs = c * kAggChunk, ce = min(cs + kAggChunk, E);
    uint4* st = s_stage[warp][b];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const uint32_t j = cs + lane + 32 * k;
      if (j < ce) cp_async16(st + lane + 32 * k, X16 + ld_index(col + j, pol_idx));
    }
  };
  auto row_range = [&](uint32_t r0, uint32_t& rb, uint32_t& re) {
    const uint32_t ri = r0 + lane;
    rb = ri < V ? __ldg(off + ri) : E;
    re = ri < V ? __ldg(off + ri + 1) : E;
  };
  // the pipeline holds chunk c (summed next), c1 and c2; each chunk's first
  // row is loaded two chunks ahead and its first 32 row ranges one ahead
  uint32_t c = take(), c1 = take();
  uint32_t r0c = 0, rbc = E, rec = E, r0n = 0;
  if (c < nchunks) {
    issue(c, 0);
    r0c = __ldg(first_row + c);
    row_range(r0c, rbc, rec);
  }
  cp_async_commit();
  if (c1 < nchunks) {
    issue(c1, 1);
    r0n = __ldg(first_row + c1);
  }
  cp_async_commit();
  int b = 0;
  while (c < nchunks) {
    const uint32_t c2 = take();
    if (c2 < nchunks) issue(c2, b == 0 ? 2 : b - 1);  // the tile summed last time
    cp_async_commit();
    uint32_t rbn = E, ren = E;
    if (c1 < nchunks) row_range(r0n, rbn, ren);
    const uint32_t r0nn = c2 < nchunks ? __ldg(first_row + c2) : 0u;
    cp_async_wait<2>();  // this lane's copies of chunk c (the oldest of three groups) have landed
    __syncwarp();        // and so have the other lanes'
    const uint4* st = s_stage[warp][b];
    const uint32_t cs = c * kAggChunk, ce = min(cs + kAggChunk, E);
    uint32_t rb = rbc, re = rec;
    for (uint32_t r0 = r0c; r0 < V;) {
      const uint32_t ri = r0 + lane;
      const bool in = rb < ce;  // row r0 + lane starts inside the chunk (lane 0 always)
      const int nrows = __popc(__ballot_sync(0xffffffffu, in));
      const uint32_t b0 = max(rb, cs), e0 = in ? min(re, ce) : b0;
      const bool whole = rb >= cs && re <= ce;
      const bool longseg = in && e0 - b0 > 32u;
      if (in && !longseg) {
        float acc[PER];
#pragma unroll
        for (int i = 0; i < PER; ++i) acc[i] = 0.f;
        for (uint32_t j = b0; j < e0; ++j) add_row<T, PER>(acc, st[j - cs]);
        put_row<D, PER>(Z, ri, 0, acc, whole);
      }
      for (unsigned lb = __ballot_sync(0xffffffffu, longseg); lb; lb &= lb - 1) {
        const int q = __ffs(lb) - 1;
        const uint32_t qb = __shfl_sync(0xffffffffu, b0, q), qe = __shfl_sync(0xffffffffu, e0, q);
        const bool qw = __shfl_sync(0xffffffffu, whole ? 1 : 0, q) != 0;
        float acc[PER];
#pragma unroll
        for (int i = 0; i < PER; ++i) acc[i] = 0.f;
        for (uint32_t j = qb + lane; j < qe; j += 32) add_row<T, PER>(acc, st[j - cs]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
          for (int i = 0; i < PER; ++i) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
        if (lane == 0) put_row<D, PER>(Z, r0 + q, 0, acc, qw);
      }
      if (nrows < 32) break;  // the chunk ended inside these rows
      r0 += 32;
      row_range(r0, rb, re);
    }
    __syncwarp();  // every lane is done with the tile before it is refilled
    c = c1;
    c1 = c2;
    b = b == 2 ? 0 : b + 1;
    r0c = r0n;
    rbc = rbn;
    rec = ren;
    r0n = r0nn;
  }
  cp_async_wait<0>();
}

// ---- tensor-core, TMA and mbarrier primitives --------------------------------
__device__ __forceinline__ void mma_bf16_16x8x16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                                 uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void ldmatrix_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// waits for the barrier's phase; the hardware may suspend the thread for a
// while inside one try_wait, so the wake-up follows the phase change at once
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// bounded wait: false when the phase did not complete within kWaitLimitNs of
// the global timer
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > kWaitLimitNs) return false;
  return true;
}
__device__ __forceinline__ void tma_load_rows(void* dst, const CUtensorMap* map, int row, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(0), "r"(row), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tma_store_rows(const CUtensorMap* map, const void* src, int row) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(map), "r"(0),
               "r"(row), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// A 16-node tile of 64 BF16 values per node as TMA lands it with the 128-byte
// swizzle: node r's 16-byte chunk c sits at r*128 + ((c ^ (r & 7)) * 16)
// (the buffer is 1024-byte aligned).
__device__ __forceinline__ uint32_t swz(uint32_t base, int r, int c) {
  return base + (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4));
}

// Weight fragments of the dense product in mma B-fragment order:
// frag[ks][nt][lane] = (W[k0][n], W[k0+1][n]), (W[k0+8][n], W[k0+9][n]) with
// n = nt*8 + lane/4, k0 = ks*16 + 2*(lane%4); rows k of the stacked [Ws; Wn]
// past its end are zero.  One 8-byte shared load per mma, conflict-free.
__device__ void load_dense_frags(uint2* frag, int ksteps, const __nv_bfloat16* __restrict__ ws, int din,
                                 const __nv_bfloat16* __restrict__ wn, int dmsg) {
  const int K = din + dmsg;
  for (int i = threadIdx.x; i < ksteps * 8 * 32; i += blockDim.x) {
    const int ks = i / 256, nt = (i / 32) % 8, l = i % 32;
    const int n = nt * 8 + (l >> 2), k0 = ks * 16 + (l & 3) * 2;
    auto wk = [&](int k) {
      if (k < din) return __bfloat162float(ws[(size_t)k * kH + n]);
      if (k < K) return __bfloat162float(wn[(size_t)(k - din) * kH + n]);
      return 0.f;
    };
    frag[i] = make_uint2(pack_bf16x2(wk(k0), wk(k0 + 1)), pack_bf16x2(wk(k0 + 8), wk(k0 + 9)));
  }
}
// U (64 x 8) as B fragments of the message product: frag[ks][lane], 4 k-steps
__device__ void load_msg_frags(uint2* frag, const __nv_bfloat16* __restrict__ u) {
  for (int i = threadIdx.x; i < 4 * 32; i += blockDim.x) {
    const int ks = i / 32, l = i % 32;
    const int n = l >> 2, k0 = ks * 16 + (l & 3) * 2;
    auto uk = [&](int k) { return __bfloat162float(u[(size_t)k * kR + n]); };
    frag[i] = make_uint2(pack_bf16x2(uk(k0), uk(k0 + 1)), pack_bf16x2(uk(k0 + 8), uk(k0 + 9)));
  }
}

// Shared epilogue of a 16-node tile (rows r0 .. r0+15; lane = 4g + t holds
// rows g and g+8, columns nt*8 + 2t, +1 of every n-tile):
//   h = bf16(relu(acc + b)); optionally H out by a TMA store of a swizzled
//   staging tile; then either the next message M = bf16(inv * (h U)) or the
//   head y = h . w_o + b_o.
struct DenseOut {
  const CUtensorMap* map_h;     // hidden-state output (null: not stored)
  const uint2* ufrag;           // message projection (null: last layer)
  const float* bias;            // 64 (shared)
  const float* wo;              // 65 (shared; last layer)
  const float* inv;             // 1/outdeg
  __nv_bfloat16* M;             // next message, V x 8
  float* y;                     // head output, V
  uint32_t V;
};

__device__ __forceinline__ void dense_epilogue(const DenseOut& o, float (&acc)[8][4], uint32_t r0,
                                               unsigned char* stage, int lane) {
  const int g = lane >> 2, t = lane & 3;
  uint32_t hp[8][2];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int c = nt * 8 + t * 2;
    const float b0 = o.bias[c], b1 = o.bias[c + 1];
    hp[nt][0] = pack_bf16x2(fmaxf(acc[nt][0] + b0, 0.f), fmaxf(acc[nt][1] + b1, 0.f));
    hp[nt][1] = pack_bf16x2(fmaxf(acc[nt][2] + b0, 0.f), fmaxf(acc[nt][3] + b1, 0.f));
  }
  if (o.map_h) {
    // the previous tile's store must have read the staging tile
    if (lane == 0) bulk_wait_read_all();
    __syncwarp();
    const uint32_t sb = smem_u32(stage);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      asm volatile("st.shared.b32 [%0], %1;\n" ::"r"(swz(sb, g, nt) + 4 * t), "r"(hp[nt][0]) : "memory");
      asm volatile("st.shared.b32 [%0], %1;\n" ::"r"(swz(sb, g + 8, nt) + 4 * t), "r"(hp[nt][1]) : "memory");
    }
    fence_async_smem();
    __syncwarp();
    if (lane == 0) {
      tma_store_rows(o.map_h, stage, (int)r0);
      bulk_commit();
    }
  }
  const uint32_t ra = r0 + g, rb = r0 + g + 8;
  if (o.ufrag) {
    float m[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const uint2 bb = o.ufrag[kk * 32 + lane];
      mma_bf16_16x8x16(m, hp[2 * kk][0], hp[2 * kk][1], hp[2 * kk + 1][0], hp[2 * kk + 1][1], bb.x, bb.y);
    }
    if (ra < o.V) {
      const float s = __ldg(o.inv + ra);
      *reinterpret_cast<uint32_t*>(o.M + (size_t)ra * kR + 2 * t) = pack_bf16x2(m[0] * s, m[1] * s);
    }
    if (rb < o.V) {
      const float s = __ldg(o.inv + rb);
      *reinterpret_cast<uint32_t*>(o.M + (size_t)rb * kR + 2 * t) = pack_bf16x2(m[2] * s, m[3] * s);
    }
  } else {
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = nt * 8 + t * 2;
      s0 += bf16_lo(hp[nt][0]) * o.wo[c] + bf16_hi(hp[nt][0]) * o.wo[c + 1];
      s1 += bf16_lo(hp[nt][1]) * o.wo[c] + bf16_hi(hp[nt][1]) * o.wo[c + 1];
    }
    s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
    s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
    if (t == 0) {
      if (ra < o.V) o.y[ra] = s0 + o.wo[kH];
      if (rb < o.V) o.y[rb] = s1 + o.wo[kH];
    }
  }
}

// Shared-memory layout of the dense kernels: kDenseWarps per-warp areas of
// kWarpSmem bytes (1024-aligned) -- [x tile 0 | x tile 1 | H staging | aggregate
// tile 0 | aggregate tile 1 | 2 mbarriers] -- then the weight fragments, U
// fragments, bias and head.
constexpr int kXBytes = kTile * kH * 2;   // 2048
constexpr int kABytes = kTile * kR * 4;   // 512
constexpr int kDenseFragBytes = 5 * 8 * 32 * 8;
constexpr int kMsgFragBytes = 4 * 32 * 8;
constexpr size_t kDenseSmem = 1024 + kDenseWarps * kWarpSmem + kDenseFragBytes + kMsgFragBytes + (kH + kH + 1) * 4;

struct DenseSmem {
  unsigned char* warp_area;
  uint2* frag;
  uint2* ufrag;
  float* bias;
  float* wo;
};
__device__ __forceinline__ DenseSmem dense_smem(unsigned char* raw) {
  DenseSmem d;
  const uint32_t a = smem_u32(raw);
  d.warp_area = raw + (((a + 1023u) & ~1023u) - a);
  d.frag = reinterpret_cast<uint2*>(d.warp_area + kDenseWarps * kWarpSmem);
  d.ufrag = d.frag + kDenseFragBytes / 8;
  d.bias = reinterpret_cast<float*>(d.ufrag + kMsgFragBytes / 8);
  d.wo = d.bias + kH;
  return d;
}

// Layer 0: [F | A_0] (4 + 4 FP32 values per node, read directly; one k-step)
// times [Ws_0; Wn_0], then the epilogue (H_0 by TMA store, M_1).
__global__ void __launch_bounds__(kDenseWarps * 32) k_gnn_dense0(const __grid_constant__ CUtensorMap map_h,
                                                                  const float* __restrict__ F,
                                                                  const float* __restrict__ A0,
                                                                  const __nv_bfloat16* __restrict__ w,
                                                                  const float* __restrict__ inv, uint32_t V,
                                                                  uint32_t ntiles, __nv_bfloat16* __restrict__ M1) {
  extern __shared__ unsigned char smem_raw[];
  const DenseSmem S = dense_smem(smem_raw);
  load_dense_frags(S.frag, 1, w + ws_offset(0), kF, w + wn_offset(0), kF);
  load_msg_frags(S.ufrag, w + layer_offset(1));
  for (int i = threadIdx.x; i < kH; i += blockDim.x) S.bias[i] = __bfloat162float(w[bias_offset(0) + i]);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  unsigned char* stage = S.warp_area + warp * kWarpSmem + 2 * kXBytes;
  DenseOut o{&map_h, S.ufrag, S.bias, nullptr, inv, M1, nullptr, V};
  for (uint32_t tile = blockIdx.x * kDenseWarps + warp; tile < ntiles; tile += gridDim.x * kDenseWarps) {
    const uint32_t r0 = tile * kTile, ra = r0 + g, rb = ra + 8;
    // k = 2t, 2t+1: features for t < 2, aggregate for t = 2, 3; k >= 8 zero
    const float* srca = t < 2 ? F + (size_t)ra * kF + 2 * t : A0 + (size_t)ra * kF + 2 * (t - 2);
    const float* srcb = t < 2 ? F + (size_t)rb * kF + 2 * t : A0 + (size_t)rb * kF + 2 * (t - 2);
    const float2 va = ra < V ? __ldg(reinterpret_cast<const float2*>(srca)) : make_float2(0.f, 0.f);
    const float2 vb = rb < V ? __ldg(reinterpret_cast<const float2*>(srcb)) : make_float2(0.f, 0.f);
    const uint32_t a0 = pack_bf16x2(va.x, va.y), a1 = pack_bf16x2(vb.x, vb.y);
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
      const uint2 bb = S.frag[nt * 32 + lane];
      mma_bf16_16x8x16(acc[nt], a0, a1, 0u, 0u, bb.x, bb.y);
    }
    dense_epilogue(o, acc, r0, stage, lane);
    __syncwarp();
  }
  if (lane == 0) bulk_wait_all();
}

// Layers 1 and 2: [H_{l-1} | A_l] (64 BF16 + 8 FP32 values per node; five
// k-steps) times [Ws_l; Wn_l].  Per warp, the next tile's hidden rows (TMA
// tensor load, 128-byte swizzle, fragments by ldmatrix) and aggregates (bulk
// copy) land while the current tile computes.  LAST: the head instead of a
// next message, and H_2 is stored only when store_h (training).
template <int LAST>
__global__ void __launch_bounds__(kDenseWarps * 32) k_gnn_dense_mid(
    const __grid_constant__ CUtensorMap map_x, const __grid_constant__ CUtensorMap map_h,
    const float* __restrict__ A, const __nv_bfloat16* __restrict__ w, int layer, const float* __restrict__ inv,
    uint32_t V, uint32_t ntiles, int store_h, __nv_bfloat16* __restrict__ M_next, float* __restrict__ y,
    unsigned int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  const DenseSmem S = dense_smem(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  // per-warp area: x tiles at wa + b*kXBytes, the H staging tile, aggregate
  // tiles at abase + b*kABytes, two mbarriers
  unsigned char* wa = S.warp_area + warp * kWarpSmem;
  unsigned char* stage = wa + 2 * kXBytes;
  unsigned char* abase = wa + 3 * kXBytes;
  uint64_t* bar = reinterpret_cast<uint64_t*>(wa + 3 * kXBytes + 2 * kABytes);
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  load_dense_frags(S.frag, 5, w + ws_offset(layer), kH, w + wn_offset(layer), kR);
  if (!LAST) load_msg_frags(S.ufrag, w + layer_offset(layer + 1));
  for (int i = threadIdx.x; i < kH; i += blockDim.x) S.bias[i] = __bfloat162float(w[bias_offset(layer) + i]);
  if (LAST)
    for (int i = threadIdx.x; i <= kH; i += blockDim.x) S.wo[i] = __bfloat162float(w[kHeadOffset + i]);
  __syncthreads();
  DenseOut o{store_h ? &map_h : nullptr, LAST ? nullptr : S.ufrag, S.bias, S.wo, inv, M_next, y, V};
  const uint32_t nw = gridDim.x * kDenseWarps;
  const uint32_t first = blockIdx.x * kDenseWarps + warp;
  auto issue = [&](uint32_t tile, int b) {
    mbar_expect_tx(&bar[b], kXBytes + kABytes);
    tma_load_rows(wa + b * kXBytes, &map_x, (int)(tile * kTile), &bar[b]);
    bulk_load(abase + b * kABytes, A + (size_t)tile * kTile * kR, kABytes, &bar[b]);
  };
  if (first < ntiles && lane == 0) issue(first, 0);
  uint32_t i = 0;
  for (uint32_t tile = first; tile < ntiles; tile += nw, ++i) {
    const int b = i & 1;
    const bool more = tile + nw < ntiles;  // the next tile's load is issued now, waited for next iteration
    if (more && lane == 0) issue(tile + nw, b ^ 1);
    if (!mbar_wait(&bar[b], (i >> 1) & 1)) {
      // record the failure, let the load already issued for the next tile land
      // (bounded), and leave the loop
      if (lane == 0) atomicExch(err, 1u);
      if (more) mbar_wait(&bar[b ^ 1], ((i + 1) >> 1) & 1);
      break;
    }
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
    const uint32_t xb = smem_u32(wa + b * kXBytes);
    const float* at = reinterpret_cast<const float*>(abase + b * kABytes);
    const int q = lane >> 3, rr = (lane & 7) + (q & 1) * 8;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      uint32_t a0, a1, a2, a3;
      ldmatrix_x4(swz(xb, rr, 2 * ks + (q >> 1)), a0, a1, a2, a3);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const uint2 bb = S.frag[(ks * 8 + nt) * 32 + lane];
        mma_bf16_16x8x16(acc[nt], a0, a1, a2, a3, bb.x, bb.y);
      }
    }
    {  // aggregate columns: k = 64 + 2t, 2t+1 (rows g, g+8); k >= 72 zero
      const float2 va = *reinterpret_cast<const float2*>(at + g * kR + 2 * t);
      const float2 vb = *reinterpret_cast<const float2*>(at + (g + 8) * kR + 2 * t);
      const uint32_t a0 = pack_bf16x2(va.x, va.y), a1 = pack_bf16x2(vb.x, vb.y);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const uint2 bb = S.frag[(4 * 8 + nt) * 32 + lane];
        mma_bf16_16x8x16(acc[nt], a0, a1, 0u, 0u, bb.x, bb.y);
      }
    }
    dense_epilogue(o, acc, tile * kTile, stage, lane);
    __syncwarp();
  }
  if (lane == 0) bulk_wait_all();
}

// ---- inference: the dense layers with the hidden states kept in registers ----
// Inference needs no hidden state after the layer that uses it, so k_gnn_infer
// recomputes them instead of storing them: for its 16-node tile a warp runs
// layer 0 from [F | A_0], then layer 1 from [H_0 | A_1], ... up to layer L,
// each layer's BF16 output fragments becoming the next layer's A fragments
// directly (an m16n8k16 accumulator pair is an A-fragment register).  It then
// writes the next layer's message M_{L+1} = bf16(inv (H_L U_{L+1})) (L < 2) or
// the head y (L = 2).  Every product is the training kernels' (same fragments,
// same k-step order), so inference equals the training forward pass bit for
// bit; the per-node traffic is F, the aggregates A_0..A_L and the output
// (16 to 100 bytes) instead of a 128-byte hidden row read and written per layer.
constexpr int kInferWarps = 8;

// bias + ReLU + BF16 of an accumulator tile into packed pairs
__device__ __forceinline__ void relu_pack(const float (&acc)[8][4], const float* bias, int t, uint32_t (&hp)[8][2]) {
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int c = nt * 8 + t * 2;
    const float b0 = bias[c], b1 = bias[c + 1];
    hp[nt][0] = pack_bf16x2(fmaxf(acc[nt][0] + b0, 0.f), fmaxf(acc[nt][1] + b1, 0.f));
    hp[nt][1] = pack_bf16x2(fmaxf(acc[nt][2] + b0, 0.f), fmaxf(acc[nt][3] + b1, 0.f));
  }
}

template <int L>
__global__ void __launch_bounds__(kInferWarps * 32) k_gnn_infer(const float* __restrict__ F,
                                                                const float* __restrict__ A0,
                                                                const float* __restrict__ A1,
                                                                const float* __restrict__ A2,
                                                                const __nv_bfloat16* __restrict__ w,
                                                                const float* __restrict__ inv, uint32_t V,
                                                                uint32_t ntiles, __nv_bfloat16* __restrict__ M_next,
                                                                float* __restrict__ y) {
  __shared__ uint2 s_f0[8 * 32];                   // layer 0: one k-step
  __shared__ uint2 s_f[L > 0 ? L : 1][5 * 8 * 32];  // layers 1..L: five k-steps
  __shared__ uint2 s_u[4 * 32];                    // U of layer L+1 (L < 2)
  __shared__ float s_bias[L + 1][kH];
  __shared__ float s_wo[kH + 1];
  load_dense_frags(s_f0, 1, w + ws_offset(0), kF, w + wn_offset(0), kF);
  for (int l = 1; l <= L; ++l) load_dense_frags(s_f[l - 1], 5, w + ws_offset(l), kH, w + wn_offset(l), kR);
  if (L < kLayers - 1) load_msg_frags(s_u, w + layer_offset(L + 1));
  for (int i = threadIdx.x; i < (L + 1) * kH; i += blockDim.x)
    s_bias[i / kH][i % kH] = __bfloat162float(w[bias_offset(i / kH) + i % kH]);
  if (L == kLayers - 1)
    for (int i = threadIdx.x; i <= kH; i += blockDim.x) s_wo[i] = __bfloat162float(w[kHeadOffset + i]);
  __syncthreads();
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  for (uint32_t tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < ntiles;
       tile += gridDim.x * kInferWarps) {
    const uint32_t ra = tile * kTile + g, rb = ra + 8;
    const bool va = ra < V, vb = rb < V;
    uint32_t hp[8][2];
    {  // layer 0: k = 2t, 2t+1 from F (t < 2) or A_0 (t = 2, 3)
      const float* pa = t < 2 ? F + (size_t)ra * kF + 2 * t : A0 + (size_t)ra * kF + 2 * (t - 2);
      const float* pb = t < 2 ? F + (size_t)rb * kF + 2 * t : A0 + (size_t)rb * kF + 2 * (t - 2);
      const float2 xa = va ? __ldg(reinterpret_cast<const float2*>(pa)) : make_float2(0.f, 0.f);
      const float2 xb = vb ? __ldg(reinterpret_cast<const float2*>(pb)) : make_float2(0.f, 0.f);
      const uint32_t a0 = pack_bf16x2(xa.x, xa.y), a1 = pack_bf16x2(xb.x, xb.y);
      float acc[8][4];
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
        const uint2 bb = s_f0[nt * 32 + lane];
        mma_bf16_16x8x16(acc[nt], a0, a1, 0u, 0u, bb.x, bb.y);
      }
      relu_pack(acc, s_bias[0], t, hp);
    }
#pragma unroll
    for (int l = 1; l <= L; ++l) {
      const float* A = l == 1 ? A1 : A2;
      const uint2* fr = s_f[l - 1];
      float acc[8][4];
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
          const uint2 bb = fr[(ks * 8 + nt) * 32 + lane];
          mma_bf16_16x8x16(acc[nt], hp[2 * ks][0], hp[2 * ks][1], hp[2 * ks + 1][0], hp[2 * ks + 1][1], bb.x, bb.y);
        }
      const float2 xa = va ? __ldg(reinterpret_cast<const float2*>(A + (size_t)ra * kR + 2 * t)) : make_float2(0.f, 0.f);
      const float2 xb = vb ? __ldg(reinterpret_cast<const float2*>(A + (size_t)rb * kR + 2 * t)) : make_float2(0.f, 0.f);
      const uint32_t a0 = pack_bf16x2(xa.x, xa.y), a1 = pack_bf16x2(xb.x, xb.y);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const uint2 bb = fr[(4 * 8 + nt) * 32 + lane];
        mma_bf16_16x8x16(acc[nt], a0, a1, 0u, 0u, bb.x, bb.y);
      }
      relu_pack(acc, s_bias[l], t, hp);
    }
    if (L < kLayers - 1) {
      float m[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const uint2 bb = s_u[kk * 32 + lane];
        mma_bf16_16x8x16(m, hp[2 * kk][0], hp[2 * kk][1], hp[2 * kk + 1][0], hp[2 * kk + 1][1], bb.x, bb.y);
      }
      if (va) {
        const float sc = __ldg(inv + ra);
        *reinterpret_cast<uint32_t*>(M_next + (size_t)ra * kR + 2 * t) = pack_bf16x2(m[0] * sc, m[1] * sc);
      }
      if (vb) {
        const float sc = __ldg(inv + rb);
        *reinterpret_cast<uint32_t*>(M_next + (size_t)rb * kR + 2 * t) = pack_bf16x2(m[2] * sc, m[3] * sc);
      }
    } else {
      float s0 = 0.f, s1 = 0.f;
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const int c = nt * 8 + t * 2;
        s0 += bf16_lo(hp[nt][0]) * s_wo[c] + bf16_hi(hp[nt][0]) * s_wo[c + 1];
        s1 += bf16_lo(hp[nt][1]) * s_wo[c] + bf16_hi(hp[nt][1]) * s_wo[c + 1];
      }
      s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
      s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
      s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
      s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
      if (t == 0) {
        if (va) y[ra] = s0 + s_wo[kH];
        if (vb) y[rb] = s1 + s_wo[kH];
      }
    }
  }
}

// ---- inference on the 5th-generation tensor cores (tcgen05, TMEM) -----------
// The same computation as k_gnn_infer, for tiles of 128 nodes per CTA: one
// thread per node row builds the layer's A operand in shared memory (the
// 128-byte-swizzled K-major layout the tensor core reads through a matrix
// descriptor), thread 0 issues tcgen05.mma with the FP32 accumulator in tensor
// memory (128 lanes = the tile's rows, 64 columns), tcgen05.commit arrives on
// an mbarrier, and every thread reads its row's 64 accumulators back with
// tcgen05.ld for the epilogue (bias, ReLU, BF16), which writes the next
// layer's A operand.  Layer 0 is one K=16 step over [F | A_0 | 0]; layers 1
// and 2 are four K=16 steps over the hidden tile plus one over [A_l | 0]; the
// message product H U is one more N=16 MMA into columns 64-79.  Weights sit in
// shared memory as N x K K-major swizzled tiles for the whole kernel.
constexpr int kTcRows = 128;
constexpr int kTcThreads = 128;
constexpr uint32_t kTcCols = 128;  // TMEM columns: [0, 64) hidden accumulator, [64, 80) message accumulator
constexpr uint32_t kTileBytes128 = kTcRows * 128;  // a 128-row, 128-byte-row swizzled tile
constexpr uint32_t kWTileBytes = 64 * 128;         // a 64-row weight tile
constexpr uint32_t kUTileBytes = 16 * 128;         // the 16-row message-weight tile

__host__ __device__ constexpr uint32_t tc_smem_bytes(int L) {
  // H, AG, B0, (Ws, Wn) per layer 1..L, U, bias (L+1) x 64, head 65, mbarrier + TMEM address
  return kTileBytes128 * 2 + kWTileBytes + 2 * kWTileBytes * (uint32_t)L + kUTileBytes + (uint32_t)(L + 1) * kH * 4 +
         (kH + 1) * 4 + 64;
}

// byte offset of element (row, k) of a K-major tile with 128-byte rows and the
// 128-byte swizzle (16-byte chunk k/8 of row r stored at chunk (k/8) ^ (r % 8))
__device__ __forceinline__ uint32_t sw128_off(uint32_t row, uint32_t k) {
  return row * 128u + ((((k >> 3) ^ (row & 7u)) & 7u) << 4) + (k & 7u) * 2u;
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart; start address in 16-byte units
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// instruction descriptor: BF16 A and B (K-major), FP32 accumulator, M = 128
__host__ __device__ constexpr uint32_t tc_idesc(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// one BF16 weight into a swizzled N x K tile: tile[n][k] = value
__device__ __forceinline__ void put_w(unsigned char* tile, uint32_t n, uint32_t k, float v) {
  *reinterpret_cast<__nv_bfloat16*>(tile + sw128_off(n, k)) = __float2bfloat16_rn(v);
}
// 16 bytes (8 BF16) into chunk c of row r of a swizzled tile
__device__ __forceinline__ void put_chunk(unsigned char* tile, uint32_t r, uint32_t c, uint4 v) {
  *reinterpret_cast<uint4*>(tile + r * 128u + (((c ^ (r & 7u)) & 7u) << 4)) = v;
}

// accumulators of one layer -> bias, ReLU, BF16 (packed pairs, column order)
__device__ __forceinline__ void tc_layer_out(uint32_t taddr, const float* bias, uint32_t (&hp)[32]) {
  float a[32];
  tc_ld32(taddr, a);
  float b[32];
  tc_ld32(taddr + 32, b);
  tc_wait_ld();
#pragma unroll
  for (int i = 0; i < 16; ++i) hp[i] = pack_bf16x2(fmaxf(a[2 * i] + bias[2 * i], 0.f), fmaxf(a[2 * i + 1] + bias[2 * i + 1], 0.f));
#pragma unroll
  for (int i = 0; i < 16; ++i)
    hp[16 + i] = pack_bf16x2(fmaxf(b[2 * i] + bias[32 + 2 * i], 0.f), fmaxf(b[2 * i + 1] + bias[33 + 2 * i], 0.f));
}

template <int L>
__global__ void __launch_bounds__(kTcThreads, 1) k_gnn_infer_tc(const float* __restrict__ F,
                                                                 const float* __restrict__ A0,
                                                                 const float* __restrict__ A1,
                                                                 const float* __restrict__ A2,
                                                                 const __nv_bfloat16* __restrict__ w,
                                                                 const float* __restrict__ inv, uint32_t V,
                                                                 uint32_t ntiles, __nv_bfloat16* __restrict__ M_next,
                                                                 float* __restrict__ y, unsigned int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t a0 = smem_u32(smem_raw);
  unsigned char* base = smem_raw + (((a0 + 1023u) & ~1023u) - a0);
  unsigned char* tH = base;
  unsigned char* tAG = base + kTileBytes128;
  unsigned char* tB0 = base + 2 * kTileBytes128;
  unsigned char* tBs[3] = {nullptr, nullptr, nullptr};
  unsigned char* tBn[3] = {nullptr, nullptr, nullptr};
  uint32_t off = 2 * kTileBytes128 + kWTileBytes;
#pragma unroll
  for (int l = 1; l <= L; ++l) {
    tBs[l] = base + off;
    off += kWTileBytes;
    tBn[l] = base + off;
    off += kWTileBytes;
  }
  unsigned char* tBu = base + off;
  off += kUTileBytes;
  float* s_bias = reinterpret_cast<float*>(base + off);
  off += (L + 1) * kH * 4;
  float* s_wo = reinterpret_cast<float*>(base + off);
  off += (kH + 1) * 4;
  off = (off + 7u) & ~7u;
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + off);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(base + off + 8);
  const int tid = threadIdx.x, warp = tid >> 5;

  // weights as N x K tiles: B0 = [Ws_0; Wn_0; 0]^T (K = 16), Ws_l^T (K = 64),
  // Wn_l^T padded to K = 16, U^T padded to N = 16
  for (int i = tid; i < 64 * 64; i += kTcThreads) {
    const uint32_t n = (uint32_t)i / 64, k = (uint32_t)i % 64;
    if (k < 16) {
      const float v = k < (uint32_t)kF ? __bfloat162float(w[ws_offset(0) + k * kH + n])
                      : k < 2u * kF   ? __bfloat162float(w[wn_offset(0) + (k - kF) * kH + n])
                                      : 0.f;
      put_w(tB0, n, k, v);
    }
#pragma unroll
    for (int l = 1; l <= L; ++l) {
      put_w(tBs[l], n, k, __bfloat162float(w[ws_offset(l) + k * kH + n]));
      if (k < 16) put_w(tBn[l], n, k, k < (uint32_t)kR ? __bfloat162float(w[wn_offset(l) + k * kH + n]) : 0.f);
    }
    if (L < kLayers - 1 && n < 16) put_w(tBu, n, k, n < (uint32_t)kR ? __bfloat162float(w[layer_offset(L + 1) + k * kR + n]) : 0.f);
  }
  for (int i = tid; i < (L + 1) * kH; i += kTcThreads) s_bias[i] = __bfloat162float(w[bias_offset(i / kH) + i % kH]);
  for (int i = tid; i <= kH; i += kTcThreads) s_wo[i] = __bfloat162float(w[kHeadOffset + i]);
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(s_tmem)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const uint32_t tlane = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's lane quarter
  const uint32_t sH = smem_u32(tH), sAG = smem_u32(tAG), sB0 = smem_u32(tB0), sBu = smem_u32(tBu);
  uint32_t phase = 0;
  bool ok = true;
  // issue the MMAs (thread 0), wait for them (every thread, bounded)
  auto sync_operands = [&]() {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  };
  auto finish = [&]() {
    if (tid == 0) tc_commit(bar);
    // a block-wide vote, so every thread leaves the tile loop together if a wait timed out
    ok = __syncthreads_and(mbar_wait(bar, phase) ? 1 : 0) != 0;
    phase ^= 1u;
    tc_fence_after();
  };
  // a tile's per-row inputs (F, A_0 and the aggregates of layers 1..L), loaded
  // one tile ahead so that their latency overlaps the current tile
  struct RowIn {
    float4 f, a0, a1[2], a2[2];
  };
  auto load_row = [&](uint32_t tile, RowIn& in) {
    const uint32_t rr = tile * kTcRows + (uint32_t)tid;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const bool v = tile < ntiles && rr < V;
    in.f = v ? __ldg(reinterpret_cast<const float4*>(F) + rr) : z;
    in.a0 = v ? __ldg(reinterpret_cast<const float4*>(A0) + rr) : z;
    in.a1[0] = in.a1[1] = in.a2[0] = in.a2[1] = z;
    if (L >= 1 && v) {
      in.a1[0] = __ldg(reinterpret_cast<const float4*>(A1 + (size_t)rr * kR));
      in.a1[1] = __ldg(reinterpret_cast<const float4*>(A1 + (size_t)rr * kR + 4));
    }
    if (L >= 2 && v) {
      in.a2[0] = __ldg(reinterpret_cast<const float4*>(A2 + (size_t)rr * kR));
      in.a2[1] = __ldg(reinterpret_cast<const float4*>(A2 + (size_t)rr * kR + 4));
    }
  };
  RowIn cur, nxt;
  load_row(blockIdx.x, cur);
  for (uint32_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const uint32_t r = tile * kTcRows + (uint32_t)tid;
    const bool valid = r < V;
    load_row(tile + gridDim.x, nxt);
    {  // layer 0 operand: [F | A_0] as 8 BF16, then zeros (K = 16)
      const float4 f = cur.f, a = cur.a0;
      put_chunk(tAG, tid, 0, make_uint4(pack_bf16x2(f.x, f.y), pack_bf16x2(f.z, f.w), pack_bf16x2(a.x, a.y),
                                        pack_bf16x2(a.z, a.w)));
      put_chunk(tAG, tid, 1, make_uint4(0u, 0u, 0u, 0u));
    }
    sync_operands();
    if (tid == 0) tc_mma(tmem, sw128_desc(sAG), sw128_desc(sB0), tc_idesc(64), 0);
    finish();
    if (!ok) break;
    uint32_t hp[32];
    tc_layer_out(tlane, s_bias, hp);
#pragma unroll
    for (int l = 1; l <= L; ++l) {
      // the hidden tile and [A_l | 0]
      tc_fence_before();
      __syncthreads();  // every thread has read the accumulators and the previous operands are consumed
#pragma unroll
      for (int c = 0; c < 8; ++c) put_chunk(tH, tid, c, make_uint4(hp[4 * c], hp[4 * c + 1], hp[4 * c + 2], hp[4 * c + 3]));
      const float4 x0 = l == 1 ? cur.a1[0] : cur.a2[0], x1 = l == 1 ? cur.a1[1] : cur.a2[1];
      put_chunk(tAG, tid, 0, make_uint4(pack_bf16x2(x0.x, x0.y), pack_bf16x2(x0.z, x0.w), pack_bf16x2(x1.x, x1.y),
                                        pack_bf16x2(x1.z, x1.w)));
      sync_operands();
      if (tid == 0) {
        const uint32_t sBs = smem_u32(tBs[l]), sBn = smem_u32(tBn[l]);
#pragma unroll
        for (int k = 0; k < 4; ++k) tc_mma(tmem, sw128_desc(sH + 32 * k), sw128_desc(sBs + 32 * k), tc_idesc(64), k > 0);
        tc_mma(tmem, sw128_desc(sAG), sw128_desc(sBn), tc_idesc(64), 1);
      }
      finish();
      if (!ok) break;
      tc_layer_out(tlane, s_bias + l * kH, hp);
    }
    if (!ok) break;
    if (L < kLayers - 1) {
      tc_fence_before();
      __syncthreads();
#pragma unroll
      for (int c = 0; c < 8; ++c) put_chunk(tH, tid, c, make_uint4(hp[4 * c], hp[4 * c + 1], hp[4 * c + 2], hp[4 * c + 3]));
      sync_operands();
      if (tid == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) tc_mma(tmem + 64, sw128_desc(sH + 32 * k), sw128_desc(sBu + 32 * k), tc_idesc(16), k > 0);
      }
      finish();
      if (!ok) break;
      float m[8];
      tc_ld8(tlane + 64, m);
      tc_wait_ld();
      if (valid) {
        const float sc = __ldg(inv + r);
        *reinterpret_cast<uint4*>(M_next + (size_t)r * kR) =
            make_uint4(pack_bf16x2(m[0] * sc, m[1] * sc), pack_bf16x2(m[2] * sc, m[3] * sc),
                       pack_bf16x2(m[4] * sc, m[5] * sc), pack_bf16x2(m[6] * sc, m[7] * sc));
      }
    } else {
      float acc = 0.f;
#pragma unroll
      for (int i = 0; i < 32; ++i) acc += bf16_lo(hp[i]) * s_wo[2 * i] + bf16_hi(hp[i]) * s_wo[2 * i + 1];
      if (valid) y[r] = acc + s_wo[kH];
    }
    tc_fence_before();
    __syncthreads();  // the tile's operands and accumulators are free for the next tile
    tc_fence_after();
    cur = nxt;
  }
  if (!ok && tid == 0) atomicExch(err, 1u);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTcCols) : "memory");
}

// ---- inference on tcgen05 with four tiles in flight per SM ---------------------
// The products and epilogues of k_gnn_infer_tc, scheduled so that the tensor
// core and the epilogue overlap: one CTA of two warpgroups per SM, each
// warpgroup driving two 128-node tiles ("slots") with their own TMEM columns
// (128 each, 512 in all), operand tiles and mbarrier.  A warpgroup visits its
// slots in turn: it waits for the slot's MMAs, reads the accumulators, runs
// the epilogue, writes the next operand and issues the next MMAs, then moves
// to the other slot while those run.  A slot's inputs for its next stage (the
// next aggregate, or the next tile's features) are loaded right after its MMAs
// are issued.  Weights sit in shared memory once per CTA.
constexpr int kTc2Threads = 256;
constexpr uint32_t kTc2Cols = 512;

__host__ __device__ constexpr uint32_t tc2_smem_bytes(int L) {
  // 4 slots x (H, AG), B0, (Ws, Wn) per layer 1..L, U, bias, head, 4 mbarriers + TMEM address
  return 8 * kTileBytes128 + kWTileBytes + 2 * kWTileBytes * (uint32_t)L + kUTileBytes + (uint32_t)(L + 1) * kH * 4 +
         (kH + 1) * 4 + 64;
}

__device__ __forceinline__ void wg_sync(int wg) { asm volatile("bar.sync %0, 128;\n" ::"r"(1 + wg) : "memory"); }
// 1 when v holds in every thread of the warpgroup (a named-barrier reduction)
__device__ __forceinline__ int wg_all(int wg, int v) {
  int r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.s32 q, %1, 0;\n barrier.cta.red.and.pred p, %2, 128, q;\n selp.s32 %0, 1, 0, p;\n}\n"
      : "=r"(r)
      : "r"(v), "r"(1 + wg)
      : "memory");
  return r;
}

template <int L>
__global__ void __launch_bounds__(kTc2Threads, 1) k_gnn_infer_tc2(const float* __restrict__ F,
                                                                   const float* __restrict__ A0,
                                                                   const float* __restrict__ A1,
                                                                   const float* __restrict__ A2,
                                                                   const __nv_bfloat16* __restrict__ w,
                                                                   const float* __restrict__ inv, uint32_t V,
                                                                   uint32_t ntiles, __nv_bfloat16* __restrict__ M_next,
                                                                   float* __restrict__ y, unsigned int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t a0 = smem_u32(smem_raw);
  unsigned char* base = smem_raw + (((a0 + 1023u) & ~1023u) - a0);
  unsigned char* tB0 = base + 8 * kTileBytes128;
  uint32_t off = 8 * kTileBytes128 + kWTileBytes;
  unsigned char* tBs[3] = {nullptr, nullptr, nullptr};
  unsigned char* tBn[3] = {nullptr, nullptr, nullptr};
#pragma unroll
  for (int l = 1; l <= L; ++l) {
    tBs[l] = base + off;
    off += kWTileBytes;
    tBn[l] = base + off;
    off += kWTileBytes;
  }
  unsigned char* tBu = base + off;
  off += kUTileBytes;
  float* s_bias = reinterpret_cast<float*>(base + off);
  off += (L + 1) * kH * 4;
  float* s_wo = reinterpret_cast<float*>(base + off);
  off += (kH + 1) * 4;
  off = (off + 7u) & ~7u;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + off);  // one per slot
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(base + off + 32);
  const int tid = threadIdx.x;
  for (int i = tid; i < 64 * 64; i += kTc2Threads) {
    const uint32_t n = (uint32_t)i / 64, k = (uint32_t)i % 64;
    if (k < 16) {
      const float v = k < (uint32_t)kF ? __bfloat162float(w[ws_offset(0) + k * kH + n])
                      : k < 2u * kF   ? __bfloat162float(w[wn_offset(0) + (k - kF) * kH + n])
                                      : 0.f;
      put_w(tB0, n, k, v);
    }
#pragma unroll
    for (int l = 1; l <= L; ++l) {
      put_w(tBs[l], n, k, __bfloat162float(w[ws_offset(l) + k * kH + n]));
      if (k < 16) put_w(tBn[l], n, k, k < (uint32_t)kR ? __bfloat162float(w[wn_offset(l) + k * kH + n]) : 0.f);
    }
    if (L < kLayers - 1 && n < 16) put_w(tBu, n, k, n < (uint32_t)kR ? __bfloat162float(w[layer_offset(L + 1) + k * kR + n]) : 0.f);
  }
  for (int i = tid; i < (L + 1) * kH; i += kTc2Threads) s_bias[i] = __bfloat162float(w[bias_offset(i / kH) + i % kH]);
  for (int i = tid; i <= kH; i += kTc2Threads) s_wo[i] = __bfloat162float(w[kHeadOffset + i]);
  if (tid == 0) {
    for (int q = 0; q < 4; ++q) mbar_init(&bars[q], 1);
    mbar_fence_init();
  }
  if ((tid >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(s_tmem)),
                 "r"(kTc2Cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const int wg = tid >> 7, t = tid & 127;
  const bool leader = t == 0;
  const uint32_t lane_off = (uint32_t)(((tid >> 5) & 3) * 32) << 16;  // this warp's TMEM lane quarter
  const uint32_t sB0 = smem_u32(tB0), sBu = smem_u32(tBu);
  const uint32_t nslots = gridDim.x * 4;
  // per-slot state (slot j of this warpgroup is CTA slot q = 2 wg + j); the
  // loops over j are unrolled, so these stay in registers
  uint32_t tile[2] = {0u, 0u}, stage[2] = {0u, 0u}, phase[2] = {0u, 0u};
  bool live[2] = {false, false};
  float4 pf[2][2] = {};  // inputs of the slot's next stage: [A_l] or the next tile's [F, A_0]
  float pinv[2] = {0.f, 0.f};
  bool ok = true;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  auto load2 = [&](const float* p, uint32_t row, int width, float4& u, float4& v) {
    // width 4: one float4 (F or A_0, in u); width 8: two (an 8-wide aggregate)
    u = v = z4;
    if (row >= V) return;
    if (width == 4) {
      u = __ldg(reinterpret_cast<const float4*>(p) + row);
    } else {
      u = __ldg(reinterpret_cast<const float4*>(p + (size_t)row * kR));
      v = __ldg(reinterpret_cast<const float4*>(p + (size_t)row * kR + 4));
    }
  };
  // a tile's first operand [F | A_0 | 0] from the prefetched inputs, then its layer-0 MMA
  auto start_tile = [&](int j) {
    const int q = 2 * wg + j;
    unsigned char* tAG = base + (2 * q + 1) * kTileBytes128;
    const float4 f = pf[j][0], a = pf[j][1];
    put_chunk(tAG, t, 0, make_uint4(pack_bf16x2(f.x, f.y), pack_bf16x2(f.z, f.w), pack_bf16x2(a.x, a.y),
                                    pack_bf16x2(a.z, a.w)));
    put_chunk(tAG, t, 1, make_uint4(0u, 0u, 0u, 0u));
    fence_async_smem();
    tc_fence_before();
    wg_sync(wg);
    tc_fence_after();
    if (leader) {
      tc_mma(tmem + (uint32_t)q * 128u, sw128_desc(smem_u32(tAG)), sw128_desc(sB0), tc_idesc(64), 0);
      tc_commit(&bars[q]);
    }
    stage[j] = 0;
    const uint32_t row = tile[j] * kTcRows + (uint32_t)t;
    if (L >= 1) {
      load2(A1, row, 8, pf[j][0], pf[j][1]);
    } else {  // layer 0 is the last hidden layer: the next tile's features, this row's scale
      const uint32_t nrow = (tile[j] + nslots) * kTcRows + (uint32_t)t;
      float4 dummy;
      load2(F, nrow, 4, pf[j][0], dummy);
      load2(A0, nrow, 4, pf[j][1], dummy);
      pinv[j] = row < V ? __ldg(inv + row) : 0.f;
    }
  };
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    tile[j] = (uint32_t)(blockIdx.x * 4 + 2 * wg + j);
    live[j] = tile[j] < ntiles;
    if (live[j]) {
      float4 dummy;
      const uint32_t row = tile[j] * kTcRows + (uint32_t)t;
      load2(F, row, 4, pf[j][0], dummy);
      load2(A0, row, 4, pf[j][1], dummy);
      start_tile(j);
    }
  }
  while (ok && (live[0] || live[1])) {
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (!ok || !live[j]) continue;
      const int q = 2 * wg + j;
      unsigned char* tH = base + (2 * q) * kTileBytes128;
      unsigned char* tAG = tH + kTileBytes128;
      const uint32_t col = tmem + (uint32_t)q * 128u;
      ok = wg_all(wg, mbar_wait(&bars[q], phase[j]) ? 1 : 0) != 0;
      phase[j] ^= 1u;
      if (!ok) break;
      tc_fence_after();
      const uint32_t taddr = col + lane_off;
      const uint32_t row = tile[j] * kTcRows + (uint32_t)t;
      const bool valid = row < V;
      bool done = false;
      if (stage[j] <= (uint32_t)L) {  // hidden layer stage[j] is in the accumulators
        uint32_t hp[32];
        tc_layer_out(taddr, s_bias + stage[j] * kH, hp);
        if (stage[j] < (uint32_t)L) {  // operands of layer stage+1: H and [A_(stage+1) | 0]
          const uint32_t l = stage[j] + 1;
          // the slot's last MMAs are complete (its mbarrier), so its operand
          // tiles are free; the barrier below orders every thread's reads of
          // the accumulators before the next MMAs overwrite them
#pragma unroll
          for (int c = 0; c < 8; ++c) put_chunk(tH, t, c, make_uint4(hp[4 * c], hp[4 * c + 1], hp[4 * c + 2], hp[4 * c + 3]));
          const float4 x0 = pf[j][0], x1 = pf[j][1];
          put_chunk(tAG, t, 0, make_uint4(pack_bf16x2(x0.x, x0.y), pack_bf16x2(x0.z, x0.w), pack_bf16x2(x1.x, x1.y),
                                          pack_bf16x2(x1.z, x1.w)));
          fence_async_smem();
          tc_fence_before();
          wg_sync(wg);
          tc_fence_after();
          if (leader) {
            const uint32_t sBs = smem_u32(l == 1 ? tBs[1] : tBs[L]), sBn = smem_u32(l == 1 ? tBn[1] : tBn[L]);
            const uint32_t sH = smem_u32(tH), sAG = smem_u32(tAG);
#pragma unroll
            for (int k = 0; k < 4; ++k) tc_mma(col, sw128_desc(sH + 32 * k), sw128_desc(sBs + 32 * k), tc_idesc(64), k > 0);
            tc_mma(col, sw128_desc(sAG), sw128_desc(sBn), tc_idesc(64), 1);
            tc_commit(&bars[q]);
          }
          stage[j] = l;
          if (l < (uint32_t)L) {
            load2(A2, row, 8, pf[j][0], pf[j][1]);
          } else {  // the last hidden layer is running: the next tile's features, this row's scale
            const uint32_t nrow = (tile[j] + nslots) * kTcRows + (uint32_t)t;
            float4 dummy;
            load2(F, nrow, 4, pf[j][0], dummy);
            load2(A0, nrow, 4, pf[j][1], dummy);
            pinv[j] = valid ? __ldg(inv + row) : 0.f;
          }
        } else if (L < kLayers - 1) {  // the message product H U_(L+1)
#pragma unroll
          for (int c = 0; c < 8; ++c) put_chunk(tH, t, c, make_uint4(hp[4 * c], hp[4 * c + 1], hp[4 * c + 2], hp[4 * c + 3]));
          fence_async_smem();
          tc_fence_before();
          wg_sync(wg);
          tc_fence_after();
          if (leader) {
            const uint32_t sH = smem_u32(tH);
#pragma unroll
            for (int k = 0; k < 4; ++k) tc_mma(col + 64, sw128_desc(sH + 32 * k), sw128_desc(sBu + 32 * k), tc_idesc(16), k > 0);
            tc_commit(&bars[q]);
          }
          stage[j] = (uint32_t)L + 1;
        } else {  // the head
          float acc = 0.f;
#pragma unroll
          for (int i = 0; i < 32; ++i) acc += bf16_lo(hp[i]) * s_wo[2 * i] + bf16_hi(hp[i]) * s_wo[2 * i + 1];
          if (valid) y[row] = acc + s_wo[kH];
          done = true;
        }
      } else {  // the message accumulators
        float m[8];
        tc_ld8(taddr + 64, m);
        tc_wait_ld();
        if (valid) {
          const float sc = pinv[j];
          *reinterpret_cast<uint4*>(M_next + (size_t)row * kR) =
              make_uint4(pack_bf16x2(m[0] * sc, m[1] * sc), pack_bf16x2(m[2] * sc, m[3] * sc),
                         pack_bf16x2(m[4] * sc, m[5] * sc), pack_bf16x2(m[6] * sc, m[7] * sc));
        }
        done = true;
      }
      if (done) {  // the slot's next tile (start_tile's barrier orders the accumulator reads)
        tile[j] += nslots;
        live[j] = tile[j] < ntiles;
        if (live[j]) start_tile(j);
      }
    }
  }
  if (!ok && t == 0) atomicExch(err, 1u);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if ((tid >> 5) == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTc2Cols) : "memory");
}

// ---- dense layer backward (data): dP = dOut * (Out > 0); dX = dP Ws^T (DIN),
// dA = dP Wn^T (DM) (the BF16 roundings of the forward operands pass the
// gradient straight through).  dP is written back in place of dOut for the
// weight-gradient kernel.
template <int DIN, int DM>
__global__ void __launch_bounds__(256) k_gnn_dense_bwd_data(float* __restrict__ dOut,
                                                            const __nv_bfloat16* __restrict__ Out,
                                                            const __nv_bfloat16* __restrict__ ws,
                                                            const __nv_bfloat16* __restrict__ wn, uint32_t V,
                                                            float* __restrict__ dX, float* __restrict__ dA) {
  __shared__ float s_ws[DIN][kH];
  __shared__ float s_wn[DM][kH];
  for (int i = threadIdx.x; i < DIN * kH; i += blockDim.x) s_ws[i / kH][i % kH] = __bfloat162float(ws[i]);
  for (int i = threadIdx.x; i < DM * kH; i += blockDim.x) s_wn[i / kH][i % kH] = __bfloat162float(wn[i]);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < V; v += nw) {
    float* d = dOut + (size_t)v * kH;
    const __nv_bfloat16* o = Out + (size_t)v * kH;
    const float p0 = __bfloat162float(o[lane]) > 0.f ? d[lane] : 0.f;
    const float p1 = __bfloat162float(o[lane + 32]) > 0.f ? d[lane + 32] : 0.f;
    d[lane] = p0;
    d[lane + 32] = p1;
    // output k of dX / dA: sum_j dP[j] W[k][j]; lane handles k = lane, lane+32
    float x0 = 0.f, x1 = 0.f, a0 = 0.f;
#pragma unroll 8
    for (int j = 0; j < kH; ++j) {
      const float pj = __shfl_sync(0xffffffffu, j < 32 ? p0 : p1, j & 31);
      if (lane < DIN) x0 += pj * s_ws[lane][j];
      if (lane + 32 < DIN) x1 += pj * s_ws[lane + 32][j];
      if (lane < DM) a0 += pj * s_wn[lane][j];
    }
    if (lane < DIN) dX[(size_t)v * DIN + lane] = x0;
    if (lane + 32 < DIN) dX[(size_t)v * DIN + lane + 32] = x1;
    if (lane < DM) dA[(size_t)v * DM + lane] = a0;
  }
}

// ---- dense layer backward (weights): dWs += X^T dP, dWn += bf16(A)^T dP,
// db += sum dP -- the operands the forward pass multiplied (X = bf16(F) for
// layer 0, the BF16 hidden state otherwise).  Each block folds a tile of nodes
// in shared memory, then adds its partial into the global FP32 gradient
// ([Ws | Wn | b] of the layer) with one atomic per weight.
template <int DIN, int DM, class XT>
__global__ void __launch_bounds__(256) k_gnn_dense_bwd_weight(const XT* __restrict__ X, const float* __restrict__ A,
                                                              const float* __restrict__ dP, uint32_t V,
                                                              float* __restrict__ grad) {
  constexpr int TILE = 32;
  __shared__ float s_x[TILE][DIN];
  __shared__ float s_a[TILE][DM];
  __shared__ float s_p[TILE][kH];
  constexpr int PS = (DIN * kH + 255) / 256;
  constexpr int PN = (DM * kH + 255) / 256;
  float gs[PS], gn[PN], gb = 0.f;
#pragma unroll
  for (int r = 0; r < PS; ++r) gs[r] = 0.f;
#pragma unroll
  for (int r = 0; r < PN; ++r) gn[r] = 0.f;
  for (uint32_t base = blockIdx.x * TILE; base < V; base += gridDim.x * TILE) {
    const uint32_t cnt = min((uint32_t)TILE, V - base);
    __syncthreads();
    for (int i = threadIdx.x; i < TILE * DIN; i += blockDim.x) {
      const uint32_t n = i / DIN;
      s_x[n][i % DIN] = n < cnt ? bf16_round(to_f32(X[(size_t)(base + n) * DIN + i % DIN])) : 0.f;
    }
    for (int i = threadIdx.x; i < TILE * DM; i += blockDim.x) {
      const uint32_t n = i / DM;
      s_a[n][i % DM] = n < cnt ? bf16_round(A[(size_t)(base + n) * DM + i % DM]) : 0.f;
    }
    for (int i = threadIdx.x; i < TILE * kH; i += blockDim.x) {
      const uint32_t n = i / kH;
      s_p[n][i % kH] = n < cnt ? dP[(size_t)(base + n) * kH + i % kH] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < PS; ++r) {
      const int idx = threadIdx.x + r * 256;
      if (idx < DIN * kH) {
        const int k = idx / kH, j = idx % kH;
        float s1 = 0.f;
        for (int n = 0; n < TILE; ++n) s1 += s_x[n][k] * s_p[n][j];
        gs[r] += s1;
      }
    }
#pragma unroll
    for (int r = 0; r < PN; ++r) {
      const int idx = threadIdx.x + r * 256;
      if (idx < DM * kH) {
        const int k = idx / kH, j = idx % kH;
        float s2 = 0.f;
        for (int n = 0; n < TILE; ++n) s2 += s_a[n][k] * s_p[n][j];
        gn[r] += s2;
      }
    }
    if (threadIdx.x < kH)
      for (int n = 0; n < TILE; ++n) gb += s_p[n][threadIdx.x];
  }
#pragma unroll
  for (int r = 0; r < PS; ++r) {
    const int idx = threadIdx.x + r * 256;
    if (idx < DIN * kH) atomicAdd(grad + idx, gs[r]);
  }
#pragma unroll
  for (int r = 0; r < PN; ++r) {
    const int idx = threadIdx.x + r * 256;
    if (idx < DM * kH) atomicAdd(grad + DIN * kH + idx, gn[r]);
  }
  if (threadIdx.x < kH) atomicAdd(grad + DIN * kH + DM * kH + threadIdx.x, gb);
}

// ---- message backward: with dQ = inv * agg^T(dA) (the gradient of Q = H U),
// dH_prev = dX + dQ U^T (in place of dX) and dU += H_prev^T dQ.  One warp per
// node, lane j owns columns j and j+32; the block folds its warps' dU in
// shared memory and adds it with one atomic per weight.
__global__ void __launch_bounds__(256) k_gnn_msg_bwd(const float* __restrict__ dQ,
                                                     const __nv_bfloat16* __restrict__ Hp,
                                                     const __nv_bfloat16* __restrict__ u, uint32_t V,
                                                     float* __restrict__ dX, float* __restrict__ gradU) {
  __shared__ float s_u[kH][kR];
  __shared__ float s_g[8][kH * kR];
  for (int i = threadIdx.x; i < kH * kR; i += blockDim.x) s_u[i / kR][i % kR] = __bfloat162float(u[i]);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float g0[kR], g1[kR];
#pragma unroll
  for (int k = 0; k < kR; ++k) g0[k] = g1[k] = 0.f;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < V; v += nw) {
    const float4 qa = __ldg(reinterpret_cast<const float4*>(dQ + (size_t)v * kR));
    const float4 qb = __ldg(reinterpret_cast<const float4*>(dQ + (size_t)v * kR + 4));
    const float q[kR] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w};
    const float h0 = __bfloat162float(Hp[(size_t)v * kH + lane]);
    const float h1 = __bfloat162float(Hp[(size_t)v * kH + lane + 32]);
    float d0 = dX[(size_t)v * kH + lane], d1 = dX[(size_t)v * kH + lane + 32];
#pragma unroll
    for (int k = 0; k < kR; ++k) {
      d0 += q[k] * s_u[lane][k];
      d1 += q[k] * s_u[lane + 32][k];
      g0[k] += h0 * q[k];
      g1[k] += h1 * q[k];
    }
    dX[(size_t)v * kH + lane] = d0;
    dX[(size_t)v * kH + lane + 32] = d1;
  }
#pragma unroll
  for (int k = 0; k < kR; ++k) {
    s_g[warp][lane * kR + k] = g0[k];
    s_g[warp][(lane + 32) * kR + k] = g1[k];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kH * kR; i += blockDim.x) {
    float s = 0.f;
    for (int w8 = 0; w8 < (int)(blockDim.x >> 5); ++w8) s += s_g[w8][i];
    atomicAdd(gradU + i, s);
  }
}

// ---- loss and head backward -------------------------------------------------
// mode 0: loss = mean over live nodes of (y - t)^2, t = log(n pr)
//         dy = 2 (y - t) / n
// mode 1: loss = KL(pr || x0) with x0 = softmax(y) over live nodes
//              = sum_v pr(v) (log pr(v) - (y(v) - ymax) + log S),  S = sum exp(y - ymax)
//         dy = x0 - pr   (pr sums to 1)
// then dH = dy w_o, dw_o = sum dy H, db_o = sum dy.  The loss is summed in FP64.
__global__ void __launch_bounds__(256) k_gnn_head_bwd(const float* __restrict__ y, const float* __restrict__ t,
                                                      const double* __restrict__ pr, const double* __restrict__ x0,
                                                      const float* __restrict__ ymax, const double* __restrict__ stot,
                                                      const __nv_bfloat16* __restrict__ H,
                                                      const __nv_bfloat16* __restrict__ wo,
                                                      const uint32_t* __restrict__ out_deg, uint32_t V, float inv_n,
                                                      int mode, float* __restrict__ dH, float* __restrict__ grad_head,
                                                      double* __restrict__ loss) {
  __shared__ float s_g[kH + 1];
  __shared__ double s_loss;
  if (threadIdx.x <= kH) s_g[threadIdx.x] = 0.f;
  if (threadIdx.x == 0) s_loss = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const float w0 = __bfloat162float(wo[2 * lane]), w1 = __bfloat162float(wo[2 * lane + 1]);
  const double lse = mode == 1 ? log(*stot) + (double)*ymax : 0.0;  // log sum exp(y)
  float g0 = 0.f, g1 = 0.f, gb = 0.f;
  double ls = 0.0;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < V; v += nw) {
    const bool live = out_deg[v] != kDeletedDegree;
    float dy = 0.f;
    if (live) {
      if (mode == 0) {
        const float r = y[v] - t[v];
        dy = 2.f * r * inv_n;
        ls += (double)(r * r * inv_n);
      } else {
        const double p = pr[v];
        dy = (float)(x0[v] - p);
        if (p > 0.0) ls += p * (log(p) - (double)y[v] + lse);
      }
    }
    const uint32_t h = __ldg(reinterpret_cast<const uint32_t*>(H + (size_t)v * kH) + lane);
    *reinterpret_cast<float2*>(dH + (size_t)v * kH + 2 * lane) = make_float2(dy * w0, dy * w1);
    g0 += dy * bf16_lo(h);
    g1 += dy * bf16_hi(h);
    gb += dy;
  }
  atomicAdd(&s_g[2 * lane], g0);
  atomicAdd(&s_g[2 * lane + 1], g1);
  if (lane == 0) {
    atomicAdd(&s_g[kH], gb);
    atomicAdd(&s_loss, ls);
  }
  __syncthreads();
  if (threadIdx.x <= kH) atomicAdd(grad_head + threadIdx.x, s_g[threadIdx.x]);
  if (threadIdx.x == 0) atomicAdd(loss, s_loss);
}

// ---- start vector: x0 = exp(y) / sum exp(y) over live nodes (FP64) ------------
__global__ void __launch_bounds__(256) k_gnn_softmax_max(const float* __restrict__ y, const uint32_t* __restrict__ out_deg,
                                                         uint32_t V, float* __restrict__ ymax) {
  float m = -INFINITY;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    if (out_deg[v] != kDeletedDegree) m = fmaxf(m, y[v]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) {
    // float max via integer compare (values may be negative)
    int* a = reinterpret_cast<int*>(ymax);
    int old = *a, assumed;
    do {
      assumed = old;
      if (__int_as_float(assumed) >= m) break;
      old = atomicCAS(a, assumed, __float_as_int(m));
    } while (old != assumed);
  }
}
__global__ void __launch_bounds__(256) k_gnn_softmax_exp(const float* __restrict__ y, const uint32_t* __restrict__ out_deg,
                                                         uint32_t V, const float* __restrict__ ymax,
                                                         double* __restrict__ x, double* __restrict__ part) {
  __shared__ double s_red[8];
  const double m = (double)*ymax;
  double s = 0.0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const double e = out_deg[v] != kDeletedDegree ? exp((double)y[v] - m) : 0.0;
    x[v] = e;
    s += e;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_red[w];
    part[blockIdx.x] = t;
  }
}
__global__ void __launch_bounds__(256) k_gnn_softmax_scale(double* __restrict__ x, uint32_t V,
                                                           const double* __restrict__ part, uint32_t nparts,
                                                           double* __restrict__ tot_out) {
  __shared__ double s_tot;
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (uint32_t i = 0; i < nparts; ++i) t += part[i];  // fixed order
    s_tot = t;
    if (tot_out && blockIdx.x == 0) *tot_out = t;
  }
  __syncthreads();
  const double inv = s_tot > 0.0 ? 1.0 / s_tot : 0.0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) x[v] *= inv;
}

// ---- training target t = log(n * pr) for live nodes ---------------------------
__global__ void k_gnn_target(const double* __restrict__ pr, const uint32_t* __restrict__ out_deg, uint32_t V, double n,
                             float* __restrict__ t) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    t[v] = out_deg[v] != kDeletedDegree ? (float)log(fmax(pr[v] * n, 1e-30)) : 0.f;
}

// ---- Adam on the FP32 masters, then the BF16 copy -----------------------------
__global__ void k_gnn_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ s,
                           __nv_bfloat16* __restrict__ pb, int n, float lr, float b1, float b2, float eps, float c1,
                           float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float si = b2 * s[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    s[i] = si;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(si / c2) + eps);
    p[i] = pi;
    pb[i] = __float2bfloat16_rn(pi);
  }
}
__global__ void k_gnn_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ pb, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) pb[i] = __float2bfloat16_rn(p[i]);
}

__global__ void k_fill_f32(float* __restrict__ p, uint32_t n, float v) {
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) p[i] = v;
}

unsigned g1d(uint64_t n) {
  uint64_t g = (n + 255) / 256;
  const uint64_t cap = (uint64_t)sm_count() * 8;
  return (unsigned)std::max<uint64_t>(1, std::min(g, cap));
}
unsigned gwarp(uint64_t n) { return g1d(n * 32); }
// weight-gradient grid: one block per 32-node tile, at most two per SM (each
// block ends with one atomic per weight, so fewer blocks = less contention)
unsigned gtile(uint64_t n) {
  const uint64_t tiles = (n + 31) / 32;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)sm_count() * 2));
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda); resolved once.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tensor map of a [rows][64] BF16 hidden-state array: 16-row x 64-column
// boxes (2 KB), 128-byte swizzle.  rows is a multiple of 16, so no box reaches
// past the array.
int hidden_map(CUtensorMap* m, void* base, uint64_t rows) {
  if (reinterpret_cast<uintptr_t>(base) & 127u) return fail(ZOGCU_ERR_INTERNAL, "hidden-state array is not 128-byte aligned");
  auto enc = tensor_map_encoder();
  if (!enc) return fail(ZOGCU_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t dims[2] = {(cuuint64_t)kH, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)kH * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kH, (cuuint32_t)kTile};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ZOGCU_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return ZOGCU_OK;
}

// Dense-kernel grid: the CTAs resident at once (kDenseSmem each), at most one
// tile per warp.  The occupancy of each kernel is looked up once.
unsigned dense_grid(const void* kernel, uint32_t ntiles) {
  static std::mutex mu;
  static std::vector<std::pair<const void*, int>> known;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    for (const auto& k : known)
      if (k.first == kernel) per_sm = k.second;
    if (!per_sm) {
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDenseSmem);
      int n = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kDenseWarps * 32, kDenseSmem);
      per_sm = std::max(n, 1);
      known.emplace_back(kernel, per_sm);
    }
  }
  const uint64_t want = ((uint64_t)ntiles + kDenseWarps - 1) / kDenseWarps;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sm_count() * per_sm));
}

}  // namespace
}  // namespace zogcu

using namespace zogcu;

struct zogcu_gnn {
  int device = 0;
  DevArray p, pb, m, s, g, loss, err;  // masters, BF16 copy, Adam moments, gradient, loss (FP64), kernel error flag
  uint64_t step = 0;
  // activations of the largest graph seen so far (about 430 bytes per node),
  // reused by later calls until the model is destroyed
  mutable WorkCache acts;
};

namespace zogcu {
namespace {

// Activations of one forward pass over a graph (kept for the backward pass):
// features F, 1/outdeg, messages M_l and aggregates A_l, hidden states H_l in
// BF16 (rows padded to a multiple of 16 for the tile loads), output y.
struct GnnActs {
  uint32_t Vp = 0;  // rows of the padded arrays
  DevBuf F, inv, y, t, ctr, rows, M0;
  DevBuf M[kLayers];   // M[1], M[2]: V x 8 BF16
  DevBuf A[kLayers];   // A[0]: V x 4, A[1], A[2]: Vp x 8 (FP32)
  DevBuf H[kLayers];   // Vp x 64 BF16
  CUtensorMap mapH[kLayers];
  // from the model's cache when the lease holds it, else per call; H[2] only
  // when the backward pass needs it
  int alloc(uint32_t V, WorkLease& L, bool train) {
    const size_t Vs = std::max<uint32_t>(V, 1);
    Vp = (uint32_t)(((uint64_t)V + kTile - 1) / kTile * kTile);
    if (Vp == 0) Vp = kTile;
    ZOGCU_TRY(L.get(F, 0, Vs * kF * 4));
    ZOGCU_TRY(L.get(inv, 1, Vs * 4));
    ZOGCU_TRY(L.get(y, 2, Vs * 4));
    ZOGCU_TRY(L.get(ctr, 3, 16));
    ZOGCU_TRY(L.get(M0, 4, Vs * kF * 4));
    ZOGCU_TRY(L.get(A[0], 5, Vs * kF * 4));
    for (int l = 1; l < kLayers; ++l) {
      ZOGCU_TRY(L.get(M[l], 5 + l, Vs * kR * 2));
      ZOGCU_TRY(L.get(A[l], 7 + l, (size_t)Vp * kR * 4));
      // the dense kernels copy 512-byte aggregate tiles with bulk copies
      if (reinterpret_cast<uintptr_t>(A[l].ptr) & 15u) return fail(ZOGCU_ERR_INTERNAL, "aggregate array is not 16-byte aligned");
    }
    // hidden states: stored for the backward pass only (inference recomputes them)
    if (train)
      for (int l = 0; l < kLayers; ++l) {
        ZOGCU_TRY(L.get(H[l], 10 + l, (size_t)Vp * kH * 2));
        ZOGCU_TRY(hidden_map(&mapH[l], H[l].ptr, Vp));
      }
    return ZOGCU_OK;
  }
};

// The in-CSR a forward pass runs over: the graph's own, or (inference) the
// PageRank schedule's degree-ranked view -- nodes renumbered by out-degree,
// descending, so the most gathered messages form a dense prefix that stays in
// L2, and each row keeping its arcs in the original order, so every aggregate
// equals the original-order one bit for bit.
struct GView {
  const uint32_t* off;   // in-CSR offsets (V + 1)
  const uint32_t* col;   // sources of each row
  const uint32_t* deg;   // out-degree (kDeletedDegree for deleted slots)
  uint32_t V;
  uint32_t E;
  uint64_t n_live;
};
GView original_view(const Graph* g) {
  return GView{g->in_off32.as<uint32_t>(), g->in_col.as<uint32_t>(), g->out_deg.as<uint32_t>(), g->V, (uint32_t)g->E,
               g->n_live};
}
GView ranked_view(const Graph* g) {
  const PrSchedule& P = g->pr;
  return GView{P.off.as<uint32_t>(), P.col.as<uint32_t>(), P.deg.as<uint32_t>(), g->V, (uint32_t)g->E, g->n_live};
}

// x_out[v] = x_ranked[rank(v)]: a ranked-order vector back in node order
__global__ void k_gnn_unrank(const double* __restrict__ xr, const uint32_t* __restrict__ rank, uint32_t V,
                             double* __restrict__ x) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) x[v] = xr[rank[v]];
}
__global__ void k_gnn_unrank_f(const float* __restrict__ yr, const uint32_t* __restrict__ rank, uint32_t V,
                               float* __restrict__ y) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) y[v] = yr[rank[v]];
}

// First row of every kChunk-arc chunk of the in-CSR (transpose = 0) or the
// out-CSR (transpose = 1), into `rows` (allocated here).
int chunk_rows(const Graph* g, bool transpose, DevBuf& rows, cudaStream_t s) {
  const uint32_t E = (uint32_t)g->E;
  const uint64_t chunks = ((uint64_t)E + kChunk - 1) / kChunk;
  ZOGCU_TRY(rows.alloc(std::max<uint64_t>(chunks, 1) * 4, s));
  if (chunks == 0) return ZOGCU_OK;
  const uint32_t* off = (transpose ? g->out_off32 : g->in_off32).as<uint32_t>();
  k_chunk_rows<<<g1d(chunks), 256, 0, s>>>(off, g->V, E, kChunk, rows.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  return ZOGCU_OK;
}

// Z = agg(X) (forward, in-CSR) or Z = inv * agg^T(X) (transpose, out-CSR);
// `ctr` is a device word for the chunk counter, `rows` the chunks' first rows.
// Z (zrows x D, zrows >= V) is zeroed first.
template <class T, int D>
int spmm(const Graph* g, bool transpose, const float* inv, const T* X, float* Z, size_t zrows, uint32_t* ctr,
         const DevBuf& rows, cudaStream_t s) {
  const uint32_t V = g->V;
  const uint32_t E = (uint32_t)g->E;
  ZOGCU_CUDA(cudaMemsetAsync(Z, 0, zrows * D * 4, s));
  if (E == 0) return ZOGCU_OK;
  const uint32_t* off = (transpose ? g->out_off32 : g->in_off32).as<uint32_t>();
  const uint32_t* col = (transpose ? g->out_col : g->in_col).as<uint32_t>();
  const uint64_t chunks = ((uint64_t)E + kChunk - 1) / kChunk;
  ZOGCU_CUDA(cudaMemsetAsync(ctr, 0, 4, s));
  k_gnn_spmm<T, D><<<gwarp(chunks), 256, 0, s>>>(off, col, inv, X, V, E, transpose ? 1 : 0, Z, ctr,
                                                 rows.as<uint32_t>());
  return ZOGCU_OK;
}

// The aggregate's gathers go straight to shared memory (k_gnn_agg16_async)
// unless ZOGCU_GNN_AGG_ASYNC=0 selects the register-staged k_gnn_agg16; both
// compute the same sums in the same order.
bool agg_async_on() {
  const char* e = std::getenv("ZOGCU_GNN_AGG_ASYNC");
  return !(e && e[0] == '0');
}

// First row of every kAggChunk-arc chunk of a view's in-CSR, into `rows`.
int chunk_rows_view(const GView& gv, DevBuf& rows, cudaStream_t s) {
  const uint64_t chunks = ((uint64_t)gv.E + kAggChunk - 1) / kAggChunk;
  ZOGCU_TRY(rows.alloc(std::max<uint64_t>(chunks, 1) * 4, s));
  if (chunks == 0) return ZOGCU_OK;
  k_chunk_rows<<<g1d(chunks), 256, 0, s>>>(gv.off, gv.V, gv.E, kAggChunk, rows.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  return ZOGCU_OK;
}

// Z = agg(X) over a view's in-CSR for 16-byte messages (k_gnn_agg16); Z
// (zrows x D, zrows >= V) is zeroed first.
template <class T, int D>
int aggregate(const GView& gv, const T* X, float* Z, size_t zrows, uint32_t* ctr, const DevBuf& rows, cudaStream_t s) {
  ZOGCU_CUDA(cudaMemsetAsync(Z, 0, zrows * D * 4, s));
  if (gv.E == 0) return ZOGCU_OK;
  const uint64_t chunks = ((uint64_t)gv.E + kAggChunk - 1) / kAggChunk;
  static int per_sm = 0;  // resident CTAs per SM (per template instance)
  if (!per_sm) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_gnn_agg16<T, D>, kAggWarps * 32, 0);
    per_sm = std::max(n, 1);
  }
  const uint64_t want = (chunks + kAggWarps - 1) / kAggWarps;
  if (agg_async_on()) {
    static int per_sm_async = 0;
    if (!per_sm_async) {
      int n = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_gnn_agg16_async<T, D>, kAggWarps * 32, 0);
      per_sm_async = std::max(n, 1);
    }
    const unsigned grid =
        (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sm_count() * per_sm_async));
    k_gnn_agg16_async<T, D><<<grid, kAggWarps * 32, 0, s>>>(gv.off, gv.col, X, gv.V, gv.E, Z, rows.as<uint32_t>());
    ZOGCU_CUDA(cudaGetLastError());
    return ZOGCU_OK;
  }
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sm_count() * per_sm));
  k_gnn_agg16<T, D><<<grid, kAggWarps * 32, 0, s>>>(gv.off, gv.col, X, gv.V, gv.E, Z, ctr, rows.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  return ZOGCU_OK;
}

// The tcgen05 inference kernels: dynamic shared memory of at least 60 KB so
// that at most three CTAs share an SM (their 3 x 128 TMEM columns fit the
// SM's 512); ZOGCU_GNN_TC=1 selects them (the mma.sync kernels otherwise).
// 0: the mma.sync kernels; 1: the one-tile tcgen05 kernels; 2: the four-slot
// tcgen05 kernels (ZOGCU_GNN_TC)
int gnn_tc_mode() {
  const char* e = std::getenv("ZOGCU_GNN_TC");
  return (e && (e[0] == '1' || e[0] == '2')) ? e[0] - '0' : 0;
}

template <int L>
int launch_infer_tc(const float* F, const float* A0, const float* A1, const float* A2, const __nv_bfloat16* w,
                    const float* inv, uint32_t V, __nv_bfloat16* M_next, float* y, unsigned int* err, cudaStream_t s) {
  static int per_sm = 0;  // per template instance; the same on every B200
  const uint32_t smem = std::max<uint32_t>(tc_smem_bytes(L) + 1024, 60u * 1024);
  if (!per_sm) {
    ZOGCU_CUDA(cudaFuncSetAttribute(k_gnn_infer_tc<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int n = 0;
    ZOGCU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_gnn_infer_tc<L>, kTcThreads, smem));
    if (n < 1 || (uint32_t)n * kTcCols > 512u) return fail(ZOGCU_ERR_INTERNAL, "tcgen05 kernel occupancy exceeds tensor memory");
    per_sm = n;
  }
  const uint32_t ntiles = (V + kTcRows - 1) / kTcRows;
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ntiles, (uint64_t)sm_count() * per_sm));
  k_gnn_infer_tc<L><<<grid, kTcThreads, smem, s>>>(F, A0, A1, A2, w, inv, V, ntiles, M_next, y, err);
  ZOGCU_CUDA(cudaGetLastError());
  return ZOGCU_OK;
}

// The four-slot tcgen05 kernels: one CTA per SM (its shared memory allows no
// second one), which owns all 512 TMEM columns.
template <int L>
int launch_infer_tc2(const float* F, const float* A0, const float* A1, const float* A2, const __nv_bfloat16* w,
                     const float* inv, uint32_t V, __nv_bfloat16* M_next, float* y, unsigned int* err, cudaStream_t s) {
  static bool checked = false;  // per template instance
  const uint32_t smem = tc2_smem_bytes(L) + 1024;
  if (!checked) {
    ZOGCU_CUDA(cudaFuncSetAttribute(k_gnn_infer_tc2<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int n = 0;
    ZOGCU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_gnn_infer_tc2<L>, kTc2Threads, smem));
    if (n != 1) return fail(ZOGCU_ERR_INTERNAL, "four-slot tcgen05 kernel must run one CTA per SM");
    checked = true;
  }
  const uint32_t ntiles = (V + kTcRows - 1) / kTcRows;
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((ntiles + 3) / 4, (uint64_t)sm_count()));
  k_gnn_infer_tc2<L><<<grid, kTc2Threads, smem, s>>>(F, A0, A1, A2, w, inv, V, ntiles, M_next, y, err);
  ZOGCU_CUDA(cudaGetLastError());
  return ZOGCU_OK;
}

// Forward pass; with train the last hidden state is stored for the backward
// pass.  err: device word the dense kernels raise when a tile load timed out.
int gnn_forward(const zogcu_gnn* M, const GView& g, GnnActs& act, bool train, cudaStream_t s) {
  const uint32_t V = g.V;
  const __nv_bfloat16* w = M->pb.as<__nv_bfloat16>();
  uint32_t* ctr = act.ctr.as<uint32_t>();
  unsigned int* err = M->err.as<unsigned int>();
  const uint32_t ntiles = act.Vp / kTile;
  k_gnn_features<<<g1d(V), 256, 0, s>>>(g.off, g.deg, V, 1.f / (float)std::max<uint64_t>(g.n_live, 1),
                                        act.F.as<float>(), act.inv.as<float>(), act.M0.as<float>());
  const float* inv = act.inv.as<float>();
  const float* F = act.F.as<float>();
  ZOGCU_TRY(chunk_rows_view(g, act.rows, s));
  ZOGCU_TRY((aggregate<float, kF>(g, act.M0.as<float>(), act.A[0].as<float>(), V, ctr, act.rows, s)));
  if (!train) {
    // inference: the dense layers recompute the hidden states in registers
    const unsigned ig = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>(((uint64_t)ntiles + kInferWarps - 1) / kInferWarps, (uint64_t)sm_count() * 8));
    const float* A0 = act.A[0].as<float>();
    const float* A1 = act.A[1].as<float>();
    const float* A2 = act.A[2].as<float>();
    const int tcm = gnn_tc_mode();
    const bool tc = tcm != 0;
    __nv_bfloat16* M1 = act.M[1].as<__nv_bfloat16>();
    __nv_bfloat16* M2 = act.M[2].as<__nv_bfloat16>();
    float* yv = act.y.as<float>();
    if (tc) {
      if (tcm == 2) ZOGCU_TRY(launch_infer_tc2<0>(F, A0, A1, A2, w, inv, V, M1, nullptr, err, s));
      else ZOGCU_TRY(launch_infer_tc<0>(F, A0, A1, A2, w, inv, V, M1, nullptr, err, s));
    } else {
      k_gnn_infer<0><<<ig, kInferWarps * 32, 0, s>>>(F, A0, A1, A2, w, inv, V, ntiles, M1, nullptr);
      ZOGCU_CUDA(cudaGetLastError());
    }
    ZOGCU_TRY((aggregate<__nv_bfloat16, kR>(g, M1, act.A[1].as<float>(), act.Vp, ctr, act.rows, s)));
    if (tc) {
      if (tcm == 2) ZOGCU_TRY(launch_infer_tc2<1>(F, A0, A1, A2, w, inv, V, M2, nullptr, err, s));
      else ZOGCU_TRY(launch_infer_tc<1>(F, A0, A1, A2, w, inv, V, M2, nullptr, err, s));
    } else {
      k_gnn_infer<1><<<ig, kInferWarps * 32, 0, s>>>(F, A0, A1, A2, w, inv, V, ntiles, M2, nullptr);
      ZOGCU_CUDA(cudaGetLastError());
    }
    ZOGCU_TRY((aggregate<__nv_bfloat16, kR>(g, M2, act.A[2].as<float>(), act.Vp, ctr, act.rows, s)));
    if (tc) {
      if (tcm == 2) ZOGCU_TRY(launch_infer_tc2<2>(F, A0, A1, A2, w, inv, V, nullptr, yv, err, s));
      else ZOGCU_TRY(launch_infer_tc<2>(F, A0, A1, A2, w, inv, V, nullptr, yv, err, s));
    } else {
      k_gnn_infer<2><<<ig, kInferWarps * 32, 0, s>>>(F, A0, A1, A2, w, inv, V, ntiles, nullptr, yv);
      ZOGCU_CUDA(cudaGetLastError());
    }
    return ZOGCU_OK;
  }
  // training: hidden states stored (TMA tile loads and stores) for the backward pass
  k_gnn_dense0<<<dense_grid((const void*)k_gnn_dense0, ntiles), kDenseWarps * 32, kDenseSmem, s>>>(
      act.mapH[0], F, act.A[0].as<float>(), w, inv, V, ntiles, act.M[1].as<__nv_bfloat16>());
  ZOGCU_CUDA(cudaGetLastError());
  for (int l = 1; l < kLayers; ++l) {
    ZOGCU_TRY((aggregate<__nv_bfloat16, kR>(g, act.M[l].as<__nv_bfloat16>(), act.A[l].as<float>(), act.Vp, ctr,
                                            act.rows, s)));
    if (l < kLayers - 1) {
      k_gnn_dense_mid<0><<<dense_grid((const void*)k_gnn_dense_mid<0>, ntiles), kDenseWarps * 32, kDenseSmem, s>>>(
          act.mapH[l - 1], act.mapH[l], act.A[l].as<float>(), w, l, inv, V, ntiles, 1,
          act.M[l + 1].as<__nv_bfloat16>(), nullptr, err);
    } else {
      k_gnn_dense_mid<1><<<dense_grid((const void*)k_gnn_dense_mid<1>, ntiles), kDenseWarps * 32, kDenseSmem, s>>>(
          act.mapH[l - 1], act.mapH[l], act.A[l].as<float>(), w, l, inv, V, ntiles, 1, nullptr,
          act.y.as<float>(), err);
    }
    ZOGCU_CUDA(cudaGetLastError());
  }
  return ZOGCU_OK;
}

// Reads and clears the dense kernels' error word (after the stream finished).
int check_dense_error(const zogcu_gnn* M, cudaStream_t s) {
  unsigned int e = 0;
  ZOGCU_CUDA(cudaMemcpyAsync(&e, M->err.ptr, 4, cudaMemcpyDeviceToHost, s));
  ZOGCU_CUDA(cudaStreamSynchronize(s));
  if (e) {
    ZOGCU_CUDA(cudaMemsetAsync(M->err.ptr, 0, 4, s));
    return fail(ZOGCU_ERR_INTERNAL, "warm-start dense layer: a tile load did not complete");
  }
  return ZOGCU_OK;
}

// x = softmax(y) over live nodes (FP64), with ymax and S = sum exp(y - ymax)
// left in device scalars.
struct Softmax {
  DevBuf ymax, part, stot;
  unsigned grid = 1;
  int run(const GView& g, const float* y, double* x, cudaStream_t s) {
    const uint32_t V = g.V;
    grid = g1d(V);
    ZOGCU_TRY(ymax.alloc(16, s));
    ZOGCU_TRY(stot.alloc(16, s));
    ZOGCU_TRY(part.alloc((size_t)grid * 8, s));
    // -inf: every live y is larger; the CAS loop below only raises it
    k_fill_f32<<<1, 32, 0, s>>>(ymax.as<float>(), 1, -INFINITY);
    k_gnn_softmax_max<<<grid, 256, 0, s>>>(y, g.deg, V, ymax.as<float>());
    k_gnn_softmax_exp<<<grid, 256, 0, s>>>(y, g.deg, V, ymax.as<float>(), x, part.as<double>());
    k_gnn_softmax_scale<<<grid, 256, 0, s>>>(x, V, part.as<double>(), grid, stot.as<double>());
    ZOGCU_CUDA(cudaGetLastError());
    return ZOGCU_OK;
  }
};

// Loss and gradient (into M->g, zeroed first) of one graph with target
// PageRank pr (device, FP64).  mode 0 = MSE on log(n pr), 1 = KL(pr || softmax(y)).
int gnn_backward(zogcu_gnn* M, const Graph* g, GnnActs& act, const double* d_pr, int mode, cudaStream_t s) {
  const uint32_t V = g->V;
  const size_t Vs = std::max<uint32_t>(V, 1);
  const __nv_bfloat16* w = M->pb.as<__nv_bfloat16>();
  float* grad = M->g.as<float>();
  ZOGCU_CUDA(cudaMemsetAsync(grad, 0, (size_t)kNumParams * 4, s));
  ZOGCU_CUDA(cudaMemsetAsync(M->loss.ptr, 0, 8, s));
  Softmax sm;
  DevBuf xq;
  if (mode == 0) {
    ZOGCU_TRY(act.t.alloc(Vs * 4, s));
    k_gnn_target<<<g1d(V), 256, 0, s>>>(d_pr, g->out_deg.as<uint32_t>(), V, (double)g->n_live, act.t.as<float>());
  } else {
    ZOGCU_TRY(xq.alloc(Vs * 8, s));
    ZOGCU_TRY(sm.run(original_view(g), act.y.as<float>(), xq.as<double>(), s));
  }
  DevBuf dH, dX, dA, dQ;
  ZOGCU_TRY(dH.alloc(Vs * kH * 4, s));
  ZOGCU_TRY(dX.alloc(Vs * kH * 4, s));
  ZOGCU_TRY(dA.alloc(Vs * kR * 4, s));
  ZOGCU_TRY(dQ.alloc(Vs * kR * 4, s));
  const float inv_n = 1.f / (float)std::max<uint64_t>(g->n_live, 1);
  float* pdH = dH.as<float>();
  float* pdX = dX.as<float>();
  uint32_t* ctr = act.ctr.as<uint32_t>();
  DevBuf out_rows;
  ZOGCU_TRY(chunk_rows(g, true, out_rows, s));
  k_gnn_head_bwd<<<gwarp(V), 256, 0, s>>>(act.y.as<float>(), act.t.as<float>(), d_pr, xq.as<double>(),
                                          sm.ymax.as<float>(), sm.stot.as<double>(),
                                          act.H[kLayers - 1].as<__nv_bfloat16>(), w + kHeadOffset,
                                          g->out_deg.as<uint32_t>(), V, inv_n, mode, pdH, grad + kHeadOffset,
                                          M->loss.as<double>());
  for (int l = kLayers - 1; l >= 1; --l) {
    k_gnn_dense_bwd_data<kH, kR><<<gwarp(V), 256, 0, s>>>(pdH, act.H[l].as<__nv_bfloat16>(), w + ws_offset(l),
                                                          w + wn_offset(l), V, pdX, dA.as<float>());
    k_gnn_dense_bwd_weight<kH, kR, __nv_bfloat16><<<gtile(V), 256, 0, s>>>(
        act.H[l - 1].as<__nv_bfloat16>(), act.A[l].as<float>(), pdH, V, grad + ws_offset(l));
    // dQ = inv * agg^T(dA): the gradient of H_{l-1} U_l
    ZOGCU_TRY((spmm<float, kR>(g, true, act.inv.as<float>(), dA.as<float>(), dQ.as<float>(), V, ctr, out_rows, s)));
    // dH_{l-1} = dX + dQ U^T (into dX), dU += H_{l-1}^T dQ
    k_gnn_msg_bwd<<<g1d((uint64_t)V * 32), 256, 0, s>>>(dQ.as<float>(), act.H[l - 1].as<__nv_bfloat16>(),
                                                        w + layer_offset(l), V, pdX, grad + layer_offset(l));
    std::swap(pdH, pdX);
  }
  k_gnn_dense_bwd_data<kF, kF><<<gwarp(V), 256, 0, s>>>(pdH, act.H[0].as<__nv_bfloat16>(), w + ws_offset(0),
                                                        w + wn_offset(0), V, pdX, dA.as<float>());
  k_gnn_dense_bwd_weight<kF, kF, float><<<gtile(V), 256, 0, s>>>(act.F.as<float>(), act.A[0].as<float>(), pdH, V,
                                                                  grad + ws_offset(0));
  ZOGCU_CUDA(cudaGetLastError());
  return ZOGCU_OK;
}

// Glorot-uniform initial weights from a seeded SplitMix64 stream, each matrix
// with its own fan (rows + columns) in flat-layout order; biases zero.
void gnn_init_host(uint64_t seed, std::vector<float>& p) {
  p.assign(kNumParams, 0.f);
  uint64_t st = seed;
  auto next = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  auto fill = [&](int off, int rows, int cols) {
    const float a = std::sqrt(6.f / (float)(rows + cols));
    for (int i = 0; i < rows * cols; ++i) p[off + i] = a * ((float)((next() >> 40) * (1.0 / 16777216.0)) * 2.f - 1.f);
  };
  for (int l = 0; l < kLayers; ++l) {
    if (l > 0) fill(layer_offset(l), layer_in(l), layer_msg(l));
    fill(ws_offset(l), layer_in(l), kH);
    fill(wn_offset(l), layer_msg(l), kH);
  }
  fill(kHeadOffset, kH, 1);
}

}  // namespace
}  // namespace zogcu

extern "C" {

int zogcu_gnn_num_params(void) { return kNumParams; }

int zogcu_gnn_create(uint64_t seed, zogcu_gnn** out) {
  if (!out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "out is null");
  *out = nullptr;
  int dev;
  ZOGCU_TRY(ensure_device(&dev));
  std::unique_ptr<zogcu_gnn> M(new (std::nothrow) zogcu_gnn());
  if (!M) return fail(ZOGCU_ERR_OUT_OF_MEMORY, "host allocation failed");
  M->device = dev;
  ZOGCU_TRY(M->p.alloc(kNumParams * 4));
  ZOGCU_TRY(M->pb.alloc(kNumParams * 2 + 16));
  ZOGCU_TRY(M->m.alloc(kNumParams * 4));
  ZOGCU_TRY(M->s.alloc(kNumParams * 4));
  ZOGCU_TRY(M->g.alloc(kNumParams * 4));
  ZOGCU_TRY(M->loss.alloc(16));
  ZOGCU_TRY(M->err.alloc(16));
  std::vector<float> h;
  gnn_init_host(seed, h);
  ZOGCU_CUDA(cudaMemcpy(M->p.ptr, h.data(), kNumParams * 4, cudaMemcpyHostToDevice));
  ZOGCU_CUDA(cudaMemset(M->m.ptr, 0, kNumParams * 4));
  ZOGCU_CUDA(cudaMemset(M->s.ptr, 0, kNumParams * 4));
  ZOGCU_CUDA(cudaMemset(M->err.ptr, 0, 16));
  k_gnn_to_bf16<<<g1d(kNumParams), 256>>>(M->p.as<float>(), M->pb.as<__nv_bfloat16>(), kNumParams);
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_CUDA(cudaDeviceSynchronize());
  *out = M.release();
  return ZOGCU_OK;
}

int zogcu_gnn_destroy(zogcu_gnn* M) {
  if (!M) return ZOGCU_OK;
  cudaSetDevice(M->device);
  delete M;
  return ZOGCU_OK;
}

int zogcu_gnn_get_params(const zogcu_gnn* M, float* out) {
  if (!M || !out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  ZOGCU_CUDA(cudaMemcpy(out, M->p.ptr, kNumParams * 4, cudaMemcpyDeviceToHost));
  return ZOGCU_OK;
}

int zogcu_gnn_set_params(zogcu_gnn* M, const float* in) {
  if (!M || !in) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  ZOGCU_CUDA(cudaSetDevice(M->device));
  ZOGCU_CUDA(cudaMemcpy(M->p.ptr, in, kNumParams * 4, cudaMemcpyHostToDevice));
  k_gnn_to_bf16<<<g1d(kNumParams), 256>>>(M->p.as<float>(), M->pb.as<__nv_bfloat16>(), kNumParams);
  ZOGCU_CUDA(cudaGetLastError());
  ZOGCU_CUDA(cudaDeviceSynchronize());
  return ZOGCU_OK;
}

// Loss and gradient for one graph (target: PageRank vector, host, length V).
int zogcu_gnn_loss_grad(zogcu_gnn* M, zogcu_graph* G, const double* target_pr, int loss_kind, float* loss,
                        float* grad_out) {
  if (!M || !G || !target_pr) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  if (loss_kind != ZOGCU_GNN_LOSS_LOG_MSE && loss_kind != ZOGCU_GNN_LOSS_KL)
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "unknown loss kind");
  const Graph* g = &G->g;
  ZOGCU_CUDA(cudaSetDevice(M->device));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(nullptr));
  DevBuf pr;
  ZOGCU_TRY(pr.alloc((size_t)std::max<uint32_t>(g->V, 1) * 8, sg.s));
  ZOGCU_CUDA(cudaMemcpyAsync(pr.ptr, target_pr, (size_t)g->V * 8, cudaMemcpyHostToDevice, sg.s));
  WorkLease lease(&M->acts, sg.s);
  GnnActs act;
  ZOGCU_TRY(act.alloc(g->V, lease, true));
  if (!g->offsets32) return fail(ZOGCU_ERR_TOO_LARGE, "the warm-start network needs fewer than 2^32 arcs");
  ZOGCU_TRY(gnn_forward(M, original_view(g), act, true, sg.s));
  ZOGCU_TRY(gnn_backward(M, g, act, pr.as<double>(), loss_kind, sg.s));
  double l = 0.0;
  ZOGCU_CUDA(cudaMemcpyAsync(&l, M->loss.ptr, 8, cudaMemcpyDeviceToHost, sg.s));
  if (grad_out) ZOGCU_CUDA(cudaMemcpyAsync(grad_out, M->g.ptr, kNumParams * 4, cudaMemcpyDeviceToHost, sg.s));
  ZOGCU_TRY(check_dense_error(M, sg.s));
  if (loss) *loss = (float)l;
  return ZOGCU_OK;
}

// One Adam step on one graph; the target PageRank vector is a device pointer.
int zogcu_gnn_train_step(zogcu_gnn* M, zogcu_graph* G, const double* d_target_pr, int loss_kind, float lr,
                         float* loss) {
  if (!M || !G || !d_target_pr) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  if (loss_kind != ZOGCU_GNN_LOSS_LOG_MSE && loss_kind != ZOGCU_GNN_LOSS_KL)
    return fail(ZOGCU_ERR_INVALID_ARGUMENT, "unknown loss kind");
  const Graph* g = &G->g;
  ZOGCU_CUDA(cudaSetDevice(M->device));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(nullptr));
  WorkLease lease(&M->acts, sg.s);
  GnnActs act;
  ZOGCU_TRY(act.alloc(g->V, lease, true));
  if (!g->offsets32) return fail(ZOGCU_ERR_TOO_LARGE, "the warm-start network needs fewer than 2^32 arcs");
  ZOGCU_TRY(gnn_forward(M, original_view(g), act, true, sg.s));
  ZOGCU_TRY(gnn_backward(M, g, act, d_target_pr, loss_kind, sg.s));
  M->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)M->step), c2 = 1.f - std::pow(b2, (float)M->step);
  k_gnn_adam<<<g1d(kNumParams), 256, 0, sg.s>>>(M->p.as<float>(), M->g.as<float>(), M->m.as<float>(), M->s.as<float>(),
                                                M->pb.as<__nv_bfloat16>(), kNumParams, lr, b1, b2, 1e-8f, c1, c2);
  ZOGCU_CUDA(cudaGetLastError());
  double l = 0.0;
  ZOGCU_CUDA(cudaMemcpyAsync(&l, M->loss.ptr, 8, cudaMemcpyDeviceToHost, sg.s));
  ZOGCU_TRY(check_dense_error(M, sg.s));
  if (loss) *loss = (float)l;
  return ZOGCU_OK;
}

// Start vector (length V, sums to 1 over live nodes) into x0 (device pointer
// when device_out != 0), on `stream` (NULL = a private stream).
int zogcu_gnn_predict(const zogcu_gnn* M, zogcu_graph* G, double* x0, int device_out, void* stream,
                      float* raw_out) {
  if (!M || !G || !x0) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  Graph* g = &G->g;
  const uint32_t V = g->V;
  if (!g->offsets32) return fail(ZOGCU_ERR_TOO_LARGE, "the warm-start network needs fewer than 2^32 arcs");
  ZOGCU_CUDA(cudaSetDevice(M->device));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(stream));
  // inference runs in the degree-ranked view the PageRank solver uses (built
  // once per graph and shared with it)
  ZOGCU_TRY(ensure_pr_schedule(g, sg.s));
  const GView gv = ranked_view(g);
  WorkLease lease(&M->acts, sg.s);
  GnnActs act;
  ZOGCU_TRY(act.alloc(V, lease, false));
  ZOGCU_TRY(gnn_forward(M, gv, act, false, sg.s));
  const size_t Vs = std::max<uint32_t>(V, 1);
  DevBuf xr, xd, yr;
  ZOGCU_TRY(xr.alloc(Vs * 8, sg.s));
  Softmax sm;
  ZOGCU_TRY(sm.run(gv, act.y.as<float>(), xr.as<double>(), sg.s));
  double* xo = x0;
  if (!device_out) {
    ZOGCU_TRY(xd.alloc(Vs * 8, sg.s));
    xo = xd.as<double>();
  }
  const uint32_t* rank = g->pr.rank.as<uint32_t>();
  k_gnn_unrank<<<g1d(V), 256, 0, sg.s>>>(xr.as<double>(), rank, V, xo);
  ZOGCU_CUDA(cudaGetLastError());
  if (!device_out) ZOGCU_CUDA(cudaMemcpyAsync(x0, xo, (size_t)V * 8, cudaMemcpyDeviceToHost, sg.s));
  if (raw_out) {
    ZOGCU_TRY(yr.alloc(Vs * 4, sg.s));
    k_gnn_unrank_f<<<g1d(V), 256, 0, sg.s>>>(act.y.as<float>(), rank, V, yr.as<float>());
    ZOGCU_CUDA(cudaGetLastError());
    ZOGCU_CUDA(cudaMemcpyAsync(raw_out, yr.ptr, (size_t)V * 4, cudaMemcpyDeviceToHost, sg.s));
  }
  ZOGCU_TRY(check_dense_error(M, sg.s));
  return ZOGCU_OK;
}

// Versioned weight file: magic, version, parameter count, then the BF16 weights.
int zogcu_gnn_save(const zogcu_gnn* M, const char* path) {
  if (!M || !path) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<uint16_t> h(kNumParams);
  ZOGCU_CUDA(cudaMemcpy(h.data(), M->pb.ptr, kNumParams * 2, cudaMemcpyDeviceToHost));
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(ZOGCU_ERR_IO, std::string("cannot write ") + path);
  const uint32_t hdr[3] = {kGnnMagic, kGnnVersion, (uint32_t)kNumParams};
  const bool ok = std::fwrite(hdr, 4, 3, f) == 3 && std::fwrite(h.data(), 2, h.size(), f) == h.size();
  std::fclose(f);
  return ok ? ZOGCU_OK : fail(ZOGCU_ERR_IO, "short write");
}

int zogcu_gnn_load(const char* path, zogcu_gnn** out) {
  if (!path || !out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(ZOGCU_ERR_IO, std::string("cannot open ") + path);
  uint32_t hdr[3] = {0, 0, 0};
  std::vector<uint16_t> h(kNumParams);
  const bool ok = std::fread(hdr, 4, 3, f) == 3 && hdr[0] == kGnnMagic && hdr[1] == kGnnVersion &&
                  hdr[2] == (uint32_t)kNumParams && std::fread(h.data(), 2, h.size(), f) == h.size();
  std::fclose(f);
  if (!ok) return fail(ZOGCU_ERR_IO, std::string("not a version-2 warm-start weight file: ") + path);
  std::vector<float> p(kNumParams);
  for (int i = 0; i < kNumParams; ++i) {
    const uint32_t bits = (uint32_t)h[i] << 16;
    std::memcpy(&p[i], &bits, 4);
  }
  zogcu_gnn* M = nullptr;
  ZOGCU_TRY(zogcu_gnn_create(0, &M));
  const int rc = zogcu_gnn_set_params(M, p.data());
  if (rc != ZOGCU_OK) {
    zogcu_gnn_destroy(M);
    return rc;
  }
  *out = M;
  return ZOGCU_OK;
}

}  // extern "C"
