// gnn.cu -- the learned PageRank warm start: a small message-passing network
// whose prediction is only the start vector of the power iteration, which
// then runs to the same residual (so the plain method alone decides the result).
//
// Model (hidden width 64; FP32 master weights, BF16 weights and BF16 operands
// in the dense layers, FP32 accumulation everywhere):
//   features  F(v) = [log(1+indeg), log(1+outdeg), outdeg == 0, 1/n]   (FP32)
//   layer l   A_l = agg(H_{l-1})                                        (FP32 sums)
//             H_l = bf16(relu(bf16(H_{l-1}) Ws_l + bf16(A_l) Wn_l + b_l)),  H_0 = F
//   head      y(v) = H_3(v) . w_o + b_o   (a prediction of log(n * pr(v)))
//   start     x0(v) = exp(y(v)) / sum_u exp(y(u))  (positive, sums to 1)
// where agg(H)(v) = sum over in-neighbours u of H(u) / max(outdeg(u), 1) --
// the PageRank propagation operator, so each layer can learn one weighted
// power step.  Training minimises KL(pr || x0) (or the mean squared error of
// y against log(n pr)) on PageRank vectors that the plain method computes;
// the BF16 roundings pass gradients straight through.  Every kernel below is
// hand-written: the SpMM aggregate and its transpose, the dense layer on the
// tensor cores (mma.m16n8k16 BF16) with its data and weight gradients, the
// head, the softmax and Adam; the gradients are checked against a CPU oracle
// that torch autograd pins.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "common.cuh"

namespace zogcu {
namespace {

constexpr int kH = 64;     // hidden width
constexpr int kF = 4;      // input features
constexpr int kLayers = 3;
constexpr uint32_t kGnnMagic = 0x5A4F474E;  // "ZOGN"
constexpr uint32_t kGnnVersion = 1;

// Flat parameter layout: per layer [Ws (din x 64) | Wn (din x 64) | b (64)], then [w_o (64) | b_o].
constexpr int layer_in(int l) { return l == 0 ? kF : kH; }
constexpr int layer_size(int l) { return 2 * layer_in(l) * kH + kH; }
constexpr int layer_offset(int l) { return l == 0 ? 0 : layer_offset(l - 1) + layer_size(l - 1); }
constexpr int kHeadOffset = layer_offset(kLayers);
constexpr int kNumParams = kHeadOffset + kH + 1;

__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---- features and inverse out-degrees -----------------------------------------
__global__ void k_gnn_features(const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ out_deg, uint32_t V,
                               float inv_n, float* __restrict__ F, float* __restrict__ inv_deg) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t od = out_deg[v];
    const bool deleted = od == kDeletedDegree;
    const float id = (float)(in_off[v + 1] - in_off[v]);
    F[(size_t)v * kF + 0] = deleted ? 0.f : log1pf(id);
    F[(size_t)v * kF + 1] = deleted ? 0.f : log1pf((float)od);
    F[(size_t)v * kF + 2] = (!deleted && od == 0) ? 1.f : 0.f;
    F[(size_t)v * kF + 3] = deleted ? 0.f : inv_n;
    inv_deg[v] = (deleted || od == 0) ? 0.f : 1.f / (float)od;
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

// ---- SpMM aggregate: Z(v) = sum over row v of H(u) * w(u)  [* inv(v) when transposed]
// Forward: in-CSR, w(u) = 1/outdeg(u).  Backward (transpose of the forward
// operator): out-CSR, w = 1, and the row sum scaled by 1/outdeg(v).
//
// Work split: the arcs are cut into chunks of kChunk arcs that warps take from
// a shared counter (so a hub row is shared by many warps and no warp holds a
// fixed share of slow chunks); the first row of every chunk is precomputed
// (k_chunk_rows).  A row that crosses a chunk boundary is added with atomics,
// a row inside one chunk is stored directly.  Each arc's feature row (D
// values of T) is read 16 bytes per lane by LPA = D*sizeof(T)/16 lanes, and a
// chunk runs in one of two modes:
//   * rows mode (the chunk holds several rows, none long): each group of LPA
//     lanes owns one row and walks its arcs, 32/LPA rows in flight per warp,
//     four independent gathers in flight per group;
//   * arcs mode (one or two rows, or a long segment): the whole warp walks
//     each row's arcs 32/LPA at a time (indices and weights loaded once,
//     coalesced, and broadcast by shuffles), then folds the groups.
// Sums are FP32.  With accumulate == 0 the caller zeroes Z first (rows that
// hold no arc of any chunk are never visited).
constexpr uint32_t kChunk = 128;

__global__ void k_chunk_rows(const uint32_t* __restrict__ off, uint32_t V, uint32_t E, uint32_t* __restrict__ first_row) {
  const uint32_t nchunks = (uint32_t)(((uint64_t)E + kChunk - 1) / kChunk);
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x) {
    const uint32_t cs = c * kChunk;
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
__device__ __forceinline__ void add_row(float (&acc)[PER], const uint4 x, float w) {
  if (sizeof(T) == 4) {
    acc[0] += __uint_as_float(x.x) * w;
    acc[1] += __uint_as_float(x.y) * w;
    acc[2] += __uint_as_float(x.z) * w;
    acc[3] += __uint_as_float(x.w) * w;
  } else {
    acc[0] += bf16_lo(x.x) * w;
    acc[1] += bf16_hi(x.x) * w;
    acc[2 % PER] += bf16_lo(x.y) * w;
    acc[3 % PER] += bf16_hi(x.y) * w;
    acc[4 % PER] += bf16_lo(x.z) * w;
    acc[5 % PER] += bf16_hi(x.z) * w;
    acc[6 % PER] += bf16_lo(x.w) * w;
    acc[7 % PER] += bf16_hi(x.w) * w;
  }
}

// writes or adds one row's PER values held by one lane
template <int D, int PER>
__device__ __forceinline__ void put_row(float* __restrict__ Z, uint32_t r, int sub, float (&acc)[PER], bool whole,
                                        int accumulate) {
  float* z = Z + (size_t)r * D + sub * PER;
  if (whole) {
#pragma unroll
    for (int i = 0; i < PER; i += 4) {
      float4 o = accumulate ? *reinterpret_cast<float4*>(z + i) : make_float4(0.f, 0.f, 0.f, 0.f);
      o.x += acc[i];
      o.y += acc[i + 1];
      o.z += acc[i + 2];
      o.w += acc[i + 3];
      *reinterpret_cast<float4*>(z + i) = o;
    }
  } else {
#pragma unroll
    for (int i = 0; i < PER; ++i) atomicAdd(z + i, acc[i]);
  }
}

template <class T, int D>
__global__ void __launch_bounds__(256) k_gnn_spmm(const uint32_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                  const float* __restrict__ inv_deg, const T* __restrict__ H,
                                                  uint32_t V, uint32_t E, int transpose, float* __restrict__ Z,
                                                  int accumulate, uint32_t* __restrict__ next_chunk,
                                                  const uint32_t* __restrict__ first_row) {
  constexpr int PER = 16 / (int)sizeof(T);  // values per lane
  constexpr int LPA = D / PER;              // lanes per arc
  constexpr int APW = 32 / LPA;             // arcs per warp step = rows per warp in rows mode
  static_assert(LPA >= 1 && LPA <= 32 && 32 % LPA == 0, "row width");
  const int lane = threadIdx.x & 31, sub = lane % LPA, grp = lane / LPA;
  const uint4* __restrict__ H16 = reinterpret_cast<const uint4*>(H);
  const uint32_t nchunks = (uint32_t)(((uint64_t)E + kChunk - 1) / kChunk);
  for (;;) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(next_chunk, 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= nchunks) break;
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
            float w[4];
            uint4 x[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) u[k] = __ldg(col + j + k);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              w[k] = transpose ? 1.f : __ldg(inv_deg + u[k]);
              x[k] = __ldg(H16 + (size_t)u[k] * LPA + sub);
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) add_row<T, PER>(acc, x[k], w[k]);
          }
          for (; j < e; ++j) {
            const uint32_t u = __ldg(col + j);
            add_row<T, PER>(acc, __ldg(H16 + (size_t)u * LPA + sub), transpose ? 1.f : __ldg(inv_deg + u));
          }
          const uint32_t r = r0 + q;
          if (transpose) {
            const float sc = __ldg(inv_deg + r);
#pragma unroll
            for (int i = 0; i < PER; ++i) acc[i] *= sc;
          }
          put_row<D, PER>(Z, r, sub, acc, qb >= cs && qe <= ce, accumulate);
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
            uint32_t u_l = 0;
            float w_l = 0.f;
            if ((uint32_t)lane < n) {
              u_l = __ldg(col + j0 + lane);
              w_l = transpose ? 1.f : __ldg(inv_deg + u_l);
            }
#pragma unroll 4
            for (uint32_t k = 0; k < n; k += APW) {
              const uint32_t idx = k + grp;
              const uint32_t u = __shfl_sync(0xffffffffu, u_l, idx & 31);
              const float w = __shfl_sync(0xffffffffu, w_l, idx & 31);
              if (idx < n) add_row<T, PER>(acc, __ldg(H16 + (size_t)u * LPA + sub), w);
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
            put_row<D, PER>(Z, r, sub, acc, qb >= cs && qe <= ce, accumulate);
          }
        }
      }
      if (nrows < 32) break;  // the chunk ended inside these rows
      r0 += 32;
    }
  }
}

// ---- dense layer forward on the tensor cores ---------------------------------
// Out = bf16(relu([X | A] W + b)) with W = [Ws ; Wn] (2*DIN x 64, BF16) and the
// operands [X | A] rounded to BF16; products accumulate in FP32
// (mma.m16n8k16, BF16 in, FP32 out).  Each warp computes 16-node tiles: A
// fragments come straight from global memory (row g / g+8, columns
// 2t, 2t+1, 2t+8, 2t+9 of each 16-wide k-step), the weight fragments sit in
// shared memory in fragment order (one conflict-free 8-byte load per mma),
// and the epilogue adds the bias, applies ReLU and stores BF16 pairs.
__device__ __forceinline__ void mma_bf16_16x8x16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                                 uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// elements (k, k+1) of row `row` of [X | A] as a BF16 pair (k even; 0 past 2*DIN)
template <int DIN, class XT>
__device__ __forceinline__ uint32_t dense_pair(const XT* __restrict__ X, const float* __restrict__ A, uint32_t row,
                                               bool valid, int k) {
  if (!valid || k >= 2 * DIN) return 0u;
  if (k < DIN) {
    if (sizeof(XT) == 2) return __ldg(reinterpret_cast<const uint32_t*>(X + (size_t)row * DIN + k));
    const float2 v = __ldg(reinterpret_cast<const float2*>(X + (size_t)row * DIN + k));
    return pack_bf16x2(v.x, v.y);
  }
  const float2 v = __ldg(reinterpret_cast<const float2*>(A + (size_t)row * DIN + (k - DIN)));
  return pack_bf16x2(v.x, v.y);
}

template <int DIN, class XT>
__global__ void __launch_bounds__(256) k_gnn_dense_fwd(const XT* __restrict__ X, const float* __restrict__ A,
                                                       const __nv_bfloat16* __restrict__ w, uint32_t V,
                                                       __nv_bfloat16* __restrict__ Out) {
  constexpr int K = 2 * DIN;
  constexpr int KS = (K + 15) / 16;  // k-steps
  __shared__ uint2 s_b[KS][8][32];  // weight fragments: [k-step][n-tile][lane]
  __shared__ float s_bias[kH];
  for (int i = threadIdx.x; i < KS * 8 * 32; i += blockDim.x) {
    const int ks = i / 256, nt = (i / 32) % 8, l = i % 32;
    const int n = nt * 8 + (l >> 2), k0 = ks * 16 + (l & 3) * 2;
    auto wk = [&](int k) { return k < K ? __bfloat162float(w[(size_t)k * kH + n]) : 0.f; };
    s_b[ks][nt][l] = make_uint2(pack_bf16x2(wk(k0), wk(k0 + 1)), pack_bf16x2(wk(k0 + 8), wk(k0 + 9)));
  }
  for (int i = threadIdx.x; i < kH; i += blockDim.x) s_bias[i] = __bfloat162float(w[(size_t)K * kH + i]);
  __syncthreads();
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const uint32_t tiles = (V + 15) / 16;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < tiles; tile += nw) {
    const uint32_t r0 = tile * 16 + g, r1 = r0 + 8;
    const bool v0 = r0 < V, v1 = r1 < V;
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
      const int k = ks * 16 + t * 2;
      const uint32_t a0 = dense_pair<DIN>(X, A, r0, v0, k);
      const uint32_t a1 = dense_pair<DIN>(X, A, r1, v1, k);
      const uint32_t a2 = dense_pair<DIN>(X, A, r0, v0, k + 8);
      const uint32_t a3 = dense_pair<DIN>(X, A, r1, v1, k + 8);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const uint2 bb = s_b[ks][nt][lane];
        mma_bf16_16x8x16(acc[nt], a0, a1, a2, a3, bb.x, bb.y);
      }
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = nt * 8 + t * 2;
      const float b0 = s_bias[c], b1 = s_bias[c + 1];
      if (v0)
        *reinterpret_cast<uint32_t*>(Out + (size_t)r0 * kH + c) =
            pack_bf16x2(fmaxf(acc[nt][0] + b0, 0.f), fmaxf(acc[nt][1] + b1, 0.f));
      if (v1)
        *reinterpret_cast<uint32_t*>(Out + (size_t)r1 * kH + c) =
            pack_bf16x2(fmaxf(acc[nt][2] + b0, 0.f), fmaxf(acc[nt][3] + b1, 0.f));
    }
  }
}

// ---- dense layer backward (data): dP = dOut * (Out > 0); dX = dP Ws^T, dA = dP Wn^T
// (the BF16 rounding of the forward operands passes the gradient straight
// through).  dP is written back in place of dOut for the weight-gradient kernel.
template <int DIN>
__global__ void __launch_bounds__(256) k_gnn_dense_bwd_data(float* __restrict__ dOut,
                                                            const __nv_bfloat16* __restrict__ Out,
                                                            const __nv_bfloat16* __restrict__ w, uint32_t V,
                                                            float* __restrict__ dX, float* __restrict__ dA) {
  __shared__ float s_ws[DIN][kH];
  __shared__ float s_wn[DIN][kH];
  for (int i = threadIdx.x; i < DIN * kH; i += blockDim.x) {
    s_ws[i / kH][i % kH] = __bfloat162float(w[i]);
    s_wn[i / kH][i % kH] = __bfloat162float(w[DIN * kH + i]);
  }
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
    float x0 = 0.f, x1 = 0.f, a0 = 0.f, a1 = 0.f;
#pragma unroll 8
    for (int j = 0; j < kH; ++j) {
      const float pj = __shfl_sync(0xffffffffu, j < 32 ? p0 : p1, j & 31);
      if (lane < DIN) {
        x0 += pj * s_ws[lane][j];
        a0 += pj * s_wn[lane][j];
      }
      if (lane + 32 < DIN) {
        x1 += pj * s_ws[lane + 32][j];
        a1 += pj * s_wn[lane + 32][j];
      }
    }
    if (lane < DIN) {
      dX[(size_t)v * DIN + lane] = x0;
      dA[(size_t)v * DIN + lane] = a0;
    }
    if (lane + 32 < DIN) {
      dX[(size_t)v * DIN + lane + 32] = x1;
      dA[(size_t)v * DIN + lane + 32] = a1;
    }
  }
}

// ---- dense layer backward (weights): dWs += bf16(X)^T dP, dWn += bf16(A)^T dP,
// db += sum dP -- the operands the forward pass multiplied.  Each block folds
// a tile of nodes in shared memory, then adds its partial into the global FP32
// gradient with one atomic per weight.
template <int DIN, class XT>
__global__ void __launch_bounds__(256) k_gnn_dense_bwd_weight(const XT* __restrict__ X, const float* __restrict__ A,
                                                              const float* __restrict__ dP, uint32_t V,
                                                              float* __restrict__ grad) {
  constexpr int TILE = 32;
  __shared__ float s_x[TILE][DIN];
  __shared__ float s_a[TILE][DIN];
  __shared__ float s_p[TILE][kH];
  // thread t owns outputs (k, j) = (t / kH + r * 256 / kH, t % kH) for r < DIN*kH/256
  constexpr int PER = (DIN * kH + 255) / 256;
  float gs[PER], gn[PER], gb = 0.f;
#pragma unroll
  for (int r = 0; r < PER; ++r) gs[r] = gn[r] = 0.f;
  for (uint32_t base = blockIdx.x * TILE; base < V; base += gridDim.x * TILE) {
    const uint32_t cnt = min((uint32_t)TILE, V - base);
    __syncthreads();
    for (int i = threadIdx.x; i < TILE * DIN; i += blockDim.x) {
      const uint32_t n = i / DIN;
      s_x[n][i % DIN] = n < cnt ? bf16_round(to_f32(X[(size_t)(base + n) * DIN + i % DIN])) : 0.f;
      s_a[n][i % DIN] = n < cnt ? bf16_round(A[(size_t)(base + n) * DIN + i % DIN]) : 0.f;
    }
    for (int i = threadIdx.x; i < TILE * kH; i += blockDim.x) {
      const uint32_t n = i / kH;
      s_p[n][i % kH] = n < cnt ? dP[(size_t)(base + n) * kH + i % kH] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < PER; ++r) {
      const int idx = threadIdx.x + r * 256;
      if (idx < DIN * kH) {
        const int k = idx / kH, j = idx % kH;
        float s1 = 0.f, s2 = 0.f;
        for (int n = 0; n < TILE; ++n) {
          s1 += s_x[n][k] * s_p[n][j];
          s2 += s_a[n][k] * s_p[n][j];
        }
        gs[r] += s1;
        gn[r] += s2;
      }
    }
    if (threadIdx.x < kH)
      for (int n = 0; n < TILE; ++n) gb += s_p[n][threadIdx.x];
  }
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int idx = threadIdx.x + r * 256;
    if (idx < DIN * kH) {
      atomicAdd(grad + idx, gs[r]);
      atomicAdd(grad + DIN * kH + idx, gn[r]);
    }
  }
  if (threadIdx.x < kH) atomicAdd(grad + 2 * DIN * kH + threadIdx.x, gb);
}

// ---- head forward: y = H3 . w_o + b_o ----------------------------------------
__global__ void __launch_bounds__(256) k_gnn_head(const __nv_bfloat16* __restrict__ H,
                                                  const __nv_bfloat16* __restrict__ wo, uint32_t V,
                                                  float* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const float w0 = __bfloat162float(wo[2 * lane]), w1 = __bfloat162float(wo[2 * lane + 1]);
  const float bo = __bfloat162float(wo[kH]);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < V; v += nw) {
    const uint32_t h = __ldg(reinterpret_cast<const uint32_t*>(H + (size_t)v * kH) + lane);
    float s = bf16_lo(h) * w0 + bf16_hi(h) * w1;
    s = warp_sumf(s);
    if (lane == 0) y[v] = s + bo;
  }
}

// ---- loss and head backward -------------------------------------------------
// mode 0: loss = mean over live nodes of (y - t)^2, t = log(n pr)
//         dy = 2 (y - t) / n
// mode 1: loss = KL(pr || x0) with x0 = softmax(y) over live nodes
//              = sum_v pr(v) (log pr(v) - (y(v) - ymax) + log S),  S = sum exp(y - ymax)
//         dy = x0 - pr   (pr sums to 1)
// then dH3 = dy w_o, dw_o = sum dy H3, db_o = sum dy.  The loss is summed in FP64.
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

}  // namespace
}  // namespace zogcu

using namespace zogcu;

struct zogcu_gnn {
  int device = 0;
  DevArray p, pb, m, s, g, loss;   // masters, BF16 copy, Adam moments, gradient, loss (FP64)
  uint64_t step = 0;
  // activations of the largest graph seen so far (about 940 bytes per node),
  // reused by later calls until the model is destroyed
  mutable WorkCache acts;
};

namespace zogcu {
namespace {

// Activations of one forward pass over a graph (kept for the backward pass):
// features F and aggregates A in FP32, hidden states H in BF16.
struct GnnActs {
  DevBuf F, inv, y, t, ctr, rows;
  DevBuf H[kLayers], A[kLayers];
  // from the model's cache when the lease holds it, else per call
  int alloc(uint32_t V, WorkLease& L) {
    const size_t Vs = std::max<uint32_t>(V, 1);
    ZOGCU_TRY(L.get(F, 0, Vs * kF * 4));
    ZOGCU_TRY(L.get(inv, 1, Vs * 4));
    ZOGCU_TRY(L.get(y, 2, Vs * 4));
    ZOGCU_TRY(L.get(ctr, 3, 16));
    for (int l = 0; l < kLayers; ++l) {
      ZOGCU_TRY(L.get(H[l], 4 + l, Vs * kH * 2));
      ZOGCU_TRY(L.get(A[l], 4 + kLayers + l, Vs * (size_t)layer_in(l) * 4));
    }
    return ZOGCU_OK;
  }
};

// First row of every kChunk-arc chunk of the in-CSR (transpose = 0) or the
// out-CSR (transpose = 1), into `rows` (allocated here).
int chunk_rows(const Graph* g, bool transpose, DevBuf& rows, cudaStream_t s) {
  const uint32_t E = (uint32_t)g->E;
  const uint64_t chunks = ((uint64_t)E + kChunk - 1) / kChunk;
  ZOGCU_TRY(rows.alloc(std::max<uint64_t>(chunks, 1) * 4, s));
  if (chunks == 0) return ZOGCU_OK;
  const uint32_t* off = (transpose ? g->out_off32 : g->in_off32).as<uint32_t>();
  k_chunk_rows<<<g1d(chunks), 256, 0, s>>>(off, g->V, E, rows.as<uint32_t>());
  ZOGCU_CUDA(cudaGetLastError());
  return ZOGCU_OK;
}

// Z = agg(X) (forward, in-CSR) or Z (+)= agg^T(X) (transpose, out-CSR);
// `ctr` is a device word for the chunk counter, `rows` the chunks' first rows.
template <class T, int D>
int spmm(const Graph* g, bool transpose, const float* inv, const T* X, float* Z, bool accumulate, uint32_t* ctr,
         const DevBuf& rows, cudaStream_t s) {
  const uint32_t V = g->V;
  const uint32_t E = (uint32_t)g->E;
  if (!accumulate) ZOGCU_CUDA(cudaMemsetAsync(Z, 0, (size_t)V * D * 4, s));
  if (E == 0) return ZOGCU_OK;
  const uint32_t* off = (transpose ? g->out_off32 : g->in_off32).as<uint32_t>();
  const uint32_t* col = (transpose ? g->out_col : g->in_col).as<uint32_t>();
  const uint64_t chunks = ((uint64_t)E + kChunk - 1) / kChunk;
  ZOGCU_CUDA(cudaMemsetAsync(ctr, 0, 4, s));
  k_gnn_spmm<T, D><<<gwarp(chunks), 256, 0, s>>>(off, col, inv, X, V, E, transpose ? 1 : 0, Z, accumulate ? 1 : 0,
                                                 ctr, rows.as<uint32_t>());
  return ZOGCU_OK;
}

unsigned gtile16(uint32_t V) { return gwarp(((uint64_t)V + 15) / 16); }

int gnn_forward(const zogcu_gnn* M, const Graph* g, GnnActs& act, cudaStream_t s) {
  const uint32_t V = g->V;
  if (!g->offsets32) return fail(ZOGCU_ERR_TOO_LARGE, "the warm-start network needs fewer than 2^32 arcs");
  const uint32_t* ioff = g->in_off32.as<uint32_t>();
  const __nv_bfloat16* w = M->pb.as<__nv_bfloat16>();
  uint32_t* ctr = act.ctr.as<uint32_t>();
  k_gnn_features<<<g1d(V), 256, 0, s>>>(ioff, g->out_deg.as<uint32_t>(), V, 1.f / (float)std::max<uint64_t>(g->n_live, 1),
                                        act.F.as<float>(), act.inv.as<float>());
  const float* inv = act.inv.as<float>();
  ZOGCU_TRY(chunk_rows(g, false, act.rows, s));
  ZOGCU_TRY((spmm<float, kF>(g, false, inv, act.F.as<float>(), act.A[0].as<float>(), false, ctr, act.rows, s)));
  k_gnn_dense_fwd<kF, float><<<gtile16(V), 256, 0, s>>>(act.F.as<float>(), act.A[0].as<float>(), w + layer_offset(0), V,
                                                        act.H[0].as<__nv_bfloat16>());
  for (int l = 1; l < kLayers; ++l) {
    const __nv_bfloat16* X = act.H[l - 1].as<__nv_bfloat16>();
    ZOGCU_TRY((spmm<__nv_bfloat16, kH>(g, false, inv, X, act.A[l].as<float>(), false, ctr, act.rows, s)));
    k_gnn_dense_fwd<kH, __nv_bfloat16><<<gtile16(V), 256, 0, s>>>(X, act.A[l].as<float>(), w + layer_offset(l), V,
                                                                  act.H[l].as<__nv_bfloat16>());
  }
  k_gnn_head<<<gwarp(V), 256, 0, s>>>(act.H[kLayers - 1].as<__nv_bfloat16>(), w + kHeadOffset, V, act.y.as<float>());
  ZOGCU_CUDA(cudaGetLastError());
  return ZOGCU_OK;
}

// x = softmax(y) over live nodes (FP64), with ymax and S = sum exp(y - ymax)
// left in device scalars.
struct Softmax {
  DevBuf ymax, part, stot;
  unsigned grid = 1;
  int run(const Graph* g, const float* y, double* x, cudaStream_t s) {
    const uint32_t V = g->V;
    grid = g1d(V);
    ZOGCU_TRY(ymax.alloc(16, s));
    ZOGCU_TRY(stot.alloc(16, s));
    ZOGCU_TRY(part.alloc((size_t)grid * 8, s));
    // -inf: every live y is larger; the CAS loop below only raises it
    k_fill_f32<<<1, 32, 0, s>>>(ymax.as<float>(), 1, -INFINITY);
    k_gnn_softmax_max<<<grid, 256, 0, s>>>(y, g->out_deg.as<uint32_t>(), V, ymax.as<float>());
    k_gnn_softmax_exp<<<grid, 256, 0, s>>>(y, g->out_deg.as<uint32_t>(), V, ymax.as<float>(), x, part.as<double>());
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
    ZOGCU_TRY(sm.run(g, act.y.as<float>(), xq.as<double>(), s));
  }
  DevBuf dH, dX, dA;
  ZOGCU_TRY(dH.alloc(Vs * kH * 4, s));
  ZOGCU_TRY(dX.alloc(Vs * kH * 4, s));
  ZOGCU_TRY(dA.alloc(Vs * kH * 4, s));
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
    const __nv_bfloat16* wl = w + layer_offset(l);
    k_gnn_dense_bwd_data<kH><<<gwarp(V), 256, 0, s>>>(pdH, act.H[l].as<__nv_bfloat16>(), wl, V, pdX, dA.as<float>());
    k_gnn_dense_bwd_weight<kH, __nv_bfloat16><<<gtile(V), 256, 0, s>>>(
        act.H[l - 1].as<__nv_bfloat16>(), act.A[l].as<float>(), pdH, V, grad + layer_offset(l));
    // gradient of H_{l-1}: dX + agg^T(dA); dX becomes the next layer's dH
    ZOGCU_TRY((spmm<float, kH>(g, true, act.inv.as<float>(), dA.as<float>(), pdX, true, ctr, out_rows, s)));
    std::swap(pdH, pdX);
  }
  k_gnn_dense_bwd_data<kF><<<gwarp(V), 256, 0, s>>>(pdH, act.H[0].as<__nv_bfloat16>(), w, V, pdX, dA.as<float>());
  k_gnn_dense_bwd_weight<kF, float><<<gtile(V), 256, 0, s>>>(act.F.as<float>(), act.A[0].as<float>(), pdH, V, grad);
  ZOGCU_CUDA(cudaGetLastError());
  return ZOGCU_OK;
}

// Glorot-uniform initial weights from a seeded SplitMix64 stream.
void gnn_init_host(uint64_t seed, std::vector<float>& p) {
  p.assign(kNumParams, 0.f);
  uint64_t st = seed;
  auto next = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  auto uni = [&]() { return (float)((next() >> 40) * (1.0 / 16777216.0)) * 2.f - 1.f; };
  for (int l = 0; l < kLayers; ++l) {
    const int din = layer_in(l);
    const float a = std::sqrt(6.f / (float)(din + kH));
    float* base = p.data() + layer_offset(l);
    for (int i = 0; i < 2 * din * kH; ++i) base[i] = a * uni();
  }
  const float a = std::sqrt(6.f / (float)(kH + 1));
  for (int i = 0; i < kH; ++i) p[kHeadOffset + i] = a * uni();
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
  std::vector<float> h;
  gnn_init_host(seed, h);
  ZOGCU_CUDA(cudaMemcpy(M->p.ptr, h.data(), kNumParams * 4, cudaMemcpyHostToDevice));
  ZOGCU_CUDA(cudaMemset(M->m.ptr, 0, kNumParams * 4));
  ZOGCU_CUDA(cudaMemset(M->s.ptr, 0, kNumParams * 4));
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
  ZOGCU_TRY(act.alloc(g->V, lease));
  ZOGCU_TRY(gnn_forward(M, g, act, sg.s));
  ZOGCU_TRY(gnn_backward(M, g, act, pr.as<double>(), loss_kind, sg.s));
  double l = 0.0;
  ZOGCU_CUDA(cudaMemcpyAsync(&l, M->loss.ptr, 8, cudaMemcpyDeviceToHost, sg.s));
  if (grad_out) ZOGCU_CUDA(cudaMemcpyAsync(grad_out, M->g.ptr, kNumParams * 4, cudaMemcpyDeviceToHost, sg.s));
  ZOGCU_CUDA(cudaStreamSynchronize(sg.s));
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
  ZOGCU_TRY(act.alloc(g->V, lease));
  ZOGCU_TRY(gnn_forward(M, g, act, sg.s));
  ZOGCU_TRY(gnn_backward(M, g, act, d_target_pr, loss_kind, sg.s));
  M->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)M->step), c2 = 1.f - std::pow(b2, (float)M->step);
  k_gnn_adam<<<g1d(kNumParams), 256, 0, sg.s>>>(M->p.as<float>(), M->g.as<float>(), M->m.as<float>(), M->s.as<float>(),
                                                M->pb.as<__nv_bfloat16>(), kNumParams, lr, b1, b2, 1e-8f, c1, c2);
  ZOGCU_CUDA(cudaGetLastError());
  double l = 0.0;
  ZOGCU_CUDA(cudaMemcpyAsync(&l, M->loss.ptr, 8, cudaMemcpyDeviceToHost, sg.s));
  ZOGCU_CUDA(cudaStreamSynchronize(sg.s));
  if (loss) *loss = (float)l;
  return ZOGCU_OK;
}

// Start vector (length V, sums to 1 over live nodes) into x0 (device pointer
// when device_out != 0), on `stream` (NULL = a private stream).
int zogcu_gnn_predict(const zogcu_gnn* M, zogcu_graph* G, double* x0, int device_out, void* stream,
                      float* raw_out) {
  if (!M || !G || !x0) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  const Graph* g = &G->g;
  const uint32_t V = g->V;
  ZOGCU_CUDA(cudaSetDevice(M->device));
  StreamGuard sg;
  ZOGCU_TRY(sg.init(stream));
  WorkLease lease(&M->acts, sg.s);
  GnnActs act;
  ZOGCU_TRY(act.alloc(V, lease));
  ZOGCU_TRY(gnn_forward(M, g, act, sg.s));
  DevBuf xd;
  double* xo = x0;
  if (!device_out) {
    ZOGCU_TRY(xd.alloc((size_t)std::max<uint32_t>(V, 1) * 8, sg.s));
    xo = xd.as<double>();
  }
  Softmax sm;
  ZOGCU_TRY(sm.run(g, act.y.as<float>(), xo, sg.s));
  if (!device_out) ZOGCU_CUDA(cudaMemcpyAsync(x0, xo, (size_t)V * 8, cudaMemcpyDeviceToHost, sg.s));
  if (raw_out) ZOGCU_CUDA(cudaMemcpyAsync(raw_out, act.y.ptr, (size_t)V * 4, cudaMemcpyDeviceToHost, sg.s));
  ZOGCU_CUDA(cudaStreamSynchronize(sg.s));
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
  if (!ok) return fail(ZOGCU_ERR_IO, std::string("not a version-1 warm-start weight file: ") + path);
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
