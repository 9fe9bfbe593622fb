// Host-side run coding of sorted arc sources (used by the chunked upload in
// graph.cu): a chunk of non-decreasing sources is fixed by its source range
// [s0, s1] and the position where each source's run starts.  Plain C++ with
// no CUDA, so the check can be compiled and tested on its own.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

namespace zogcu {

constexpr int kScanThreads = 16;  // host threads that check one chunk

// Checks from[a, b) of a chunk whose first and last sources are s0 and s1
// (every element non-decreasing from its predecessor and at most s1) and, for
// each position k in [a, b) where the source rises from q to v, writes
// off[u - s0] = k for u in (q, v].  Every such u lies in (s0, s1], so no
// write leaves off[1 .. s1 - s0] even when the check fails part way.  Eight
// sources at a time are compared with their predecessors (SSE2 where the host
// has it): a block without a rise costs no branch per source.
inline bool scan_runs(const uint32_t* from, uint64_t a, uint64_t b, uint32_t s0, uint32_t s1, uint32_t* off) {
  uint32_t p = a ? from[a - 1] : s0;
  if (p < s0 || p > s1) return false;
  auto one = [&](uint64_t k) -> bool {
    const uint32_t v = from[k];
    if (v == p) return true;
    if (v < p || v > s1) return false;
    for (uint32_t u = p + 1; u <= v; ++u) off[u - s0] = (uint32_t)k;
    p = v;
    return true;
  };
  uint64_t i = a;
  if (i < b && !one(i++)) return false;  // from here on from[i - 1] is inside the array
#if defined(__SSE2__)
  const __m128i sign = _mm_set1_epi32((int)0x80000000u);
  for (; i + 8 <= b; i += 8) {
    const __m128i x0 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(from + i));
    const __m128i x1 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(from + i + 4));
    const __m128i y0 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(from + i - 1));
    const __m128i y1 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(from + i + 3));
    const int rise = ~(_mm_movemask_ps(_mm_castsi128_ps(_mm_cmpeq_epi32(x0, y0))) |
                       (_mm_movemask_ps(_mm_castsi128_ps(_mm_cmpeq_epi32(x1, y1))) << 4)) & 0xFF;
    if (!rise) continue;  // all eight equal their predecessors, hence p
    const int fall =
        _mm_movemask_ps(_mm_castsi128_ps(_mm_cmplt_epi32(_mm_xor_si128(x0, sign), _mm_xor_si128(y0, sign)))) |
        (_mm_movemask_ps(_mm_castsi128_ps(_mm_cmplt_epi32(_mm_xor_si128(x1, sign), _mm_xor_si128(y1, sign)))) << 4);
    if (fall) return false;
    for (int m = rise; m; m &= m - 1) {
      const int j = __builtin_ctz(m);
      const uint32_t v = from[i + j], q = from[i + j - 1];
      if (v > s1) return false;
      for (uint32_t u = q + 1; u <= v; ++u) off[u - s0] = (uint32_t)(i + j);
    }
    p = from[i + 7];
  }
#endif
  for (; i < b; ++i)
    if (!one(i)) return false;
  return true;
}

// Offsets of the runs of from[0, n): off[j] = the first position holding a
// source >= s0 + j, for j = 0 .. s1 - s0 + 1 (off[0] = 0, off[s1 - s0 + 1] = n),
// where s0 = from[0] and s1 = from[n - 1].  `prev` is the source before the
// chunk (-1 for none).  Returns false, with off partly written, unless the
// chunk is non-decreasing from prev and every source is < V.  Host threads
// take equal parts of the chunk.
inline bool encode_runs(const uint32_t* from, uint64_t n, int64_t prev, uint32_t V, uint32_t* off) {
  const uint32_t s0 = from[0], s1 = from[n - 1];
  if ((int64_t)s0 < prev || s1 < s0 || s1 >= V) return false;
  std::atomic<bool> ok{true};
  const int T = (int)std::max(1u, std::min((unsigned)kScanThreads, std::thread::hardware_concurrency()));
  const uint64_t part = (n + T - 1) / T;
  std::vector<std::thread> th;
  for (int t = 1; t < T; ++t) {
    const uint64_t a = std::min(n, part * t), b = std::min(n, part * (t + 1));
    if (a >= b) continue;
    auto work = [&, a, b] {
      if (!scan_runs(from, a, b, s0, s1, off)) ok = false;
    };
    try {
      th.emplace_back(work);
    } catch (...) {  // no thread to be had: this part on the calling thread
      work();
    }
  }
  if (!scan_runs(from, 0, std::min(n, part), s0, s1, off)) ok = false;
  for (auto& x : th) x.join();
  if (!ok) return false;
  off[0] = 0;
  off[s1 - s0 + 1] = (uint32_t)n;
  return true;
}

}  // namespace zogcu
