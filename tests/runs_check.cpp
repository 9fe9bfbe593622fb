// Checks the host run coding of sorted sources (zog_b200/csrc/runs.h) against
// a plain loop on random chunks: sorted, sorted with one swap, unsorted, with
// sources >= V, with gaps and long runs, and with a source before the chunk
// that is larger than its first (a fall across the chunk boundary).  Prints
// "runs ok" and exits 0 when every case agrees.
#include <cstdio>
#include <random>
#include <vector>

#include "runs.h"

// the offsets by a plain loop, or false when the chunk cannot be coded
static bool plain_runs(const std::vector<uint32_t>& f, int64_t prev, uint32_t V, std::vector<uint32_t>& off) {
  const uint64_t n = f.size();
  const uint32_t s0 = f[0], s1 = f[n - 1];
  if ((int64_t)s0 < prev || s1 < s0 || s1 >= V) return false;
  for (uint64_t i = 1; i < n; ++i)
    if (f[i] < f[i - 1]) return false;
  off.assign((size_t)(s1 - s0) + 2, 0);
  uint64_t i = 0;
  for (uint64_t u = s0; u <= (uint64_t)s1 + 1; ++u) {
    while (i < n && f[i] < u) ++i;
    off[u - s0] = (uint32_t)i;
  }
  return true;
}

int main() {
  std::mt19937_64 r(20261204);
  int coded = 0, refused = 0;
  for (int c = 0; c < 4000; ++c) {
    const uint64_t n = 1 + r() % (c < 3000 ? 300 : 20000);
    const uint32_t V = 1 + (uint32_t)(r() % (c % 3 == 0 ? 40 : 5000));
    std::vector<uint32_t> f(n);
    for (auto& x : f) x = (uint32_t)(r() % (V + (r() % 8 == 0 ? 3 : 0)));
    const int shape = (int)(r() % 6);
    if (shape != 0) std::sort(f.begin(), f.end());
    if (shape == 2 && n > 2) std::swap(f[r() % n], f[r() % n]);
    const int64_t prev = (r() % 4 == 0) ? (int64_t)(r() % (V + 1)) : -1;
    std::vector<uint32_t> want;
    const bool w = plain_runs(f, prev, V, want);
    std::vector<uint32_t> got((size_t)V + 8, 0xDEADBEEFu);
    const bool g = zogcu::encode_runs(f.data(), n, prev, V, got.data());
    if (g != w) {
      std::printf("case %d: coded %d, expected %d (n %llu, V %u)\n", c, (int)g, (int)w, (unsigned long long)n, V);
      return 1;
    }
    if (g) {
      ++coded;
      for (size_t k = 0; k < want.size(); ++k)
        if (got[k] != want[k]) {
          std::printf("case %d: off[%zu] = %u, expected %u\n", c, k, got[k], want[k]);
          return 1;
        }
      for (size_t k = want.size(); k < got.size(); ++k)
        if (got[k] != 0xDEADBEEFu) {
          std::printf("case %d: wrote past the offsets at %zu\n", c, k);
          return 1;
        }
    } else {
      ++refused;
      // a refused chunk may leave offsets written, but only inside off[1 .. s1 - s0]
      const uint32_t s0 = f[0], s1 = f[n - 1];
      const size_t hi = s1 >= s0 ? (size_t)(s1 - s0) : 0;
      for (size_t k = 0; k < got.size(); ++k)
        if ((k == 0 || k > hi) && got[k] != 0xDEADBEEFu) {
          std::printf("case %d: refused chunk wrote off[%zu]\n", c, k);
          return 1;
        }
    }
  }
  if (coded < 1000 || refused < 1000) {
    std::printf("too few cases of a kind: %d coded, %d refused\n", coded, refused);
    return 1;
  }
  std::printf("runs ok\n");
  return 0;
}
