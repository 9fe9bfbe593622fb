// io.cu -- edge-list reader that builds the device graph directly.
//
// Reference: nif_read_edgelist (lib/zog/.Elixir.Zog.ResourceGraph.zig:896-990)
// and addParsedEdges (:859-894).  Semantics kept:
//   * lines are trimmed of ' ', '\t', '\r'; empty lines and lines starting
//     with '#' are skipped; fields split on ' ', '\t' and ',';
//   * a "source target" header (case-insensitive) is skipped;
//   * the third field is the weight, 1.0 when absent or unparsable;
//   * integer_labels: both ids parse as u32 (lines that do not parse are
//     skipped) and the node count is max id + 1, so gaps become isolated
//     placeholder nodes; otherwise string labels get ids in order of first
//     appearance;
//   * directed: arcs are added in file order; undirected: edges are stably
//     sorted by their (min, max) pair, later duplicates of a pair are dropped,
//     and each pair adds from->to then to->from (one arc for a self-loop).
// Instead of materialising an ArrayGraph, the parsed arcs (in the order the
// reference would insert them) go straight to the device CSR builder -- the
// loader path that skips the linked-list build.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <string_view>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace zogcu {

namespace {

inline bool is_trim(char c) { return c == ' ' || c == '\t' || c == '\r'; }
inline bool is_sep(char c) { return c == ' ' || c == '\t' || c == ','; }

// std.fmt.parseInt(u32, s, 10): optional '+', digits with '_' separators
// between digits, no overflow.
bool parse_u32(std::string_view s, uint32_t* out) {
  size_t i = 0;
  if (!s.empty() && s[0] == '+') i = 1;
  if (i >= s.size()) return false;
  uint64_t acc = 0;
  bool digit = false;
  for (; i < s.size(); ++i) {
    const char c = s[i];
    if (c == '_') {
      if (!digit || i + 1 >= s.size() || s[i + 1] == '_') return false;
      continue;
    }
    if (c < '0' || c > '9') return false;
    acc = acc * 10 + (uint64_t)(c - '0');
    if (acc > 0xFFFFFFFFull) return false;
    digit = true;
  }
  if (!digit) return false;
  *out = (uint32_t)acc;
  return true;
}

bool iequals(std::string_view a, const char* b) {
  const size_t n = std::strlen(b);
  if (a.size() != n) return false;
  for (size_t i = 0; i < n; ++i) {
    char x = a[i], y = b[i];
    if (x >= 'A' && x <= 'Z') x = (char)(x - 'A' + 'a');
    if (x != y) return false;
  }
  return true;
}

struct Parsed {
  uint32_t from, to;
};

}  // namespace

}  // namespace zogcu

using namespace zogcu;

extern "C" int zogcu_read_edgelist(const char* path, int directed, int integer_labels, zogcu_graph** out,
                                   uint32_t* next_id_out, char** labels_out, uint64_t* labels_len) {
  if (!path || !out || !next_id_out) return fail(ZOGCU_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (labels_out) *labels_out = nullptr;
  if (labels_len) *labels_len = 0;
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(ZOGCU_ERR_IO, std::string("cannot open ") + path + ": " + std::strerror(errno));
  std::string buf;
  {
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (sz < 0) {
      std::fclose(f);
      return fail(ZOGCU_ERR_IO, "cannot size file");
    }
    buf.resize((size_t)sz);
    if (sz && std::fread(&buf[0], 1, (size_t)sz, f) != (size_t)sz) {
      std::fclose(f);
      return fail(ZOGCU_ERR_IO, "short read");
    }
    std::fclose(f);
  }
  std::vector<Parsed> edges;
  edges.reserve(buf.size() / 8);
  std::unordered_map<std::string_view, uint32_t> label_to_id;
  std::vector<std::string_view> labels;
  uint64_t next_id = 0;
  const char* p = buf.data();
  const char* end = p + buf.size();
  while (p < end) {
    const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
    const char* le = nl ? nl : end;
    const char* b = p;
    const char* e = le;
    p = nl ? nl + 1 : end;
    while (b < e && is_trim(*b)) ++b;
    while (e > b && is_trim(e[-1])) --e;
    if (b == e || *b == '#') continue;
    std::string_view parts[3];
    int np = 0;
    const char* q = b;
    while (q < e && np < 3) {
      while (q < e && is_sep(*q)) ++q;
      const char* r = q;
      while (r < e && !is_sep(*r)) ++r;
      if (r > q) parts[np++] = std::string_view(q, (size_t)(r - q));
      q = r;
    }
    if (np < 2) continue;
    if (iequals(parts[0], "source") && iequals(parts[1], "target")) continue;
    uint32_t s = 0, d = 0;
    if (integer_labels) {
      if (!parse_u32(parts[0], &s) || !parse_u32(parts[1], &d)) continue;
      const uint64_t mx = std::max(s, d);
      if (mx >= next_id) next_id = mx + 1;
    } else {
      for (int k = 0; k < 2; ++k) {
        auto it = label_to_id.find(parts[k]);
        uint32_t id;
        if (it != label_to_id.end()) {
          id = it->second;
        } else {
          if (next_id >= 0xFFFFFFFFull) return fail(ZOGCU_ERR_TOO_LARGE, "too many labels");
          id = (uint32_t)next_id++;
          label_to_id.emplace(parts[k], id);
          labels.push_back(parts[k]);
        }
        (k == 0 ? s : d) = id;
      }
    }
    edges.push_back({s, d});
  }
  if (next_id > 0xFFFFFFFFull) return fail(ZOGCU_ERR_TOO_LARGE, "node id space exceeds u32");
  // arcs in the reference's insertion order
  std::vector<uint32_t> src, dst;
  if (directed) {
    src.resize(edges.size());
    dst.resize(edges.size());
    for (size_t i = 0; i < edges.size(); ++i) {
      src[i] = edges[i].from;
      dst[i] = edges[i].to;
    }
  } else {
    std::stable_sort(edges.begin(), edges.end(), [](const Parsed& x, const Parsed& y) {
      const uint32_t xl = std::min(x.from, x.to), xh = std::max(x.from, x.to);
      const uint32_t yl = std::min(y.from, y.to), yh = std::max(y.from, y.to);
      return xl != yl ? xl < yl : xh < yh;
    });
    src.reserve(edges.size() * 2);
    dst.reserve(edges.size() * 2);
    uint64_t plo = ~0ull, phi = ~0ull;
    for (const Parsed& ed : edges) {
      const uint32_t lo = std::min(ed.from, ed.to), hi = std::max(ed.from, ed.to);
      if (lo == plo && hi == phi) continue;
      src.push_back(ed.from);
      dst.push_back(ed.to);
      if (ed.from != ed.to) {
        src.push_back(ed.to);
        dst.push_back(ed.from);
      }
      plo = lo;
      phi = hi;
    }
  }
  zogcu_graph* g = nullptr;
  int rc = zogcu_graph_create_from_edges((uint32_t)next_id, src.data(), dst.data(), nullptr, src.size(), &g);
  if (rc != ZOGCU_OK) return rc;
  *out = g;
  *next_id_out = (uint32_t)next_id;
  if (!integer_labels && labels_out) {
    size_t total = 0;
    for (auto& l : labels) total += l.size() + 1;
    char* lb = static_cast<char*>(std::malloc(total + 1));
    if (!lb) {
      zogcu_graph_destroy(g);
      *out = nullptr;
      return fail(ZOGCU_ERR_OUT_OF_MEMORY, "label buffer");
    }
    size_t k = 0;
    for (size_t i = 0; i < labels.size(); ++i) {
      if (i) lb[k++] = '\n';
      std::memcpy(lb + k, labels[i].data(), labels[i].size());
      k += labels[i].size();
    }
    lb[k] = '\0';
    *labels_out = lb;
    if (labels_len) *labels_len = k;
  }
  return ZOGCU_OK;
}
