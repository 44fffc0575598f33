// Seeded synthetic inputs in the reference's file formats.
//
// The reference benchmarks on external SNAP-style social graphs that are not
// available here, so tests and the benchmark use Barabasi-Albert power-law
// graphs of the same shapes instead.  This library builds them fast enough for
// the 4M-vertex / 35M-edge case and writes every input format the reference
// reads:
//   <data>.in            "V E" header, then one "u v w" line per undirected
//                        edge (read_input_graph,
//                        code/PrunedDP++/include/graph_hash_of_mixed_weighted_read_for_GSTP.h:15-66)
//   <data>_beg_pos.bin   V+1 x int64 row offsets
//   <data>_csr.bin       E x int64 neighbour ids
//   <data>_weight.bin    E x int64 weights (graph ctor,
//                        code/TrimCDP-WB/include/graph.hpp:12-118)
// Group (.g) and query (.csv) files are small and written by the Python side.
//
// The BA model: start from a star on m+1 vertices; every later vertex attaches
// to m distinct earlier vertices drawn with probability proportional to their
// degree (the "repeated endpoints" list).  An optional random Hamiltonian path
// is added on top.  Multi-edges are removed (first weight kept), self loops are
// never produced.  Each CSR row is sorted by neighbour id, which is the order
// the reference's text loader produces.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct Rng {  // xoshiro256** seeded by splitmix64
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) {
      x += 0x9E3779B97F4A7C15ull;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      s[i] = z ^ (z >> 31);
    }
  }
  static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
  uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  // uniform in [0, n)
  uint64_t below(uint64_t n) {
    return (uint64_t)(((unsigned __int128)next() * n) >> 64);
  }
};

struct Graph {
  int64_t V = 0;
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  std::vector<int32_t> w;
};

}  // namespace

extern "C" {

typedef struct gstgen_graph gstgen_graph;

// Builds a BA(V, m) graph with integer weights uniform in [wmin, wmax].
// spanning_path != 0 adds a random path through all vertices.
// Returns 0 on success, -1 on bad arguments.
int gstgen_ba(int64_t V, int m, int wmin, int wmax, int spanning_path,
              uint64_t seed, gstgen_graph** out) {
  if (!out || V < 2 || m < 1 || m >= V || wmin > wmax || V > (int64_t)INT32_MAX)
    return -1;
  Rng rng(seed);
  std::vector<uint64_t> keys;  // (min << 32 | max), undirected
  keys.reserve((size_t)(m * V + (spanning_path ? V : 0)));
  std::vector<int32_t> rep;
  rep.reserve((size_t)(2 * m * V));
  for (int i = 1; i <= m; ++i) {
    keys.push_back(((uint64_t)0 << 32) | (uint32_t)i);
    rep.push_back(0);
    rep.push_back(i);
  }
  std::vector<int32_t> picked(m);
  for (int64_t src = m + 1; src < V; ++src) {
    int got = 0;
    while (got < m) {
      int32_t t = rep[rng.below(rep.size())];
      bool dup = false;
      for (int j = 0; j < got; ++j)
        if (picked[j] == t) { dup = true; break; }
      if (!dup) picked[got++] = t;
    }
    for (int j = 0; j < m; ++j) {
      keys.push_back(((uint64_t)(uint32_t)picked[j] << 32) | (uint32_t)src);
      rep.push_back(picked[j]);
      rep.push_back((int32_t)src);
    }
  }
  std::vector<int32_t>().swap(rep);
  if (spanning_path) {
    std::vector<int32_t> perm(V);
    for (int64_t i = 0; i < V; ++i) perm[i] = (int32_t)i;
    for (int64_t i = V - 1; i > 0; --i) std::swap(perm[i], perm[rng.below(i + 1)]);
    for (int64_t i = 0; i + 1 < V; ++i) {
      uint32_t a = perm[i], b = perm[i + 1];
      if (a > b) std::swap(a, b);
      keys.push_back(((uint64_t)a << 32) | b);
    }
  }
  // weights are drawn per generated edge in generation order, then duplicates
  // are dropped keeping the first occurrence (stable sort)
  const uint64_t span = (uint64_t)(wmax - wmin + 1);
  std::vector<std::pair<uint64_t, int32_t>> ew(keys.size());
  for (size_t i = 0; i < keys.size(); ++i)
    ew[i] = {keys[i], (int32_t)(wmin + (int64_t)rng.below(span))};
  std::vector<uint64_t>().swap(keys);
  std::stable_sort(ew.begin(), ew.end(),
                   [](const std::pair<uint64_t, int32_t>& x,
                      const std::pair<uint64_t, int32_t>& y) { return x.first < y.first; });
  size_t n = 0;
  for (size_t i = 0; i < ew.size(); ++i)
    if (n == 0 || ew[n - 1].first != ew[i].first) ew[n++] = ew[i];
  ew.resize(n);

  Graph* g = new Graph;
  g->V = V;
  g->rowptr.assign(V + 1, 0);
  for (auto& e : ew) {
    g->rowptr[(e.first >> 32) + 1]++;
    g->rowptr[(e.first & 0xffffffffu) + 1]++;
  }
  for (int64_t i = 0; i < V; ++i) g->rowptr[i + 1] += g->rowptr[i];
  g->col.resize(g->rowptr[V]);
  g->w.resize(g->rowptr[V]);
  std::vector<int64_t> fill(g->rowptr.begin(), g->rowptr.end() - 1);
  // scatter both directions; every row is sorted by neighbour id afterwards
  for (auto& e : ew) {
    uint32_t a = (uint32_t)(e.first >> 32), b = (uint32_t)(e.first & 0xffffffffu);
    g->col[fill[a]] = (int32_t)b;
    g->w[fill[a]++] = e.second;
    g->col[fill[b]] = (int32_t)a;
    g->w[fill[b]++] = e.second;
  }
  std::vector<std::pair<uint64_t, int32_t>>().swap(ew);
  std::vector<std::pair<int32_t, int32_t>> row;
  for (int64_t v = 0; v < V; ++v) {
    int64_t b = g->rowptr[v], e = g->rowptr[v + 1];
    row.clear();
    for (int64_t j = b; j < e; ++j) row.push_back({g->col[j], g->w[j]});
    std::sort(row.begin(), row.end());
    for (int64_t j = b; j < e; ++j) {
      g->col[j] = row[j - b].first;
      g->w[j] = row[j - b].second;
    }
  }
  *out = reinterpret_cast<gstgen_graph*>(g);
  return 0;
}

int64_t gstgen_num_vertices(const gstgen_graph* h) {
  return h ? reinterpret_cast<const Graph*>(h)->V : -1;
}

// number of directed CSR entries (twice the undirected edge count)
int64_t gstgen_num_arcs(const gstgen_graph* h) {
  return h ? reinterpret_cast<const Graph*>(h)->rowptr.back() : -1;
}

int gstgen_copy_csr(const gstgen_graph* h, int64_t* rowptr, int32_t* col, int32_t* w) {
  if (!h) return -1;
  const Graph* g = reinterpret_cast<const Graph*>(h);
  if (rowptr) std::memcpy(rowptr, g->rowptr.data(), sizeof(int64_t) * (g->V + 1));
  if (col) std::memcpy(col, g->col.data(), sizeof(int32_t) * g->col.size());
  if (w) std::memcpy(w, g->w.data(), sizeof(int32_t) * g->w.size());
  return 0;
}

void gstgen_free(gstgen_graph* h) { delete reinterpret_cast<Graph*>(h); }

// Writes "<prefix>.in": header "V E" (E = undirected edges), then "u v w"
// once per undirected edge (u < v), single spaces.
int gstgen_write_in(const char* file, int64_t V, const int64_t* rowptr,
                    const int32_t* col, const int32_t* w) {
  FILE* f = std::fopen(file, "w");
  if (!f) return -1;
  std::vector<char> buf(1 << 22);
  std::setvbuf(f, buf.data(), _IOFBF, buf.size());
  std::fprintf(f, "%lld %lld\n", (long long)V, (long long)(rowptr[V] / 2));
  char line[64];
  for (int64_t u = 0; u < V; ++u) {
    for (int64_t j = rowptr[u]; j < rowptr[u + 1]; ++j) {
      if (col[j] > u) {
        int n = std::snprintf(line, sizeof line, "%lld %d %d\n", (long long)u, col[j], w[j]);
        std::fwrite(line, 1, n, f);
      }
    }
  }
  return std::fclose(f) == 0 ? 0 : -1;
}

// Writes the int64 binary CSR triplet <prefix>_beg_pos.bin, _csr.bin, _weight.bin.
int gstgen_write_bin(const char* prefix, int64_t V, const int64_t* rowptr,
                     const int32_t* col, const int32_t* w) {
  std::string p(prefix);
  const int64_t E = rowptr[V];
  FILE* f = std::fopen((p + "_beg_pos.bin").c_str(), "wb");
  if (!f) return -1;
  size_t ok = std::fwrite(rowptr, sizeof(int64_t), V + 1, f);
  std::fclose(f);
  if (ok != (size_t)(V + 1)) return -1;
  std::vector<int64_t> tmp(E);
  for (int64_t j = 0; j < E; ++j) tmp[j] = col[j];
  f = std::fopen((p + "_csr.bin").c_str(), "wb");
  if (!f) return -1;
  ok = std::fwrite(tmp.data(), sizeof(int64_t), E, f);
  std::fclose(f);
  if (ok != (size_t)E) return -1;
  for (int64_t j = 0; j < E; ++j) tmp[j] = w[j];
  f = std::fopen((p + "_weight.bin").c_str(), "wb");
  if (!f) return -1;
  ok = std::fwrite(tmp.data(), sizeof(int64_t), E, f);
  std::fclose(f);
  return ok == (size_t)E ? 0 : -1;
}

}  // extern "C"
