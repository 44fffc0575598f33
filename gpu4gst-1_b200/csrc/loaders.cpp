// Readers for the reference's input formats (host side of the C ABI).
//
// Each reader mirrors the behaviour of the reference loader it replaces
// (cited per function) with two differences: errors are returned as a status
// instead of getchar()+exit(1), and malformed content is rejected instead of
// being indexed out of bounds.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <utility>
#include <vector>

#include "gst_b200.h"
#include "status.hpp"

namespace {

bool read_file(const char* path, std::string& out) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  out.resize(n > 0 ? (size_t)n : 0);
  size_t got = n > 0 ? std::fread(&out[0], 1, (size_t)n, f) : 0;
  std::fclose(f);
  return got == out.size();
}

// Splits the buffer into lines (without '\n' / '\r').
template <class F>
void for_each_line(const std::string& buf, F f) {
  size_t i = 0, n = buf.size();
  while (i < n) {
    size_t j = buf.find('\n', i);
    if (j == std::string::npos) j = n;
    size_t e = j;
    while (e > i && (buf[e - 1] == '\r')) --e;
    if (!f(buf.data() + i, buf.data() + e)) return;
    i = j + 1;
  }
}

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// Parses whitespace-separated integers of [b, e) into out; false on junk.
bool parse_ints(const char* b, const char* e, std::vector<long long>& out) {
  out.clear();
  const char* p = b;
  while (p < e) {
    while (p < e && is_space(*p)) ++p;
    if (p >= e) break;
    bool neg = false;
    if (*p == '-' || *p == '+') {
      neg = *p == '-';
      ++p;
    }
    if (p >= e || *p < '0' || *p > '9') return false;
    long long v = 0;
    while (p < e && *p >= '0' && *p <= '9') {
      v = v * 10 + (*p - '0');
      if (v > (1ll << 40)) return false;
      ++p;
    }
    // tolerate a fractional part (the reference parses the header with stod)
    if (p < e && *p == '.') {
      ++p;
      while (p < e && *p >= '0' && *p <= '9') ++p;
    }
    if (p < e && !is_space(*p)) return false;
    out.push_back(neg ? -v : v);
  }
  return true;
}

template <class T>
T* dup_array(const std::vector<T>& v) {
  T* p = static_cast<T*>(std::malloc(sizeof(T) * (v.size() ? v.size() : 1)));
  if (p && !v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
  return p;
}

}  // namespace

extern "C" {

// read_input_graph (code/PrunedDP++/include/graph_hash_of_mixed_weighted_read_for_GSTP.h:15-66):
// first token of line 1 is V; every later line with three integers "u v w"
// adds both directions; each adjacency row is sorted by (neighbour, weight).
gst_status gst_read_input_graph(const char* file, gst_csr* out) {
  if (!file || !out) return gst::fail(GST_E_INVALID, "gst_read_input_graph: null argument");
  std::memset(out, 0, sizeof *out);
  std::string buf;
  if (!read_file(file, buf)) return gst::fail(GST_E_IO, std::string("cannot open ") + file);
  long long V = -1;
  std::vector<long long> tok;
  std::vector<std::pair<int32_t, int32_t>> ends;  // (u, v) per line
  std::vector<int32_t> wts;
  bool bad = false;
  std::string why;
  bool first = true;
  for_each_line(buf, [&](const char* b, const char* e) {
    if (first) {
      first = false;
      if (!parse_ints(b, e, tok) || tok.empty() || tok[0] < 0 || tok[0] > INT32_MAX) {
        bad = true;
        why = "header must start with the vertex count";
        return false;
      }
      V = tok[0];
      return true;
    }
    if (!parse_ints(b, e, tok)) {
      bad = true;
      why = "non-integer token in edge line";
      return false;
    }
    if (tok.size() != 3) return true;  // the reference skips lines without 3 fields
    if (tok[0] < 0 || tok[0] >= V || tok[1] < 0 || tok[1] >= V) {
      bad = true;
      why = "edge endpoint out of range";
      return false;
    }
    if (tok[2] < 0 || tok[2] >= (1ll << 30)) {
      bad = true;
      why = "edge weight outside [0, 2^30)";
      return false;
    }
    ends.push_back({(int32_t)tok[0], (int32_t)tok[1]});
    wts.push_back((int32_t)tok[2]);
    return true;
  });
  if (first) return gst::fail(GST_E_FORMAT, std::string(file) + ": empty file");
  if (bad) return gst::fail(GST_E_FORMAT, std::string(file) + ": " + why);
  std::vector<int64_t> rowptr(V + 1, 0);
  for (auto& p : ends) {
    rowptr[p.first + 1]++;
    rowptr[p.second + 1]++;
  }
  for (long long i = 0; i < V; ++i) rowptr[i + 1] += rowptr[i];
  const int64_t E = rowptr[V];
  std::vector<std::pair<int32_t, int32_t>> adj(E);
  std::vector<int64_t> fill(rowptr.begin(), rowptr.end() - 1);
  for (size_t i = 0; i < ends.size(); ++i) {
    adj[fill[ends[i].first]++] = {ends[i].second, wts[i]};
    adj[fill[ends[i].second]++] = {ends[i].first, wts[i]};
  }
  for (long long v = 0; v < V; ++v) std::sort(adj.begin() + rowptr[v], adj.begin() + rowptr[v + 1]);
  std::vector<int32_t> col(E), w(E);
  for (int64_t j = 0; j < E; ++j) {
    col[j] = adj[j].first;
    w[j] = adj[j].second;
  }
  out->V = V;
  out->E = E;
  out->rowptr = dup_array(rowptr);
  out->col = dup_array(col);
  out->w = dup_array(w);
  if (!out->rowptr || !out->col || !out->w) {
    gst_csr_free(out);
    return gst::fail(GST_E_NOMEM, "host allocation failed");
  }
  return GST_OK;
}

// graph<long,long,long,...> constructor (code/TrimCDP-WB/include/graph.hpp:12-118):
// V = size(beg_pos)/8 - 1, E = beg_pos[V]; ids and weights narrowed to int32.
gst_status gst_read_binary_csr(const char* beg_file, const char* csr_file, const char* weight_file,
                               gst_csr* out) {
  if (!beg_file || !csr_file || !weight_file || !out)
    return gst::fail(GST_E_INVALID, "gst_read_binary_csr: null argument");
  std::memset(out, 0, sizeof *out);
  std::string b, c, w;
  if (!read_file(beg_file, b)) return gst::fail(GST_E_IO, std::string("cannot open ") + beg_file);
  if (!read_file(csr_file, c)) return gst::fail(GST_E_IO, std::string("cannot open ") + csr_file);
  if (!read_file(weight_file, w)) return gst::fail(GST_E_IO, std::string("cannot open ") + weight_file);
  if (b.size() < 16 || b.size() % 8) return gst::fail(GST_E_FORMAT, "beg_pos file size is not (V+1) x 8");
  const int64_t V = (int64_t)(b.size() / 8) - 1;
  const int64_t* bp = reinterpret_cast<const int64_t*>(b.data());
  const int64_t E = bp[V];
  if (bp[0] != 0 || E < 0 || (int64_t)c.size() < E * 8 || (int64_t)w.size() < E * 8)
    return gst::fail(GST_E_FORMAT, "csr/weight files shorter than beg_pos[V] entries");
  if (V > INT32_MAX) return gst::fail(GST_E_UNSUPPORTED, "more than 2^31-1 vertices");
  for (int64_t i = 0; i < V; ++i)
    if (bp[i + 1] < bp[i]) return gst::fail(GST_E_FORMAT, "beg_pos is not non-decreasing");
  const int64_t* cp = reinterpret_cast<const int64_t*>(c.data());
  const int64_t* wp = reinterpret_cast<const int64_t*>(w.data());
  std::vector<int32_t> col(E), wt(E);
  for (int64_t j = 0; j < E; ++j) {
    if (cp[j] < 0 || cp[j] >= V) return gst::fail(GST_E_FORMAT, "neighbour id out of range");
    if (wp[j] < 0 || wp[j] >= (1ll << 30)) return gst::fail(GST_E_FORMAT, "weight outside [0, 2^30)");
    col[j] = (int32_t)cp[j];
    wt[j] = (int32_t)wp[j];
  }
  std::vector<int64_t> rowptr(bp, bp + V + 1);
  out->V = V;
  out->E = E;
  out->rowptr = dup_array(rowptr);
  out->col = dup_array(col);
  out->w = dup_array(wt);
  if (!out->rowptr || !out->col || !out->w) {
    gst_csr_free(out);
    return gst::fail(GST_E_NOMEM, "host allocation failed");
  }
  return GST_OK;
}

// read_Group (graph_hash_of_mixed_weighted_read_for_GSTP.h:116-171): "gK:v v v",
// group index K-1, members sorted ascending.
gst_status gst_read_groups(const char* file, gst_groups* out) {
  if (!file || !out) return gst::fail(GST_E_INVALID, "gst_read_groups: null argument");
  std::memset(out, 0, sizeof *out);
  std::string buf;
  if (!read_file(file, buf)) return gst::fail(GST_E_IO, std::string("cannot open ") + file);
  std::vector<std::vector<int32_t>> groups;
  std::vector<long long> tok;
  bool bad = false;
  std::string why;
  for_each_line(buf, [&](const char* b, const char* e) {
    while (b < e && is_space(*b)) ++b;
    if (b == e) return true;  // blank line
    const char* colon = static_cast<const char*>(std::memchr(b, ':', e - b));
    if (!colon || *b != 'g') {
      bad = true;
      why = "group line must look like gK:v v v";
      return false;
    }
    if (!parse_ints(b + 1, colon, tok) || tok.size() != 1 || tok[0] < 1 || tok[0] > INT32_MAX) {
      bad = true;
      why = "bad group label";
      return false;
    }
    size_t g = (size_t)(tok[0] - 1);
    if (!parse_ints(colon + 1, e, tok)) {
      bad = true;
      why = "bad group member";
      return false;
    }
    if (groups.size() <= g) groups.resize(g + 1);
    auto& m = groups[g];
    m.clear();
    for (long long x : tok) {
      if (x < 0 || x > INT32_MAX) {
        bad = true;
        why = "group member out of range";
        return false;
      }
      m.push_back((int32_t)x);
    }
    std::sort(m.begin(), m.end());
    return true;
  });
  if (bad) return gst::fail(GST_E_FORMAT, std::string(file) + ": " + why);
  std::vector<int64_t> ptr(groups.size() + 1, 0);
  for (size_t g = 0; g < groups.size(); ++g) ptr[g + 1] = ptr[g] + (int64_t)groups[g].size();
  std::vector<int32_t> mem;
  mem.reserve(ptr.back());
  for (auto& g : groups) mem.insert(mem.end(), g.begin(), g.end());
  out->n = (int64_t)groups.size();
  out->ptr = dup_array(ptr);
  out->members = dup_array(mem);
  if (!out->ptr || !out->members) {
    gst_groups_free(out);
    return gst::fail(GST_E_NOMEM, "host allocation failed");
  }
  return GST_OK;
}

// read_inquire (graph_hash_of_mixed_weighted_read_for_GSTP.h:172-218): one query
// per line, space-separated group ids.
gst_status gst_read_queries(const char* file, gst_queries* out) {
  if (!file || !out) return gst::fail(GST_E_INVALID, "gst_read_queries: null argument");
  std::memset(out, 0, sizeof *out);
  std::string buf;
  if (!read_file(file, buf)) return gst::fail(GST_E_IO, std::string("cannot open ") + file);
  std::vector<int64_t> ptr{0};
  std::vector<int32_t> ids;
  std::vector<long long> tok;
  bool bad = false;
  for_each_line(buf, [&](const char* b, const char* e) {
    if (!parse_ints(b, e, tok)) {
      bad = true;
      return false;
    }
    if (tok.empty()) return true;
    for (long long x : tok) {
      if (x < 0 || x > INT32_MAX) {
        bad = true;
        return false;
      }
      ids.push_back((int32_t)x);
    }
    ptr.push_back((int64_t)ids.size());
    return true;
  });
  if (bad) return gst::fail(GST_E_FORMAT, std::string(file) + ": query lines must hold group ids");
  out->n = (int64_t)ptr.size() - 1;
  out->ptr = dup_array(ptr);
  out->ids = dup_array(ids);
  if (!out->ptr || !out->ids) {
    gst_queries_free(out);
    return gst::fail(GST_E_NOMEM, "host allocation failed");
  }
  return GST_OK;
}

void gst_csr_free(gst_csr* g) {
  if (!g) return;
  std::free(g->rowptr);
  std::free(g->col);
  std::free(g->w);
  std::memset(g, 0, sizeof *g);
}

void gst_groups_free(gst_groups* g) {
  if (!g) return;
  std::free(g->ptr);
  std::free(g->members);
  std::memset(g, 0, sizeof *g);
}

void gst_queries_free(gst_queries* q) {
  if (!q) return;
  std::free(q->ptr);
  std::free(q->ids);
  std::memset(q, 0, sizeof *q);
}

}  // extern "C"
