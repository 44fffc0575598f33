// Host scheduler and C ABI of the GST engine.
//
// The engine keeps the graph and the groups resident in HBM and owns one
// device arena, carved into per-query slabs (DP table, dirty masks, frontier
// lists, chunk list, witness buffers).  Queries are admitted into slots; every
// device round advances all admitted queries at once (batching), and the
// rounds are replayed from one captured CUDA graph.  Slots whose query
// finished are harvested between graph launches, their tree is rebuilt on the
// device, their slab is cleaned and cached for the next query of the same
// shape, and waiting queries are admitted (continuous batching).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine_dev.cuh"
#include "kernels.cuh"
#include "status.hpp"

namespace gst {

std::string& last_error_text() {
  thread_local std::string s;
  return s;
}

#define GST_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(GST_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

// ---------------------------------------------------------------------------
// Arena: first-fit allocator over one device allocation, with coalescing.
// ---------------------------------------------------------------------------
class Arena {
 public:
  void reset(size_t bytes) {
    free_.clear();
    if (bytes) free_[0] = bytes;
    size_ = bytes;
  }
  // returns offset or SIZE_MAX
  size_t alloc(size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        size_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > bytes) free_[off + bytes] = len - bytes;
        return off;
      }
    }
    return SIZE_MAX;
  }
  void release(size_t off, size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t size() const { return size_; }

 private:
  std::map<size_t, size_t> free_;
  size_t size_ = 0;
};

struct Shape {
  int k, L;
  bool operator<(const Shape& o) const { return k != o.k ? k < o.k : L < o.L; }
};

struct Slab {
  Shape shape{};
  size_t off = 0, bytes = 0;
  int32_t* table = nullptr;
  unsigned long long* mask = nullptr;
  uint32_t* queue = nullptr;
  uint32_t* touched = nullptr;
  uint32_t* tflag = nullptr;
  uint32_t* dead = nullptr;
  int32_t* sd = nullptr;
  Chunk* chunks = nullptr;
  int32_t* lbtab = nullptr;
  int32_t* wstack = nullptr;
  int32_t* wedges = nullptr;
  long long chunk_cap = 0, wcap = 0;
};

struct Request {
  uint64_t ticket = 0;
  std::vector<int32_t> groups;  // distinct group ids
  int D = -1;
  std::atomic<bool> done{false};
  gst_status status = GST_OK;
  gst_result result{};
  cudaEvent_t t0 = nullptr;
  std::chrono::steady_clock::time_point t_submit, t_admit;
};

class Engine {
 public:
  ~Engine() { shutdown(); }

  gst_status init(const gst_engine_config* cfg) {
    gst_engine_config c{};
    if (cfg) c = *cfg;
    device_ = c.device;
    max_slots_ = c.max_slots > 0 ? std::min(c.max_slots, MAXSLOTS) : MAXSLOTS;
    max_rounds_override_ = c.max_rounds > 0 ? c.max_rounds : 0;
    profile_ = c.profile != 0;
    bucket_shift_ = c.bucket_shift > 0 ? std::min(c.bucket_shift, 30) : 30;
    rounds_per_poll_ = c.rounds_per_poll > 0 ? c.rounds_per_poll : 8;
    if (const char* w = std::getenv("GST_WATCHDOG_S")) watchdog_s_ = std::max(1e-4, std::atof(w));
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
      return fail(GST_E_CUDA, "no CUDA device visible");
    if (device_ < 0 || device_ >= n) return fail(GST_E_INVALID, "device ordinal out of range");
    GST_CUDA(cudaSetDevice(device_));
    cudaDeviceProp prop;
    GST_CUDA(cudaGetDeviceProperties(&prop, device_));
    num_sms_ = prop.multiProcessorCount;
    {  // the grow kernel runs one resident wave: grid = SMs x resident blocks
      int a = 0, b = 0, c3 = 0;
      GST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_grow_t<8>, GROW_WARPS * 32, 0));
      GST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_grow_t<16>, GROW_WARPS * 32, 0));
      GST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c3, k_grow_t<32>, GROW_WARPS * 32, 0));
      grow_grid_[0] = num_sms_ * std::max(a, 1);
      grow_grid_[1] = num_sms_ * std::max(b, 1);
      grow_grid_[2] = num_sms_ * std::max(c3, 1);
    }
    std::memset(&tuning_, 0, sizeof tuning_);
    tuning_.grow_lanes = GROW_LANES_DEFAULT;
    tuning_.rounds_per_poll = rounds_per_poll_;
    tuning_.max_slots = max_slots_;
    tuning_.overlap = 1;
    for (int k = 0; k <= MAXK; ++k) {
      tuning_.chunk_pairs[k][0] = tuning_.chunk_pairs[k][1] = 1024;
      tuning_.bucket_mult[k] = 1;
    }
    GST_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    GST_CUDA(cudaStreamCreateWithFlags(&stream2_, cudaStreamNonBlocking));  // the grow branch (overlap = 2)
    GST_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
    GST_CUDA(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
    SubsetTables st;
    fill_subset_tables(st);
    GST_CUDA(cudaMemcpyToSymbol(c_sub, &st, sizeof st));
    GST_CUDA(cudaMalloc(&d_slots_, sizeof(Slot) * MAXSLOTS));
    GST_CUDA(cudaMemset(d_slots_, 0, sizeof(Slot) * MAXSLOTS));
    GST_CUDA(cudaMalloc(&d_plan_, sizeof(Plan)));
    GST_CUDA(cudaMemset(d_plan_, 0, sizeof(Plan)));
    GST_CUDA(cudaMalloc(&d_status_, sizeof(SlotStatus) * MAXSLOTS));
    GST_CUDA(cudaMallocHost(&h_status_, sizeof(SlotStatus) * MAXSLOTS));
    GST_CUDA(cudaMalloc(&d_list_, sizeof(int) * MAXSLOTS));
    GST_CUDA(cudaMallocHost(&h_list_, sizeof(int) * MAXSLOTS));
    GST_CUDA(cudaMallocHost(&h_slot_, sizeof(Slot) * MAXSLOTS));  // admission staging, one per slot
    GST_CUDA(cudaMallocHost(&h_harv_, sizeof(Slot) * MAXSLOTS));  // harvest read-back
    size_t fr = 0, tot = 0;
    GST_CUDA(cudaMemGetInfo(&fr, &tot));
    arena_request_ = c.arena_bytes > 0 ? (size_t)c.arena_bytes
                                       : (size_t)((c.arena_fraction > 0 ? c.arena_fraction : 0.85) * fr);
    slot_busy_.assign(MAXSLOTS, 0);
    slot_req_.assign(MAXSLOTS, nullptr);
    slot_slab_.resize(MAXSLOTS);
    return GST_OK;
  }

  void shutdown() {
    if (device_ < 0) return;
    if (broken_) {  // device work still running: freeing would block on it
      device_ = -1;
      return;
    }
    cudaSetDevice(device_);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
    for (auto* p : {(void*)d_slots_, (void*)d_plan_, (void*)d_status_, (void*)d_list_, (void*)arena_,
                    (void*)d_rowptr_, (void*)d_adj_, (void*)d_gptr_, (void*)d_gmem_})
      if (p) cudaFree(p);
    for (auto* p : {(void*)h_status_, (void*)h_list_, (void*)h_slot_, (void*)h_harv_, (void*)h_wedges_})
      if (p) cudaFreeHost(p);
    if (stream_) cudaStreamDestroy(stream_);
    if (stream2_) cudaStreamDestroy(stream2_);
    if (ev_fork_) cudaEventDestroy(ev_fork_);
    if (ev_join_) cudaEventDestroy(ev_join_);
    d_slots_ = nullptr;
    arena_ = nullptr;
    device_ = -1;
  }

  gst_status load_graph(int64_t V, const int64_t* rowptr, const int32_t* col, const int32_t* w) {
    if (V <= 0 || !rowptr || !col || !w) return fail(GST_E_INVALID, "graph: empty or null arrays");
    if (V > INT32_MAX) return fail(GST_E_UNSUPPORTED, "graph: more than 2^31-1 vertices");
    if (rowptr[0] != 0) return fail(GST_E_INVALID, "graph: rowptr[0] must be 0");
    const int64_t E = rowptr[V];
    if (E < 0 || E >= (int64_t)UINT32_MAX) return fail(GST_E_UNSUPPORTED, "graph: edge count outside [0, 2^32)");
    std::vector<int2> adj(E);
    for (int64_t v = 0; v < V; ++v)
      if (rowptr[v + 1] < rowptr[v]) return fail(GST_E_INVALID, "graph: rowptr not non-decreasing");
    for (int64_t j = 0; j < E; ++j) {
      if (col[j] < 0 || col[j] >= V) return fail(GST_E_INVALID, "graph: neighbour id out of range");
      if (w[j] < 0 || w[j] >= (1 << 30)) return fail(GST_E_INVALID, "graph: weight outside [0, 2^30)");
      adj[j] = make_int2(col[j], w[j]);
    }
    std::lock_guard<std::mutex> lk(mu_);
    if (busy_) return fail(GST_E_STATE, "graph: engine is serving");
    GST_CUDA(cudaSetDevice(device_));
    if (d_rowptr_) cudaFree(d_rowptr_);
    if (d_adj_) cudaFree(d_adj_);
    d_rowptr_ = nullptr;
    d_adj_ = nullptr;
    GST_CUDA(cudaMalloc(&d_rowptr_, sizeof(long long) * (V + 1)));
    GST_CUDA(cudaMalloc(&d_adj_, sizeof(int2) * std::max<int64_t>(E, 1)));
    GST_CUDA(cudaMemcpy(d_rowptr_, rowptr, sizeof(long long) * (V + 1), cudaMemcpyHostToDevice));
    if (E) GST_CUDA(cudaMemcpy(d_adj_, adj.data(), sizeof(int2) * E, cudaMemcpyHostToDevice));
    V_ = V;
    E_ = E;
    {  // bucket width of the cost-ordered grows: the typical lightest edge
      double sum = 0;
      int64_t n = 0;
      for (int64_t v = 0; v < V; ++v) {
        if (rowptr[v + 1] == rowptr[v]) continue;
        int mn = INT32_MAX;
        for (int64_t j = rowptr[v]; j < rowptr[v + 1]; ++j) mn = std::min(mn, w[j]);
        sum += mn;
        ++n;
      }
      delta_ = std::max(1, (int)(n ? sum / n + 0.5 : 1));
    }
    cache_.clear();
    drop_graph_exec();  // the captured rounds hold the old graph's pointers
    return setup_arena();
  }

  gst_status load_groups(int64_t n, const int64_t* ptr, const int32_t* mem) {
    if (n < 0 || !ptr || (n > 0 && !mem)) return fail(GST_E_INVALID, "groups: null arrays");
    if (V_ == 0) return fail(GST_E_STATE, "groups: load the graph first");
    if (ptr[0] != 0) return fail(GST_E_INVALID, "groups: ptr[0] must be 0");
    for (int64_t g = 0; g < n; ++g)
      if (ptr[g + 1] < ptr[g]) return fail(GST_E_INVALID, "groups: ptr not non-decreasing");
    const int64_t M = ptr[n];
    for (int64_t j = 0; j < M; ++j)
      if (mem[j] < 0 || mem[j] >= V_) return fail(GST_E_INVALID, "groups: member id out of range");
    std::lock_guard<std::mutex> lk(mu_);
    if (busy_) return fail(GST_E_STATE, "groups: engine is serving");
    GST_CUDA(cudaSetDevice(device_));
    if (d_gptr_) cudaFree(d_gptr_);
    if (d_gmem_) cudaFree(d_gmem_);
    d_gptr_ = nullptr;
    d_gmem_ = nullptr;
    GST_CUDA(cudaMalloc(&d_gptr_, sizeof(long long) * (n + 1)));
    GST_CUDA(cudaMalloc(&d_gmem_, sizeof(int32_t) * std::max<int64_t>(M, 1)));
    GST_CUDA(cudaMemcpy(d_gptr_, ptr, sizeof(long long) * (n + 1), cudaMemcpyHostToDevice));
    if (M) GST_CUDA(cudaMemcpy(d_gmem_, mem, sizeof(int32_t) * M, cudaMemcpyHostToDevice));
    G_ = n;
    drop_graph_exec();
    gsize_.assign(ptr, ptr + n + 1);
    gfirst_.resize(n);
    for (int64_t g = 0; g < n; ++g) gfirst_[g] = ptr[g + 1] > ptr[g] ? mem[ptr[g]] : -1;
    return GST_OK;
  }

  // ---- request intake -------------------------------------------------------
  // Validates a query and either answers it on the host (trivial cases) or
  // queues it.  Returns the request.
  std::shared_ptr<Request> make_request(const int32_t* ids, int k, int D, gst_status* st) {
    auto r = std::make_shared<Request>();
    r->t_submit = r->t_admit = std::chrono::steady_clock::now();
    r->D = D;
    *st = GST_OK;
    if (!ids || k <= 0) { *st = fail(GST_E_INVALID, "query: no group ids"); return nullptr; }
    if (D > GST_MAX_D) { *st = fail(GST_E_UNSUPPORTED, "query: D above GST_MAX_D"); return nullptr; }
    if (D < -1) D = -1, r->D = -1;
    if (V_ == 0 || G_ == 0 || !d_gptr_) { *st = fail(GST_E_STATE, "query: graph and groups not loaded"); return nullptr; }
    for (int i = 0; i < k; ++i) {
      if (ids[i] < 0 || ids[i] >= G_) { *st = fail(GST_E_INVALID, "query: group id out of range"); return nullptr; }
      if (std::find(r->groups.begin(), r->groups.end(), ids[i]) == r->groups.end())
        r->groups.push_back(ids[i]);
    }
    if ((int)r->groups.size() > MAXK) {
      *st = fail(GST_E_UNSUPPORTED, "query: more than GST_MAX_K distinct groups");
      return nullptr;
    }
    bool empty_group = false;
    for (int gid : r->groups) empty_group |= gsize_[gid + 1] == gsize_[gid];
    if (empty_group) {
      finish_infeasible(*r);
    } else if (r->groups.size() == 1) {
      r->result.cost = 0;
      r->result.feasible = 1;
      r->result.root = gfirst_[r->groups[0]];
      r->result.n_edges = 0;
      r->result.edges = nullptr;
      r->done = true;
    }
    return r;
  }

  static void finish_infeasible(Request& r) {
    r.result.cost = GST_REF_INF;
    r.result.feasible = 0;
    r.result.root = -1;
    r.result.n_edges = 0;
    r.result.edges = nullptr;
    r.done = true;
  }

  // ---- running ----------------------------------------------------------------
  // Runs until every request in `reqs` is done (batch / single solve).
  gst_status run(std::vector<std::shared_ptr<Request>>& reqs) {
    std::lock_guard<std::mutex> lk(mu_);
    if (busy_) return fail(GST_E_STATE, "engine is serving; use the server API");
    if (broken_) return fail(GST_E_STATE, "engine is unusable after a device wait timed out");
    GST_CUDA(cudaSetDevice(device_));
    if (!ev_run0_) {
      GST_CUDA(cudaEventCreate(&ev_run0_));
      GST_CUDA(cudaEventCreate(&ev_run1_));
    }
    std::memset(&prof_, 0, sizeof prof_);
    GST_CUDA(cudaEventRecord(ev_run0_, stream_));
    // largest tables first (longest-processing-time order): the queries that
    // hold the most memory start early and the small ones fill the gaps,
    // instead of a large query starting last and running alone at the end
    std::vector<std::pair<size_t, std::shared_ptr<Request>>> order;
    for (auto& r : reqs)
      if (r && !r->done) {
        const Shape sh{(int)r->groups.size(), r->D < 0 ? 1 : r->D + 1};
        order.emplace_back(slab_bytes(sh, nullptr), r);
      }
    std::stable_sort(order.begin(), order.end(),
                     [](const auto& a, const auto& b) { return a.first > b.first; });
    for (auto& o : order) pending_.push_back(o.second);
    while (true) {
      gst_status s = step();
      if (s != GST_OK) return s;
      if (pending_.empty() && active_ == 0) break;
    }
    GST_CUDA(cudaEventRecord(ev_run1_, stream_));
    GST_CUDA(cudaEventSynchronize(ev_run1_));
    float ms = 0;
    GST_CUDA(cudaEventElapsedTime(&ms, ev_run0_, ev_run1_));
    prof_.run_ms = ms;
    return GST_OK;
  }

  gst_profile profile() const { return prof_; }

  gst_status set_tuning(const gst_tuning& t) {
    std::lock_guard<std::mutex> lk(mu_);
    if (busy_) return fail(GST_E_STATE, "tuning: engine is serving");
    if (t.grow_lanes && t.grow_lanes != 8 && t.grow_lanes != 16 && t.grow_lanes != 32)
      return fail(GST_E_INVALID, "tuning: grow_lanes must be 8, 16 or 32");
    if (t.overlap < 0 || t.overlap > 2) return fail(GST_E_INVALID, "tuning: overlap must be 1 or 2");
    if (t.rounds_per_poll < 0 || t.max_slots < 0 || t.max_slots > MAXSLOTS)
      return fail(GST_E_INVALID, "tuning: rounds_per_poll or max_slots out of range");
    for (int k = 0; k <= MAXK; ++k) {
      if (t.chunk_pairs[k][0] < 0 || t.chunk_pairs[k][1] < 0 || t.chunk_pairs[k][0] > (1 << 20) ||
          t.chunk_pairs[k][1] > (1 << 20) || t.bucket_mult[k] < 0 || t.bucket_mult[k] > (1 << 16))
        return fail(GST_E_INVALID, "tuning: chunk_pairs or bucket_mult out of range");
    }
    if (t.grow_lanes) tuning_.grow_lanes = t.grow_lanes;
    if (t.overlap) tuning_.overlap = t.overlap;
    if (t.rounds_per_poll) tuning_.rounds_per_poll = rounds_per_poll_ = t.rounds_per_poll;
    if (t.max_slots) tuning_.max_slots = max_slots_ = t.max_slots;
    for (int k = 0; k <= MAXK; ++k) {
      for (int h = 0; h < 2; ++h)
        if (t.chunk_pairs[k][h]) tuning_.chunk_pairs[k][h] = t.chunk_pairs[k][h];
      if (t.bucket_mult[k]) tuning_.bucket_mult[k] = t.bucket_mult[k];
    }
    drop_graph_exec();  // the captured rounds hold the old launch shapes
    return GST_OK;
  }

  gst_tuning tuning() const { return tuning_; }

  // One scheduling step: admit, run rounds_per_poll rounds, harvest.
  gst_status step() {
    gst_status s = admit();
    if (s != GST_OK) return s;
    if (active_ == 0) {
      if (!pending_.empty()) {  // nothing admitted and nothing running: cannot fit
        auto r = pending_.front();
        pending_.pop_front();
        r->status = fail(GST_E_NOMEM, "query does not fit the device arena");
        r->done = true;
      }
      return GST_OK;
    }
    s = launch_rounds();
    if (s != GST_OK) return s;
    return harvest();
  }

  void bind_device() { cudaSetDevice(device_); }

  // Marks every queued request failed (after a device error in serving).
  void abort_all(const std::string& why) {
    for (auto& r : pending_) {
      r->status = GST_E_CUDA;
      r->done = true;
    }
    pending_.clear();
    for (int t = 0; t < MAXSLOTS; ++t)
      if (slot_busy_[t]) {
        slot_req_[t]->status = GST_E_CUDA;
        slot_req_[t]->done = true;
        slot_busy_[t] = 0;
        slot_req_[t] = nullptr;
      }
    active_ = 0;
    (void)why;
  }

  std::mutex mu_;
  bool busy_ = false;  // a server thread owns the scheduler
  std::deque<std::shared_ptr<Request>> pending_;
  int active_ = 0;
  int max_rounds_override_ = 0;

 private:
  size_t slab_bytes(Shape sh, Slab* out) const {
    const size_t V = (size_t)V_, E = (size_t)E_;
    const size_t W = (size_t)1 << sh.k, L = (size_t)sh.L;
    const size_t nq = sh.L == 1 ? 4 : L;      // plain: near 0/1, far 2/3
    const size_t planes = sh.L == 1 ? 2 : L;  // plain: near and far dirty planes
    Slab s;
    s.shape = sh;
    s.chunk_cap = (long long)(V + E / 32 + 64);
    s.wcap = (long long)(2 * V + 64);
    size_t off = 0;
    auto take = [&](size_t bytes) {
      size_t o = off;
      off += (bytes + 255) & ~size_t(255);
      return o;
    };
    size_t o_table = take(V * W * L * 4);
    size_t o_mask = take(planes * V * 8);
    size_t o_queue = take(nq * V * 4);
    size_t o_touched = take(V * 4);
    size_t o_tflag = take(V * 4);
    size_t o_dead = take((V + 31) / 32 * 4);
    size_t o_sd = take(V * 32);
    size_t o_chunks = take((size_t)s.chunk_cap * sizeof(Chunk));
    size_t o_lbtab = take((size_t)sh.k * sh.k * W * 4 + (size_t)sh.k * W * 4);
    size_t o_wstack = take((size_t)s.wcap * 16);
    size_t o_wedges = take((size_t)s.wcap * 12);
    if (out) {
      *out = s;
      out->bytes = off;
      // offsets stored in pointers until placed
      out->table = reinterpret_cast<int32_t*>(o_table);
      out->mask = reinterpret_cast<unsigned long long*>(o_mask);
      out->queue = reinterpret_cast<uint32_t*>(o_queue);
      out->touched = reinterpret_cast<uint32_t*>(o_touched);
      out->tflag = reinterpret_cast<uint32_t*>(o_tflag);
      out->dead = reinterpret_cast<uint32_t*>(o_dead);
      out->sd = reinterpret_cast<int32_t*>(o_sd);
      out->chunks = reinterpret_cast<Chunk*>(o_chunks);
      out->lbtab = reinterpret_cast<int32_t*>(o_lbtab);
      out->wstack = reinterpret_cast<int32_t*>(o_wstack);
      out->wedges = reinterpret_cast<int32_t*>(o_wedges);
    }
    return off;
  }

  gst_status setup_arena() {
    if (arena_) cudaFree(arena_);
    arena_ = nullptr;
    size_t fr = 0, tot = 0;
    GST_CUDA(cudaMemGetInfo(&fr, &tot));
    size_t want = std::min(arena_request_, (size_t)(fr * 0.95));
    want &= ~size_t(255);
    while (want >= (1u << 20)) {
      if (cudaMalloc(&arena_, want) == cudaSuccess) break;
      cudaGetLastError();
      arena_ = nullptr;
      want = want * 3 / 4;
    }
    if (!arena_) return fail(GST_E_NOMEM, "cannot allocate the device arena");
    arena_bytes_ = want;
    arena_alloc_.reset(want);
    return GST_OK;
  }

  void drop_graph_exec() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
  }

  void clear_slab_cache() {
    for (auto& kv : cache_)
      for (auto& s : kv.second) arena_alloc_.release(s.off, s.bytes);
    cache_.clear();
  }

  // A clean slab of the shape: cached, or carved and initialised.
  bool acquire_slab(Shape sh, Slab* out, bool evict = true) {
    auto it = cache_.find(sh);
    if (it != cache_.end() && !it->second.empty()) {
      *out = it->second.back();
      it->second.pop_back();
      return true;
    }
    Slab s;
    size_t bytes = slab_bytes(sh, &s);
    size_t off = arena_alloc_.alloc(bytes);
    if (off == SIZE_MAX) {  // evict cached slabs of other shapes and retry
      if (!evict) return false;
      clear_slab_cache();
      off = arena_alloc_.alloc(bytes);
      if (off == SIZE_MAX) return false;
    }
    char* base = arena_ + off;
    auto place = [&](auto*& p) { p = reinterpret_cast<std::remove_reference_t<decltype(p)>>(base + reinterpret_cast<size_t>(p)); };
    place(s.table);
    place(s.mask);
    place(s.queue);
    place(s.touched);
    place(s.tflag);
    place(s.dead);
    place(s.sd);
    place(s.chunks);
    place(s.lbtab);
    place(s.wstack);
    place(s.wedges);
    s.off = off;
    s.bytes = bytes;
    const size_t V = (size_t)V_, W = (size_t)1 << sh.k, L = (size_t)sh.L;
    if (cudaMemsetAsync(s.table, 0x3f, V * W * L * 4, stream_) != cudaSuccess ||
        cudaMemsetAsync(s.mask, 0, (sh.L == 1 ? 2 : L) * V * 8, stream_) != cudaSuccess ||
        cudaMemsetAsync(s.tflag, 0, V * 4, stream_) != cudaSuccess ||
        cudaMemsetAsync(s.dead, 0, (V + 31) / 32 * 4, stream_) != cudaSuccess ||
        cudaMemsetAsync(s.sd, 0x3f, V * 32, stream_) != cudaSuccess) {
      arena_alloc_.release(off, bytes);
      return false;
    }
    *out = s;
    return true;
  }

  // Waits for the engine stream with a deadline.  A round sequence that does
  // not finish within watchdog_s_ seconds (far above any legitimate poll
  // interval) turns into GST_E_CUDA instead of blocking the caller for good;
  // the engine is then unusable and the process should exit, which ends the
  // device work with its context.
  gst_status wait_stream() {
    if (!ev_poll_) GST_CUDA(cudaEventCreateWithFlags(&ev_poll_, cudaEventDisableTiming));
    GST_CUDA(cudaEventRecord(ev_poll_, stream_));
    const auto t0 = std::chrono::steady_clock::now();
    for (int spin = 0;; ++spin) {
      const cudaError_t q = cudaEventQuery(ev_poll_);
      if (q == cudaSuccess) return GST_OK;
      if (q != cudaErrorNotReady) return fail(GST_E_CUDA, std::string("engine stream: ") + cudaGetErrorString(q));
      if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > watchdog_s_) {
        broken_ = true;
        return fail(GST_E_CUDA, "engine stream did not finish within " + std::to_string(watchdog_s_) +
                                    " s (GST_WATCHDOG_S); the engine is unusable");
      }
      if (spin > 2000) std::this_thread::sleep_for(std::chrono::microseconds(100));
      else std::this_thread::yield();
    }
  }

  // Admits pending queries into free slots while their slabs fit.  When the
  // first pending query does not fit yet, later ones that fit are admitted
  // past it (the memory it waits for is not freed any sooner by idling),
  // but at most kMaxBypass times in a row, so it cannot starve.
  static constexpr int kMaxBypass = 256;
  gst_status admit() {
    size_t pi = 0;
    while (pi < pending_.size()) {
      int t = -1;
      for (int i = 0; i < max_slots_; ++i)
        if (!slot_busy_[i]) { t = i; break; }
      if (t < 0) break;
      auto r = pending_[pi];
      const int k = (int)r->groups.size();
      Shape sh{k, r->D < 0 ? 1 : r->D + 1};
      Slab sb;
      if (!acquire_slab(sh, &sb, /*evict=*/pi == 0)) {
        if (pi == 0 && active_ == 0) {  // cannot fit even alone
          pending_.pop_front();
          r->status = fail(GST_E_NOMEM, "query needs more than the device arena");
          r->done = true;
          continue;
        }
        if (pi == 0 && bypassed_ >= kMaxBypass) break;  // let the front one have the memory
        ++pi;
        continue;
      }
      pending_.erase(pending_.begin() + (std::ptrdiff_t)pi);
      bypassed_ = pi == 0 ? 0 : bypassed_ + 1;
      pi = 0;
      r->t_admit = std::chrono::steady_clock::now();
      Slot& q = h_slot_[t];  // its previous copy finished: the slot was harvested after a sync
      std::memset(&q, 0, sizeof q);
      q.table = sb.table;
      q.mask = sb.mask;
      q.queue = sb.queue;
      q.touched = sb.touched;
      q.tflag = sb.tflag;
      q.dead = sb.dead;
      q.sd = sb.sd;
      q.chunks = sb.chunks;
      q.lbtab = sb.lbtab;
      q.wstack = sb.wstack;
      q.wedges = sb.wedges;
      // merge lists borrow the witness stack (>= 8 V bytes, used only after the last merge)
      q.live[0] = reinterpret_cast<uint32_t*>(sb.wstack);
      q.live[1] = q.live[0] + V_;
      q.chunk_cap = sb.chunk_cap;
      q.wcap = sb.wcap;
      q.k = k;
      q.W = 1 << k;
      q.L = sh.L;
      q.D = r->D;
      for (int i = 0; i < k; ++i) q.groups[i] = r->groups[i];
      q.max_rounds = max_rounds_override_;
      q.phase = PH_ACTIVE;
      q.action = A_INIT;
      q.s = 1;
      q.d = 0;
      q.cur = 0;
      q.best = INF;
      q.R1 = INF / 2;
      q.answer = ~0ull;
      q.delta = delta_ * tuning_.bucket_mult[k];  // plain: first bucket opens at the seeds (cost 0)
      q.bshift = bucket_shift_;
      q.chunk_pairs = tuning_.chunk_pairs[k][r->D >= 0 ? 1 : 0];
      q.T = 0;
      q.next_min = INF;
      q.fcur = 2;
      GST_CUDA(cudaMemcpyAsync(d_slots_ + t, &q, sizeof(Slot), cudaMemcpyHostToDevice, stream_));
      prof_.h2d_bytes += sizeof(Slot);
      if (!r->t0) GST_CUDA(cudaEventCreate(&r->t0));
      GST_CUDA(cudaEventRecord(r->t0, stream_));
      Graph g = graph();
      k_init_seeds<<<64, 256, 0, stream_>>>(d_slots_, t, g);
      k_init_base<<<64, 256, 0, stream_>>>(d_slots_, t, g);
      GST_CUDA(cudaGetLastError());
      prof_.kernel_launches += 2;
      slot_busy_[t] = 1;
      slot_req_[t] = r;
      slot_slab_[t] = sb;
      ++active_;
      nslots_hw_ = std::max(nslots_hw_, t + 1);
    }
    return GST_OK;
  }

  Graph graph() const {
    Graph g;
    g.rowptr = d_rowptr_;
    g.adj = d_adj_;
    g.gptr = d_gptr_;
    g.gmem = d_gmem_;
    g.V = V_;
    g.E = E_;
    g.G = G_;
    return g;
  }

  // One round.  The merge branch (lbprep, merge) and the grow branch (prep,
  // ctl_b, grow) touch disjoint slots: with overlap = 2 they are forked onto
  // two streams after ctl_a and joined before the next round.
  void enqueue_round(cudaStream_t st, int i) {
    Graph g = graph();
    const int grid = num_sms_ * 4;
    const bool fork = tuning_.overlap == 2;
    k_ctl_a<<<1, MAXSLOTS, 0, st>>>(d_slots_, max_slots_, d_plan_, d_status_);
    cudaStream_t sg = st;
    if (fork) {
      cudaEventRecord(ev_fork_, st);
      cudaStreamWaitEvent(stream2_, ev_fork_, 0);
      sg = stream2_;
    }
    k_lbprep<<<std::min(max_slots_, 256), 256, 0, st>>>(d_slots_, d_plan_, g);
    if (profile_) cudaEventRecordWithFlags(ev_prof_[4 * i + 0], st, cudaEventRecordExternal);
    k_merge_t<false><<<grid, MERGE_THREADS, 0, st>>>(d_slots_, d_plan_, g);
    k_merge_t<true><<<grid, MERGE_THREADS, 0, st>>>(d_slots_, d_plan_, g);
    if (profile_) cudaEventRecordWithFlags(ev_prof_[4 * i + 1], st, cudaEventRecordExternal);
    k_prep<<<grid, 256, 0, sg>>>(d_slots_, d_plan_, g);
    k_ctl_b<<<1, MAXSLOTS, 0, sg>>>(d_slots_, d_plan_, 32 / tuning_.grow_lanes);
    if (profile_) cudaEventRecordWithFlags(ev_prof_[4 * i + 2], sg, cudaEventRecordExternal);
    switch (tuning_.grow_lanes) {
      case 8: k_grow_t<8><<<grow_grid_[0], GROW_WARPS * 32, 0, sg>>>(d_slots_, d_plan_, g); break;
      case 32: k_grow_t<32><<<grow_grid_[2], GROW_WARPS * 32, 0, sg>>>(d_slots_, d_plan_, g); break;
      default: k_grow_t<16><<<grow_grid_[1], GROW_WARPS * 32, 0, sg>>>(d_slots_, d_plan_, g); break;
    }
    if (profile_) cudaEventRecordWithFlags(ev_prof_[4 * i + 3], sg, cudaEventRecordExternal);
    if (fork) {
      cudaEventRecord(ev_join_, stream2_);
      cudaStreamWaitEvent(st, ev_join_, 0);
    }
  }

  gst_status launch_rounds() {
    if (!graph_exec_ || graph_rounds_ != rounds_per_poll_ || graph_slots_ != max_slots_) {
      if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
      graph_exec_ = nullptr;
      cudaGraph_t gr;
      if (profile_) {
        for (auto ev : ev_prof_) if (ev) cudaEventDestroy(ev);
        ev_prof_.assign(4 * rounds_per_poll_, nullptr);
        for (auto& ev : ev_prof_) GST_CUDA(cudaEventCreate(&ev));
      }
      GST_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      for (int i = 0; i < rounds_per_poll_; ++i) enqueue_round(stream_, i);
      GST_CUDA(cudaStreamEndCapture(stream_, &gr));
      GST_CUDA(cudaGraphInstantiate(&graph_exec_, gr, 0));
      cudaGraphDestroy(gr);
      graph_rounds_ = rounds_per_poll_;
      graph_slots_ = max_slots_;
    }
    GST_CUDA(cudaGraphLaunch(graph_exec_, stream_));
    k_publish<<<(max_slots_ + 255) / 256, 256, 0, stream_>>>(d_slots_, max_slots_, d_status_);
    GST_CUDA(cudaMemcpyAsync(h_status_, d_status_, sizeof(SlotStatus) * max_slots_,
                             cudaMemcpyDeviceToHost, stream_));
    if (gst_status st = wait_stream(); st != GST_OK) return st;
    prof_.rounds += rounds_per_poll_;
    prof_.kernel_launches += 7 * rounds_per_poll_ + 1;
    prof_.d2h_bytes += sizeof(SlotStatus) * max_slots_;
    if (profile_) {
      for (int i = 0; i < rounds_per_poll_; ++i) {
        float a = 0, b = 0;
        GST_CUDA(cudaEventElapsedTime(&a, ev_prof_[4 * i + 0], ev_prof_[4 * i + 1]));
        GST_CUDA(cudaEventElapsedTime(&b, ev_prof_[4 * i + 2], ev_prof_[4 * i + 3]));
        prof_.merge_ms += a;
        prof_.grow_ms += b;
      }
      prof_.merge_launches += rounds_per_poll_;
      prof_.grow_launches += rounds_per_poll_;
    }
    return GST_OK;
  }

  gst_status harvest() {
    std::vector<int> fin;
    for (int t = 0; t < max_slots_; ++t)
      if (slot_busy_[t] && (h_status_[t].phase == PH_DONE || h_status_[t].phase == PH_ERROR))
        fin.push_back(t);
    if (fin.empty()) return GST_OK;
    cudaEvent_t t1;
    GST_CUDA(cudaEventCreate(&t1));
    GST_CUDA(cudaEventRecord(t1, stream_));
    GST_CUDA(cudaEventSynchronize(t1));
    std::vector<int> wit;
    for (int t : fin)
      if (h_status_[t].phase == PH_DONE && (h_status_[t].answer >> 32) < (unsigned long long)INF)
        wit.push_back(t);
    Graph g = graph();
    if (!wit.empty()) {
      std::memcpy(h_list_, wit.data(), sizeof(int) * wit.size());
      GST_CUDA(cudaMemcpyAsync(d_list_, h_list_, sizeof(int) * wit.size(), cudaMemcpyHostToDevice, stream_));
      k_witness<<<(int)wit.size(), 256, 0, stream_>>>(d_slots_, d_list_, (int)wit.size(), g);
      k_validate<<<(int)wit.size(), 256, 0, stream_>>>(d_slots_, d_list_, (int)wit.size(), g);
      GST_CUDA(cudaGetLastError());
      prof_.kernel_launches += 2;
      prof_.h2d_bytes += sizeof(int) * wit.size();
    }
    // one read-back of the slot array, then one batch of tree-edge copies
    GST_CUDA(cudaMemcpyAsync(h_harv_, d_slots_, sizeof(Slot) * nslots_hw_, cudaMemcpyDeviceToHost, stream_));
    GST_CUDA(cudaStreamSynchronize(stream_));
    prof_.d2h_bytes += sizeof(Slot) * nslots_hw_;
    std::vector<size_t> woff(fin.size() + 1, 0);
    for (size_t i = 0; i < fin.size(); ++i) {
      const Slot& q = h_harv_[fin[i]];
      const bool tree = q.phase == PH_DONE && q.err == ERR_NONE && (q.answer >> 32) < (unsigned long long)INF;
      woff[i + 1] = woff[i] + (tree ? 3 * (size_t)q.nwedges : 0);
    }
    const size_t wtot = woff[fin.size()];
    if (wtot > wedge_cap_) {
      if (h_wedges_) cudaFreeHost(h_wedges_);
      h_wedges_ = nullptr;
      wedge_cap_ = 0;
      const size_t cap = std::max(wtot, (size_t)1 << 16);
      GST_CUDA(cudaMallocHost(&h_wedges_, sizeof(int32_t) * cap));
      wedge_cap_ = cap;
    }
    for (size_t i = 0; i < fin.size(); ++i) {
      const size_t n = woff[i + 1] - woff[i];
      if (n) GST_CUDA(cudaMemcpyAsync(h_wedges_ + woff[i], h_harv_[fin[i]].wedges, sizeof(int32_t) * n,
                                      cudaMemcpyDeviceToHost, stream_));
      prof_.d2h_bytes += sizeof(int32_t) * n;
    }
    if (wtot) GST_CUDA(cudaStreamSynchronize(stream_));
    for (size_t fi = 0; fi < fin.size(); ++fi) {
      const int t = fin[fi];
      auto r = slot_req_[t];
      const Slot q = h_harv_[t];
      gst_result& res = r->result;
      std::memset(&res, 0, sizeof res);
      res.root = -1;
      float ms = 0;
      GST_CUDA(cudaEventElapsedTime(&ms, r->t0, t1));
      res.stats.device_ms = ms;
      res.stats.rounds = q.rounds;
      res.stats.frontier = (int64_t)q.st_frontier;
      res.stats.relax = (int64_t)q.st_relax;
      res.stats.improve = (int64_t)q.st_improve;
      res.stats.merges = (int64_t)q.st_merges;
      res.stats.merge_items = (int64_t)q.st_mitems;
      res.stats.merge_passed = (int64_t)q.st_mpassed;
      res.stats.touched = q.ntouched;
      if (q.phase == PH_ERROR || q.err != ERR_NONE) {
        static const char* why[] = {"", "chunk list overflow", "frontier list overflow",
                                    "tree reconstruction failed", "tree reconstruction buffer overflow",
                                    "round limit exceeded", "tree check failed"};
        static const char* tree_why[] = {"", "an edge is not in the graph with that weight",
                                         "an edge is listed twice", "the edges are not one tree",
                                         "a queried group has no vertex in the tree",
                                         "the edge weights do not sum to the cost",
                                         "hop diameter above D", "tree larger than the check's scratch"};
        std::string msg = std::string("device: ") + (q.err >= 0 && q.err <= 6 ? why[q.err] : "error");
        if (q.err == ERR_TREE && q.terr > 0 && q.terr <= 7) msg += std::string(": ") + tree_why[q.terr];
        r->status = fail(GST_E_LIMIT, msg);
        res.cost = GST_REF_INF;
      } else if ((q.answer >> 32) >= (unsigned long long)INF) {
        res.cost = GST_REF_INF;
        res.feasible = 0;
      } else {
        res.cost = (int64_t)(q.answer >> 32);
        res.feasible = 1;
        res.root = (int32_t)(q.answer & 0xffffffffu);
        // k_validate checked the edges (distinct, a tree of the cost's weight)
        const int ne = q.nwedges;
        const int32_t* e = h_wedges_ + woff[fi];
        res.n_edges = ne;
        res.edges = nullptr;
        if (ne) {
          res.edges = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * 3 * (size_t)ne));
          for (int x = 0; x < ne; ++x) {
            res.edges[3 * x] = std::min(e[3 * x], e[3 * x + 1]);
            res.edges[3 * x + 1] = std::max(e[3 * x], e[3 * x + 1]);
            res.edges[3 * x + 2] = e[3 * x + 2];
          }
        }
        r->status = GST_OK;
      }
      // clean the slab for reuse and free the slot: row by row when few
      // vertices were touched, else plain memsets of the whole slab arrays
      const Slab& sb = slot_slab_[t];
      if ((int64_t)q.ntouched * 4 < V_) {
        k_reset<<<num_sms_ * 2, 256, 0, stream_>>>(d_slots_, t, g);
        prof_.kernel_launches += 1;
      } else {
        const size_t V = (size_t)V_, W = (size_t)1 << sb.shape.k, L = (size_t)sb.shape.L;
        GST_CUDA(cudaMemsetAsync(sb.table, 0x3f, V * W * L * 4, stream_));
        GST_CUDA(cudaMemsetAsync(sb.mask, 0, (L == 1 ? 2 : L) * V * 8, stream_));
        GST_CUDA(cudaMemsetAsync(sb.tflag, 0, V * 4, stream_));
        GST_CUDA(cudaMemsetAsync(sb.dead, 0, (V + 31) / 32 * 4, stream_));
        GST_CUDA(cudaMemsetAsync(sb.sd, 0x3f, V * 32, stream_));
      }
      k_free_slot<<<1, 1, 0, stream_>>>(d_slots_, t);
      GST_CUDA(cudaGetLastError());
      prof_.kernel_launches += 1;
      cache_[slot_slab_[t].shape].push_back(slot_slab_[t]);
      slot_busy_[t] = 0;
      slot_req_[t] = nullptr;
      --active_;
      {
        using ms = std::chrono::duration<double, std::milli>;
        const auto now = std::chrono::steady_clock::now();
        res.stats.queue_ms = ms(r->t_admit - r->t_submit).count();
        res.stats.latency_ms = ms(now - r->t_submit).count();
      }
      r->done = true;
    }
    cudaEventDestroy(t1);
    GST_CUDA(cudaStreamSynchronize(stream_));
    return GST_OK;
  }

  int device_ = -1;
  int num_sms_ = 0;
  int grow_grid_[3] = {0, 0, 0};  // one resident wave of k_grow_t<8 / 16 / 32>
  gst_tuning tuning_{};
  int max_slots_ = 256;
  int rounds_per_poll_ = 8;
  cudaStream_t stream_ = nullptr;
  cudaStream_t stream2_ = nullptr;
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
  Slot* d_slots_ = nullptr;
  Plan* d_plan_ = nullptr;
  SlotStatus* d_status_ = nullptr;
  SlotStatus* h_status_ = nullptr;
  int* d_list_ = nullptr;
  int* h_list_ = nullptr;
  Slot* h_slot_ = nullptr;
  Slot* h_harv_ = nullptr;
  int32_t* h_wedges_ = nullptr;
  size_t wedge_cap_ = 0;
  long long* d_rowptr_ = nullptr;
  int2* d_adj_ = nullptr;
  long long* d_gptr_ = nullptr;
  int32_t* d_gmem_ = nullptr;
  int64_t V_ = 0, E_ = 0, G_ = 0;
  int delta_ = 1;
  int bucket_shift_ = 30;
  std::vector<int64_t> gsize_;
  std::vector<int32_t> gfirst_;
  char* arena_ = nullptr;
  size_t arena_request_ = 0, arena_bytes_ = 0;
  Arena arena_alloc_;
  std::map<Shape, std::vector<Slab>> cache_;
  std::vector<char> slot_busy_;
  std::vector<std::shared_ptr<Request>> slot_req_;
  std::vector<Slab> slot_slab_;
  int nslots_hw_ = 0;
  int bypassed_ = 0;  // admissions past a pending front query that did not fit
  cudaGraphExec_t graph_exec_ = nullptr;
  int graph_rounds_ = 0, graph_slots_ = 0;
  bool profile_ = false;
  std::vector<cudaEvent_t> ev_prof_;
  cudaEvent_t ev_run0_ = nullptr, ev_run1_ = nullptr;
  cudaEvent_t ev_poll_ = nullptr;
  double watchdog_s_ = 120.0;
  bool broken_ = false;  // a device wait timed out: refuse further work
  gst_profile prof_{};
};

}  // namespace gst

// ===========================================================================
// C ABI
// ===========================================================================
using gst::Engine;
using gst::Request;

struct gst_engine {
  Engine eng;
};

struct gst_server {
  gst_engine* e = nullptr;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv_in, cv_out;
  bool stop = false;
  uint64_t next = 1;
  std::deque<std::shared_ptr<Request>> inbox;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> all;
};

extern "C" {

const char* gst_last_error(void) { return gst::last_error_text().c_str(); }

int64_t gst_sizeof(const char* type_name) {
  if (!type_name) return -1;
  const std::string n(type_name);
  if (n == "gst_result") return (int64_t)sizeof(gst_result);
  if (n == "gst_stats") return (int64_t)sizeof(gst_stats);
  if (n == "gst_engine_config") return (int64_t)sizeof(gst_engine_config);
  if (n == "gst_profile") return (int64_t)sizeof(gst_profile);
  if (n == "gst_tuning") return (int64_t)sizeof(gst_tuning);
  if (n == "gst_csr") return (int64_t)sizeof(gst_csr);
  if (n == "gst_groups") return (int64_t)sizeof(gst_groups);
  if (n == "gst_queries") return (int64_t)sizeof(gst_queries);
  return -1;
}

gst_status gst_engine_create(const gst_engine_config* cfg, gst_engine** out) {
  if (!out) return gst::fail(GST_E_INVALID, "gst_engine_create: null out");
  *out = nullptr;
  auto* e = new gst_engine;
  gst_status s = e->eng.init(cfg);
  if (s != GST_OK) {
    delete e;
    return s;
  }
  *out = e;
  return GST_OK;
}

void gst_engine_destroy(gst_engine* e) { delete e; }

gst_status gst_engine_load_graph(gst_engine* e, int64_t V, const int64_t* rowptr, const int32_t* col,
                                 const int32_t* w) {
  if (!e) return gst::fail(GST_E_INVALID, "null engine");
  return e->eng.load_graph(V, rowptr, col, w);
}

gst_status gst_engine_load_groups(gst_engine* e, int64_t n, const int64_t* ptr, const int32_t* members) {
  if (!e) return gst::fail(GST_E_INVALID, "null engine");
  return e->eng.load_groups(n, ptr, members);
}

gst_status gst_engine_set_tuning(gst_engine* e, const gst_tuning* t) {
  if (!e || !t) return gst::fail(GST_E_INVALID, "gst_engine_set_tuning: null argument");
  return e->eng.set_tuning(*t);
}

gst_status gst_engine_get_tuning(gst_engine* e, gst_tuning* out) {
  if (!e || !out) return gst::fail(GST_E_INVALID, "gst_engine_get_tuning: null argument");
  *out = e->eng.tuning();
  return GST_OK;
}

gst_status gst_engine_profile(gst_engine* e, gst_profile* out) {
  if (!e || !out) return gst::fail(GST_E_INVALID, "gst_engine_profile: null argument");
  *out = e->eng.profile();
  return GST_OK;
}

void gst_result_free(gst_result* r) {
  if (!r) return;
  std::free(r->edges);
  r->edges = nullptr;
  r->n_edges = 0;
}

static void hand_out(Request& r, gst_result* out) {
  *out = r.result;
  r.result.edges = nullptr;  // ownership moves to the caller
  r.result.n_edges = 0;
  if (r.t0) {
    cudaEventDestroy(r.t0);
    r.t0 = nullptr;
  }
}

gst_status gst_solve(gst_engine* e, const int32_t* group_ids, int k, int D, gst_result* out) {
  if (!e || !out) return gst::fail(GST_E_INVALID, "gst_solve: null argument");
  std::memset(out, 0, sizeof *out);
  gst_status st;
  auto r = e->eng.make_request(group_ids, k, D, &st);
  if (!r) return st;
  std::vector<std::shared_ptr<Request>> v{r};
  st = e->eng.run(v);
  if (st != GST_OK) return st;
  hand_out(*r, out);
  return r->status;
}

gst_status gst_solve_batch(gst_engine* e, int64_t n, const int64_t* ptr, const int32_t* ids,
                           const int32_t* D, gst_result* out, gst_status* status_out) {
  if (!e || !ptr || !ids || !out || n < 0) return gst::fail(GST_E_INVALID, "gst_solve_batch: null argument");
  std::vector<std::shared_ptr<Request>> reqs(n);
  std::vector<gst_status> sts(n, GST_OK);
  for (int64_t i = 0; i < n; ++i) {
    std::memset(&out[i], 0, sizeof out[i]);
    out[i].cost = GST_REF_INF;
    out[i].root = -1;
    const int64_t b = ptr[i], en = ptr[i + 1];
    if (en < b) {
      sts[i] = gst::fail(GST_E_INVALID, "batch: bad ptr");
      continue;
    }
    reqs[i] = e->eng.make_request(ids + b, (int)(en - b), D ? D[i] : -1, &sts[i]);
  }
  gst_status st = e->eng.run(reqs);
  if (st != GST_OK) return st;
  for (int64_t i = 0; i < n; ++i) {
    if (reqs[i]) {
      hand_out(*reqs[i], &out[i]);
      sts[i] = reqs[i]->status;
    }
    if (status_out) status_out[i] = sts[i];
  }
  return GST_OK;
}

// ---- serving -------------------------------------------------------------------

static void server_loop(gst_server* s) {
  Engine& eng = s->e->eng;
  eng.bind_device();
  while (true) {
    std::vector<std::shared_ptr<Request>> taken;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_in.wait(lk, [&] { return s->stop || !s->inbox.empty() || eng.active_ > 0 || !eng.pending_.empty(); });
      if (s->stop && s->inbox.empty() && eng.active_ == 0 && eng.pending_.empty()) break;
      while (!s->inbox.empty()) {
        taken.push_back(s->inbox.front());
        s->inbox.pop_front();
      }
    }
    for (auto& r : taken)
      if (!r->done) eng.pending_.push_back(r);
    if (eng.step() != GST_OK) {  // device failure: fail everything in flight
      std::lock_guard<std::mutex> lk(s->mu);
      eng.abort_all(gst::last_error_text());
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);  // publish completions to waiters
    }
    s->cv_out.notify_all();
  }
  s->cv_out.notify_all();
}

gst_status gst_server_start(gst_engine* e, gst_server** out) {
  if (!e || !out) return gst::fail(GST_E_INVALID, "gst_server_start: null argument");
  {
    std::lock_guard<std::mutex> lk(e->eng.mu_);
    if (e->eng.busy_) return gst::fail(GST_E_STATE, "a server is already running");
    e->eng.busy_ = true;
  }
  auto* s = new gst_server;
  s->e = e;
  s->th = std::thread(server_loop, s);
  *out = s;
  return GST_OK;
}

gst_status gst_server_submit(gst_server* s, const int32_t* group_ids, int k, int D, uint64_t* ticket) {
  if (!s || !ticket) return gst::fail(GST_E_INVALID, "gst_server_submit: null argument");
  gst_status st;
  auto r = s->e->eng.make_request(group_ids, k, D, &st);
  if (!r) return st;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return gst::fail(GST_E_STATE, "server is stopping");
    r->ticket = s->next++;
    *ticket = r->ticket;
    s->all[r->ticket] = r;
    s->inbox.push_back(r);
  }
  s->cv_in.notify_all();
  return GST_OK;
}

gst_status gst_server_wait(gst_server* s, uint64_t ticket, double timeout_ms, gst_result* out) {
  if (!s || !out) return gst::fail(GST_E_INVALID, "gst_server_wait: null argument");
  std::memset(out, 0, sizeof *out);
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return gst::fail(GST_E_STATE, "unknown or already collected ticket");
  auto r = it->second;
  auto pred = [&] { return r->done.load(); };
  if (timeout_ms < 0) {
    s->cv_out.wait(lk, pred);
  } else if (!s->cv_out.wait_for(lk, std::chrono::microseconds((long long)(timeout_ms * 1000)), pred)) {
    return gst::fail(GST_E_TIMEOUT, "result not ready");
  }
  s->all.erase(it);
  hand_out(*r, out);
  return r->status;
}

void gst_server_stop(gst_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_in.notify_all();
  if (s->th.joinable()) s->th.join();
  {
    std::lock_guard<std::mutex> lk(s->e->eng.mu_);
    s->e->eng.busy_ = false;
  }
  delete s;
}

}  // extern "C"
