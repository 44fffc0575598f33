// gst_solve_noalloc: one query solved without allocating any memory.
//
// Some callers cannot allocate: code that runs while a caller-owned memory
// pool must not grow (a serving process that reserved all HBM up front), code
// inside allocation-free sections of a host framework, or plugin hosts that
// forbid cudaMalloc/cudaFree after start-up.  For them this entry point takes
// the graph and groups as device pointers the caller already owns, returns
// the cost and root in host variables, and keeps every piece of scratch state
// (DP table, dirty masks, frontier lists, chunk list, control blocks) in one
// file-scope static device array of GST_NOALLOC_SCRATCH_BYTES.  It runs the
// same round kernels as the engine, launched directly (no CUDA graph, whose
// instantiation allocates).
//
// The array is part of this library's device image: every GPU that loads the
// library holds it until the process exits.  All calls share it and it keeps
// the previous call's contents, so each call re-initialises what must start
// cleared.  Calls that overlapped on the GPU would race on it, so a call holds
// a process-wide lock from its first device operation until its work has
// finished (calls from several host threads, or for several streams, run one
// after another).  The first call on a device does a one-time set-up on that device
// (symbol address lookup, subset tables); make that first
// call before any stream capture.  Every call checks a token that the set-up
// wrote into this library's device memory: a context that was reset and
// re-created has lost it, so the set-up runs again there.
//
// Device waits are bounded like the engine's: a wait that does not end within
// GST_WATCHDOG_S seconds (environment variable, default 120) fails the call
// with GST_E_CUDA, and later calls on that device are refused, since the
// scratch array may still be in use by the unfinished work.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "status.hpp"  // gst::fail: the library's shared error text

// This translation unit instantiates its own copy of the round kernels and
// of the subset tables under a private namespace, so that the engine's
// definitions are left untouched.
#define gst gst_noalloc
#include "engine_dev.cuh"
#include "kernels.cuh"
#undef gst

namespace gst_noalloc {
using gst::fail;
namespace {

constexpr size_t kScratchBytes = GST_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];
// Written by the set-up; a module loaded into a fresh context starts at 0.
constexpr unsigned kSetupToken = 0x6e6f616cu;
static __device__ unsigned g_setup_token;

struct DeviceSetup {
  bool done = false;
  bool broken = false;            // a device wait ran out: refuse further calls
  unsigned char* base = nullptr;  // device address of g_scratch
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;

// Symbol address of the scratch array, subset tables and the set-up token,
// with the device current.
gst_status setup_device(int dev, DeviceSetup& s) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
  if (e != cudaSuccess) return fail(GST_E_CUDA, std::string("noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  SubsetTables t;
  fill_subset_tables(t);
  e = cudaMemcpyToSymbol(c_sub, &t, sizeof t);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_setup_token, &kSetupToken, sizeof kSetupToken);
  if (e != cudaSuccess) return fail(GST_E_CUDA, std::string("noalloc: set-up: ") + cudaGetErrorString(e));
  s.base = static_cast<unsigned char*>(p);
  s.done = true;
  (void)dev;
  return GST_OK;
}

double watchdog_seconds() {
  const char* w = std::getenv("GST_WATCHDOG_S");
  const double x = w ? std::atof(w) : 120.0;
  return x > 1e-4 ? x : 1e-4;
}

// Waits for the stream with a deadline (no event: nothing is created).
gst_status wait_stream(cudaStream_t st, DeviceSetup& ds) {
  const double limit = watchdog_seconds();
  const auto t0 = std::chrono::steady_clock::now();
  for (int spin = 0;; ++spin) {
    const cudaError_t q = cudaStreamQuery(st);
    if (q == cudaSuccess) return GST_OK;
    if (q != cudaErrorNotReady) return fail(GST_E_CUDA, std::string("noalloc: ") + cudaGetErrorString(q));
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit) {
      ds.broken = true;
      return fail(GST_E_CUDA, "noalloc: device work did not finish within " + std::to_string(limit) +
                                  " s (GST_WATCHDOG_S); further calls on this device are refused");
    }
    if (spin > 2000) std::this_thread::sleep_for(std::chrono::microseconds(100));
    else std::this_thread::yield();
  }
}

// Bucket width of the cost-ordered grows, as the engine computes it at graph
// load: the mean over vertices with edges of their lightest edge weight,
// rounded, at least 1.  acc[0] = sum, acc[1] = count (cleared by the caller).
__global__ void k_delta_sum(Graph g, unsigned long long* acc) {
  unsigned long long sum = 0, cnt = 0;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < g.V;
       v += (long long)gridDim.x * blockDim.x) {
    const long long b = g.rowptr[v], e = g.rowptr[v + 1];
    if (e == b) continue;
    int mn = INT32_MAX;
    for (long long j = b; j < e; ++j) mn = imin(mn, g.adj[j].y);
    sum += (unsigned long long)mn;
    ++cnt;
  }
  for (int o = 16; o; o >>= 1) {
    sum += __shfl_down_sync(0xffffffffu, sum, o);
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  if ((threadIdx.x & 31) == 0 && cnt) {
    atomicAdd(&acc[0], sum);
    atomicAdd(&acc[1], cnt);
  }
}

__global__ void k_delta_set(Slot* q, const unsigned long long* acc) {
  const double m = acc[1] ? (double)acc[0] / (double)acc[1] : 1.0;
  const int d = (int)(m + 0.5);
  q->delta = d > 1 ? d : 1;
}

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace gst_noalloc

extern "C" gst_status gst_solve_noalloc(int64_t V, int64_t E, const int64_t* d_rowptr, const int32_t* d_adj,
                                        int64_t n_groups, const int64_t* d_group_ptr,
                                        const int32_t* d_group_members, const int32_t* group_ids, int k,
                                        int D, void* stream, int64_t* cost_out, int32_t* root_out) {
  using namespace gst_noalloc;
  if (!d_rowptr || !d_adj || !d_group_ptr || !d_group_members || !group_ids || !cost_out || !root_out ||
      V <= 0 || E < 0 || k <= 0)
    return fail(GST_E_INVALID, "noalloc: null pointer or empty input");
  if (V > INT32_MAX || E >= (int64_t)UINT32_MAX) return fail(GST_E_UNSUPPORTED, "noalloc: graph too large");
  if (D > GST_MAX_D) return fail(GST_E_UNSUPPORTED, "noalloc: D above GST_MAX_D");
  if (D < 0) D = -1;
  int32_t groups[MAXK];
  int kk = 0;
  for (int i = 0; i < k; ++i) {
    if (group_ids[i] < 0 || group_ids[i] >= n_groups) return fail(GST_E_INVALID, "noalloc: group id out of range");
    bool dup = false;
    for (int j = 0; j < kk; ++j) dup |= groups[j] == group_ids[i];
    if (dup) continue;
    if (kk == MAXK) return fail(GST_E_UNSUPPORTED, "noalloc: more than GST_MAX_K distinct groups");
    groups[kk++] = group_ids[i];
  }
  *cost_out = GST_REF_INF;
  *root_out = -1;
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return fail(GST_E_CUDA, std::string("noalloc: ") + cudaGetErrorString(ce));
  if (dev < 0 || dev >= kMaxDevices) return fail(GST_E_INVALID, "noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_setup_mu);  // one call per process at a time: they share the array
  DeviceSetup& ds = g_setup[dev];
  if (ds.broken) return fail(GST_E_STATE, "noalloc: an earlier call on this device timed out");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!ds.done) {
    gst_status st = setup_device(dev, ds);
    if (st != GST_OK) return st;
  }
  unsigned char* base = ds.base;

  // group offsets (two per queried group) and the set-up token, in one wait
  int64_t goff[MAXK][2];
  unsigned token = 0;
  for (int i = 0; i < kk && ce == cudaSuccess; ++i)
    ce = cudaMemcpyAsync(goff[i], d_group_ptr + groups[i], sizeof goff[i], cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaMemcpyFromSymbolAsync(&token, g_setup_token, sizeof token, 0, cudaMemcpyDeviceToHost, s);
  if (ce != cudaSuccess) return fail(GST_E_CUDA, std::string("noalloc: ") + cudaGetErrorString(ce));
  if (gst_status st = wait_stream(s, ds); st != GST_OK) return st;
  if (token != kSetupToken) {  // the context was reset since the set-up
    gst_status st = setup_device(dev, ds);
    if (st != GST_OK) return st;
    base = ds.base;
  }
  for (int i = 0; i < kk; ++i)
    if (goff[i][1] == goff[i][0]) return GST_OK;  // an empty group: infeasible
  if (kk == 1) {  // one group: any member is a tree of cost 0
    int32_t m = 0;
    ce = cudaMemcpyAsync(&m, d_group_members + goff[0][0], sizeof m, cudaMemcpyDeviceToHost, s);
    if (ce != cudaSuccess) return fail(GST_E_CUDA, std::string("noalloc: ") + cudaGetErrorString(ce));
    if (gst_status st = wait_stream(s, ds); st != GST_OK) return st;
    *cost_out = 0;
    *root_out = m;
    return GST_OK;
  }

  // carve the scratch array
  const size_t W = (size_t)1 << kk, L = D < 0 ? 1 : (size_t)D + 1, nq = D < 0 ? 4 : L;
  const size_t planes = D < 0 ? 2 : L;  // plain: near and far dirty planes
  const size_t chunk_cap = (size_t)V + (size_t)E / 32 + 64;
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += up256(bytes); return o; };
  const size_t o_slot = take(sizeof(Slot));
  const size_t o_plan = take(sizeof(Plan));
  const size_t o_status = take(sizeof(SlotStatus));
  const size_t o_table = take((size_t)V * W * L * 4);
  const size_t o_mask = take(planes * (size_t)V * 8);
  const size_t o_queue = take(nq * (size_t)V * 4);
  const size_t o_touched = take((size_t)V * 4);
  const size_t o_tflag = take((size_t)V * 4);
  const size_t o_dead = take(((size_t)V + 31) / 32 * 4);
  const size_t o_sd = take((size_t)V * 32);
  const size_t o_chunks = take(chunk_cap * sizeof(Chunk));
  const size_t o_lbtab = take((size_t)kk * kk * W * 4 + (size_t)kk * W * 4);
  const size_t o_live = take(2 * (size_t)V * 4);
  const size_t o_acc = take(2 * sizeof(unsigned long long));
  if (off > kScratchBytes)
    return fail(GST_E_NOMEM, "noalloc: query needs " + std::to_string(off >> 20) + " MiB of scratch, above the " +
                                 std::to_string(kScratchBytes >> 20) + " MiB static maximum");
  Slot* d_slot = reinterpret_cast<Slot*>(base + o_slot);
  Plan* d_plan = reinterpret_cast<Plan*>(base + o_plan);
  SlotStatus* d_status = reinterpret_cast<SlotStatus*>(base + o_status);

  Slot q;
  std::memset(&q, 0, sizeof q);
  q.table = reinterpret_cast<int32_t*>(base + o_table);
  q.mask = reinterpret_cast<unsigned long long*>(base + o_mask);
  q.queue = reinterpret_cast<uint32_t*>(base + o_queue);
  q.touched = reinterpret_cast<uint32_t*>(base + o_touched);
  q.tflag = reinterpret_cast<uint32_t*>(base + o_tflag);
  q.dead = reinterpret_cast<uint32_t*>(base + o_dead);
  q.sd = reinterpret_cast<int32_t*>(base + o_sd);
  q.chunks = reinterpret_cast<Chunk*>(base + o_chunks);
  q.lbtab = reinterpret_cast<int32_t*>(base + o_lbtab);
  q.live[0] = reinterpret_cast<uint32_t*>(base + o_live);
  q.live[1] = q.live[0] + V;
  q.wstack = nullptr;
  q.wedges = nullptr;
  q.chunk_cap = (long long)chunk_cap;
  q.wcap = 0;
  q.k = kk;
  q.W = (int)W;
  q.L = (int)L;
  q.D = D;
  for (int i = 0; i < kk; ++i) q.groups[i] = groups[i];
  q.phase = PH_ACTIVE;
  q.action = A_INIT;
  q.s = 1;
  q.cur = 0;
  q.best = INF;
  q.R1 = INF / 2;
  q.answer = ~0ull;
  q.delta = 1;  // replaced on the device by k_delta_set before the first round
  q.bshift = 30;
  q.chunk_pairs = 1024;
  q.T = 0;
  q.next_min = INF;
  q.fcur = 2;

  // what must start cleared: the table (INF), dirty masks, touched flags, plan
  ce = cudaMemsetAsync(base + o_table, 0x3f, (size_t)V * W * L * 4, s);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(base + o_mask, 0, planes * (size_t)V * 8, s);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(base + o_tflag, 0, (size_t)V * 4, s);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(base + o_dead, 0, ((size_t)V + 31) / 32 * 4, s);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(base + o_sd, 0x3f, (size_t)V * 32, s);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(d_plan, 0, sizeof(Plan), s);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(base + o_acc, 0, 2 * sizeof(unsigned long long), s);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(d_slot, &q, sizeof q, cudaMemcpyHostToDevice, s);
  if (ce != cudaSuccess) return fail(GST_E_CUDA, std::string("noalloc: ") + cudaGetErrorString(ce));
  if (gst_status st = wait_stream(s, ds); st != GST_OK) return st;  // q lives on this stack frame

  Graph g;
  g.rowptr = reinterpret_cast<const long long*>(d_rowptr);
  g.adj = reinterpret_cast<const int2*>(d_adj);
  g.gptr = reinterpret_cast<const long long*>(d_group_ptr);
  g.gmem = d_group_members;
  g.V = V;
  g.E = E;
  g.G = n_groups;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = nsm * 4;
  unsigned long long* d_acc = reinterpret_cast<unsigned long long*>(base + o_acc);
  k_delta_sum<<<grid, 256, 0, s>>>(g, d_acc);
  k_delta_set<<<1, 1, 0, s>>>(d_slot, d_acc);
  k_init_seeds<<<64, 256, 0, s>>>(d_slot, 0, g);
  k_init_base<<<64, 256, 0, s>>>(d_slot, 0, g);
  const long long max_rounds = 4ll * V * (long long)L + 1000;  // far above any DP's need
  SlotStatus hs;
  long long rounds = 0;
  for (;;) {
    for (int r = 0; r < 8; ++r) {
      k_ctl_a<<<1, MAXSLOTS, 0, s>>>(d_slot, 1, d_plan, d_status);
      k_lbprep<<<1, 256, 0, s>>>(d_slot, d_plan, g);
      k_merge_t<false><<<grid, MERGE_THREADS, 0, s>>>(d_slot, d_plan, g);
      k_merge_t<true><<<grid, MERGE_THREADS, 0, s>>>(d_slot, d_plan, g);
      k_prep<<<grid, 256, 0, s>>>(d_slot, d_plan, g);
      k_ctl_b<<<1, MAXSLOTS, 0, s>>>(d_slot, d_plan, 32 / GROW_LANES_DEFAULT);
      k_grow_t<GROW_LANES_DEFAULT><<<grid, GROW_WARPS * 32, 0, s>>>(d_slot, d_plan, g);
    }
    rounds += 8;
    k_publish<<<1, 32, 0, s>>>(d_slot, 1, d_status);
    ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&hs, d_status, sizeof hs, cudaMemcpyDeviceToHost, s);
    if (ce != cudaSuccess) return fail(GST_E_CUDA, std::string("noalloc: ") + cudaGetErrorString(ce));
    if (gst_status st = wait_stream(s, ds); st != GST_OK) return st;
    if (hs.phase == PH_DONE || hs.phase == PH_ERROR) break;
    if (rounds > max_rounds) return fail(GST_E_LIMIT, "noalloc: round limit exceeded");
  }
  if (hs.phase == PH_ERROR || hs.err != ERR_NONE) return fail(GST_E_LIMIT, "noalloc: device-side bound hit");
  if ((hs.answer >> 32) < (unsigned long long)INF) {
    *cost_out = (int64_t)(hs.answer >> 32);
    *root_out = (int32_t)(hs.answer & 0xffffffffu);
  }
  return GST_OK;
}
