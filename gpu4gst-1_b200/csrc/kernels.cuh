// Round kernels of the GST engine (sm_100a).
//
// A query runs the DP layer by layer over |S| (the "layered DPBF"):
//   layer 1   k singleton shortest-path trees grown from the group members
//             (the one-label distances of dis0_init_1, code/TrimCDP/src/DPQ.cu:241-271);
//   lbprep    group-to-group bounds and Held-Karp path table for the tour
//             lower bounds (host W/W1 tables of code/TrimCDP/src/DPQ.cu:409-483,
//             LB_procedure of code/PrunedDP++/include/CPUNONHOP.h:436-496);
//   layer s   subset join at every touched vertex (merge,
//             code/TrimCDP/src/DPQ.cu:140-170) followed by frontier edge
//             relaxation until no state of the layer improves (grow, :112-137);
//   layer k   join of the full set at every vertex: the answer.
// The D- variants carry a depth label per state (code/D-TrimCDP/src/DPQ.cu:62-120):
// grow moves label l to l+1 (l < D); merging labels l1, l2 needs l1 + l2 <= D and
// yields max(l1, l2).  Tables hold the best cost found with that label; a value
// is only stored when it beats every smaller label, so prefix minima over labels
// are the costs "with depth at most l".
//
// Pruning (all admissible, so every optimal derivation survives):
//   * grow sources must cost at most best/2 (optimal-tree decomposition,
//     PrunedDP++ Theorem 1, CPUNONHOP.h:795);
//   * a state is dropped when cost + lb(v, S) > best, lb the max of the
//     one-label bound and the two tour bounds of LB_procedure (rounded up:
//     the tree cost is an integer at least half the tour);
//   * a vertex whose whole-tree lower bound exceeds best is dropped from the
//     later merges (live lists) and, for the plain problem, from grows and
//     preps (dead bitmap): no tree of cost <= best passes through it;
//   * after an untruncated layer 1, a missing singleton entry means the group
//     is out of reach, so every (v, S) containing it is skipped.
// All kernels run on a fixed grid and read their work sizes from device
// memory, so a round (ctl_a, then the merge branch lbprep, merge, merge_wide
// and the grow branch prep, ctl_b, grow, which touch disjoint slots) can be
// captured once in a CUDA graph and replayed.  Finished slots get k_witness
// (tree rebuild) and k_validate (tree check).
#pragma once
#include <cuda_runtime.h>

#include "engine_dev.cuh"

namespace gst {

__constant__ SubsetTables c_sub;

constexpr int GROW_WARPS = 8;
// The grow is bound by the latency of dependent random reads, so resident
// warps matter more than pairs in flight per lane.  With no call in the
// relaxation loop it needs 64 registers: 4 blocks of 8 warps per SM
// (measured best; 6 blocks at 40 registers spill onto the loop).
constexpr int GROW_MIN_BLOCKS = 4;
constexpr int GROW_QUEUE = 128;  // improving candidates queued per warp
// Lanes per chunk (a template parameter of k_grow_t: 8, 16 or 32; 16 unless
// a tuning says otherwise): a warp relaxes 32 / lanes chunks side by side, so
// the per-chunk latency (descriptor, source row, dirty sets) overlaps.
constexpr int GROW_LANES_DEFAULT = 16;

__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }
__device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }

// Largest j in [0, n) with off[j] <= g (off[0] = 0, off[n] = total > g).
__device__ __forceinline__ int seg_search(const long long* off, int n, long long g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void touch(Slot& q, uint32_t u) {
  if (q.tflag[u] == 0 && atomicExch(&q.tflag[u], 1u) == 0u) {
    int p = atomicAdd(&q.ntouched, 1);
    q.touched[p] = u;
  }
}

// Marks (u, rank r, label l) dirty and enqueues u on the list qi if it was clean.
__device__ __forceinline__ void mark_dirty(Slot& q, long long V, uint32_t u, int r, int mi, int qi) {
  unsigned long long* mp = &q.mask[(long long)mi * V + u];
  // within a grow or merge pass bits are only set, so a bit seen set stays set
  if ((*(volatile unsigned long long*)mp >> r) & 1ull) return;
  unsigned long long om = atomicOr(mp, 1ull << r);
  if (om == 0ull) {
    int pos = atomicAdd(&q.qcount[qi], 1);
    if (pos < V) q.queue[(long long)qi * V + pos] = u;
    else q.err = ERR_QUEUE_CAP;
  }
}

// Plain problem: marks (u, rank r) with cost c dirty in the near plane if c is
// below the bucket bound T, else in the far plane (and far list).
__device__ __forceinline__ void mark_plain(Slot& q, long long V, uint32_t u, int r, int c) {
  if (c < q.T) {
    mark_dirty(q, V, u, r, 0, q.cur ^ 1);
  } else {
    unsigned long long* mp = &q.mask[V + u];
    if (!((*(volatile unsigned long long*)mp >> r) & 1ull)) {
      const unsigned long long om = atomicOr(mp, 1ull << r);
      if (om == 0ull) {
        const int pos = atomicAdd(&q.qcount[q.fcur], 1);
        if (pos < V) q.queue[(long long)q.fcur * V + pos] = u;
        else q.err = ERR_QUEUE_CAP;
      }
    }
    // next_min only decreases during the pass: skip the contended atomic
    // unless this cost can lower it
    if (c < *(volatile int*)&q.next_min) atomicMin(&q.next_min, c);
  }
}

// Distance lower bound of v to singleton group i: entries above R1 only tell
// that the distance exceeds R1.
__device__ __forceinline__ int clip_dist(int d, int R1) { return d > R1 ? R1 + 1 : d; }

// Tour / one-label lower bound for completing (v, S) given the clipped
// singleton distances dist[0..k) of v (LB_procedure, CPUNONHOP.h:436-496).
// The loops walk the set bits of the complement X of S, so every lane of a
// layer (same |S|) runs the same (k - |S|)^2 iterations.  ceil(t / 2) is
// monotone in t, so the tour bound rounds its minimum once.
__device__ __forceinline__ int lower_bound(const int* dist, int k, int W, int S,
                                           const int32_t* lbtab, long long lim) {
  // Callers only ask whether the bound exceeds lim, so the parts are taken
  // cheapest first (one-label O(m), W2 tour O(m), pairwise tour O(m^2), m =
  // |X|) and the first that exceeds lim ends the evaluation; a bound <= lim
  // is the exact maximum of the three.  Unsigned 32-bit sums: every term is
  // at most INF, and three of them stay below 2^32.
  const int Xs = (W - 1) ^ S;
  if (Xs == 0) return 0;
  unsigned one = 0, mind = INF;
  for (int x = Xs; x; x &= x - 1) {
    const unsigned d = (unsigned)dist[__ffs(x) - 1];
    one = one > d ? one : d;
    mind = mind < d ? mind : d;
  }
  unsigned lb = one;
  if ((long long)lb > lim) return (int)(lb < INF ? lb : INF);
  const int32_t* W2 = lbtab + (size_t)k * k * W + Xs;
  for (int x = Xs; x; x &= x - 1) {
    const int i = __ffs(x) - 1;
    const unsigned t2 = ((unsigned)dist[i] + (unsigned)W2[i * W] + mind + 1u) >> 1;
    if (t2 > lb) lb = t2;
  }
  if ((long long)lb > lim) return (int)(lb < INF ? lb : INF);
  unsigned t1 = 2u * INF;
  for (int x = Xs; x; x &= x - 1) {
    const int i = __ffs(x) - 1;
    const unsigned di = (unsigned)dist[i];
    const int32_t* Pi = lbtab + (size_t)i * k * W + Xs;
    for (int y = Xs; y; y &= y - 1) {
      const int jj = __ffs(y) - 1;
      const unsigned t = di + (unsigned)Pi[jj * W] + (unsigned)dist[jj];
      if (t < t1) t1 = t;
    }
  }
  const unsigned lb1 = (t1 + 1u) >> 1;
  if (lb1 > lb && lb1 < INF) lb = lb1;
  return (int)(lb < INF ? lb : INF);
}

// Cheap lower bound of a tree that contains v and touches every group: the
// one-label bound and the W2 tour bound of lower_bound with S empty (O(k);
// the pairwise tour bound is left out).
__device__ __forceinline__ int full_bound(const int* dist, int k, int W, const int32_t* lbtab) {
  const int full = W - 1;
  int one = 0, mind = INF;
  for (int i = 0; i < k; ++i) {
    one = imax(one, dist[i]);
    mind = imin(mind, dist[i]);
  }
  long long lb = one;
  const int32_t* W2 = lbtab + (size_t)k * k * W + full;
  for (int i = 0; i < k; ++i) {
    const long long t2 = ((long long)dist[i] + W2[i * W] + mind + 1) >> 1;
    if (t2 > lb) lb = t2;
  }
  return (int)(lb < INF ? lb : INF);
}

// ---------------------------------------------------------------------------
// Admission: seed the singleton states of the group members.
// ---------------------------------------------------------------------------
__global__ void k_init_seeds(Slot* slots, int t, Graph g) {
  Slot& q = slots[t];
  const int k = q.k, L = q.L, rowlen = q.W * q.L;
  long long total = 0;
  for (int i = 0; i < k; ++i) total += g.gptr[q.groups[i] + 1] - g.gptr[q.groups[i]];
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total;
       x += (long long)gridDim.x * blockDim.x) {
    long long rem = x;
    int i = 0;
    for (; i < k; ++i) {
      long long n = g.gptr[q.groups[i] + 1] - g.gptr[q.groups[i]];
      if (rem < n) break;
      rem -= n;
    }
    uint32_t v = (uint32_t)g.gmem[g.gptr[q.groups[i]] + rem];
    q.table[(long long)v * rowlen + (1 + i) * L + 0] = 0;
    touch(q, v);
    if (q.D >= 0) mark_dirty(q, g.V, v, i, 0, 0);
    else mark_plain(q, g.V, v, i, 0);
  }
  (void)L;
}

// Base states: cost 0 for every S inside groupset(v) (CPUNONHOP.h:594-624).
__global__ void k_init_base(Slot* slots, int t, Graph g) {
  Slot& q = slots[t];
  const int k = q.k, W = q.W, L = q.L, rowlen = W * L;
  const int n = q.ntouched;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    uint32_t v = q.touched[x];
    int32_t* row = q.table + (long long)v * rowlen;
    int gs = 0;
    for (int i = 0; i < k; ++i)
      if (row[(1 + i) * L] == 0) gs |= 1 << i;
    for (int S = gs; S > 0; S = (S - 1) & gs)
      if (__popc(S) >= 2) row[c_sub.sidx[k][S] * L] = 0;
    if (gs == W - 1) atomicMin(&q.best, 0);
  }
}

// ---------------------------------------------------------------------------
// Control: advance every slot's state machine and lay out this round's work.
// One block of MAXSLOTS threads.
// ---------------------------------------------------------------------------
__global__ void k_ctl_a(Slot* slots, int nslots, Plan* plan, SlotStatus* status) {
  __shared__ long long s_scan[2][MAXSLOTS];
  __shared__ int s_cnt[3][MAXSLOTS];
  const int t = threadIdx.x;
  int act = A_NONE;
  long long n_merge = 0, n_prep = 0;
  if (t < nslots) {
    Slot& q = slots[t];
    if (q.phase == PH_ACTIVE) {
      const bool hop = q.D >= 0;
      const int pa = q.action;
      q.rounds++;
      if (q.err != ERR_NONE || (q.max_rounds > 0 && q.rounds > q.max_rounds)) {
        if (q.err == ERR_NONE) q.err = ERR_ROUNDS;
        q.phase = PH_ERROR;
      } else {
        bool done = false;
        switch (pa) {
          case A_INIT: if (hop) q.d = 0; break;
          case A_GROW:
            if (!hop) {
              q.qcount[q.farround ? (q.fcur ^ 1) : q.cur] = 0;  // the list this round consumed
              q.cur ^= 1;
            } else {
              q.qcount[q.d] = 0;
              q.d += 1;
            }
            break;
          case A_MERGE: if (hop) q.d = 0; q.sd_ready = 1; break;
          case A_MERGEFULL: q.phase = PH_DONE; done = true; break;
          default: break;
        }
        q.nchunks = 0;
        q.farround = 0;
        if (!done) {
          if (pa == A_LBPREP) {
            q.s = 2;
            act = (q.k == 2) ? A_MERGEFULL : A_MERGE;
          } else {
            bool more;
            if (!hop) {
              more = q.qcount[q.cur] > 0;
              if (!more && q.qcount[q.fcur] > 0) {
                // the bucket is drained: open the next one at the cheapest
                // waiting state and drain the far list into it
                const int width = q.best < INF ? imax(q.delta, q.best >> q.bshift) : q.delta;
                q.T = q.next_min + width;
                q.next_min = INF;
                q.fcur ^= 1;
                q.farround = 1;
                more = true;
              }
            } else {
              while (q.d < q.D && q.qcount[q.d] == 0) q.d++;
              more = q.d < q.D;
            }
            if (more) {
              act = A_GROW;
            } else if (q.s == 1) {
              act = A_LBPREP;
            } else {
              q.s += 1;
              act = (q.s == q.k) ? A_MERGEFULL : A_MERGE;
            }
          }
          if (act == A_MERGE || act == A_MERGEFULL) {
            // one item per (listed vertex, set of the layer): the previous
            // merge's live list plus the vertices touched since it was cut
            if (q.s == 2 || hop) {
              // D-queries visit every touched vertex: their best is rarely
              // finite early enough for the liveness test to drop any
              q.lr = 0;
              q.nlr = 0;
              q.mt0 = 0;
            } else {
              q.lr ^= 1;
              q.nlr = q.nlw;
              q.mt0 = q.mt1;
            }
            q.nlw = 0;
            q.mt1 = q.ntouched;
            n_merge = (long long)(q.nlr + q.mt1 - q.mt0) * (c_sub.loff[q.k][q.s + 1] - c_sub.loff[q.k][q.s]);
          }
          if (act == A_GROW) n_prep = hop ? q.qcount[q.d] : q.qcount[q.farround ? (q.fcur ^ 1) : q.cur];
          // plain layers >= 2: consult the dead bitmap in prep and grow once
          // the last merge dropped most of the vertices it visited (the
          // bitmap read is an extra dependent step for live targets)
          q.use_dead = !hop && q.s >= 2 && 2LL * q.nlw < (long long)q.nlr + q.mt1 - q.mt0;
        }
      }
      q.action = act;
    }
    status[t].phase = q.phase;
    status[t].err = q.err;
    status[t].answer = q.answer;
  }
  // compact the slot list of each action with block-wide inclusive scans
  const int f0 = (act == A_LBPREP), f1 = (act == A_MERGE || act == A_MERGEFULL), f2 = (act == A_GROW);
  const int n_wide = __syncthreads_count(f1 && slots[t < nslots ? t : 0].L > 6);
  if (t == 0) plan->n_wide_merge = n_wide;
  s_cnt[0][t] = f0;
  s_cnt[1][t] = f1;
  s_cnt[2][t] = f2;
  s_scan[0][t] = f1 ? n_merge : 0;
  s_scan[1][t] = f2 ? n_prep : 0;
  __syncthreads();
  for (int off = 1; off < MAXSLOTS; off <<= 1) {
    long long a0 = 0, a1 = 0;
    int c0 = 0, c1 = 0, c2 = 0;
    if (t >= off) {
      a0 = s_scan[0][t - off]; a1 = s_scan[1][t - off];
      c0 = s_cnt[0][t - off]; c1 = s_cnt[1][t - off]; c2 = s_cnt[2][t - off];
    }
    __syncthreads();
    s_scan[0][t] += a0; s_scan[1][t] += a1;
    s_cnt[0][t] += c0; s_cnt[1][t] += c1; s_cnt[2][t] += c2;
    __syncthreads();
  }
  if (f0) plan->lb_slots[s_cnt[0][t] - 1] = t;
  if (f1) {
    const int p = s_cnt[1][t] - 1;
    plan->merge_slots[p] = t;
    plan->merge_off[p] = s_scan[0][t] - n_merge;
  }
  if (f2) {
    const int p = s_cnt[2][t] - 1;
    plan->grow_slots[p] = t;
    plan->prep_off[p] = s_scan[1][t] - n_prep;
  }
  if (t == MAXSLOTS - 1) {
    plan->n_lb = s_cnt[0][t];
    plan->n_merge = s_cnt[1][t];
    plan->n_grow = s_cnt[2][t];
    plan->merge_off[s_cnt[1][t]] = s_scan[0][t];
    plan->prep_off[s_cnt[2][t]] = s_scan[1][t];
  }
}

// Chunk offsets of the grow slots, after the prep pass.
__global__ void k_ctl_b(Slot* slots, Plan* plan, int cpw) {
  __shared__ long long s_scan[MAXSLOTS];
  const int t = threadIdx.x;
  const int n = plan->n_grow;
  long long c = 0;
  if (t < n) {
    Slot& q = slots[plan->grow_slots[t]];
    c = q.nchunks;
    if (c > q.chunk_cap) { q.err = ERR_CHUNK_CAP; c = 0; }
    c = (c + cpw - 1) / cpw;  // grow units: cpw chunks each (one warp)
  }
  s_scan[t] = c;
  __syncthreads();
  for (int off = 1; off < MAXSLOTS; off <<= 1) {
    long long a = t >= off ? s_scan[t - off] : 0;
    __syncthreads();
    s_scan[t] += a;
    __syncthreads();
  }
  if (t < n) plan->chunk_off[t] = s_scan[t] - c;
  if (t == MAXSLOTS - 1) plan->chunk_off[n] = s_scan[t];
}

// ---------------------------------------------------------------------------
// Lower-bound tables after the singleton layer (one block per slot).
// vv[i][j]  lower bound of dist(g_i, g_j) from the clipped singleton distances
//           of the members of g_i (virtual_node_distances, CPUNONHOP.h:175-210);
// P[i][j][X] cheapest visiting order of the groups of X from i to j (Held-Karp
//           over vv, the W table of CPUNONHOP.h:269-386 / DPQ.cu:445-472);
// W2[i][X]  min over j of P[i][j][X] (CPUNONHOP.h:568-587).
// ---------------------------------------------------------------------------
__global__ void k_lbprep(Slot* slots, const Plan* plan, Graph g) {
  __shared__ int s_vv[MAXK * MAXK];
  __shared__ int s_P[MAXK * MAXK * MAXW];
  for (int j = blockIdx.x; j < plan->n_lb; j += gridDim.x) {
    Slot& q = slots[plan->lb_slots[j]];
    const int k = q.k, W = q.W, L = q.L, rowlen = W * L;
    const int R1 = q.best >= INF ? INF / 2 : q.best / 2;
    __syncthreads();
    for (int x = threadIdx.x; x < k * k; x += blockDim.x) s_vv[x] = INF;
    for (int x = threadIdx.x; x < k * k * W; x += blockDim.x) s_P[x] = INF;
    __syncthreads();
    for (int i = 0; i < k; ++i) {
      const long long b = g.gptr[q.groups[i]], e = g.gptr[q.groups[i] + 1];
      for (long long m = b + threadIdx.x; m < e; m += blockDim.x) {
        const int32_t* row = q.table + (long long)g.gmem[m] * rowlen;
        for (int jj = 0; jj < k; ++jj) {
          int dmin = INF;
          for (int l = 0; l < L; ++l) dmin = imin(dmin, row[(1 + jj) * L + l]);
          atomicMin(&s_vv[i * k + jj], clip_dist(dmin, R1));
        }
      }
    }
    __syncthreads();
    {  // both directions bound the same distance
      int a = 0, b = 0;
      if (threadIdx.x < k * k) {
        a = s_vv[threadIdx.x];
        b = s_vv[(threadIdx.x % k) * k + threadIdx.x / k];
      }
      __syncthreads();
      if (threadIdx.x < k * k) s_vv[threadIdx.x] = imax(a, b);
    }
    if (threadIdx.x < k) s_P[(threadIdx.x * k + threadIdx.x) * W + (1 << threadIdx.x)] = 0;
    __syncthreads();
    for (int X = 1; X < W; ++X) {
      for (int x = threadIdx.x; x < k * k; x += blockDim.x) {
        int i = x / k, jj = x % k;
        if (!((X >> i) & 1) || !((X >> jj) & 1)) continue;
        int cur = s_P[(i * k + jj) * W + X];
        if (cur >= INF) continue;
        for (int l = 0; l < k; ++l) {
          if ((X >> l) & 1) continue;
          int cand = cur + s_vv[jj * k + l];
          if (cand < INF) atomicMin(&s_P[(i * k + l) * W + (X | (1 << l))], cand);
        }
      }
      __syncthreads();
    }
    for (int x = threadIdx.x; x < k * k * W; x += blockDim.x) q.lbtab[x] = s_P[x];
    for (int x = threadIdx.x; x < k * W; x += blockDim.x) {
      int i = x / W, X = x % W;
      int m = INF;
      for (int jj = 0; jj < k; ++jj) m = imin(m, s_P[(i * k + jj) * W + X]);
      q.lbtab[k * k * W + x] = m;
    }
    if (threadIdx.x == 0) q.R1 = R1;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Merge: subset join of layer s.  One thread per (touched vertex, set of the
// layer); the vertex's row is read through L1 (the threads of one vertex are
// adjacent, so its row is fetched once).  LT is the compile-time label count
// (1 = plain); 0 handles any count.
// ---------------------------------------------------------------------------
constexpr int MERGE_THREADS = 256;
constexpr int DIST_STRIDE = MAXK + (MAXK % 2 == 0 ? 1 : 0);  // odd, >= MAXK

// Segmented (by key, keys contiguous in lane order) reductions; the first lane
// of each segment ends with the result.
__device__ __forceinline__ unsigned long long seg_min_u64(unsigned long long v, unsigned long long key) {
  const int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long ov = __shfl_down_sync(0xffffffffu, v, o);
    const unsigned long long ok = __shfl_down_sync(0xffffffffu, key, o);
    if (lane + o < 32 && ok == key && ov < v) v = ov;
  }
  return v;
}
__device__ __forceinline__ unsigned long long seg_or_u64(unsigned long long v, unsigned long long key) {
  const int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long ov = __shfl_down_sync(0xffffffffu, v, o);
    const unsigned long long ok = __shfl_down_sync(0xffffffffu, key, o);
    if (lane + o < 32 && ok == key) v |= ov;
  }
  return v;
}
__device__ __forceinline__ unsigned long long seg_add_u64(unsigned long long v, unsigned long long key) {
  const int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long ov = __shfl_down_sync(0xffffffffu, v, o);
    const unsigned long long ok = __shfl_down_sync(0xffffffffu, key, o);
    if (lane + o < 32 && ok == key) v += ov;
  }
  return v;
}
__device__ __forceinline__ bool seg_head(unsigned long long key) {
  const int lane = threadIdx.x & 31;
  const unsigned long long pk = __shfl_up_sync(0xffffffffu, key, 1);
  return lane == 0 || pk != key;
}

// Inclusive add-scan of x over lanes with equal key; segments must be runs of
// consecutive lanes.  Every lane of the warp must call it.
__device__ __forceinline__ int seg_iscan(int x, unsigned long long key) {
  const int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    const unsigned long long ky = __shfl_up_sync(0xffffffffu, key, o);
    if (lane >= o && ky == key) x += y;
  }
  return x;
}

// Reserves x consecutive entries of *counter per lane with one atomicAdd per
// run of equal keys (the run's last lane adds the run's total and passes the
// base on).  counter may differ between runs; lanes with x = 0 get an unused
// position.  Every lane of the warp must call it.  A warp with nothing to
// reserve returns after one vote; a warp of one key scans without keys.
__device__ __forceinline__ int seg_reserve(int* counter, int x, unsigned long long key) {
  if (!__any_sync(0xffffffffu, x != 0)) return 0;
  const int lane = threadIdx.x & 31;
  const unsigned long long kf = __shfl_sync(0xffffffffu, key, 0), kl = __shfl_sync(0xffffffffu, key, 31);
  int incl, tail;
  if (kf == kl) {
    incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    tail = 31;
  } else {
    incl = seg_iscan(x, key);
    tail = 31 - __clz(__match_any_sync(0xffffffffu, key));
  }
  int base = 0;
  if (lane == tail && incl > 0) base = atomicAdd(counter, incl);
  base = __shfl_sync(0xffffffffu, base, tail);
  return base + incl - x;
}

// Merged costs M[0..L) (prefix minima over labels) of set S at a vertex row.
// sidx: the subset -> index map of this k (in shared memory: lanes look up
// different subsets, which the constant cache would serialise).  With a
// compile-time label count LT > 1 the bound is D = LT - 1, so the label
// pairing below indexes registers.
template <int LT>
__device__ __forceinline__ void merge_costs(const int32_t* row, const uint8_t* sidx, int S, int Lrt, int Drt,
                                            int* M) {
  const int L = LT > 0 ? LT : Lrt;
  const int D = LT > 0 ? LT - 1 : Drt;
  const int base = sidx[S] * L;
  {
    int m = INF;
#pragma unroll
    for (int l = 0; l < (LT > 0 ? LT : MAXL); ++l) {
      if (LT == 0 && l >= L) break;
      m = imin(m, row[base + l]);
      M[l] = m;
    }
  }
  // each unordered split once: S1 holds the highest group of S, S2 = S ^ S1
  // is a non-empty part of the rest (2^(s-1) - 1 iterations, none wasted)
  const int top = 1 << (31 - __clz(S));
  const int rest = S ^ top;
  for (int T = (rest - 1) & rest; rest != 0; T = (T - 1) & rest) {
    const int S1 = top | T, S2 = rest ^ T;
    const int i1 = sidx[S1] * L, i2 = sidx[S2] * L;
    if (LT == 1) {
      M[0] = imin(M[0], row[i1] + row[i2]);
    } else {
      int a[LT > 0 ? LT : MAXL], b[LT > 0 ? LT : MAXL];
      int ma = INF, mb = INF;
      if (LT > 1 && LT % 2 == 0) {
        // an even label count keeps a set's labels 8-byte aligned: pairs per load
        const int2* r1 = reinterpret_cast<const int2*>(row + i1);
        const int2* r2 = reinterpret_cast<const int2*>(row + i2);
#pragma unroll
        for (int h = 0; h < (LT > 1 ? LT / 2 : 1); ++h) {
          const int2 x = r1[h], y = r2[h];
          ma = imin(ma, x.x);
          mb = imin(mb, y.x);
          a[2 * h] = ma;
          b[2 * h] = mb;
          ma = imin(ma, x.y);
          mb = imin(mb, y.y);
          a[2 * h + 1] = ma;
          b[2 * h + 1] = mb;
        }
      } else {
#pragma unroll
        for (int l = 0; l < (LT > 0 ? LT : MAXL); ++l) {
          if (LT == 0 && l >= L) break;
          ma = imin(ma, row[i1 + l]);
          mb = imin(mb, row[i2 + l]);
          a[l] = ma;
          b[l] = mb;
        }
      }
#pragma unroll
      for (int l = 0; l < (LT > 0 ? LT : MAXL); ++l) {
        if (LT == 0 && l >= L) break;
        const int m2 = imin(l, D - l);
        M[l] = imin(M[l], imin(a[l] + b[m2], a[m2] + b[l]));
      }
    }
    if (T == 0) break;
  }
#pragma unroll
  for (int l = 1; l < (LT > 0 ? LT : MAXL); ++l) {
    if (LT == 0 && l >= L) break;
    M[l] = imin(M[l], M[l - 1]);
  }
}

// Adds a run of merge statistics to slot t (nothing for t < 0).
__device__ __forceinline__ void flush_merge_counts(Slot* slots, int t, unsigned long long items,
                                                   unsigned long long passed, unsigned long long splits) {
  if (t < 0) return;
  if (items) atomicAdd(&slots[t].st_mitems, items);
  if (passed) atomicAdd(&slots[t].st_mpassed, passed);
  if (splits) atomicAdd(&slots[t].st_merges, splits);
}

// Returns whether the split loop ran (false: the lower-bound pre-filter
// rejected the item).  vdist: the vertex's clipped singleton distances and
// vmiss: the groups with no singleton entry at the vertex, both computed
// once per vertex by the lanes that share it.
template <int LT>
__device__ __forceinline__ bool merge_item(Slot& q, int t, uint32_t v, int r, int S, const uint8_t* sidx,
                                           const int* vdist, unsigned vmiss, Graph& g, unsigned long long* ans,
                                           unsigned long long* dirty0, int* dmin) {
  const int k = q.k, W = q.W, L = LT > 0 ? LT : q.L, rowlen = W * L, D = q.D, s = q.s;
  const bool hop = D >= 0;
  const int lo = c_sub.loff[k][s];
  int32_t* row = q.table + (long long)v * rowlen;
  const int best = *(volatile int*)&q.best;
  // R1 >= INF / 2: layer 1 ran untruncated (best was still unknown), so a
  // missing singleton entry means the group is out of reach (for a D-query:
  // more than D hops away) and every state (v, S) holding it is infinite
  const bool reach_known = q.R1 >= INF / 2;
  int lbv = 0;
  if (s < k) {
    // a tree rooted at v that covers S reaches every group of S, so its cost
    // is at least max_{i in S} dist_i(v): skip the split loop when even that
    // cannot pass the lower-bound test
    if (reach_known && (vmiss & (unsigned)S)) return false;
    int need = 0;
    for (int x = S; x; x &= x - 1) need = imax(need, vdist[__ffs(x) - 1]);
    lbv = lower_bound(vdist, k, W, S, q.lbtab, (long long)best - need);
    if ((long long)need + lbv > best) return false;
  } else {
    // full join: the answer at v is a tree rooted at v touching every group
    if (reach_known && vmiss) return false;
    if (full_bound(vdist, k, W, q.lbtab) > best) return false;
  }
  int M[LT > 0 ? LT : MAXL];
  merge_costs<LT>(row, sidx, S, L, D, M);
  if (s == k) {
    const int a = M[L - 1];
    if (a < INF) *ans = ((unsigned long long)(unsigned)a << 32) | (unsigned long long)v;
    return true;
  }
  for (int l = 0; l < L; ++l) {
    const int val = M[l];
    if (val >= INF) continue;
    if (l > 0 && val >= M[l - 1]) continue;     // no better than a smaller label
    if ((long long)val + lbv > best) continue;  // cannot be part of an optimum
    const long long idx = (long long)(lo + r) * L + l;
    if (val < row[idx]) row[idx] = val;
    // star upper bound: the cheapest path to every missing group
    long long ub = val;
    const int hl = hop ? imin(l, D - l) : 0;
    for (int i = 0; i < k && ub < INF; ++i)
      if (!((S >> i) & 1)) {
        int dm = INF;
        for (int x = 0; x <= hl; ++x) dm = imin(dm, row[(1 + i) * L + x]);
        ub += dm;
      }
    if (ub < best) atomicMin(&q.best, (int)ub);
    if (2LL * val <= best && (!hop || l < D)) {
      if (!hop) {  // plain: aggregated per vertex by the caller
        *dirty0 |= 1ull << r;
        *dmin = imin(*dmin, val);
      } else {
        mark_dirty(q, g.V, v, r, l, l);
      }
    }
  }
  (void)t;
  return true;
}

// 4 blocks per SM (64 registers, no spills): 25% faster than the 3 that 78
// registers allow, on C2 and C4.  Label counts up to 6 (D <= 5) are
// compile-time cases of k_merge; larger ones (D >= 6) run in k_merge_wide,
// whose run-time label loops need more registers than the kernel of the
// common cases may use without spilling.  Each kernel skips the other's
// items; k_merge_wide returns at once when no merging slot needs it.
template <bool WIDE>
__global__ void __launch_bounds__(MERGE_THREADS, 4)
k_merge_t(Slot* slots, const Plan* plan, Graph g) {
  __shared__ long long s_off[MAXSLOTS + 1];
  __shared__ int s_slot[MAXSLOTS];
  __shared__ uint8_t s_sidx[MAXK + 1][MAXW], s_sof[MAXK + 1][MAXW];
  // singleton distances of the vertex whose items start at a lane (the lower
  // bound indexes them by set bit, which would put a register array in local
  // memory), and the vertex's unreachable-group mask
  __shared__ int s_vdist[MERGE_THREADS * DIST_STRIDE];
  __shared__ unsigned s_vmiss[MERGE_THREADS];
  const int lane = threadIdx.x & 31;
  const int wbase = threadIdx.x - lane;
  const int nm = plan->n_merge;
  if (nm == 0 || (WIDE && plan->n_wide_merge == 0)) return;
  for (int x = threadIdx.x; x <= nm; x += blockDim.x) s_off[x] = plan->merge_off[x];
  for (int x = threadIdx.x; x < nm; x += blockDim.x) s_slot[x] = plan->merge_slots[x];
  for (int x = threadIdx.x; x < (MAXK + 1) * MAXW; x += blockDim.x) {
    (&s_sidx[0][0])[x] = (&c_sub.sidx[0][0])[x];
    (&s_sof[0][0])[x] = (&c_sub.sof[0][0])[x];
  }
  __syncthreads();
  const long long total = s_off[nm];
  const long long stride = (long long)gridDim.x * blockDim.x;
  // every lane of a warp iterates the same number of times (shuffles below)
  const long long span = (total + 31) & ~31ll;
  int acc_slot = -1;  // warp-uniform statistics run (see the loop's end)
  unsigned long long acc_items = 0, acc_passed = 0, acc_splits = 0;
  for (long long gi = blockIdx.x * (long long)blockDim.x + threadIdx.x; gi < span; gi += stride) {
    unsigned long long ans = ~0ull, dirty = 0, key = ~0ull;
    int dmin = INF;
    int t = -1;
    uint32_t v = 0;
    unsigned long long nsplit = 0;
    int alive = 0;
    int r = 0;  // rank of the item's set in the layer
    if (gi < total) {
      const int j = seg_search(s_off, nm, gi);
      t = s_slot[j];
      Slot& q = slots[t];
      if (WIDE == (q.L > 6)) {
        const int k = q.k, s = q.s;
        const int nS = c_sub.loff[k][s + 1] - c_sub.loff[k][s];
        const long long local = gi - s_off[j];
        int vi;
        if (local < (1ll << 32)) {  // 32-bit division unless a slot holds 2^32 items
          const unsigned l32 = (unsigned)local, q32 = l32 / (unsigned)nS;
          vi = (int)q32;
          r = (int)(l32 - q32 * (unsigned)nS);
        } else {
          vi = (int)(local / nS);
          r = (int)(local % nS);
        }
        v = vi < q.nlr ? q.live[q.lr][vi] : q.touched[q.mt0 + vi - q.nlr];
        key = ((unsigned long long)(unsigned)t << 32) | (unsigned)vi;
      } else {
        t = -1;  // the other merge kernel's item
      }
    }
    // The items of one vertex are consecutive lanes (a segment of equal key).
    // Its lanes split the k singleton minima between them (each over the L
    // labels) and leave them, clipped, in the head lane's shared slot, with
    // the groups that have no entry in the head's miss mask.
    const unsigned seg = __match_any_sync(0xffffffffu, key);
    const int head = __ffs(seg) - 1;
    const int* vdist = s_vdist + (wbase + head) * DIST_STRIDE;
    s_vmiss[threadIdx.x] = 0u;
    __syncwarp();
    if (t >= 0) {
      const Slot& q = slots[t];
      const int k = q.k, L = q.L, R1 = q.R1;
      const int off = __popc(seg & ((1u << lane) - 1)), seglen = __popc(seg);
      int32_t* sdv = q.sd + (long long)v * 8;
      unsigned mm = 0;
      // D-queries read the minima from sd once it is filled (one sector
      // instead of k * L row entries); plain rows hold one label, whose
      // singleton entries share a sector the split loop reads anyway
      if (q.sd_ready && L > 1) {
        for (int i = off; i < k; i += seglen) {
          const int dm = sdv[i];
          s_vdist[(wbase + head) * DIST_STRIDE + i] = clip_dist(dm, R1);
          if (dm >= INF) mm |= 1u << i;
        }
      } else {
        const int32_t* row = q.table + (long long)v * ((long long)q.W * L);
        const bool first = !q.sd_ready;  // the query's first merge: layer 1 is final, keep its minima
        for (int i = off; i < k; i += seglen) {
          int dm = INF;
          for (int l = 0; l < L; ++l) dm = imin(dm, row[(1 + i) * L + l]);
          if (first) sdv[i] = dm;
          s_vdist[(wbase + head) * DIST_STRIDE + i] = clip_dist(dm, R1);
          if (dm >= INF) mm |= 1u << i;
        }
      }
      if (mm) atomicOr(&s_vmiss[wbase + head], mm);
    }
    __syncwarp();
    if (t >= 0) {
      Slot& q = slots[t];
      const int k = q.k, s = q.s;
      const int S = s_sof[k][c_sub.loff[k][s] + r];
      const uint8_t* sidx = s_sidx[k];
      const unsigned vmiss = s_vmiss[wbase + head];
      bool ev = false;
      if (WIDE) {
        ev = merge_item<0>(q, t, v, r, S, sidx, vdist, vmiss, g, &ans, &dirty, &dmin);
      } else {
        switch (q.L) {
          case 1: ev = merge_item<1>(q, t, v, r, S, sidx, vdist, vmiss, g, &ans, &dirty, &dmin); break;
          case 2: ev = merge_item<2>(q, t, v, r, S, sidx, vdist, vmiss, g, &ans, &dirty, &dmin); break;
          case 3: ev = merge_item<3>(q, t, v, r, S, sidx, vdist, vmiss, g, &ans, &dirty, &dmin); break;
          case 4: ev = merge_item<4>(q, t, v, r, S, sidx, vdist, vmiss, g, &ans, &dirty, &dmin); break;
          case 5: ev = merge_item<5>(q, t, v, r, S, sidx, vdist, vmiss, g, &ans, &dirty, &dmin); break;
          default: ev = merge_item<6>(q, t, v, r, S, sidx, vdist, vmiss, g, &ans, &dirty, &dmin); break;
        }
      }
      if (ev) nsplit = (1ull << (__popc(S) - 1)) - 1;
      // the vertex stays on the next layer's list while a tree through it
      // can still cost <= best (best only falls, so a dropped vertex never
      // returns)
      if (r == 0 && s < k && q.D < 0) {
        alive = full_bound(vdist, k, q.W, q.lbtab) <= *(volatile int*)&q.best;
        if (!alive) atomicOr(&q.dead[v >> 5], 1u << (v & 31));
      }
    }
    // Warp epilogue.  The segment reductions and heads use full-warp
    // shuffles, so every lane evaluates them; each is skipped after one vote
    // when no lane of the warp has anything to contribute.
    const unsigned long long skey = t < 0 ? ~0ull : (unsigned long long)(unsigned)t;
    // answers (full join only): one atomicMin per (warp, slot)
    if (__any_sync(0xffffffffu, ans != ~0ull)) {
      const unsigned long long amin = seg_min_u64(ans, skey);
      const bool shead = seg_head(skey);  // every lane: a full-warp shuffle
      if (t >= 0 && shead && amin != ~0ull) atomicMin(&slots[t].answer, amin);
    }
    // plain seeds: one atomicOr (and at most one enqueue) per (warp, vertex),
    // into the far plane; the next grow round opens the first bucket at the
    // cheapest seed
    if (__any_sync(0xffffffffu, dirty != 0ull)) {
      const bool vhead = seg_head(key);
      const unsigned long long dor = seg_or_u64(dirty, key);
      const unsigned long long dm = seg_min_u64((unsigned long long)(unsigned)dmin, key);
      if (t >= 0 && vhead && dor) {
        Slot& q = slots[t];
        const unsigned long long om = atomicOr(&q.mask[g.V + v], dor);
        if (om == 0ull) {
          const int pos = atomicAdd(&q.qcount[q.fcur], 1);
          if (pos < g.V) q.queue[(long long)q.fcur * g.V + pos] = v;
          else q.err = ERR_QUEUE_CAP;
        }
        if ((int)dm < *(volatile int*)&q.next_min) atomicMin(&q.next_min, (int)dm);
      }
    }
    // statistics (items visited, items past the pre-filter, splits): warp
    // sums accumulated while the warp stays on one slot and flushed when it
    // changes (one atomic per counter and run instead of per iteration); a
    // warp spanning slots adds each slot's segment directly
    {
      const int tf = __shfl_sync(0xffffffffu, t, 0), tl = __shfl_sync(0xffffffffu, t, 31);
      const unsigned long long packed =
          t >= 0 ? (1ull | (nsplit ? 1ull << 8 : 0ull) | ((unsigned long long)nsplit << 16)) : 0ull;
      if (tf == tl && tf >= 0) {
        unsigned long long sum = packed;
        for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (tf != acc_slot) {
          if (lane == 0) flush_merge_counts(slots, acc_slot, acc_items, acc_passed, acc_splits);
          acc_slot = tf;
          acc_items = acc_passed = acc_splits = 0;
        }
        acc_items += sum & 0xff;
        acc_passed += (sum >> 8) & 0xff;
        acc_splits += sum >> 16;
      } else {
        const unsigned long long sum = seg_add_u64(packed, skey);
        const bool shead = seg_head(skey);  // every lane: a full-warp shuffle
        if (t >= 0 && shead) flush_merge_counts(slots, t, sum & 0xff, (sum >> 8) & 0xff, sum >> 16);
      }
    }
    // live-list append: one vertex per nS items appends, so most warps skip
    // this after one vote; the alive lanes of one slot share one atomicAdd
    const unsigned am = __ballot_sync(0xffffffffu, alive);
    if (am) {
      const int lane = threadIdx.x & 31;
      const int l0 = __ffs(am) - 1, l1 = 31 - __clz(am);
      const int t0 = __shfl_sync(0xffffffffu, t, l0), t1 = __shfl_sync(0xffffffffu, t, l1);
      if (t0 == t1) {
        int base = 0;
        if (lane == l0) base = atomicAdd(&slots[t0].nlw, __popc(am));
        base = __shfl_sync(0xffffffffu, base, l0);
        if (alive) slots[t].live[slots[t].lr ^ 1][base + __popc(am & ((1u << lane) - 1))] = v;
      } else if (alive) {
        const int pos = atomicAdd(&slots[t].nlw, 1);
        slots[t].live[slots[t].lr ^ 1][pos] = v;
      }
    }
  }
  if (lane == 0) flush_merge_counts(slots, acc_slot, acc_items, acc_passed, acc_splits);
}

// ---------------------------------------------------------------------------
// Prep: snapshot the dirty masks of this round's frontier and cut each
// vertex's adjacency into chunks of bounded work.  The far-list slots, chunk
// ranges and frontier counts are reserved once per run of same-slot lanes.
// ---------------------------------------------------------------------------
__global__ void k_prep(Slot* slots, const Plan* plan, Graph g) {
  __shared__ long long s_off[MAXSLOTS + 1];
  __shared__ int s_slot[MAXSLOTS];
  const int ng = plan->n_grow;
  if (ng == 0) return;
  for (int x = threadIdx.x; x <= ng; x += blockDim.x) s_off[x] = plan->prep_off[x];
  for (int x = threadIdx.x; x < ng; x += blockDim.x) s_slot[x] = plan->grow_slots[x];
  __syncthreads();
  const long long total = s_off[ng];
  const long long span = (total + 31) & ~31ll;  // whole warps: the reservations use shuffles
  for (long long gi = blockIdx.x * (long long)blockDim.x + threadIdx.x; gi < span;
       gi += (long long)gridDim.x * blockDim.x) {
    int t = -1, nfar = 0, nch = 0, nb = 0, fmin = INF;
    uint32_t v = 0;
    unsigned long long m = 0;
    long long eb = 0, ee = 0, ch = 1;
    if (gi < total) {
      const int j = seg_search(s_off, ng, gi);
      t = s_slot[j];
      Slot& q = slots[t];
      const bool hop = q.D >= 0;
      const bool farround = !hop && q.farround;
      const int lvl = hop ? q.d : 0;
      const int qi = hop ? q.d : (farround ? (q.fcur ^ 1) : q.cur);
      v = q.queue[(long long)qi * g.V + (gi - s_off[j])];
      const long long plane = hop ? lvl : (farround ? 1 : 0);
      m = atomicExch(&q.mask[plane * g.V + v], 0ull);
      if (m && q.use_dead && ((q.dead[v >> 5] >> (v & 31)) & 1u)) m = 0;  // no optimal tree reaches v
      if (m) {
        // keep the sets whose cost is still a valid grow source (2 * cost <= best);
        // plain problem: expand only costs below the bucket bound T and put the
        // others back on the far list (cost order: a state is expanded once it
        // is final rather than every time it improves)
        const int best = *(volatile int*)&q.best;
        const int k = q.k, L = q.L, lo = c_sub.loff[k][q.s];
        const int T = hop ? INF : q.T;
        const int32_t* src = q.table + (long long)v * q.W * L;
        unsigned long long far = 0;
        for (unsigned long long x = m; x; x &= x - 1) {
          const int r = __ffsll((long long)x) - 1;
          const int sv = src[(lo + r) * L + lvl];
          if (sv >= INF || 2LL * sv > best) {
            m &= ~(1ull << r);
          } else if (sv >= T) {
            m &= ~(1ull << r);
            far |= 1ull << r;
            fmin = imin(fmin, sv);
          }
        }
        if (far) {
          if (atomicOr(&q.mask[g.V + v], far) == 0ull) nfar = 1;
          if (fmin < *(volatile int*)&q.next_min) atomicMin(&q.next_min, fmin);
        }
        if (m) {
          eb = g.rowptr[v];
          ee = g.rowptr[v + 1];
          nb = __popcll(m);
          if (ee > eb) {
            ch = imax(32, q.chunk_pairs / nb);
            nch = (int)((ee - eb + ch - 1) / ch);
          }
        }
      }
    }
    const unsigned long long key = t < 0 ? ~0ull : (unsigned long long)t;
    Slot* qp = t < 0 ? slots : &slots[t];  // lanes past the end reserve nothing
    const int fpos = seg_reserve(&qp->qcount[t < 0 ? 0 : qp->fcur], nfar, key);
    const int cpos = seg_reserve(&qp->nchunks, nch, key);
    const unsigned long long nfr = seg_add_u64((unsigned long long)nb, key);
    const bool head = seg_head(key);  // every lane: a full-warp shuffle
    if (t < 0) continue;
    Slot& q = *qp;
    if (head && nfr) atomicAdd(&q.st_frontier, nfr);
    if (nfar) {
      if (fpos < g.V) q.queue[(long long)q.fcur * g.V + fpos] = v;
      else q.err = ERR_QUEUE_CAP;
    }
    if (nch == 0) continue;
    if (cpos + nch > q.chunk_cap) { q.err = ERR_CHUNK_CAP; continue; }
    for (int c = 0; c < nch; ++c) {
      Chunk x;
      x.v = v;
      x.eb = (uint32_t)(eb + c * ch);
      x.ee = (uint32_t)(eb + (c + 1) * ch < ee ? eb + (c + 1) * ch : ee);
      x.pad = 0;
      x.mask = m;
      q.chunks[cpos + c] = x;
    }
  }
}

// ---------------------------------------------------------------------------
// Grow: one group of GROW_LANES lanes per chunk, 32 / GROW_LANES chunks of
// one slot per warp.  Lanes walk (edge, dirty set) pairs with the set index
// fastest, so the lanes relaxing one neighbour touch adjacent words of its
// row.  Each lane relaxes two pairs per step, so two independent
// adjacency-then-target read chains are in flight per lane.  A target is read
// before the atomicMin; candidates that beat it are queued per warp in shared
// memory and handled in batches by grow_cold.
// ---------------------------------------------------------------------------

// Lower-bound test of a grow candidate (cold path: only improving candidates
// reach it), kept out of line so the relaxation loop stays small.
// dist: a per-thread scratch of k ints (shared memory: the bound indexes it
// by set bit, which would put a register array in local memory).
// The bound reads the distances of the groups outside S only, so only those
// are loaded.
// Layers >= 2 only: the singleton minima come from sd (one sector) rather
// than from the target row.
__device__ __forceinline__ bool lb_prunes(const int32_t* sdu, int k, int W, int S, int R1,
                                          const int32_t* lbtab, int nc, int best, int* dist) {
  for (int x = (W - 1) ^ S; x; x &= x - 1) {
    const int i = __ffs(x) - 1;
    dist[i] = clip_dist(sdu[i], R1);
  }
  return (long long)nc + lower_bound(dist, k, W, S, lbtab, (long long)best - nc) > best;
}

// Adds a warp's relaxation counters to its slot (one atomic pair per flush).
__device__ __forceinline__ void flush_counts(Slot& q, unsigned long long& nrel, unsigned long long& nimp) {
  for (int o = 16; o; o >>= 1) {
    nrel += __shfl_down_sync(0xffffffffu, nrel, o);
    nimp += __shfl_down_sync(0xffffffffu, nimp, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (nrel) atomicAdd(&q.st_relax, nrel);
    if (nimp) atomicAdd(&q.st_improve, nimp);
  }
  nrel = 0;
  nimp = 0;
}

// Star upper bound at a vertex that just improved a singleton entry: the
// cheapest path to every group, joined at the vertex.  With a diameter bound D
// every branch may be hl = floor(D/2) hops deep and one of them hh = ceil(D/2)
// (any two branches then span at most D hops).
__device__ __forceinline__ void star_bound(Slot& q, const int32_t* trow, int k, int L, int hl, int hh) {
  long long sum = 0, gain = 0;
  int ninf = 0;
  long long deep_only = INF;  // the one group reachable only within hh hops
  for (int i = 0; i < k; ++i) {
    int a = INF, b = INF;
    for (int l = 0; l <= hh; ++l) {
      const int x = trow[(1 + i) * L + l];
      if (l <= hl) a = imin(a, x);
      b = imin(b, x);
    }
    if (b >= INF) return;
    if (a >= INF) {
      if (++ninf > 1) return;
      deep_only = b;
    } else {
      sum += a;
      gain = gain < (long long)b - a ? gain : (long long)b - a;
    }
  }
  const long long ub = ninf ? sum + deep_only : sum + gain;
  if (ub < *(volatile int*)&q.best) atomicMin(&q.best, (int)ub);
}


// Improvement path of a queued batch of candidates (nb <= GROW_QUEUE, at most
// GROW_QUEUE / 32 per lane), each of which beat its target entry when the
// relaxation loop read it.  It runs in phases, so that a lane's stores, mask
// reads and mask atomics are in flight together instead of one candidate's
// chain after another's: the atomicMin stores; for improvements, the touch of
// a first finite entry, the lower bound and, at layer 1, the star upper bound;
// then the dirty marks of the grow sources that survive the bound.  A
// candidate that fails the bound is still stored (a real derivation cost:
// later, costlier candidates for that state stop at the plain read), but
// not marked.  The bound only decides whether a stored candidate is grown
// from, so it is skipped for candidates that are not grow sources (cost
// above best/2, or the last depth label).  Returns the improvements.
__device__ __forceinline__ unsigned grow_cold(Slot& q, long long V, const int* qu, const int* qr, const int* qc,
                                              int nb, int td, int* dist) {
  constexpr int PER = GROW_QUEUE / 32;
  const int lane = threadIdx.x & 31;
  const int k = q.k, W = q.W, L = q.L, D = q.D, s = q.s;
  const bool hop = D >= 0;
  const int best = *(volatile int*)&q.best;
  const int lo = c_sub.loff[k][s];
  int old[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int x = lane + 32 * j;
    old[j] = 0;
    if (x < nb) {
      int32_t* trow = q.table + (long long)(uint32_t)qu[x] * (W * L);
      old[j] = atomicMin(&trow[(long long)(lo + (qr[x] & 0xff)) * L + td], qc[x]);
    }
  }
  unsigned nimp = 0, mark = 0;
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int x = lane + 32 * j;
    if (x < nb && old[j] > qc[x]) {
      const uint32_t u = (uint32_t)qu[x];
      const int rS = qr[x], nc = qc[x];
      ++nimp;
      if (old[j] >= INF) touch(q, u);
      const bool source = 2LL * nc <= best && (!hop || td < D);
      if (s >= 2 && source && lb_prunes(q.sd + (long long)u * 8, k, W, rS >> 8, q.R1, q.lbtab, nc, best, dist))
        continue;
      if (s == 1 && (!hop || td <= (D + 1) / 2))
        star_bound(q, q.table + (long long)u * (W * L), k, L, hop ? D / 2 : 0, hop ? (D + 1) / 2 : 0);
      if (source) mark |= 1u << j;
    }
  }
  // dirty marks of the surviving sources: the mask words first (within a
  // pass bits are only set, so a bit seen set needs no atomic), then the
  // atomics, then the appends
  unsigned long long om[PER];
  int mi[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int x = lane + 32 * j;
    om[j] = 1ull;
    mi[j] = 0;
    if ((mark >> j) & 1u) {
      mi[j] = hop ? td : (qc[x] < q.T ? 0 : 1);
      om[j] = *(volatile unsigned long long*)&q.mask[(long long)mi[j] * V + (uint32_t)qu[x]];
    }
  }
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int x = lane + 32 * j;
    if ((mark >> j) & 1u) {
      const int r = qr[x] & 0xff;
      if ((om[j] >> r) & 1ull) om[j] = 1ull;
      else om[j] = atomicOr(&q.mask[(long long)mi[j] * V + (uint32_t)qu[x]], 1ull << r);
    }
  }
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    if (!((mark >> j) & 1u)) continue;
    const int x = lane + 32 * j;
    const uint32_t u = (uint32_t)qu[x];
    const int qi = hop ? td : (mi[j] == 0 ? (q.cur ^ 1) : q.fcur);
    if (om[j] == 0ull) {
      const int pos = atomicAdd(&q.qcount[qi], 1);
      if (pos < V) q.queue[(long long)qi * V + pos] = u;
      else q.err = ERR_QUEUE_CAP;
    }
    if (!hop && mi[j] == 1 && qc[x] < *(volatile int*)&q.next_min) atomicMin(&q.next_min, qc[x]);
  }
  return nimp;
}

template <int GROW_LANES>
__global__ void __launch_bounds__(GROW_WARPS * 32, GROW_MIN_BLOCKS)
k_grow_t(Slot* slots, const Plan* plan, Graph g) {
  constexpr int GROW_CPW = 32 / GROW_LANES;  // chunks per warp
  __shared__ long long s_off[MAXSLOTS + 1];
  __shared__ int s_slot[MAXSLOTS];
  __shared__ int s_r[GROW_WARPS][GROW_CPW * 64];
  __shared__ int s_sv[GROW_WARPS][GROW_CPW * 64];
  __shared__ int s_qu[GROW_WARPS][GROW_QUEUE], s_qr[GROW_WARPS][GROW_QUEUE], s_qc[GROW_WARPS][GROW_QUEUE];
  __shared__ int s_dist[GROW_WARPS * 32 * DIST_STRIDE];
  int* dist = s_dist + threadIdx.x * DIST_STRIDE;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int sub = lane / GROW_LANES, sl = lane % GROW_LANES;  // lane group and lane in it
  const unsigned gmask = GROW_LANES == 32 ? 0xffffffffu : ((1u << GROW_LANES) - 1) << (sub * GROW_LANES);
  const int ng = plan->n_grow;
  if (ng == 0) return;
  for (int x = threadIdx.x; x <= ng; x += blockDim.x) s_off[x] = plan->chunk_off[x];
  for (int x = threadIdx.x; x < ng; x += blockDim.x) s_slot[x] = plan->grow_slots[x];
  __syncthreads();
  const long long total = s_off[ng];
  const long long nwarps = (long long)gridDim.x * GROW_WARPS;
  unsigned long long nrel = 0, nimp = 0;  // flushed when the slot changes
  unsigned nrel32 = 0;  // this unit's relaxations (a 32-bit counter in the loop needs fewer registers)
  int cur_slot = -1;
  for (long long gi = blockIdx.x * (long long)GROW_WARPS + wib; gi < total; gi += nwarps) {
    const int j = seg_search(s_off, ng, gi);
    if (s_slot[j] != cur_slot) {
      if (cur_slot >= 0) flush_counts(slots[cur_slot], nrel, nimp);
      cur_slot = s_slot[j];
    }
    Slot& q = slots[s_slot[j]];
    // this lane group's chunk of the unit (none past the slot's last chunk)
    const long long ci = (gi - s_off[j]) * GROW_CPW + sub;
    Chunk c;
    c.v = 0; c.eb = 0; c.ee = 0; c.pad = 0; c.mask = 0ull;
    if (ci < q.nchunks) c = q.chunks[ci];
    const int k = q.k, L = q.L, rowlen = q.W * L;
    const bool hop = q.D >= 0;
    const int d = hop ? q.d : 0;
    const int td = hop ? d + 1 : 0;
    const int lo = c_sub.loff[k][q.s];
    const bool use_dead = q.use_dead;
    const int32_t* src = q.table + (long long)c.v * rowlen;
    int* gr = s_r[wib] + sub * 64;
    int* gsv = s_sv[wib] + sub * 64;
    // the chunk's dirty sets (filtered to valid grow sources by the prep pass)
    int nact = 0;
    for (int base = 0; base < 64; base += GROW_LANES) {
      const int b = base + sl;
      int r = -1, sv = INF;
      if ((c.mask >> b) & 1ull) {
        r = b;
        sv = src[(lo + r) * L + d];
      }
      const unsigned ok = (__ballot_sync(0xffffffffu, r >= 0) & gmask) >> (sub * GROW_LANES);
      if (r >= 0) {
        const int p = nact + __popc(ok & ((1u << sl) - 1));
        gr[p] = (int)c_sub.sof[k][lo + r] << 8 | r;  // (subset, rank)
        gsv[p] = sv;
      }
      nact += __popc(ok);
    }
    __syncwarp();
    const int npairs = (int)(c.ee - c.eb) * nact;
    int npmax = npairs;  // the warp runs until its largest chunk is done
    for (int o = GROW_LANES; o < 32; o <<= 1) npmax = max(npmax, __shfl_xor_sync(0xffffffffu, npmax, o));
    if (npmax > 0) {
      // pair p0 + sl = (edge / nact, set % nact), advanced incrementally by
      // GROW_LANES.  The relaxation loop makes no calls (a call's register
      // convention would cost it occupancy): candidates that beat their
      // target are queued in shared memory and handled between batches.
      const int na = nact > 0 ? nact : 1;
      const int qG = GROW_LANES / na, rG = GROW_LANES % na;
      // unsigned: CSR offsets go up to 2^32 - 1 (the loaders' limit)
      uint32_t e = c.eb + (uint32_t)(sl / na);
      int bi = sl % na;
      int p0 = 0;
      while (true) {
        int nb = 0;  // queued candidates (warp-uniform)
        // two pairs per lane per step: their adjacency and target reads are
        // independent, so each lane keeps two random reads in flight
        for (; p0 < npmax && nb <= GROW_QUEUE - 64; p0 += 2 * GROW_LANES) {
          int nc0 = INF, rS0 = 0, nc1 = INF, rS1 = 0;
          int2 a0 = make_int2(0, 0), a1 = make_int2(0, 0);
          if (p0 + sl < npairs) { a0 = __ldg(&g.adj[e]); rS0 = gr[bi]; nc0 = gsv[bi] + a0.y; ++nrel32; }
          e += qG; bi += rG; if (bi >= na) { bi -= na; ++e; }
          if (p0 + GROW_LANES + sl < npairs) { a1 = __ldg(&g.adj[e]); rS1 = gr[bi]; nc1 = gsv[bi] + a1.y; ++nrel32; }
          e += qG; bi += rG; if (bi >= na) { bi -= na; ++e; }
          if (use_dead) {
            if (nc0 < INF && ((q.dead[(uint32_t)a0.x >> 5] >> (a0.x & 31)) & 1u)) nc0 = INF;
            if (nc1 < INF && ((q.dead[(uint32_t)a1.x >> 5] >> (a1.x & 31)) & 1u)) nc1 = INF;
          }
          int cv0 = INF, cv1 = INF;
          if (nc0 < INF) {
            const int32_t* trow = q.table + (long long)a0.x * rowlen + (long long)(lo + (rS0 & 0xff)) * L;
            cv0 = trow[td]; for (int l = 0; l < td; ++l) cv0 = imin(cv0, trow[l]);
          }
          if (nc1 < INF) {
            const int32_t* trow = q.table + (long long)a1.x * rowlen + (long long)(lo + (rS1 & 0xff)) * L;
            cv1 = trow[td]; for (int l = 0; l < td; ++l) cv1 = imin(cv1, trow[l]);
          }
          const bool imp0 = nc0 < cv0, imp1 = nc1 < cv1;
          const unsigned im0 = __ballot_sync(0xffffffffu, imp0);
          if (imp0) { const int x = nb + __popc(im0 & ((1u << lane) - 1)); s_qu[wib][x] = a0.x; s_qr[wib][x] = rS0; s_qc[wib][x] = nc0; }
          nb += __popc(im0);
          const unsigned im1 = __ballot_sync(0xffffffffu, imp1);
          if (imp1) { const int x = nb + __popc(im1 & ((1u << lane) - 1)); s_qu[wib][x] = a1.x; s_qr[wib][x] = rS1; s_qc[wib][x] = nc1; }
          nb += __popc(im1);
        }
        __syncwarp();
        nimp += grow_cold(q, g.V, s_qu[wib], s_qr[wib], s_qc[wib], nb, td, dist);
        __syncwarp();
        if (p0 >= npmax) break;
      }
    }
    __syncwarp();
    nrel += nrel32;
    nrel32 = 0;
  }
  if (cur_slot >= 0) flush_counts(slots[cur_slot], nrel, nimp);
}

// ---------------------------------------------------------------------------
// Witness search: rebuild the tree of a finished slot from its table (one
// block per slot).  Every step follows an exact equality (base, smaller label,
// merge split or grow edge), so the walk ends at base states; a bounded stack
// turns any inconsistency into ERR_WITNESS instead of a hang.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int cum_at(const int32_t* row, int idx, int L, int l) {
  int m = INF;
  for (int x = 0; x <= l; ++x) m = imin(m, row[idx * L + x]);
  return m;
}

__global__ void k_witness(Slot* slots, const int* list, int n, Graph g) {
  __shared__ int s_top, s_found, s_fu, s_stop;
  __shared__ int s_x, s_S, s_l, s_C;
  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    Slot& q = slots[list[j]];
    const int k = q.k, W = q.W, L = q.L, rowlen = W * L, D = q.D;
    const bool hop = D >= 0;
    const int full = W - 1;
    if (threadIdx.x == 0) {
      s_top = 0;
      s_stop = 0;
      q.nwedges = 0;
      const unsigned long long a = q.answer;
      q.wstack[0] = (int)(a & 0xffffffffu);
      q.wstack[1] = full;
      q.wstack[2] = L - 1;
      q.wstack[3] = (int)(a >> 32);
      s_top = 1;
    }
    __syncthreads();
    long long steps = 0;
    while (true) {
      if (threadIdx.x == 0) {
        if (s_top == 0 || s_stop) {
          s_x = -1;
        } else {
          --s_top;
          s_x = q.wstack[s_top * 4 + 0];
          s_S = q.wstack[s_top * 4 + 1];
          s_l = q.wstack[s_top * 4 + 2];
          s_C = q.wstack[s_top * 4 + 3];
        }
        s_found = 0;
      }
      __syncthreads();
      if (s_x < 0) break;
      if (++steps > 8 * q.wcap) {
        if (threadIdx.x == 0) { q.err = ERR_WITNESS_CAP; s_stop = 1; }
        __syncthreads();
        continue;
      }
      const int x = s_x, S = s_S, l = s_l, C = s_C;
      const int32_t* row = q.table + (long long)x * rowlen;
      if (threadIdx.x == 0) {
        int gs = 0;
        for (int i = 0; i < k; ++i)
          if (row[(1 + i) * L] == 0) gs |= 1 << i;
        int found = 0;
        if (C == 0 && (S & gs) == S) {
          found = 1;  // base state
        } else if (hop && l > 0 && S != full && cum_at(row, c_sub.sidx[k][S], L, l - 1) == C) {
          found = 2;
          if (s_top + 1 > q.wcap) { q.err = ERR_WITNESS_CAP; s_stop = 1; }
          else {
            int* st = q.wstack + s_top * 4;
            st[0] = x; st[1] = S; st[2] = l - 1; st[3] = C;
            ++s_top;
          }
        } else {
          // merge witness at label l; the full set is not stored, so its root
          // may have been joined at any label up to l
          const int lmin = (hop && S == full) ? 0 : l;
          for (int S1 = (S - 1) & S; S1 > 0 && !found; S1 = (S1 - 1) & S) {
            const int S2 = S ^ S1;
            if (S1 < S2) continue;
            const int i1 = c_sub.sidx[k][S1], i2 = c_sub.sidx[k][S2];
            int l1 = 0, l2 = 0, c1 = INF, c2 = INF;
            if (!hop) {
              c1 = row[i1]; c2 = row[i2];
            } else {
              for (int lj = lmin; lj <= l && c1 >= INF; ++lj) {
                const int m2 = imin(lj, D - lj);
                const int a1 = cum_at(row, i1, L, lj), a2 = cum_at(row, i2, L, m2);
                const int b1 = cum_at(row, i1, L, m2), b2 = cum_at(row, i2, L, lj);
                if (a1 < INF && a2 < INF && a1 + a2 == C) { c1 = a1; c2 = a2; l1 = lj; l2 = m2; }
                else if (b1 < INF && b2 < INF && b1 + b2 == C) { c1 = b1; c2 = b2; l1 = m2; l2 = lj; }
              }
            }
            if (c1 < INF && c2 < INF && c1 + c2 == C) {
              found = 3;
              if (s_top + 2 > q.wcap) { q.err = ERR_WITNESS_CAP; s_stop = 1; }
              else {
                int* st = q.wstack + s_top * 4;
                st[0] = x; st[1] = S1; st[2] = l1; st[3] = c1;
                st[4] = x; st[5] = S2; st[6] = l2; st[7] = c2;
                s_top += 2;
              }
            }
          }
        }
        s_found = found;
        s_fu = INT32_MAX;
      }
      __syncthreads();
      if (s_found == 0 && S != full && (!hop || l > 0)) {
        // grow witness: a neighbour u with cost(u, S, l-1) + w == C
        const int idx = c_sub.sidx[k][S];
        const long long eb = g.rowptr[x], ee = g.rowptr[x + 1];
        for (long long e = eb + threadIdx.x; e < ee; e += blockDim.x) {
          const int2 a = g.adj[e];
          if (a.y > C) continue;
          const int32_t* urow = q.table + (long long)a.x * rowlen;
          const int cu = hop ? cum_at(urow, idx, L, l - 1) : urow[idx];
          if (cu < INF && cu + a.y == C) atomicMin(&s_fu, (int)(e - eb));
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          if (s_fu != INT32_MAX) {
            const int2 a = g.adj[eb + s_fu];
            if (s_top + 1 > q.wcap || q.nwedges + 1 > q.wcap) { q.err = ERR_WITNESS_CAP; s_stop = 1; }
            else {
              int* st = q.wstack + s_top * 4;
              st[0] = a.x; st[1] = S; st[2] = hop ? l - 1 : 0; st[3] = C - a.y;
              ++s_top;
              int* oe = q.wedges + q.nwedges * 3;
              oe[0] = x; oe[1] = a.x; oe[2] = a.y;
              q.nwedges++;
            }
          } else {
            q.err = ERR_WITNESS;
            s_stop = 1;
          }
        }
      } else if (s_found == 0 && threadIdx.x == 0) {
        q.err = ERR_WITNESS;
        s_stop = 1;
      }
      __syncthreads();
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Tree check of a finished slot (one block per slot, after k_witness): the
// witness edges must exist in the graph with their weights, be distinct, form
// one tree containing the root, touch every queried group, weigh exactly the
// answer's cost and, with a bound D, have hop diameter <= D.  A failure sets
// ERR_TREE and the reason, so the query fails instead of returning a tree the
// engine has not checked (the reference's check, this_is_a_feasible_solution
// of code/PrunedDP++/include/exp_CPU_nonHop.h:17-49, covers connectivity and
// groups only).  Scratch: the witness stack, idle once the walk is done.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tree_fail(Slot& q, int why) {
  if (atomicCAS(&q.terr, TE_NONE, why) == TE_NONE) q.err = ERR_TREE;
}

// Hop distances from entry `src` over the tree edges (entries are edge
// endpoints as representative indices); returns with dist filled (INF where
// unreachable).  Bellman-Ford rounds: a tree of n edges settles in <= n + 1.
__device__ void tree_bfs(const int* rep, int ne, int nent, int src, int* dist, int* s_changed) {
  for (int a = threadIdx.x; a < nent; a += blockDim.x) dist[a] = INF;
  __syncthreads();
  if (threadIdx.x == 0) dist[src] = 0;
  __syncthreads();
  for (int it = 0; it <= ne + 1; ++it) {
    if (threadIdx.x == 0) *s_changed = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < ne; i += blockDim.x) {
      const int a = rep[1 + 2 * i], b = rep[2 + 2 * i];
      const int da = dist[a], db = dist[b];
      if (da < INF && da + 1 < db) { atomicMin(&dist[b], da + 1); *s_changed = 1; }
      if (db < INF && db + 1 < da) { atomicMin(&dist[a], db + 1); *s_changed = 1; }
    }
    __syncthreads();
    const int ch = *s_changed;
    __syncthreads();
    if (!ch) break;
  }
}

__global__ void k_validate(Slot* slots, const int* list, int n, Graph g) {
  __shared__ int s_skip, s_changed, s_nv, s_far, s_maxd, s_found, s_ok;
  __shared__ long long s_sum;
  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    __syncthreads();  // the previous slot's shared values are read
    Slot& q = slots[list[j]];
    const int ne = q.nwedges;
    const int nent = 2 * ne + 1;
    if (threadIdx.x == 0) {
      s_skip = q.err != ERR_NONE;
      if (!s_skip && 3ll * nent > 4ll * q.wcap) { tree_fail(q, TE_SCRATCH); s_skip = 1; }
      s_sum = 0;
      s_nv = 0;
      s_maxd = 0;
      s_far = 0;
    }
    __syncthreads();
    if (s_skip) continue;
    const int32_t* e = q.wedges;
    const uint32_t root = (uint32_t)(q.answer & 0xffffffffu);
    const long long cost = (long long)(q.answer >> 32);
    int* ent = q.wstack;      // entry 0: the root; 1 + 2i, 2 + 2i: the ends of edge i
    int* rep = ent + nent;    // first entry holding the same vertex
    int* dist = rep + nent;   // hop distances, by representative entry
    for (int a = threadIdx.x; a < nent; a += blockDim.x) ent[a] = a == 0 ? (int)root : e[3 * ((a - 1) >> 1) + ((a - 1) & 1)];
    __syncthreads();
    for (int i = threadIdx.x; i < ne; i += blockDim.x) {
      const int u = e[3 * i], v = e[3 * i + 1], w = e[3 * i + 2];
      atomicAdd((unsigned long long*)&s_sum, (unsigned long long)(long long)w);
      for (int i2 = 0; i2 < i; ++i2) {
        const int u2 = e[3 * i2], v2 = e[3 * i2 + 1];
        if ((u2 == u && v2 == v) || (u2 == v && v2 == u)) { tree_fail(q, TE_REPEAT); break; }
      }
      // scan the shorter of the two adjacency rows (both directions are stored)
      bool ok = u >= 0 && v >= 0 && u < g.V && v < g.V && u != v;
      if (ok) {
        const long long du = g.rowptr[u + 1] - g.rowptr[u], dv = g.rowptr[v + 1] - g.rowptr[v];
        const int a = du <= dv ? u : v, b = du <= dv ? v : u;
        bool hit = false;
        for (long long x = g.rowptr[a]; x < g.rowptr[a + 1] && !hit; ++x) {
          const int2 aw = g.adj[x];
          hit = aw.x == b && aw.y == w;
        }
        ok = hit;
      }
      if (!ok) tree_fail(q, TE_EDGE);
    }
    for (int a = threadIdx.x; a < nent; a += blockDim.x) {
      int r = a;
      for (int b = 0; b < a; ++b)
        if (ent[b] == ent[a]) { r = b; break; }
      rep[a] = r;
      if (r == a) atomicAdd(&s_nv, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_sum != cost) tree_fail(q, TE_WEIGHT);
    // n distinct edges on n + 1 vertices, all reachable from the root: a tree
    if (threadIdx.x == 0 && s_nv != ne + 1) tree_fail(q, TE_SHAPE);
    tree_bfs(rep, ne, nent, 0, dist, &s_changed);
    for (int a = threadIdx.x; a < nent; a += blockDim.x) {
      if (rep[a] != a) continue;
      if (dist[a] >= INF) tree_fail(q, TE_SHAPE);
      else atomicMax(&s_maxd, dist[a]);
    }
    __syncthreads();
    if (threadIdx.x == 0) s_ok = q.D >= 0 && q.terr == TE_NONE;
    __syncthreads();
    if (s_ok) {
      // the farthest vertex from any vertex ends a longest path of a tree
      int far = 0;
      if (threadIdx.x == 0) {
        for (int a = 0; a < nent; ++a)
          if (rep[a] == a && dist[a] == s_maxd) { far = a; break; }
        s_far = far;
        s_maxd = 0;
      }
      __syncthreads();
      far = s_far;
      tree_bfs(rep, ne, nent, far, dist, &s_changed);
      for (int a = threadIdx.x; a < nent; a += blockDim.x)
        if (rep[a] == a && dist[a] < INF) atomicMax(&s_maxd, dist[a]);
      __syncthreads();
      if (threadIdx.x == 0 && s_maxd > q.D) tree_fail(q, TE_DIAMETER);
    }
    // every queried group has a member among the tree's vertices
    for (int i = 0; i < q.k; ++i) {
      if (threadIdx.x == 0) s_found = 0;
      __syncthreads();
      const long long gb = g.gptr[q.groups[i]], ge = g.gptr[q.groups[i] + 1];
      for (long long m = gb + threadIdx.x; m < ge && !s_found; m += blockDim.x) {
        const int mv = g.gmem[m];
        for (int a = 0; a < nent; ++a)
          if (rep[a] == a && ent[a] == mv) { s_found = 1; break; }
      }
      __syncthreads();
      if (threadIdx.x == 0 && !s_found) tree_fail(q, TE_COVER);
    }
    __syncthreads();
  }
}

// Publishes every slot's status after a batch of rounds.  A slot whose full
// merge ran in the last round is finished here (the transition the next
// control pass would make).
__global__ void k_publish(Slot* slots, int nslots, SlotStatus* status) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nslots) return;
  Slot& q = slots[t];
  if (q.phase == PH_ACTIVE && q.action == A_MERGEFULL && q.err == ERR_NONE) {
    q.phase = PH_DONE;
    q.action = A_NONE;
  }
  status[t].phase = q.phase;
  status[t].err = q.err;
  status[t].answer = q.answer;
}

__global__ void k_free_slot(Slot* slots, int t) {
  slots[t].phase = PH_FREE;
  slots[t].action = A_NONE;
}

// Resets the rows and flags of a finished slot so its slab can be reused.
__global__ void k_reset(Slot* slots, int t, Graph g) {
  Slot& q = slots[t];
  const int rowlen = q.W * q.L, L = q.L;
  const int n = q.ntouched;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < (long long)n * rowlen;
       x += (long long)gridDim.x * blockDim.x) {
    const uint32_t v = q.touched[x / rowlen];
    q.table[(long long)v * rowlen + (x % rowlen)] = INF;
  }
  const int planes = q.D >= 0 ? L : 2;  // plain: near and far planes
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < (long long)n * planes;
       x += (long long)gridDim.x * blockDim.x) {
    const uint32_t v = q.touched[x / planes];
    q.mask[(x % planes) * g.V + v] = 0ull;
    if (x % planes == 0) {
      q.tflag[v] = 0u;
      q.dead[v >> 5] = 0u;  // only touched vertices are ever marked
      for (int i = 0; i < 8; ++i) q.sd[(long long)v * 8 + i] = INF;  // only touched vertices are ever written
    }
  }
}

}  // namespace gst
