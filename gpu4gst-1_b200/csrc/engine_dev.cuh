// Device-side data layout and helpers of the GST engine.
//
// One query occupies a "slot".  Its DP table lives in a slab of the device
// arena:
//
//   table[v][idx(S)][l]   int32, row = W*L ints per vertex, W = 2^k, L = 1
//                          (plain) or D+1 (diameter bound D).  idx orders the
//                          2^k subsets by (popcount, value), so the sets of one
//                          layer |S| = s are contiguous in a row; l is the
//                          depth label of the D- variants, innermost so that
//                          the labels of one (v, S) share a sector.
//   mask[l][v]            uint64 dirty bits over the ranks of the current
//                          layer's sets: (v, S, l) improved and must be grown.
//                          Plain problem: plane 0 holds "near" bits (cost below
//                          the bucket bound T), plane 1 "far" bits.
//   queue[qi][v]          frontier vertex lists (plain: near lists 0/1 and far
//                          lists 2/3, ping-pong; D-: one list per depth label).
//   touched[], tflag[v]   vertices that ever held a finite entry.
//   dead[V / 32]          vertices the liveness test dropped (bitmap).
//   sd[v][8]              v's singleton minima over labels, one sector per
//                          vertex, filled by the first merge.
//   live[2][V]            merge lists: the vertices a layer's merge visits;
//                          each merge writes, for the next layer, the vertices
//                          whose whole-tree lower bound is still <= best
//                          (the witness stack's memory, idle until the end).
//   chunks[]              the current round's grow work: (v, edge range, mask).
//
// INF = 0x3f3f3f3f so that a byte memset initialises a table and the sum of
// two INF entries does not overflow int32.
#pragma once
#include <cstdint>

#include "gst_b200.h"

namespace gst {

constexpr int INF = 0x3f3f3f3f;
constexpr int MAXK = GST_MAX_K;
constexpr int MAXW = 1 << MAXK;
constexpr int MAXL = GST_MAX_D + 1;
constexpr int MAXSLOTS = 1024;
constexpr int MAXQ = MAXL + 1;  // queue lists per slot

enum Phase : int32_t { PH_FREE = 0, PH_ACTIVE = 1, PH_DONE = 2, PH_ERROR = 3 };
enum Action : int32_t {
  A_NONE = 0,
  A_INIT = 1,      // seeds written by the admission kernels
  A_GROW = 2,      // prep + relax one frontier
  A_LBPREP = 3,    // lower-bound tables after the singleton layer
  A_MERGE = 4,     // subset join of the next layer
  A_MERGEFULL = 5  // join of the full set: the answer
};
enum Err : int32_t {
  ERR_NONE = 0,
  ERR_CHUNK_CAP = 1,
  ERR_QUEUE_CAP = 2,
  ERR_WITNESS = 3,
  ERR_WITNESS_CAP = 4,
  ERR_ROUNDS = 5,
  ERR_TREE = 6  // the device check of the returned tree failed (reason in Slot::terr)
};
// Reasons of ERR_TREE (Slot::terr).
enum TreeErr : int32_t {
  TE_NONE = 0,
  TE_EDGE = 1,      // an edge is not in the graph or has another weight
  TE_REPEAT = 2,    // the derivation lists an edge twice
  TE_SHAPE = 3,     // the edges do not form one tree (cycle or disconnected)
  TE_COVER = 4,     // a queried group has no vertex in the tree
  TE_WEIGHT = 5,    // the edge weights do not sum to the cost
  TE_DIAMETER = 6,  // hop diameter above D
  TE_SCRATCH = 7    // the tree does not fit the check's scratch
};

struct Chunk {
  uint32_t v;
  uint32_t eb;  // first edge (absolute CSR index)
  uint32_t ee;  // one past the last edge
  uint32_t pad;
  unsigned long long mask;  // dirty set ranks snapshotted by the prep pass
};

struct Slot {
  // ---- set at admission --------------------------------------------------
  int32_t* table;
  unsigned long long* mask;
  uint32_t* queue;
  uint32_t* touched;
  uint32_t* tflag;
  Chunk* chunks;
  int32_t* lbtab;   // P[k][k][W] then W2[k][W]
  int32_t* wstack;  // witness search stack, 4 ints per entry
  int32_t* wedges;  // witness output, 3 ints per edge
  long long chunk_cap;
  long long wcap;
  int32_t k, W, L, D;  // D < 0: plain
  int32_t groups[MAXK];
  int32_t max_rounds;
  // ---- dynamic -------------------------------------------------------------
  int32_t phase, action;
  int32_t s;    // current layer |S|
  int32_t d;    // current depth label (D- variants)
  int32_t cur;  // current ping-pong list (plain)
  int32_t best; // upper bound: cost of a known feasible solution
  int32_t R1;   // singleton distances above R1 are only known to exceed R1
  int32_t err;
  int32_t terr;  // TreeErr of ERR_TREE
  int32_t ntouched, nchunks, nwedges;
  int32_t rounds;
  // cost-ordered grows (plain problem): states below the bucket bound T are
  // expanded from the near lists; costlier ones wait in the far list fcur
  // (next_min = their smallest cost) until the near lists run dry; farround
  // marks a round that drains the previous far list
  int32_t delta, bshift, T, next_min, fcur, farround;
  int32_t chunk_pairs;  // (edge, set) pairs per grow chunk
  int32_t qcount[MAXQ];
  // merge lists: layer s visits live[lr][0, nlr) and touched[mt0, mt1) (the
  // vertices first touched since the previous list was cut) and appends the
  // vertices that stay alive to live[lr ^ 1] (nlw entries)
  uint32_t* live[2];
  int32_t lr, nlr, nlw, mt0, mt1;
  // dead[v >> 5] bit v & 31: the merge's liveness test dropped v (plain
  // queries); grows and preps skip such vertices while use_dead is set
  uint32_t* dead;
  int32_t use_dead;
  // sd[v * 8 + i]: min over depth labels of v's singleton entry of group i
  // (INF: none), written by the query's first merge, when layer 1 is final;
  // later merges and the grow's lower bound read it instead of the row
  int32_t* sd;
  int32_t sd_ready;
  unsigned long long answer;  // (cost << 32) | root
  unsigned long long st_frontier, st_relax, st_improve, st_merges;
  unsigned long long st_mitems, st_mpassed;  // merge items visited / past the pre-filter
};

struct SlotStatus {
  int32_t phase;
  int32_t err;
  unsigned long long answer;
};

struct Plan {
  int32_t n_lb, n_merge, n_grow, n_active;
  int32_t n_wide_merge;  // merging slots with more than 6 labels (k_merge_wide)
  int32_t lb_slots[MAXSLOTS];
  int32_t merge_slots[MAXSLOTS];
  int32_t grow_slots[MAXSLOTS];
  long long merge_off[MAXSLOTS + 1];
  long long prep_off[MAXSLOTS + 1];
  long long chunk_off[MAXSLOTS + 1];
};

// Subset orderings for k = 1..MAXK (popcount, then value).
struct SubsetTables {
  uint8_t sidx[MAXK + 1][MAXW];     // S -> index
  uint8_t sof[MAXK + 1][MAXW];      // index -> S
  uint8_t loff[MAXK + 1][MAXK + 2]; // first index of layer s
};

// Fills the subset orderings: for each k, the 2^k subsets ordered by
// popcount and then by value; loff[k][s] is the index of the first set of
// popcount s (loff[k][k + 1] = 2^k).  Host code; the engine and the
// allocation-free entry point upload the same tables.
inline void fill_subset_tables(SubsetTables& t) {
  for (int k = 0; k <= MAXK; ++k)
    for (int i = 0; i < MAXW; ++i) t.sidx[k][i] = t.sof[k][i] = 0;
  for (int k = 0; k <= MAXK; ++k)
    for (int s = 0; s < MAXK + 2; ++s) t.loff[k][s] = 0;
  for (int k = 1; k <= MAXK; ++k) {
    const int W = 1 << k;
    int pos = 0;
    for (int s = 0; s <= k; ++s) {
      t.loff[k][s] = (uint8_t)pos;
      for (int S = 0; S < W; ++S)
        if (__builtin_popcount(S) == s) {
          t.sof[k][pos] = (uint8_t)S;
          t.sidx[k][S] = (uint8_t)pos;
          ++pos;
        }
    }
    t.loff[k][k + 1] = (uint8_t)W;
  }
}

struct Graph {
  const long long* rowptr;  // V+1
  const int2* adj;          // E x (neighbour, weight)
  const long long* gptr;    // groups: n+1
  const int32_t* gmem;
  long long V, E, G;
};

}  // namespace gst
