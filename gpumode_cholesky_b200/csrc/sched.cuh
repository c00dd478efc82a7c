// Matrix/tile addressing shared by the blocked-path kernels: a dense batch
// or a ragged schedule (see potrf_ragged.cu).
#pragma once

#include <stdint.h>

namespace b2p {

// Which matrix (and tile) a CTA works on: a dense batch (matrix b at b*n*n,
// tiles from blockIdx.x, matrices from blockIdx.y) or a ragged schedule
// (an item list of (list position, tile) pairs; positions map to matrix
// indices through `order`, each with its own offset and order n).
struct Sched {
  const int2* items;       // ragged panel/trail: (position, ti | tj << 16)
  const int32_t* order;    // ragged: position -> matrix index
  const int64_t* offsets;  // ragged: element offset of each matrix
  const int32_t* ns;       // ragged: order of each matrix
  int64_t count;           // dense: batch; ragged: items (panel/trail) or positions (diag)
  int n;                   // dense order
};

struct Target {
  int64_t pos;  // workspace slot (dense: b)
  int64_t mat;  // matrix index (info)
  size_t off;   // element offset of the matrix
  int n;
  int ti, tj;
};

template <bool RAGGED>
__device__ __forceinline__ Target resolve_matrix(const Sched& sc, int64_t it) {
  Target t;
  if (!RAGGED) {
    t.pos = it;
    t.mat = it;
    t.off = (size_t)it * sc.n * sc.n;
    t.n = sc.n;
  } else {
    t.pos = it;
    t.mat = sc.order[it];
    t.off = (size_t)sc.offsets[t.mat];
    t.n = sc.ns[t.mat];
  }
  t.ti = t.tj = 0;
  return t;
}

template <bool RAGGED>
__device__ __forceinline__ Target resolve_tile(const Sched& sc, int64_t it) {
  if (!RAGGED) {
    Target t = resolve_matrix<false>(sc, it);
    t.ti = blockIdx.x;
    return t;
  }
  const int2 w = sc.items[it];
  Target t = resolve_matrix<true>(sc, w.x);
  t.ti = w.y & 0xffff;
  t.tj = w.y >> 16;
  return t;
}

// Device tables of a ragged schedule (layout owned by potrf_ragged.cu).
struct RaggedTables {
  const int32_t* order;    // big-matrix list (n > 128), sorted by n descending
  const int64_t* offsets;  // per matrix
  const int32_t* ns;       // per matrix
  const int2* items;       // all panel/trail item lists, concatenated
};

// Launch parameters of one block-column step.
struct RaggedStep {
  int64_t ndiag;                // active big matrices (a prefix of the order)
  int64_t panel_beg, npanel;    // slice of items
  int64_t trail_beg, ntrail;    // slice of items
};

inline Sched dense_sched(int64_t batch, int n) {
  Sched s;
  s.items = nullptr;
  s.order = nullptr;
  s.offsets = nullptr;
  s.ns = nullptr;
  s.count = batch;
  s.n = n;
  return s;
}

inline Sched ragged_sched(const RaggedTables& t, const int2* items, int64_t count) {
  Sched s;
  s.items = items;
  s.order = t.order;
  s.offsets = t.offsets;
  s.ns = t.ns;
  s.count = count;
  s.n = 0;
  return s;
}

}  // namespace b2p
