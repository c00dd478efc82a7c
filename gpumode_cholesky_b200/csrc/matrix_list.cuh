// Addressing of the matrices one launch processes: a dense batch
// (matrix b at element b*n*n) or a ragged list (per-matrix offset and order,
// visited through an optional index permutation that groups size buckets).
#pragma once

#include <stdint.h>

namespace b2p {

struct MatrixList {
  const int64_t* offsets;  // ragged: element offset of each matrix (device)
  const int32_t* ns;       // ragged: order of each matrix (device)
  const int32_t* order;    // ragged: item -> matrix index (device), may be null
  int64_t count;           // number of items this launch visits
  int n;                   // dense: order of every matrix

  __device__ __forceinline__ void get(int64_t item, int64_t& mat, int64_t& off, int& nn) const {
    if (ns == nullptr) {
      mat = item;
      off = item * (int64_t)n * n;
      nn = n;
    } else {
      mat = order ? (int64_t)order[item] : item;
      off = offsets[mat];
      nn = ns[mat];
    }
  }
};

inline MatrixList dense_list(int64_t batch, int n) {
  MatrixList m;
  m.offsets = nullptr;
  m.ns = nullptr;
  m.order = nullptr;
  m.count = batch;
  m.n = n;
  return m;
}

}  // namespace b2p
