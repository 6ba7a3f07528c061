// Iteration order of a default-constructed std::unordered_set<std::size_t>
// (GNU libstdc++) after a sequence of insertions, without the container.
//
// The reference stores Vertex::cellIDs, Cell::edgeIDs and Cell::neighbourIDs
// in such sets (include/mesh.hpp), and their iteration order fixes the
// summation order of every gather, so a topology built without the
// containers must reproduce it.  The library keeps one singly linked list
// in which the elements of a bucket (key % bucket_count, the hash of an
// integer being the integer) are contiguous; a new key goes in front of the
// first element of its bucket, or at the front of the list when its bucket
// is empty, and a rehash re-inserts the elements in list order by the same
// rule with the new bucket count.  The bucket count after the k-th distinct
// insertion, read from the library in this image (bucket_count() after each
// insert): 13 for k <= 13, then 29, 59, 127, 257 from k = 14, 30, 60, 128.
// tests/uset_order_check.cpp compares this emulation with the container
// itself on random and ascending insertion sequences.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define O2F_USET_FN __host__ __device__ __forceinline__
#else
#define O2F_USET_FN inline
#endif

namespace o2f {

constexpr int kUsetMax = 257;  // largest set the emulation handles

O2F_USET_FN uint64_t uset_buckets(int k) {
  return k <= 13 ? 13 : k <= 29 ? 29 : k <= 59 ? 59 : k <= 127 ? 127 : 257;
}

// list[0..n) in iteration order; insert x (ignored if present).  Returns
// false if the set would exceed kUsetMax elements.
O2F_USET_FN bool uset_insert(uint64_t* list, int& n, uint64_t x) {
  for (int i = 0; i < n; ++i)
    if (list[i] == x) return true;
  if (n >= kUsetMax) return false;
  const uint64_t nb = uset_buckets(n + 1);
  if (n == 0 || uset_buckets(n) != nb) {
    // rehash: re-insert the current order with the new bucket count
    for (int m = 0; m < n; ++m) {
      const uint64_t y = list[m], b = y % nb;
      int pos = 0;
      while (pos < m && list[pos] % nb != b) ++pos;
      if (pos == m) pos = 0;  // bucket empty so far: front of the list
      for (int j = m; j > pos; --j) list[j] = list[j - 1];
      list[pos] = y;
    }
  }
  const uint64_t b = x % nb;
  int pos = 0;
  while (pos < n && list[pos] % nb != b) ++pos;
  if (pos == n) pos = 0;
  for (int j = n; j > pos; --j) list[j] = list[j - 1];
  list[pos] = x;
  ++n;
  return true;
}

}  // namespace o2f
