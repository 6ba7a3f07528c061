// CPU check of o2f::uset_insert (optimisation2forme_b200/csrc/uset_order.h):
// the emulated iteration order must equal that of std::unordered_set<std::size_t>
// after the same insertions -- random keys in narrow and wide ranges (many
// bucket collisions, duplicates), ascending sequences with random gaps (how
// the mesh build inserts cells and edges), every length up to the largest
// the emulation handles.
//
// Usage: uset_order_check [n_sequences] [seed]; exits 1 on a mismatch.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <unordered_set>
#include <vector>

#include "uset_order.h"

namespace {
uint64_t g_state = 0x2545f4914f6cdd1dull;
uint64_t next_u64() {
  uint64_t z = (g_state += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
}  // namespace

int main(int argc, char** argv) {
  const long n_seq = argc > 1 ? std::atol(argv[1]) : 200000;
  if (argc > 2) g_state = std::strtoull(argv[2], nullptr, 10);
  long bad = 0, checked = 0;
  std::vector<uint64_t> keys;
  uint64_t list[o2f::kUsetMax];
  for (long s = 0; s < n_seq; ++s) {
    const int kind = (int)(s % 4);
    // short sets dominate in meshes; every length up to the limit appears
    const int len = (s % 97 == 0) ? 1 + (int)(next_u64() % o2f::kUsetMax) : 1 + (int)(next_u64() % 16);
    keys.clear();
    uint64_t cur = next_u64() % 5000000;
    for (int i = 0; i < len; ++i) {
      uint64_t k;
      if (kind == 0) k = next_u64() % 50;                 // collisions and duplicates
      else if (kind == 1) k = next_u64() % 1000000000ull; // wide
      else if (kind == 2) k = (cur += 1 + next_u64() % 40); // ascending, small gaps
      else k = (cur += 1 + next_u64() % 3000000);          // ascending, large gaps
      keys.push_back(k);
    }
    std::unordered_set<std::size_t> ref;
    int n = 0;
    for (uint64_t k : keys) {
      ref.insert((std::size_t)k);
      if (!o2f::uset_insert(list, n, k)) {
        std::printf("emulation overflow at %d elements\n", n);
        return 1;
      }
    }
    ++checked;
    int i = 0;
    bool ok = (int)ref.size() == n;
    for (auto it = ref.begin(); ok && it != ref.end(); ++it, ++i) ok = (uint64_t)*it == list[i];
    if (!ok && bad++ < 5) {
      std::printf("MISMATCH kind %d length %d:", kind, len);
      for (uint64_t k : keys) std::printf(" %llu", (unsigned long long)k);
      std::printf("\n");
    }
  }
  std::printf("uset_order_check: %ld sequences, %ld mismatches\n", checked, bad);
  return bad == 0 ? 0 : 1;
}
