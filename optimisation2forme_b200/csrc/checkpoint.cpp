// Binary structure-of-arrays state checkpoint, alongside the reference's text
// state file (saveCellStates / loadCellStates, src/utils.cpp:29-107: a cell
// count, then one "rho rho_u rho_v E" line per cell with 17 significant
// digits).  The binary file holds the same values in the same cell order,
// exactly, in 32 bytes per cell instead of ~100 characters, and is read and
// written without formatting or parsing:
//
//   offset  size  field
//        0     8  magic "O2FSOA1\0"
//        8     4  format version (1), uint32 little-endian
//       12     4  number of fields (4: rho, rho_u, rho_v, E), uint32
//       16     8  number of cells, uint64
//       24     8  simulation time, float64
//       32     8  time steps done, uint64
//       40     8  FNV-1a 64-bit hash of the payload bytes, uint64
//       48    16  reserved, zero
//       64        payload: field-major float64 arrays [4][n_cells]
//
// The checkpoint carries the state only; the mesh it belongs to is the one
// the caller supplies (as for the reference's text file).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "checkpoint.hpp"
#include "o2f.h"
#include "solver.hpp"

namespace o2f {
namespace {

constexpr char kMagic[8] = {'O', '2', 'F', 'S', 'O', 'A', '1', '\0'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kFields = 4;
constexpr size_t kHeader = 64;

uint64_t fnv1a(const unsigned char* p, size_t n, uint64_t h = 0xcbf29ce484222325ull) {
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 0x100000001b3ull;
  }
  return h;
}

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

void put_u32(unsigned char* p, uint32_t v) {
  for (int i = 0; i < 4; ++i) p[i] = (unsigned char)(v >> (8 * i));
}
void put_u64(unsigned char* p, uint64_t v) {
  for (int i = 0; i < 8; ++i) p[i] = (unsigned char)(v >> (8 * i));
}
uint32_t get_u32(const unsigned char* p) {
  uint32_t v = 0;
  for (int i = 0; i < 4; ++i) v |= (uint32_t)p[i] << (8 * i);
  return v;
}
uint64_t get_u64(const unsigned char* p) {
  uint64_t v = 0;
  for (int i = 0; i < 8; ++i) v |= (uint64_t)p[i] << (8 * i);
  return v;
}
void put_f64(unsigned char* p, double d) {
  uint64_t v;
  std::memcpy(&v, &d, 8);
  put_u64(p, v);
}
double get_f64(const unsigned char* p) {
  const uint64_t v = get_u64(p);
  double d;
  std::memcpy(&d, &v, 8);
  return d;
}

}  // namespace

void checkpoint_write(const std::string& path, int64_t n_cells, const double* U, double time, int64_t steps) {
  if (n_cells <= 0 || !U) throw Error(O2F_ERR_ARG, "checkpoint: empty state");
  const size_t n = (size_t)n_cells;
  std::vector<unsigned char> payload(32 * n);
  for (size_t k = 0; k < kFields; ++k)
    for (size_t c = 0; c < n; ++c) put_f64(&payload[8 * (k * n + c)], U[4 * c + k]);
  unsigned char head[kHeader] = {};
  std::memcpy(head, kMagic, 8);
  put_u32(head + 8, kVersion);
  put_u32(head + 12, kFields);
  put_u64(head + 16, (uint64_t)n);
  put_f64(head + 24, time);
  put_u64(head + 32, (uint64_t)(steps < 0 ? 0 : steps));
  put_u64(head + 40, fnv1a(payload.data(), payload.size()));
  File f;
  f.f = std::fopen(path.c_str(), "wb");
  if (!f.f) throw Error(O2F_ERR_IO, "cannot open " + path + " for writing");
  if (std::fwrite(head, 1, kHeader, f.f) != kHeader ||
      std::fwrite(payload.data(), 1, payload.size(), f.f) != payload.size() || std::fflush(f.f) != 0)
    throw Error(O2F_ERR_IO, "write error in " + path);
}

void checkpoint_read(const std::string& path, int64_t n_cells, double* U, double* time, int64_t* steps) {
  if (n_cells <= 0 || !U) throw Error(O2F_ERR_ARG, "checkpoint: empty state");
  File f;
  f.f = std::fopen(path.c_str(), "rb");
  if (!f.f) throw Error(O2F_ERR_IO, "cannot open " + path + " for reading");
  unsigned char head[kHeader];
  if (std::fread(head, 1, kHeader, f.f) != kHeader) throw Error(O2F_ERR_IO, path + ": truncated header");
  if (std::memcmp(head, kMagic, 8) != 0) throw Error(O2F_ERR_IO, path + ": not an o2f state checkpoint");
  if (get_u32(head + 8) != kVersion) throw Error(O2F_ERR_IO, path + ": unsupported checkpoint version");
  if (get_u32(head + 12) != kFields) throw Error(O2F_ERR_IO, path + ": unexpected number of fields");
  const uint64_t n = get_u64(head + 16);
  if (n != (uint64_t)n_cells)
    throw Error(O2F_ERR_IO, path + ": " + std::to_string(n) + " cells in the file, " + std::to_string(n_cells) +
                                " in the mesh (check the cell order / topology)");
  std::vector<unsigned char> payload(32 * (size_t)n);
  if (std::fread(payload.data(), 1, payload.size(), f.f) != payload.size())
    throw Error(O2F_ERR_IO, path + ": truncated payload");
  unsigned char extra;
  if (std::fread(&extra, 1, 1, f.f) != 0) throw Error(O2F_ERR_IO, path + ": trailing bytes after the payload");
  if (fnv1a(payload.data(), payload.size()) != get_u64(head + 40)) throw Error(O2F_ERR_IO, path + ": checksum mismatch");
  for (size_t k = 0; k < kFields; ++k)
    for (size_t c = 0; c < (size_t)n; ++c) U[4 * c + k] = get_f64(&payload[8 * (k * (size_t)n + c)]);
  if (time) *time = get_f64(head + 24);
  if (steps) *steps = (int64_t)get_u64(head + 32);
}

}  // namespace o2f
