// Binary structure-of-arrays state checkpoint (format in checkpoint.cpp).
#pragma once

#include <cstdint>
#include <string>

namespace o2f {

// U: 4 values per cell (rho, rho_u, rho_v, E), cell order of the mesh file.
void checkpoint_write(const std::string& path, int64_t n_cells, const double* U, double time, int64_t steps);
// Throws Error(O2F_ERR_IO) for a missing, foreign, truncated, corrupted or
// mismatched (cell count) file; time and steps may be null.
void checkpoint_read(const std::string& path, int64_t n_cells, double* U, double* time, int64_t* steps);

}  // namespace o2f
