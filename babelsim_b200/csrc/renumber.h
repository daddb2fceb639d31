// Locality renumbering of mesh cells (renumber.cpp).
#pragma once

#include <vector>

namespace bsg {

// order[i] = the caller's cell that becomes internal cell i: reverse Cuthill-McKee per
// connected component when that shortens the mean |i - j| over interior faces more than
// twofold, else the identity (*applied tells which).
std::vector<int> localityOrder(int n_cells, int n_faces, const int* owner, const int* neighbour, bool* applied);

}  // namespace bsg
