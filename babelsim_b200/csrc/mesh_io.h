// Host-side BABELSIM_MESH 3 reader (src/io/mesh_reader.cpp:44-111) producing the flat
// polyhedral description that bsg_mesh_create_polyhedral takes.
#pragma once

#include "bsg_internal.h"

#include <string>
#include <vector>

namespace bsg {

struct PolyFile {
    int n_cells = 0;
    std::vector<double> vertices;        // 3 per vertex
    std::vector<int> offsets, ids;       // face rings: ids[offsets[f] .. offsets[f+1])
    std::vector<int> owner, neighbour, patch;
    std::vector<std::string> patch_names;
    std::vector<int> patch_kinds;        // PatchKind order: generic wall inlet outlet symmetry processor
};

// Reads and checks the file; throws Error(kArgument) with the reference's message on a bad file.
PolyFile readPolyFile(const std::string& path);

}  // namespace bsg
