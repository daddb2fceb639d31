// Result output in the reference's format (src/parallel/parallel_writer.cpp:42-171,
// src/io/case.cpp:228-270), so the reference's restart reader
// (src/io/field_reader.cpp:160-226) and tools read fields computed here:
//   <time_directory>/rank-0000/<field>.csv   global_id,x,y,z,value0[,value1,...] (17 digits)
//   <time_directory>/rank-0000/metadata.bs   format babelsim_result 3, time, rank, ranks, counts, fields
//   <time_directory>/rank-0000/mesh.geometry global_id,vertex_count,x,y,z,... (sorted unique cell vertices)
// One rank: every cell is owned, global ids are the cell indices.
#include "bsg_internal.h"
#include "results.h"

#include <filesystem>
#include <fstream>
#include <iomanip>
#include <set>
#include <string>
#include <vector>

namespace bsg {

void writeResults(const std::string& time_directory, const std::string& time_name, int n_vertices,
                  const double* vertices, int n_faces, const int* face_point_offsets, const int* face_point_ids,
                  const int* owner, const int* neighbour, const int* patch, int n_patches,
                  const std::vector<ResultField>& fields) {
    if (time_name.empty() || fields.empty()) fail(kArgument, "result output needs a time name and fields");
    for (const ResultField& f : fields) {
        if (f.name.empty() || !f.values) fail(kArgument, "result field is incomplete");
        if (f.components != 1 && f.components != 3 && f.components != 9)
            fail(kArgument, "result field components must be 1, 3 or 9");
    }
    const HostGeometry g = computePolyhedralGeometry(n_vertices, vertices, n_faces, face_point_offsets,
                                                     face_point_ids, owner, neighbour, patch, n_patches);
    const int N = g.n_cells;
    namespace fs = std::filesystem;
    const fs::path rank_dir = fs::path(time_directory) / "rank-0000";
    std::error_code ec;
    fs::create_directories(rank_dir, ec);
    if (ec) fail(kState, "cannot create result directory " + rank_dir.string() + ": " + ec.message());
    for (const ResultField& f : fields) {
        const fs::path path = rank_dir / (f.name + ".csv");
        std::ofstream out(path);
        if (!out) fail(kState, "cannot create field output " + path.string());
        out << "global_id,x,y,z";
        for (int c = 0; c < f.components; ++c) out << ",value" << c;
        out << '\n' << std::setprecision(17);
        for (int i = 0; i < N; ++i) {
            out << i << ',' << g.xc[3 * i] << ',' << g.xc[3 * i + 1] << ',' << g.xc[3 * i + 2];
            for (int c = 0; c < f.components; ++c) out << ',' << f.values[static_cast<std::size_t>(f.components) * i + c];
            out << '\n';
        }
        if (!out) fail(kState, "cannot write field output " + path.string());
    }
    // mesh provenance: the sorted unique vertices of each cell's faces (src/core/mesh.cpp:473-484)
    {
        std::vector<std::set<int>> cell_vertices(N);
        for (int f = 0; f < n_faces; ++f)
            for (int k = face_point_offsets[f]; k < face_point_offsets[f + 1]; ++k) {
                cell_vertices[owner[f]].insert(face_point_ids[k]);
                if (neighbour[f] >= 0) cell_vertices[neighbour[f]].insert(face_point_ids[k]);
            }
        std::ofstream geo(rank_dir / "mesh.geometry");
        if (!geo) fail(kState, "cannot create result mesh provenance");
        geo << std::setprecision(17);
        for (int i = 0; i < N; ++i) {
            geo << i << ',' << cell_vertices[i].size();
            for (int v : cell_vertices[i])
                geo << ',' << vertices[3 * v] << ',' << vertices[3 * v + 1] << ',' << vertices[3 * v + 2];
            geo << '\n';
        }
        if (!geo) fail(kState, "cannot write result mesh provenance");
    }
    std::ofstream meta(rank_dir / "metadata.bs");
    if (!meta) fail(kState, "cannot create result metadata");
    meta << "format babelsim_result 3\n"
         << "time " << time_name << '\n'
         << "rank 0\n"
         << "ranks 1\n"
         << "global_cell_count " << N << '\n'
         << "owned_cells " << N << '\n';
    for (const ResultField& f : fields)
        meta << "field " << f.name << ' ' << (f.components == 1 ? "scalar" : f.components == 3 ? "vector" : "tensor")
             << " cell\n";
    if (!meta) fail(kState, "cannot write result metadata");
}

}  // namespace bsg
