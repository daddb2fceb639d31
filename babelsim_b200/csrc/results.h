// Result output in the reference's rank-sharded format (results.cpp).
#pragma once

#include <string>
#include <vector>

namespace bsg {

struct ResultField {
    std::string name;
    int components = 1;       // 1 scalar, 3 vector, 9 tensor
    const double* values = nullptr;
};

void writeResults(const std::string& time_directory, const std::string& time_name, int n_vertices,
                  const double* vertices, int n_faces, const int* face_point_offsets, const int* face_point_ids,
                  const int* owner, const int* neighbour, const int* patch, int n_patches,
                  const std::vector<ResultField>& fields);

}  // namespace bsg
