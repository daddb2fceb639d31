// Oracle driver: runs one case through the reference's own solver function and
// writes the resulting fields, the mesh geometry the reference computed, and the
// reference's iteration timing counters.  Test infrastructure only.
//
//   babelsim-oracle <case-dir> <out-dir>
//
// The solver is the one named by case.bs; the physics loop is the reference's
// unmodified src/physics/<solver>/main.cpp.  Unlike the reference CLI, fields are
// written even when the outer loop stops at maxIterations, so a fixed number of
// SIMPLE iterations can be compared.
#include "babelsim/case.h"
#include "babelsim/application.h"
#include "internal/field_access.h"
#include "internal/mesh_access.h"

#include <mpi.h>

#include <chrono>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace babelsim {
SolverResult runSimple(Case&);
SolverResult runPiso(Case&);
SolverResult runTransientSimple(Case&);
}

namespace {
using namespace babelsim;

void writeArray(std::FILE* out, const char* name, const void* data, long long count, int width) {
    // Record: int64 name length, name, int64 element count, int64 element width, raw bytes.
    const long long len = static_cast<long long>(std::string(name).size());
    std::fwrite(&len, sizeof(len), 1, out);
    std::fwrite(name, 1, static_cast<std::size_t>(len), out);
    const long long meta[2] = {count, width};
    std::fwrite(meta, sizeof(meta), 1, out);
    if (count > 0) std::fwrite(data, static_cast<std::size_t>(width), static_cast<std::size_t>(count), out);
}

template <class Container>
void writeVector(std::FILE* out, const char* name, const Container& v) {
    writeArray(out, name, v.data(), static_cast<long long>(v.size()), static_cast<int>(sizeof(v[0])));
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <case-dir> <out-dir>\n", argv[0]);
        return 1;
    }
    MPI_Init(&argc, &argv);
    int status = 0;
    try {
        const std::filesystem::path out_dir = argv[2];
        std::filesystem::create_directories(out_dir);
        Case problem(argv[1]);
        const Mesh& mesh = problem.mesh();
        const auto& m = detail::meshData(mesh);
        {
            std::FILE* g = std::fopen((out_dir / "geometry.bin").c_str(), "wb");
            if (!g) throw std::runtime_error("cannot write geometry");
            writeVector(g, "face_owner", m.face_owner);
            writeVector(g, "face_neighbour", m.face_neighbour);
            writeVector(g, "face_patch", m.face_patch);
            writeVector(g, "face_centres", m.face_centres);
            writeVector(g, "face_area_vectors", m.face_area_vectors);
            writeVector(g, "face_areas", m.face_areas);
            writeVector(g, "face_normals", m.face_normals);
            writeVector(g, "face_owner_weights", m.face_owner_weights);
            writeVector(g, "face_orthogonal_coefficients", m.face_orthogonal_coefficients);
            writeVector(g, "face_non_orthogonal", m.face_non_orthogonal);
            writeVector(g, "face_skewness", m.face_skewness);
            writeVector(g, "cell_centres", m.cell_centres);
            writeVector(g, "cell_volumes", m.cell_volumes);
            const int orthogonal = m.orthogonal_geometry ? 1 : 0;
            writeArray(g, "orthogonal_geometry", &orthogonal, 1, sizeof(int));
            std::fclose(g);
        }
        const auto start = std::chrono::steady_clock::now();
        SolverResult result;
        if (problem.solver() == "simple") result = runSimple(problem);
        else if (problem.solver() == "piso") result = runPiso(problem);
        else if (problem.solver() == "transientSimple") result = runTransientSimple(problem);
        else throw std::invalid_argument("oracle driver does not run solver " + problem.solver());
        const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        status = static_cast<int>(result.status);
        std::FILE* f = std::fopen((out_dir / "fields.bin").c_str(), "wb");
        if (!f) throw std::runtime_error("cannot write fields");
        writeVector(f, "U", detail::fieldValues(problem.existingVectorField("U")));
        writeVector(f, "p", detail::fieldValues(problem.existingScalarField("p")));
        writeVector(f, "phi", detail::fieldValues(problem.existingFaceField("phi")));
        // turbulence fields, when the case has a model
        for (const char* name : {"k", "omega", "epsilon", "nuTilda", "mut", "muEffective"}) {
            try {
                writeVector(f, name, detail::fieldValues(problem.existingScalarField(name)));
            } catch (const std::exception&) {
            }
        }
        std::fclose(f);
        const PerformanceCounters perf = problem.localPerformance();
        std::ofstream json(out_dir / "run.json");
        json << "{\"status\": " << status << ", \"solver_seconds\": " << seconds
             << ", \"iteration_compute_seconds\": " << perf.iteration_compute_seconds
             << ", \"reported_iteration_intervals\": " << perf.reported_iteration_intervals
             << ", \"linear_solves\": " << perf.linear_solves << ", \"krylov_iterations\": " << perf.krylov_iterations
             << ", \"preconditioner_setups\": " << perf.preconditioner_setups
             << ", \"preconditioner_reuses\": " << perf.preconditioner_reuses
             << ", \"linear_solve_seconds\": " << perf.linear_solve_seconds
             << ", \"preconditioner_seconds\": " << perf.preconditioner_seconds
             << ", \"cells\": " << mesh.cellCount() << ", \"faces\": " << mesh.faceCount() << "}\n";
    } catch (const std::exception& error) {
        std::fprintf(stderr, "oracle driver: %s\n", error.what());
        MPI_Finalize();
        return 1;
    }
    MPI_Finalize();
    return status == 0 ? 0 : 2;
}
