// The reference-facing plugin for the linear-system seam: a BabelSim
// detail::ComputeBackend (src/internal/compute_backend.h:17-41) whose solves run
// on the B200 through the C ABI of libbabelsim_b200.so.
//
// Link it into a BabelSim program instead of the PETSc translation units
// (src/backend/petsc_*.cpp, petsc_session.cpp), the same link-time replacement
// the reference's tests/backend_interface_test.cpp:72-80 performs.  The mesh
// geometry the reference computed (Mesh::Storage) is handed to the device once;
// every solve passes the DiscreteEquation's LDU arrays and the unknown's host
// values, which are xyz-contiguous for Vec3 and so cross the ABI without copies.
//
// Environment: BABELSIM_B200_DEVICE selects the CUDA device (default 0).
#include "babelsim/field.h"
#include "babelsim/parallel.h"
#include "internal/compute_backend.h"
#include "internal/field_access.h"
#include "internal/mesh_access.h"

#include "babelsim_b200.h"

#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

namespace babelsim::detail {

// The PETSc session hooks the reference's runtime calls (src/internal/petsc_session.h).
void ensurePetscSession() {}
void finalizePetscSession() {}

namespace {

void check(int code, bsg_context* ctx, const char* what) {
    if (code == BSG_OK) return;
    const std::string msg = std::string(what) + ": " + (ctx ? bsg_last_error(ctx) : bsg_global_error());
    if (code == BSG_ERR_ARGUMENT) throw std::invalid_argument(msg);
    if (code == BSG_ERR_STATE) throw std::logic_error(msg);
    throw std::runtime_error(msg);
}

bsg_solver_config toConfig(const LinearSolverConfig& c) {
    bsg_solver_config r{};
    r.solver = static_cast<int32_t>(c.solver);
    r.preconditioner = static_cast<int32_t>(c.preconditioner);
    r.absolute_tolerance = c.absolute_tolerance;
    r.relative_tolerance = c.relative_tolerance;
    r.max_iterations = c.max_iterations;
    r.warm_start = c.warm_start ? 1 : 0;
    r.preconditioner_rebuild_interval = c.preconditioner_rebuild_interval;
    r.preconditioner_reuse_iteration_growth = c.preconditioner_reuse_iteration_growth;
    r.amg_max_levels = c.amg_max_levels;
    r.amg_coarse_size = c.amg_coarse_size;
    r.amg_smoothing_steps = c.amg_smoothing_steps;
    r.precision = BSG_PRECISION_FP64;
    return r;
}

SolveResult toResult(const bsg_solve_result& r) {
    return SolveResult(static_cast<SolveStatus>(r.status), r.iterations, r.initial_residual, r.final_residual,
                       r.relative_residual);
}

class B200Backend final : public ComputeBackend {
public:
    B200Backend(const Mesh& mesh, ParallelContext parallel) : m_mesh(&mesh) {
        if (parallel.size != 1)
            throw std::invalid_argument("the B200 backend solves one whole mesh per GPU (run one rank per case)");
        const char* dev = std::getenv("BABELSIM_B200_DEVICE");
        check(bsg_context_create(dev ? std::atoi(dev) : 0, &m_ctx), nullptr, "bsg_context_create");
        const auto& m = meshData(mesh);
        bsg_mesh_geometry g{};
        g.n_cells = mesh.cellCount();
        g.n_faces = mesh.faceCount();
        g.n_patches = static_cast<int32_t>(mesh.patchCount());
        g.face_owner = m.face_owner.data();
        g.face_neighbour = m.face_neighbour.data();
        g.face_patch = m.face_patch.data();
        g.face_area_vectors = &m.face_area_vectors.data()->x;
        g.face_centres = &m.face_centres.data()->x;
        g.face_areas = m.face_areas.data();
        g.face_normals = &m.face_normals.data()->x;
        g.face_owner_weights = m.face_owner_weights.data();
        g.face_orthogonal_coefficients = m.face_orthogonal_coefficients.data();
        g.face_non_orthogonal = &m.face_non_orthogonal.data()->x;
        g.face_skewness = &m.face_skewness.data()->x;
        g.cell_centres = &m.cell_centres.data()->x;
        g.cell_volumes = m.cell_volumes.data();
        g.orthogonal_geometry = m.orthogonal_geometry ? 1 : 0;
        check(bsg_mesh_create(m_ctx, &g, &m_device_mesh), m_ctx, "bsg_mesh_create");
    }
    ~B200Backend() override {
        bsg_mesh_destroy(m_device_mesh);
        bsg_context_destroy(m_ctx);
    }

    // One rank: fields are always complete (petsc_backend.cpp:288-310 without a halo).
    void synchronize(ScalarField& f) override { markHaloValid(f); }
    void synchronize(VectorField& f) override { markHaloValid(f); }
    void synchronize(TensorField& f) override { markHaloValid(f); }
    void sum(const double* local, double* global, int count) const override {
        std::memmove(global, local, sizeof(double) * static_cast<std::size_t>(count));
    }
    void maximum(const double* local, double* global, int count) const override {
        std::memmove(global, local, sizeof(double) * static_cast<std::size_t>(count));
    }
    bool all(bool local_condition) const override { return local_condition; }

    SolveResult solve(const ScalarDiscreteEquation& eq, ScalarField& x, const LinearSolverConfig& config) override {
        config.validate();
        const bsg_solver_config c = toConfig(config);
        bsg_solve_result r{};
        check(bsg_solve_ldu(m_device_mesh, &c, 1, eq.diagonal.data(), eq.upper.data(), eq.lower.data(),
                            eq.source.data(), fieldData(x), &r),
              m_ctx, "bsg_solve_ldu");
        markHaloValid(x);
        return toResult(r);
    }

    std::array<SolveResult, 3> solve(const VectorDiscreteEquation& eq, VectorField& x,
                                     const LinearSolverConfig& config) override {
        config.validate();
        const bsg_solver_config c = toConfig(config);
        bsg_solve_result r[3]{};
        check(bsg_solve_ldu(m_device_mesh, &c, 3, eq.diagonal.data(), eq.upper.data(), eq.lower.data(),
                            &eq.source.data()->x, &fieldData(x)->x, r),
              m_ctx, "bsg_solve_ldu");
        markHaloValid(x);
        return {toResult(r[0]), toResult(r[1]), toResult(r[2])};
    }

private:
    const Mesh* m_mesh;
    bsg_context* m_ctx = nullptr;
    bsg_mesh* m_device_mesh = nullptr;
};

}  // namespace

std::unique_ptr<ComputeBackend> makeComputeBackend(const Mesh& mesh, ParallelContext parallel) {
    return std::make_unique<B200Backend>(mesh, std::move(parallel));
}

}  // namespace babelsim::detail
