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
// Like PetscBackend (src/backend/petsc_backend.cpp:201-213) it keeps one
// persistent device system per equation identity, so device buffers and AMG
// hierarchies live across solves and the preconditioner lag applies, and it
// reports the same PerformanceCounters (petsc_backend.cpp:110-121, 228-286).
//
// Environment: BABELSIM_B200_DEVICE selects the CUDA device (default 0).
#include "babelsim/field.h"
#include "babelsim/parallel.h"
#include "internal/compute_backend.h"
#include "internal/field_access.h"
#include "internal/mesh_access.h"

#include "babelsim_b200.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
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
    // The reference's default coarsest size (48) is Hypre's CPU setting.  The device AMG
    // inverts its coarsest level on an 8-CTA cluster in distributed shared memory, up to
    // 440 rows, and every level it stops earlier adds three latency-bound grid-wide
    // phases to each V-cycle, so the default maps to the device default (400); an
    // explicitly configured size is passed through unchanged.
    r.amg_coarse_size = c.amg_coarse_size == LinearSolverConfig{}.amg_coarse_size ? 400 : c.amg_coarse_size;
    r.amg_smoothing_steps = c.amg_smoothing_steps;
    r.precision = BSG_PRECISION_FP64;
    return r;
}

SolveResult toResult(const bsg_solve_result& r) {
    return SolveResult(static_cast<SolveStatus>(r.status), r.iterations, r.initial_residual, r.final_residual,
                       r.relative_residual);
}

// The names PetscBackend records (petsc_backend.cpp:30-60).
const char* kspText(LinearSolverType t) {
    switch (t) {
    case LinearSolverType::ConjugateGradient: return "cg";
    case LinearSolverType::BiCGSTAB: return "bcgs";
    case LinearSolverType::GMRES: return "gmres";
    case LinearSolverType::FGMRES: return "fgmres";
    }
    return "unknown";
}
const char* pcText(PreconditionerType t) {
    switch (t) {
    case PreconditionerType::None: return "none";
    case PreconditionerType::IncompleteCholesky: return "icc";
    case PreconditionerType::Hypre: return "hypre-boomeramg";
    case PreconditionerType::GAMG: return "gamg";
    case PreconditionerType::BlockJacobi: return "bjacobi";
    case PreconditionerType::ASM: return "asm";
    case PreconditionerType::Jacobi: return "jacobi";
    }
    return "unknown";
}
const char* statusText(int32_t s) {
    return s == BSG_CONVERGED ? "converged" : s == BSG_MAX_ITERATIONS ? "maxIterations" : "numericalFailure";
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
        for (auto& entry : m_systems) bsg_system_destroy(entry.second.system);
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
        Entry& e = system(identity(eq.numerical_identity, x.name(), false), 1, config);
        bsg_solve_result r{};
        check(bsg_system_solve(e.system, &c, eq.diagonal.data(), eq.upper.data(), eq.lower.data(), eq.source.data(),
                               fieldData(x), &r),
              m_ctx, "bsg_system_solve");
        markHaloValid(x);
        return toResult(r);
    }

    std::array<SolveResult, 3> solve(const VectorDiscreteEquation& eq, VectorField& x,
                                     const LinearSolverConfig& config) override {
        config.validate();
        const bsg_solver_config c = toConfig(config);
        Entry& e = system(identity(eq.numerical_identity, x.name(), true), 3, config);
        bsg_solve_result r[3]{};
        check(bsg_system_solve(e.system, &c, eq.diagonal.data(), eq.upper.data(), eq.lower.data(),
                               &eq.source.data()->x, &fieldData(x)->x, r),
              m_ctx, "bsg_system_solve");
        markHaloValid(x);
        return {toResult(r[0]), toResult(r[1]), toResult(r[2])};
    }

    PerformanceCounters performance() const override {
        PerformanceCounters p;
        for (const auto& entry : m_systems) {
            bsg_system_counters k{};
            check(bsg_system_counters_read(entry.second.system, &k), m_ctx, "bsg_system_counters_read");
            EquationPerformanceCounters e;
            e.identity = entry.first;
            e.ksp_type = kspText(entry.second.solver);
            e.pc_type = pcText(entry.second.preconditioner);
            e.last_status = k.linear_solves ? statusText(k.last_status) : "";
            e.matrix_pattern_builds = 1;
            e.matrix_value_updates = k.matrix_value_updates;
            e.rhs_only_solves = k.rhs_only_solves;
            e.linear_solves = k.linear_solves;
            e.krylov_iterations = k.krylov_iterations;
            e.preconditioner_setups = k.preconditioner_setups;
            e.preconditioner_reuses = k.preconditioner_reuses;
            e.preconditioner_retries = k.preconditioner_retries;
            e.true_residual_checks = k.true_residual_checks;
            e.last_initial_residual = k.last_initial_residual;
            e.last_final_residual = k.last_final_residual;
            e.last_relative_residual = k.last_relative_residual;
            e.matrix_update_seconds = k.matrix_update_seconds;
            e.preconditioner_seconds = k.preconditioner_seconds;
            e.solve_seconds = k.solve_seconds;
            p.linear_solves += e.linear_solves;
            p.krylov_iterations += e.krylov_iterations;
            p.matrix_pattern_builds += e.matrix_pattern_builds;
            p.matrix_value_updates += e.matrix_value_updates;
            p.rhs_only_solves += e.rhs_only_solves;
            p.true_residual_checks += e.true_residual_checks;
            p.preconditioner_setups += e.preconditioner_setups;
            p.preconditioner_reuses += e.preconditioner_reuses;
            p.preconditioner_retries += e.preconditioner_retries;
            p.matrix_update_seconds += e.matrix_update_seconds;
            p.preconditioner_seconds += e.preconditioner_seconds;
            p.linear_solve_seconds += e.solve_seconds;
            p.equation_systems.push_back(std::move(e));
        }
        std::sort(p.equation_systems.begin(), p.equation_systems.end(),
                  [](const EquationPerformanceCounters& a, const EquationPerformanceCounters& b) {
                      return a.identity < b.identity;
                  });
        return p;
    }

private:
    struct Entry {
        bsg_system* system = nullptr;
        LinearSolverType solver = LinearSolverType::BiCGSTAB;
        PreconditionerType preconditioner = PreconditionerType::BlockJacobi;
    };

    // PetscBackend::equationIdentity (petsc_backend.cpp:201-205)
    static std::string identity(const std::string& equation, const std::string& field, bool vector) {
        return std::string(vector ? "vector:" : "scalar:") + (equation.empty() ? field : equation) + ":" + field;
    }

    Entry& system(const std::string& key, int components, const LinearSolverConfig& config) {
        auto found = m_systems.find(key);
        if (found == m_systems.end()) {
            Entry e;
            check(bsg_system_create(m_device_mesh, components, &e.system), m_ctx, "bsg_system_create");
            found = m_systems.emplace(key, e).first;
        }
        found->second.solver = config.solver;
        found->second.preconditioner = config.preconditioner;
        return found->second;
    }

    const Mesh* m_mesh;
    bsg_context* m_ctx = nullptr;
    bsg_mesh* m_device_mesh = nullptr;
    std::map<std::string, Entry> m_systems;
};

}  // namespace

std::unique_ptr<ComputeBackend> makeComputeBackend(const Mesh& mesh, ParallelContext parallel) {
    return std::make_unique<B200Backend>(mesh, std::move(parallel));
}

}  // namespace babelsim::detail
