// Sparse linear algebra on the device: DCSR matrices (diagonal + off-diagonal
// CSR), Krylov solvers with device-resident scalars, preconditioners.
#pragma once

#include <algorithm>

#include "bsg_internal.h"

#include <memory>
#include <vector>

namespace bsg {

// A square matrix in "diagonal + off-diagonal CSR" form; arrays are borrowed.
template <class T>
struct Dcsr {
    int n = 0;
    const int* ptr = nullptr;
    const int* col = nullptr;
    const T* diag = nullptr;
    const T* val = nullptr;
    long long nnz_off = 0;
};

// LinearSolverConfig (include/babelsim/solver_control.h:165-184).
struct SolverConfig {
    int solver = 1;            // 0 CG, 1 BiCGSTAB, 2 GMRES, 3 FGMRES
    int preconditioner = 4;    // PreconditionerType order
    double atol = 1e-12, rtol = 1e-8;
    int max_iterations = 1000;
    bool warm_start = false;
    int rebuild_interval = 8;
    double reuse_growth = 2.0;
    int amg_max_levels = 12, amg_coarse_size = 400, amg_smoothing_steps = 2;
    int precision = 0;         // 0 FP64, 1 FP32 inner iterations with FP64 refinement
};

// SolveResult (include/babelsim/solver_control.h:227-258).
struct SolveOutcome {
    int status = 2;            // 0 converged, 1 max iterations, 2 numerical failure
    int iterations = 0;
    double initial = 0.0, final_ = 0.0, relative = 0.0;
    int checks = 0;            // true-residual evaluations (PetscLinearSystem's true_residual_checks)
};

class AmgPreconditioner;
class KrylovSolver;

// One system of a batched persistent CG + AMG solve (KrylovSolver::solveBatch).
struct BatchSolve {
    KrylovSolver* solver = nullptr;       // owns this system's vectors, partials and solve state
    AmgPreconditioner* amg = nullptr;     // its hierarchy; level 0 is the Krylov matrix
    Dcsr<double> A{};                     // the system, for the true-residual checks
    const double* b = nullptr;
    double* x = nullptr;
    SolverConfig cfg{};
    SolveOutcome out{};
};

// One 3-component system of a batched persistent BiCGStab solve (KrylovSolver::solveVector3Batch).
struct BicgItem {
    KrylovSolver* solver = nullptr;       // owns this system's vectors, SELL copy and solve state
    Dcsr<double> A{};
    const double* b = nullptr;            // xyz-interleaved
    double* x = nullptr;
    SolverConfig cfg{};
    SolveOutcome out[3]{};
};

// When a preconditioner built for an earlier matrix version is reused (lagged), as
// PetscLinearSystem does (src/backend/petsc_linear_system.cpp:257-324, 446-470): a
// rebuild is due when rebuild_interval matrix versions or right-hand-side solves
// have passed since the last setup, or when a lagged solve needed more than
// reuse_growth times the iterations the fresh preconditioner needed; a lagged solve
// that fails is retried once with a fresh preconditioner.
struct PcReusePolicy {
    long long matrix_updates = 0, pc_matrix_update = -1, pc_setups = 0, rhs_solves = 0;
    int fresh[3] = {0, 0, 0};  // iterations of the fresh preconditioner, per right-hand side
    bool force_rebuild = true;
    // Before a solve: true when the preconditioner must be rebuilt for this matrix.
    bool needRebuild(bool matrix_changed, const SolverConfig& cfg) {
        if (matrix_changed) ++matrix_updates;
        if (!matrix_changed && !force_rebuild) return false;
        const bool reuse = pc_setups != 0 && !force_rebuild &&
                           matrix_updates - pc_matrix_update < cfg.rebuild_interval &&
                           rhs_solves < cfg.rebuild_interval;
        force_rebuild = false;
        if (!reuse) rebuilt();
        return !reuse;
    }
    void rebuilt() {
        ++pc_setups;
        pc_matrix_update = matrix_updates;
        rhs_solves = 0;
        fresh[0] = fresh[1] = fresh[2] = 0;
    }
    bool lagged() const { return pc_matrix_update != matrix_updates; }
    // After a solve of right-hand side `rhs` with `attempt_iterations` iterations of the final attempt.
    void afterSolve(int status, int attempt_iterations, int total_iterations, const SolverConfig& cfg, int rhs = 0) {
        int& f = fresh[rhs < 0 || rhs > 2 ? 0 : rhs];
        if (status == 0) {
            if (!lagged()) f = std::max(f, attempt_iterations);
            else if (attempt_iterations > cfg.reuse_growth * static_cast<double>(std::max(f, 1)))
                force_rebuild = true;
        }
        if (total_iterations > 0) ++rhs_solves;
    }
};

// Preconditioner application z = M^-1 r for a single right-hand side.
struct Preconditioner {
    virtual ~Preconditioner() = default;
    virtual void apply(Context& ctx, const double* r, double* z) = 0;
};

// Workspace and driver for solving A x = b with the reference's acceptance
// contract (src/backend/petsc_linear_system.cpp:355-481):
// ||b-Ax|| <= max(atol, rtol*max(||r0||,||b||)), zero initial guess unless
// warm_start, up to 3 true-residual restarts with a halved internal target.
class KrylovSolver {
public:
    explicit KrylovSolver(Context& ctx);
    ~KrylovSolver();
    // Scalar system; x holds the guess on entry (warm start) and the solution on exit.
    // cfg.solver selects the method: 0 CG (persistent kernel with AMG, Jacobi or no
    // preconditioner), 1 BiCGStab (point Jacobi), 2 GMRES(30), 3 FGMRES(30) (with pc).
    SolveOutcome solveScalar(const Dcsr<double>& A, const SolverConfig& cfg, Preconditioner* pc,
                             const double* b, double* x);
    // Three right-hand sides (xyz interleaved) sharing one matrix; Jacobi-preconditioned
    // BiCGStab in lockstep, one matrix read per product for all three (cfg.solver 1);
    // GMRES / FGMRES / CG solve the components one after another.
    void solveVector3(const Dcsr<double>& A, const SolverConfig& cfg, const double* b, double* x,
                      SolveOutcome out[3]);
    // One right-hand side, Jacobi-preconditioned BiCGStab (non-symmetric scalar systems:
    // transported turbulence quantities, and any scalar equation configured with kspType bcgs).
    SolveOutcome solveBicgstab(const Dcsr<double>& A, const SolverConfig& cfg, const double* b, double* x);
    // Several independent CG + AMG systems (FP64, or FP64 CG with an FP32 V-cycle) solved
    // together: each attempt of every unfinished system runs in one cooperative launch, on
    // CTAs of its own, with the same acceptance loop per system as solveScalar (true-residual
    // restarts with a halved internal target).  The true residuals of all systems are read
    // back together.  Every item's solver must be on ctx.
    static void solveBatch(Context& ctx, std::vector<BatchSolve>& items);
    // Several 3-component BiCGStab systems (Jacobi preconditioner, the momentum equations of
    // a batch) solved by the persistent BiCGStab kernel: with `batched` all unfinished systems
    // of an attempt share one cooperative launch, each on CTAs of its own; otherwise each
    // system gets the whole grid in turn.  The reference's acceptance loop per component.
    static void solveVector3Batch(Context& ctx, std::vector<BicgItem>& items, bool batched = true);
    int check_interval = 8;  // iterations between host convergence checks
    // CG with AMG, Jacobi or no preconditioner runs as one persistent cooperative
    // kernel per attempt (pcg_persistent.cu); set false to use per-kernel launches.
    bool persistent = true;
    // FP32-inner iterative refinement (precision 1): each pass asks the FP32 solve
    // for this reduction of the current FP64 residual.
    double refine_inner_rtol = 1e-5;
    int max_refinements = 12;

private:
    SolveOutcome solveRefined(const Dcsr<double>& A, const SolverConfig& cfg, AmgPreconditioner* amg, const double* b,
                              double* x);
    template <int C>
    void lockstepBicgstab(const Dcsr<double>& A, const SolverConfig& cfg, const double* b, double* x,
                          SolveOutcome out[]);
    template <int C>
    void refinedBicgstab(const Dcsr<double>& A, const SolverConfig& cfg, const double* b, double* x,
                         SolveOutcome out[]);
    SolveOutcome cgComponent(const Dcsr<double>& A, const SolverConfig& cfg, Preconditioner* pc, int c,
                             const double* b, double* x);
    SolveOutcome solvePersistent(const Dcsr<double>& A, const SolverConfig& cfg, AmgPreconditioner* amg,
                                 const double* jacobi_diag, const double* b, double* x);
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

// Workspace of the restarted GMRES / FGMRES solver (gmres.cu): the Krylov basis
// V ((m+1) x n), the preconditioned directions Z (FGMRES, m x n) and scratch.
struct GmresWorkspace {
    int restart = 30;  // m (the reference's PETSc default restart, at most 30 here)
    DeviceArray<double> V, Z, w, r, zt, bc, xc, partial, coef;
    void ensure(int n, int m, bool flexible);
};

// Restarted right-preconditioned GMRES(m) (cfg.solver 2) or FGMRES(m) (3) with the
// reference's acceptance contract; pc may be nullptr (gmres.cu).
SolveOutcome gmresSolve(Context& ctx, GmresWorkspace& ws, const Dcsr<double>& A, const SolverConfig& cfg,
                        Preconditioner* pc, const double* b, double* x);
// Component c of a C-component xyz-interleaved vector copied to (gather) or from a
// contiguous n-vector (gmres.cu).
void componentCopy(Context& ctx, int n, int C, int c, const double* in, double* out, bool gather);
// gmresSolve for component c of C xyz-interleaved right-hand sides sharing A.
SolveOutcome gmresComponent(Context& ctx, GmresWorkspace& ws, const Dcsr<double>& A, const SolverConfig& cfg,
                            Preconditioner* pc, int C, int c, const double* b, double* x);

// Jacobi preconditioner (point diagonal).
struct JacobiPreconditioner : Preconditioner {
    const double* diag = nullptr;
    int n = 0;
    void apply(Context& ctx, const double* r, double* z) override;
};

// Device SpMV y = A x for C interleaved components.
void spmv(Context& ctx, const Dcsr<double>& A, const double* x, double* y, int C);
// ||b - A x||_2 for one right-hand side, returned to the host.
double trueResidualNorm(Context& ctx, const Dcsr<double>& A, const double* b, const double* x, double* r_ws);

}  // namespace bsg
