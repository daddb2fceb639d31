// Aggregation AMG preconditioner on the device (replaces Hypre BoomerAMG /
// PETSc GAMG behind pcType hypre|gamg, src/backend/petsc_linear_system.cpp:92-115,197-231).
//
// Structure (aggregates, coarse patterns and the fine->coarse value maps) is
// built once per mesh on the host from the first matrix by pairwise matching
// of strongest couplings, applied twice per level (aggregates of up to four).
// Every later matrix version only re-runs the numeric Galerkin product
// A_c = P^T A P of piecewise-constant P on the device as fixed-order gathers,
// so the preconditioner always matches the current matrix (no lagged reuse).
// The V-cycle uses damped-Jacobi smoothing and a dense inverse on the coarsest
// level, symmetric as PCG requires.
#pragma once

#include "linalg.h"
#include "pcg_persistent.cuh"
#include "pcg_sell.cuh"

#include <vector>

namespace bsg {

class AmgPreconditioner : public Preconditioner {
public:
    AmgPreconditioner(DeviceMesh& mesh, const SolverConfig& cfg);
    ~AmgPreconditioner() override;
    // Numeric setup for matrix A (same pattern as the mesh).  The structure is
    // built on the first call.
    void update(const Dcsr<double>& A, bool numeric);
    void apply(Context& ctx, const double* r, double* z) override;
    int levels() const;
    long long coarseRows(int level) const;
    // Device-side description of the hierarchy for the persistent PCG kernel
    // (valid after update()).
    AmgView<double> deviceView() const;
    // Algorithmic bytes of one V-cycle as the persistent kernel runs it (every
    // array a phase reads or writes counted once; FP64 8 B, int32 4 B).
    double vcycleBytes() const;
    // SELL-32 views for the persistent SELL solver (pcg_sell.cuh): the level-0
    // matrix in FP64 for the Krylov products, and the V-cycle in FP64 or FP32.
    bool fp32VCycle() const { return fp32_; }
    SellMat<double> krylovMatrix() const;
    SellMat<float> krylovMatrix32() const;  // level 0 in FP32 (mixed-precision path)
    VCycleView<double> sellView64() const;
    VCycleView<float> sellView32() const;
    double sellVcycleBytes() const;
    long long krylovEntries() const;  // padded level-0 SELL entries

    struct Level;

private:
    void buildStructure(const Dcsr<double>& A);
    void uploadViews();
    DeviceMesh& mesh_;
    Context& ctx_;
    SolverConfig cfg_;
    std::vector<Level*> levels_;
    bool built_ = false;
    Dcsr<double> fine_{};
    DeviceArray<AmgLevelView<double>> d_views_;
    bool fp32_ = false;
    int passes0_ = 2, passes_ = 2;  // pairwise-matching rounds per level (level 0, coarser levels)
    DeviceArray<VLevel<double>> d_vl64_;
    DeviceArray<VLevel<float>> d_vl32_;
    DeviceArray<float> dense32_;
    // Damped-Jacobi weight and coarse-correction scale.  Piecewise-constant
    // aggregation under-corrects smooth error; scaling the coarse correction by
    // 1.8 (kept fixed, so the V-cycle stays a symmetric operator for CG) cut the
    // CG iterations of the 1M-cell Voronoi pressure systems from 81 to 23 per
    // solve together with the weight 0.85 and the coarsening stop rule below.
    double omega_ = 0.85;
    double gamma_ = 1.8;
};

// Launch the persistent PCG (pcg_persistent.cu); `jac` is the Jacobi diagonal
// when amg.levels == 0 (nullptr: no preconditioner).
void launchPersistentPcg(Context& ctx, const Dcsr<double>& A, const AmgView<double>& amg, const double* jac,
                         const double* b, double* x, double* r, double* z, double* p0, double* p1, double* q,
                         double* partial, PcgState* st);
int persistentGrid(Context& ctx);

// Jacobi PCG on caller-provided device arrays with the library's file-scope
// static scratch: allocates nothing (pcg_persistent.cu).
SolveOutcome staticJacobiPcg(int n, const int* row_ptr, const int* cols, const double* diag, const double* vals,
                             const double* b, double* x, double atol, double rtol, int max_iterations);

}  // namespace bsg
