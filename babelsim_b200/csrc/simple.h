// Steady SIMPLE outer loop on device-resident state (src/physics/simple/main.cpp:11-131).
#pragma once

#include "fvm.h"
#include "linalg.h"
#include "rans.h"

#include <memory>

namespace bsg {

class AmgPreconditioner;

struct SimpleConfig {
    double rho = 1.0, mu = 0.01, alpha_u = 0.7, alpha_p = 0.3;
    int non_orthogonal_corrections = 1;
    double mass_tolerance = 1e-8, velocity_tolerance = 1e-7, momentum_tolerance = 1e-6,
           pressure_tolerance = 1e-6;
    Options momentum, pressure;
    SolverConfig momentum_solver, pressure_solver;
};

struct SimpleReport {
    int iterations = 0;
    bool converged = false;
    int status = 1;
    double mass = 0, dU = 0, rU = 0, dP = 0, linP = 0;
    int momentum_iterations = 0, pressure_iterations = 0;
    double turbulence_change = 0, turbulence_residual = 0;
};

// One case of a batch: a contiguous cell range of the mesh that no interior face leaves.
struct SimpleSegment;

class SimpleSolver {
public:
    SimpleSolver(DeviceMesh& mesh, const SimpleConfig& cfg);
    ~SimpleSolver();
    // Several independent cases in one mesh (block-diagonal batching over a segment table):
    // case s owns cells [cell_offsets[s], cell_offsets[s+1]) and has dynamic viscosity
    // viscosity[s].  Every assembly, gradient, flux and update kernel runs once over all
    // cases; the diagnostics, the gauge and the convergence tests are per case; each case's
    // momentum system is solved on its own rows and all cases' pressure systems are solved
    // together in one persistent launch per attempt (KrylovSolver::solveBatch), each with
    // its own AMG hierarchy and preconditioner lag.  A case that has converged keeps its
    // converged state while the others continue.  Call before start(); laminar only.
    void setSegments(const std::vector<int>& cell_offsets, const std::vector<double>& viscosity);
    int segments() const { return static_cast<int>(segs_.size()); }
    const SimpleReport& segmentReport(int s) const;
    DeviceField& U() { return U_; }
    DeviceField& p() { return p_; }
    DeviceField& phi() { return phi_; }
    // Initial state: phi = flux(U) (simple/main.cpp:40).
    void start();
    // Outer iterations until converged or `max_iterations` more are done.
    SimpleReport iterate(int max_iterations);
    // Overwrite U, p, phi from host memory (caller numbering) keeping all other state.
    void loadState(const double* U, const double* p, const double* phi);
    // Wilcox-1988m k-omega eddy viscosity (rans::load with turbulenceModel kOmega); call before start().
    void enableKOmega(const KOmegaConfig& cfg);
    KOmegaModel* turbulence() { return turb_.get(); }
    const SimpleReport& report() const { return report_; }

private:
    void outerIteration();
    void outerIterationSegments();
    DeviceMesh& m_;
    Context& ctx_;
    SimpleConfig cfg_;
    DeviceField U_, p_, phi_, pP_, muEff_, rAU_, phiH_;
    std::unique_ptr<DeviceEquation> mom_, peq_;
    std::unique_ptr<KOmegaModel> turb_;
    PcReusePolicy preuse_;      // lag of the pressure AMG across matrix versions
    DeviceArray<double> divStress_;
    KrylovSolver krylov_;
    std::unique_ptr<Preconditioner> ppc_;
    Reducer red_, redU_, redPP_, redP_, redM_;  // one per diagnostic, read back together
    DeviceArray<double> Uprev_, gradP_, gradPP_, divPhiH_, pflux_, diag_ws_;
    DeviceArray<int> flags_;
    SimpleReport report_;
    bool started_ = false;
    std::vector<std::unique_ptr<SimpleSegment>> segs_;
    double* seg_pinned_ = nullptr;  // per-segment diagnostics read back together
};

}  // namespace bsg
