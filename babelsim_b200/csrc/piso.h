// Transient PISO on device-resident state (src/physics/piso/main.cpp:60-301).
#pragma once

#include "fvm.h"
#include "linalg.h"
#include "rans.h"

#include <memory>

namespace bsg {

struct PisoConfig {
    double rho = 1.0, mu = 0.01, alpha_u = 1.0;
    int max_iterations = 1;          // predictor-corrector passes per time step
    int correctors = 2, max_correctors = 2;
    double coupling_tolerance = 1.7976931348623157e308;
    int non_orthogonal_corrections = 1;
    double mass_tolerance = 1e-8, velocity_tolerance = 1e-7, momentum_tolerance = 1e-6, pressure_tolerance = 1e-6;
    int time_method = 2;             // TimeMethod: 1 Euler, 2 BDF2
    double start_time = 0.0, end_time = 1.0, delta_t = 1e-3;
    Options momentum, pressure;
    SolverConfig momentum_solver, pressure_solver;
};

// runPiso's turbulence controls (piso/main.cpp:99-120).
struct PisoTurbulenceControls {
    bool segregated = false;        // turbulenceCoupling segregated (else iterated)
    int max_iterations = 1000;      // turbulenceMaxIterations
    int correctors = 0;             // turbulenceCorrectors; <= 0: max_iterations with one PISO pass and
                                    // iterated coupling, else 1
};

struct PisoReport {
    int steps = 0;
    double time = 0.0;
    int status = 1;                  // 0 completed (end time reached), 1 running / not converged, 2 numerical failure
    bool accepted = true;
    double mass = 0, dU = 0, rU = 0, dP = 0, coupling = 0, courant_max = 0, courant_mean = 0;
    int correctors = 0, momentum_iterations = 0, pressure_iterations = 0;
    double turbulence_change = 0, turbulence_residual = 0;
    int turbulence_corrections = 0;
};

class PisoSolver {
public:
    PisoSolver(DeviceMesh& mesh, const PisoConfig& cfg);
    ~PisoSolver();
    DeviceField& U() { return U_; }
    DeviceField& p() { return p_; }
    DeviceField& phi() { return phi_; }
    // rans::load (piso/main.cpp:98-121): an eddy-viscosity model; call before start().
    void enableTurbulence(const KOmegaConfig& cfg, const PisoTurbulenceControls& controls);
    KOmegaModel* turbulence() { return turb_.get(); }
    // initializePotentialFlow (piso/main.cpp:123-146): before the first step, potential solves on the
    // initial flux imbalance correct U and phi; `initial_non_orthogonal_corrections` < 0 takes
    // nonOrthogonalCorrections.  Call before start().
    void initializePotentialFlow(int initial_non_orthogonal_corrections);
    // Initial state: phi = flux(U) with the pressure options (piso/main.cpp:122).
    void start();
    // Advance up to `steps` time steps (fewer at the end time or on a rejected step).
    PisoReport advance(int steps);
    const PisoReport& report() const { return report_; }

private:
    bool step();
    void saveHistory(double dt);
    DeviceMesh& m_;
    Context& ctx_;
    PisoConfig cfg_;
    DeviceField U_, p_, phi_, muEff_, rAU_, rAUf_, HbyA_, phiH_;
    DeviceField Uprev_lvl_, Uolder_lvl_;   // time::History<Vec3> levels
    DeviceArray<double> phi_prev_, phi_older_, flux_tmp_;
    DeviceField flux_field_;
    int levels_ = 0;
    double dt_ = 0.0, prev_dt_ = 0.0, time_ = 0.0;
    int step_ = 0;
    std::unique_ptr<DeviceEquation> mom_, peq_;
    KrylovSolver krylov_;
    std::unique_ptr<Preconditioner> ppc_;
    Reducer redR_, redU_, redP_, redM_, redC_, redCo_;
    DeviceArray<double> Uiter_, gradP_, npr_, AU_, temporal_, divPhiH_, pflux_, pprev_;
    DeviceArray<int> flags_;
    PisoReport report_;
    bool started_ = false;
    std::unique_ptr<KOmegaModel> turb_;
    PcReusePolicy preuse_;      // lag of the pressure AMG across matrix versions
    bool potential_start_ = false;
    int initial_non_orth_ = -1;
    void potentialFlowStart();
    PisoTurbulenceControls tctl_;
    DeviceArray<double> divStress_;
};

}  // namespace bsg
