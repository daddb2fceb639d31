// Wilcox-1988m k-omega on device-resident fields (src/physics/RANS/k_omega.cpp,
// model.cpp).  Derived fields (mut, the effective viscosity, the transport
// diffusivities, the deviatoric stress) are calculated fields: every pointwise
// expression is applied to the cell values and to the boundary traces of its
// operands, as the reference's calculated fields do (include/babelsim/field.h:262-320).
#pragma once

#include "fvm.h"
#include "linalg.h"

#include <memory>

namespace bsg {

// Eddy-viscosity models: kind 0 Wilcox-1988m k-omega (k_omega.cpp), kind 1
// standard k-epsilon (k_epsilon.cpp), kind 2 Spalart-Allmaras (spalart_allmaras.cpp).
// The second transported field (omega, epsilon, or nuTilda for the one-equation
// model, which has no k) uses the omega_* members of the configuration.
struct KOmegaConfig {
    int kind = 0;
    double rho = 1.0, mu = 1e-3;
    double beta_star = 0.09, beta = 3.0 / 40.0, gamma = 5.0 / 9.0, sigma_k = 0.5, sigma_omega = 0.5;
    double k_min = 1e-12, omega_min = 1e-12, viscosity_ratio_max = 1e5;
    double c_mu = 0.09, c1 = 1.44, c2 = 1.92;  // k-epsilon (sigma_k, sigma_omega = sigmaEpsilon, omega_min = epsilonMin)
    // Spalart-Allmaras (omega_min = saNuTildaMin); sa_cw1 <= 0 takes cb1/kappa^2 + (1 + cb2)/sigma
    double sa_cb1 = 0.1355, sa_cb2 = 0.622, sa_sigma = 2.0 / 3.0, sa_kappa = 0.41, sa_cw1 = 0.0, sa_cw2 = 0.3,
           sa_cw3 = 2.0, sa_cv1 = 7.1, sa_ct3 = 1.2, sa_ct4 = 0.5, wall_distance_min = 1e-12;
    double relaxation = 0.7, tolerance = 1e-6;
    Options k_options, omega_options, momentum_options;
    SolverConfig k_solver, omega_solver;
};

struct TransportResult {
    double change = 0.0;     // max relative change of omega and k
    double residual = 0.0;   // max initial normalised residual
    bool linear_converged = true;
    bool healthy = true;
    int iterations = 0;
};

class KOmegaModel {
public:
    KOmegaModel(DeviceMesh& mesh, const KOmegaConfig& cfg);
    ~KOmegaModel();
    DeviceField& k() { return k_; }
    DeviceField& omega() { return omega_; }
    // Spalart-Allmaras: the given wall distance of every cell (the reference reads it as an input field).
    void setWallDistance(const double* host);
    // Transient use (runPiso): `method` 1 Euler, 2 BDF2; saveOld stores every transported field's
    // history once per physical step, and the transport equations then take equ::ddt(rho, history).
    void setTransient(int method);
    void saveOld(double dt);
    DeviceField& effectiveViscosity() { return muEff_; }
    DeviceField& turbulentViscosity() { return mut_; }
    const KOmegaConfig& config() const { return cfg_; }
    // Constructor work of the reference model (k_omega.cpp:51-56): bound k and
    // omega with `phi` as their boundary-flux context, then mut and muEff.
    void start(const DeviceField& phi);
    // div(muEff (grad(U)^T - 2/3 tr(grad U) I)) into out (3 per cell) (model.cpp:65-69).
    void stressRemainderDivergence(DeviceField& U, double* out);
    // KOmega::solveTransport, steady (k_omega.cpp:65-125).
    TransportResult solveTransport(DeviceField& U, DeviceField& phi);

private:
    void updateViscosity();
    void boundOmega();
    void gradientWithTraces(DeviceField& U);
    DeviceMesh& m_;
    Context& ctx_;
    KOmegaConfig cfg_;
    DeviceField k_, omega_, mut_, muEff_, kDiff_, wDiff_;
    std::unique_ptr<DeviceEquation> keq_, weq_;
    KrylovSolver krylov_;
    DeviceArray<double> G_, Gtr_, T_, Ttr_, production_, wDestruction_, wProduction_, kSink_, prevK_, prevW_;
    DeviceArray<double> wallDist_, gradNt_;
    bool wall_set_ = false;
    int time_method_ = 0;
    DeviceArray<double> kPrevLvl_, kOlderLvl_, wPrevLvl_, wOlderLvl_;
    double tdt_ = 0.0, tprev_dt_ = 0.0;
    int tlevels_ = 0;
    // equ::ddt(eq, rho, history) when transient (a no-op when steady)
    void timeTerm(DeviceEquation& eq, const DeviceArray<double>& previous, const DeviceArray<double>& older);
    TransportResult solveSpalartAllmaras(DeviceField& U, DeviceField& phi);
    Reducer redW_, redK_, redDW_, redDK_;
};

}  // namespace bsg
