// Steady SIMPLE on device-resident fields: every step of the reference's outer
// iteration (src/physics/simple/main.cpp:47-127) runs as sm_100a kernels; the host
// only sequences launches and reads one small diagnostics block per iteration.
#include "bsg_device.cuh"
#include "simple.h"
#include "amg.h"

#include <cmath>
#include <cstring>

namespace bsg {
namespace {
constexpr int kBlock = 256;

// Rhie-Chow interior correction (simple/main.cpp:71-79) with linear
// interpolation: phiH += interp(rAU*gradP).Sf - interp(rAU)*snGrad(p)*|Sf|.
__global__ void kRhieChow(MeshView m, BcView bp, const double* __restrict__ rAU, const double* __restrict__ gradP,
                          const double* __restrict__ p, int diffusion, double* __restrict__ phiH) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.n_interior) return;
    const int o = m.own[f], n = m.nbr[f];
    const double w = m.w[f];
    const double ro = rAU[o], rn = rAU[n];
    double ifl = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) ifl += (w * (ro * gradP[3 * o + c]) + (1.0 - w) * (rn * gradP[3 * n + c])) * m.Sf[3 * f + c];
    const double orth = m.dcoef[f] * (p[n] - p[o]);
    double ing = orth;
    if (diffusion != 0) {
        const double fg0 = w * gradP[3 * o] + (1.0 - w) * gradP[3 * n];
        const double fg1 = w * gradP[3 * o + 1] + (1.0 - w) * gradP[3 * n + 1];
        const double fg2 = w * gradP[3 * o + 2] + (1.0 - w) * gradP[3 * n + 2];
        ing = orth + limitCorrection(orth, m.kvec[3 * f] * fg0 + m.kvec[3 * f + 1] * fg1 + m.kvec[3 * f + 2] * fg2,
                                     diffusion);
    }
    const double rAUf = w * ro + (1.0 - w) * rn;
    const double nfl = rAUf * (ing / m.area[f]) * m.area[f];
    double v = phiH[f];
    v += ifl;
    v -= nfl;
    phiH[f] = v;
}

// Traces of a calculated cell field whose constraints are the default
// zeroGradient ones: the owner value (geometry.cpp values(), field.h:264-272).
__global__ void kOwnerTrace(MeshView m, const double* __restrict__ x, double* __restrict__ trace) {
    const int fb = blockIdx.x * blockDim.x + threadIdx.x;
    if (fb < m.n_boundary) trace[fb] = x[m.bown[fb]];
}

}  // namespace

SimpleSolver::SimpleSolver(DeviceMesh& mesh, const SimpleConfig& cfg)
    : m_(mesh), ctx_(*mesh.ctx), cfg_(cfg), U_(mesh, 0, 3), p_(mesh, 0, 1), phi_(mesh, 1, 1), pP_(mesh, 0, 1),
      muEff_(mesh, 0, 1), rAU_(mesh, 0, 1), phiH_(mesh, 1, 1), krylov_(*mesh.ctx) {
    if (!(cfg.rho > 0) || !(cfg.mu > 0)) fail(kArgument, "density and dynamicViscosity must be positive");
    if (cfg.pressure.interpolation != 0 || cfg.pressure.coefInterp() != 0)
        fail(kArgument, "the device SIMPLE driver supports linear interpolation of the Rhie-Chow terms");
    std::vector<double> mu(mesh.n_cells, cfg.mu);
    muEff_.v.upload(mu, ctx_.stream);
    rAU_.calculated = true;
    rAU_.trace.resize(mesh.n_boundary);
    Uprev_.resize(3 * static_cast<std::size_t>(mesh.n_cells));
    flags_.resize(4);
    mom_ = std::make_unique<DeviceEquation>(U_, cfg.momentum);
    peq_ = std::make_unique<DeviceEquation>(pP_, cfg.pressure);
    ctx_.sync();
}

SimpleSolver::~SimpleSolver() = default;

void SimpleSolver::enableKOmega(const KOmegaConfig& cfg) {
    if (started_) fail(kState, "the turbulence model must be chosen before the fields are set");
    KOmegaConfig c = cfg;
    c.rho = cfg_.rho;
    c.mu = cfg_.mu;
    c.momentum_options = cfg_.momentum;
    turb_ = std::make_unique<KOmegaModel>(m_, c);
    divStress_.resize(3 * static_cast<std::size_t>(m_.n_cells));
}

void SimpleSolver::start() {
    // pPrime = homogeneousLike(p) (field.h:380-420)
    for (int patch = 0; patch < m_.n_patches; ++patch) {
        const int t = p_.bcs[patch].type;
        const double zero[3] = {0, 0, 0};
        pP_.setBoundary(patch, t == 0 ? 0 : (t == 4 ? 4 : 2), zero);
    }
    if (turb_) {
        // rans::load runs before phi = flux(U) (simple/main.cpp:33-40): the model sees phi = 0
        phi_.v.zero(ctx_.stream);
        turb_->start(phi_);
    }
    faceFlux(U_, cfg_.momentum.interpolation, cfg_.momentum.gradient, phi_);
    const int pcType = cfg_.pressure_solver.preconditioner;
    if (pcType == 2 || pcType == 3) ppc_ = std::make_unique<AmgPreconditioner>(m_, cfg_.pressure_solver);
    else ppc_ = std::make_unique<JacobiPreconditioner>();
    started_ = true;
    report_ = SimpleReport{};
    ctx_.sync();
}

void SimpleSolver::loadState(const double* U, const double* p, const double* phi) {
    if (!started_) fail(kState, "load_state requires a started SIMPLE solver (set_fields first)");
    const std::size_t N = m_.n_cells;
    U_.v.upload(U, 3 * N, ctx_.stream);
    p_.v.upload(p, N, ctx_.stream);
    // phi arrives in the caller's face numbering; the device keeps interior faces first.
    phi_.uploadExternal(phi);
}

SimpleReport SimpleSolver::iterate(int max_iterations) {
    if (!started_) start();
    for (int k = 0; k < max_iterations; ++k) {
        outerIteration();
        if (report_.converged || report_.status == 2) break;
    }
    return report_;
}

void SimpleSolver::outerIteration() {
    const int N = m_.n_cells;
    const MeshView mv = view(m_);
    copyAsync(ctx_, Uprev_.data(), U_.v.data(), 3LL * N);
    // Momentum assembly (simple/main.cpp:51-56).
    DeviceEquation& mom = *mom_;
    {
        BSG_PROFILE(ctx_, "momentum_assembly");
        mom.reset();
        addConvection(mom, phi_, cfg_.rho, cfg_.momentum);
        addLaplacian(mom, turb_ ? &turb_->effectiveViscosity() : &muEff_, 0.0, -1.0, cfg_.momentum);
        gradient(p_, cfg_.pressure.gradient, gradP_);
        addSource(mom, gradP_.data(), -1.0);
        if (turb_) {
            // explicit remainder of the eddy-viscosity stress (simple/main.cpp:54-56)
            turb_->stressRemainderDivergence(U_, divStress_.data());
            addSource(mom, divStress_.data(), 1.0);
        }
    }
    // rU before relaxation (simple/main.cpp:59-60).
    // The norms stay on the device and are read with the other diagnostics: a
    // non-finite rU still ends the run as a numerical failure, one sync later.
    relativeResidualNorms(mom, U_.v.data(), red_);
    relax(mom, Uprev_.data(), cfg_.alpha_u);
    scale(mom, cfg_.alpha_u);
    ratioVolume(m_, mom.diag.data(), rAU_.v.data());
    kOwnerTrace<<<gridFor(m_.n_boundary, kBlock), kBlock, 0, ctx_.stream>>>(mv, rAU_.v.data(), rAU_.trace.data());
    ctx_.launched();
    // Momentum solve (simple/main.cpp:67-68), three components on one matrix.
    Dcsr<double> A{N, m_.cf_ptr.data(), m_.cf_col.data(), mom.diag.data(), mom.val.data(),
                   2LL * m_.n_interior};
    SolveOutcome uo[3];
    krylov_.solveVector3(A, cfg_.momentum_solver, mom.src.data(), U_.v.data(), uo);
    int mom_iters = 0;
    bool mom_ok = true, mom_healthy = true;
    for (const auto& o : uo) {
        mom_iters += o.iterations;
        mom_ok = mom_ok && o.status == 0;
        mom_healthy = mom_healthy && o.status != 2 && std::isfinite(o.final_);
    }
    report_.momentum_iterations = mom_iters;
    if (!mom_healthy) { report_.status = 2; return; }
    // Rhie-Chow face flux (simple/main.cpp:71-79); p is unchanged since assembly, so gradP is reused.
    {
        BSG_PROFILE(ctx_, "rhie_chow_flux");
        faceFlux(U_, cfg_.momentum.interpolation, cfg_.momentum.gradient, phiH_);
        kRhieChow<<<gridFor(m_.n_interior, kBlock), kBlock, 0, ctx_.stream>>>(
            mv, p_.bcView(), rAU_.v.data(), gradP_.data(), p_.v.data(), cfg_.pressure.diffusion, phiH_.v.data());
        ctx_.launched();
        divFlux(phiH_, divPhiH_);
    }
    // Pressure correction (simple/main.cpp:81-93).
    BSG_CUDA(cudaMemsetAsync(pP_.v.data(), 0, sizeof(double) * N, ctx_.stream));
    const int pressure_solves = cfg_.pressure.diffusion == 0 ? 1 : cfg_.non_orthogonal_corrections + 1;
    DeviceEquation& peq = *peq_;
    bool p_ok = true;
    int p_iters = 0;
    double linP = 0.0;
    for (int corr = 0; corr < pressure_solves; ++corr) {
        {
            BSG_PROFILE(ctx_, "pressure_assembly");
            peq.reset();
            addLaplacian(peq, &rAU_, 0.0, -1.0, cfg_.pressure);
            addSource(peq, divPhiH_.data(), -1.0);
            referenceIfUnanchored(peq, 0.0, flags_.data());
        }
        Dcsr<double> P{N, m_.cf_ptr.data(), m_.cf_col.data(), peq.diag.data(), peq.val.data(), 2LL * m_.n_interior};
        if (auto* jac = dynamic_cast<JacobiPreconditioner*>(ppc_.get())) { jac->diag = peq.diag.data(); jac->n = N; }
        auto* amg = dynamic_cast<AmgPreconditioner*>(ppc_.get());
        bool lagged = false;
        if (amg) {
            BSG_PROFILE(ctx_, "amg_numeric_setup");
            amg->update(P, preuse_.needRebuild(corr == 0, cfg_.pressure_solver));
            lagged = preuse_.lagged();
        }
        SolveOutcome po = krylov_.solveScalar(P, cfg_.pressure_solver, ppc_.get(), peq.src.data(), pP_.v.data());
        int attempt = po.iterations;
        if (amg && lagged && po.status != 0) {
            // a failed lagged solve is retried once with a fresh preconditioner
            {
                BSG_PROFILE(ctx_, "amg_numeric_setup");
                amg->update(P, true);
            }
            preuse_.rebuilt();
            const int first = po.iterations;
            po = krylov_.solveScalar(P, cfg_.pressure_solver, ppc_.get(), peq.src.data(), pP_.v.data());
            attempt = po.iterations;
            po.iterations += first;
        }
        if (amg) preuse_.afterSolve(po.status, attempt, po.iterations, cfg_.pressure_solver);
        if (po.status == 2 || !std::isfinite(po.final_)) { report_.status = 2; return; }
        p_ok = p_ok && po.status == 0;
        p_iters += po.iterations;
        linP = po.relative;
    }
    report_.pressure_iterations = p_iters;
    report_.linP = linP;
    // Field updates (simple/main.cpp:95-98).
    axpyCell(ctx_, p_.v.data(), cfg_.alpha_p, pP_.v.data(), N);
    BSG_PROFILE(ctx_, "field_updates_diagnostics");
    faceFluxEquation(peq, pP_.v.data(), pflux_);
    gradient(pP_, cfg_.pressure.gradient, gradPP_);
    subtractScaledGradient(m_, U_.v.data(), rAU_.v.data(), gradPP_.data());
    addArrays(ctx_, phi_.v.data(), phiH_.v.data(), pflux_.data(), m_.n_faces);
    // turbulence transport after the flow update (simple/main.cpp:102-110)
    TransportResult tr;
    if (turb_) {
        tr = turb_->solveTransport(U_, phi_);
        report_.turbulence_change = tr.change;
        report_.turbulence_residual = tr.residual;
        if (!tr.healthy) { report_.status = 2; return; }
    }
    const bool turbulence_ok = !turb_ || (tr.linear_converged && tr.change <= turb_->config().tolerance &&
                                          tr.residual <= turb_->config().tolerance);
    // Convergence diagnostics (simple/main.cpp:112-126).
    relativeChangeNorms(ctx_, U_.v.data(), Uprev_.data(), 3LL * N, redU_);
    relativeChangeNorms(ctx_, pP_.v.data(), nullptr, N, redPP_);
    relativeChangeNorms(ctx_, p_.v.data(), nullptr, N, redP_);
    fluxBalance(m_, phi_.v.data(), redM_);
    double* h = ctx_.pinned;
    BSG_CUDA(cudaMemcpyAsync(h + 0, red_.result.data(), 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
    BSG_CUDA(cudaMemcpyAsync(h + 4, redU_.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
    BSG_CUDA(cudaMemcpyAsync(h + 6, redPP_.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
    BSG_CUDA(cudaMemcpyAsync(h + 8, redP_.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
    BSG_CUDA(cudaMemcpyAsync(h + 10, redM_.result.data(), 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
    ctx_.sync();
    const double rU = std::sqrt(h[0]) / std::max(std::sqrt(h[1]) + std::sqrt(h[2]), 1e-30);
    const double dU = std::sqrt(h[4]) / std::max(std::sqrt(h[5]), 1e-30);
    const double dP = std::sqrt(h[6]) / std::max(std::sqrt(h[9]), 1e-30);
    const double mass = h[10] / std::max(h[12], 1e-30);
    report_.rU = rU;
    if (!std::isfinite(rU)) { report_.status = 2; return; }
    report_.dU = dU;
    report_.dP = dP;
    report_.mass = mass;
    report_.iterations += 1;
    if (!(std::isfinite(dU) && std::isfinite(dP) && std::isfinite(mass))) { report_.status = 2; return; }
    const bool linear_ok = mom_ok && p_ok;
    report_.converged = linear_ok && turbulence_ok && rU <= cfg_.momentum_tolerance && dU <= cfg_.velocity_tolerance &&
                        dP <= cfg_.pressure_tolerance && mass <= cfg_.mass_tolerance;
    report_.status = report_.converged ? 0 : 1;
}

}  // namespace bsg
