// Transient PISO on device-resident fields: every step of the reference's time
// step (src/physics/piso/main.cpp:160-297) runs as sm_100a kernels; the host
// sequences launches and reads a few scalars per corrector.
#include "bsg_device.cuh"
#include "piso.h"
#include "amg.h"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>

namespace bsg {
namespace {
__global__ void kSubtract(long long n, const double* __restrict__ a, double* __restrict__ out) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i < n) out[i] -= a[i];
}

constexpr int kBlock = 256;

// temporalFluxCorrection (piso/main.cpp:19-55), times rho, interior faces only:
// e = phi_prev - flux(U_prev); c = w1 e + w2 (phi_older - flux(U_older));
// coupling = 1 if e == 0, 0 if phi_prev == 0, else max(0, 1 - |e|/|phi_prev|).
__global__ void kTemporalFlux(int n_interior, int n_faces, double rho, double w1, double w2,
                              const double* __restrict__ phi_prev, const double* __restrict__ flux_prev,
                              const double* __restrict__ phi_older, const double* __restrict__ flux_older,
                              double* __restrict__ out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    if (f >= n_interior) { out[f] = 0.0; return; }
    const double e = phi_prev[f] - flux_prev[f];
    double c = w1 * e;
    if (w2 != 0.0) c += w2 * (phi_older[f] - flux_older[f]);
    const double fp = phi_prev[f];
    double k;
    if (e == 0.0) k = 1.0;
    else if (fp == 0.0) k = 0.0;
    else k = fmax(0.0, 1.0 - fabs(e) / fabs(fp));
    out[f] = rho * (k * c);
}

// Integrated non-pressure right-hand side b + V grad(p) (piso/main.cpp:194).
__global__ void kNonPressureRhs(int n, const double* __restrict__ src, const double* __restrict__ V,
                                const double* __restrict__ gradP, double* __restrict__ npr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) npr[3 * i + c] = src[3 * i + c] + V[i] * gradP[3 * i + c];
}

// HbyA = (1/aP) (npr - A U + aP U) (piso/main.cpp:208-209).
__global__ void kHbyA(int n, const double* __restrict__ aP, const double* __restrict__ npr,
                      const double* __restrict__ AU, const double* __restrict__ U, double* __restrict__ H) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a = aP[i], inv = 1.0 / a;
#pragma unroll
    for (int c = 0; c < 3; ++c) H[3 * i + c] = inv * (npr[3 * i + c] - AU[3 * i + c] + a * U[3 * i + c]);
}

// phiH += rAUf * temporalFlux on interior faces (piso/main.cpp:214).
__global__ void kAddInteriorProduct(int n_interior, const double* __restrict__ a, const double* __restrict__ b,
                                    double* __restrict__ out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < n_interior) out[f] += a[f] * b[f];
}

// ||npr||^2, ||A U||^2, ||V gradP||^2, ||npr - A U - V gradP||^2 (piso/main.cpp:243-248).
__global__ void kCouplingNorms(int n, const double* __restrict__ npr, const double* __restrict__ AU,
                               const double* __restrict__ V, const double* __restrict__ gradP,
                               double* __restrict__ partial) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (i < n) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double a = npr[3 * i + c], b = AU[3 * i + c], s = V[i] * gradP[3 * i + c];
            const double d = a - b - s;
            v[0] += a * a; v[1] += b * b; v[2] += s * s; v[3] += d * d;
        }
    }
    blockSum<4, kBlock>(v);
    if (threadIdx.x == 0)
        for (int j = 0; j < 4; ++j) partial[4 * blockIdx.x + j] = v[j];
}

// Courant number (fvm_execution.cpp:179-204): co = 0.5 dt sum|phi_f| / V per cell;
// partials: sum co V, sum V, max co.
__global__ void kCourant(MeshView m, const double* __restrict__ phi, double dt, double* __restrict__ partial) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    double v[2] = {0.0, 0.0};
    double mx = 0.0;
    if (i < m.n_cells) {
        double s = 0.0;
        for (int k = m.cf_ptr[i]; k < m.cf_ptr[i + 1]; ++k) s += fabs(phi[m.cf_face[k]]);
        for (int fb = m.cb_ptr[i]; fb < m.cb_ptr[i + 1]; ++fb) s += fabs(phi[m.n_interior + fb]);
        const double Vi = m.V[i];
        const double co = 0.5 * dt * s / Vi;
        v[0] = co * Vi;
        v[1] = Vi;
        mx = co;
    }
    blockSum<2, kBlock>(v);
    __shared__ double smax[kBlock / 32];
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int j = 0; j < kBlock / 32; ++j) r = fmax(r, smax[j]);
        partial[3 * blockIdx.x] = v[0];
        partial[3 * blockIdx.x + 1] = v[1];
        partial[3 * blockIdx.x + 2] = r;
    }
}

__global__ void kFinish(int blocks, int nv, unsigned max_mask, const double* __restrict__ partial,
                        double* __restrict__ result) {
    const int j = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (j >= nv) return;
    const bool is_max = (max_mask >> j) & 1u;
    double r = 0.0;
    for (int b = lane; b < blocks; b += 32) {
        const double p = partial[nv * b + j];
        r = is_max ? fmax(r, p) : r + p;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double q = __shfl_down_sync(0xffffffffu, r, o);
        r = is_max ? fmax(r, q) : r + q;
    }
    if (lane == 0) result[j] = r;
}

__global__ void kOwnerTraceP(MeshView m, const double* __restrict__ x, double* __restrict__ trace) {
    const int fb = blockIdx.x * blockDim.x + threadIdx.x;
    if (fb < m.n_boundary) trace[fb] = x[m.bown[fb]];
}

template <class K, class... A>
void launch(Context& ctx, K kernel, long long n, A... args) {
    kernel<<<gridFor(n, kBlock), kBlock, 0, ctx.stream>>>(args...);
    BSG_CUDA(cudaGetLastError());
    ctx.launched();
}

void copyBoundaries(DeviceField& dst, const DeviceField& src) {
    dst.bcs = src.bcs;
    dst.bcs_dirty = true;
}

}  // namespace

PisoSolver::PisoSolver(DeviceMesh& mesh, const PisoConfig& cfg)
    : m_(mesh), ctx_(*mesh.ctx), cfg_(cfg), U_(mesh, 0, 3), p_(mesh, 0, 1), phi_(mesh, 1, 1), muEff_(mesh, 0, 1),
      rAU_(mesh, 0, 1), rAUf_(mesh, 1, 1), HbyA_(mesh, 0, 3), phiH_(mesh, 1, 1), Uprev_lvl_(mesh, 0, 3),
      Uolder_lvl_(mesh, 0, 3), flux_field_(mesh, 1, 1), krylov_(*mesh.ctx) {
    if (!(cfg.rho > 0) || !(cfg.mu > 0)) fail(kArgument, "density and dynamicViscosity must be positive");
    if (!(cfg.alpha_u > 0 && cfg.alpha_u <= 1)) fail(kArgument, "velocityRelaxation must be in (0,1]");
    if (cfg.time_method != 1 && cfg.time_method != 2) fail(kArgument, "PISO requires a transient time scheme");
    if (cfg.correctors < 1 || cfg.correctors > 100 || cfg.max_correctors < cfg.correctors || cfg.max_correctors > 100)
        fail(kArgument, "nCorrectors must be in [1,100] and maxCorrectors in [nCorrectors,100]");
    if (cfg.max_iterations < 1) fail(kArgument, "maxIterations must be positive");
    if (cfg.non_orthogonal_corrections < 0 || cfg.non_orthogonal_corrections > 20)
        fail(kArgument, "nonOrthogonalCorrections must be in [0,20]");
    if (!(cfg.delta_t > 0) || !std::isfinite(cfg.delta_t) || !(cfg.end_time >= cfg.start_time) ||
        !std::isfinite(cfg.start_time) || !std::isfinite(cfg.end_time))
        fail(kArgument, "time control is invalid");
    std::vector<double> mu(mesh.n_cells, cfg.mu);
    muEff_.v.upload(mu, ctx_.stream);
    rAU_.calculated = true;
    rAU_.trace.resize(mesh.n_boundary);
    const std::size_t N = mesh.n_cells;
    for (DeviceArray<double>* a : {&Uiter_, &gradP_, &npr_, &AU_}) a->resize(3 * N);
    pprev_.resize(N);
    for (DeviceArray<double>* a : {&phi_prev_, &phi_older_, &temporal_}) a->resize(mesh.n_faces);
    flags_.resize(4);
    mom_ = std::make_unique<DeviceEquation>(U_, cfg.momentum);
    peq_ = std::make_unique<DeviceEquation>(p_, cfg.pressure);
    time_ = cfg.start_time;
    ctx_.sync();
}

PisoSolver::~PisoSolver() = default;

void PisoSolver::enableTurbulence(const KOmegaConfig& cfg, const PisoTurbulenceControls& controls) {
    if (started_) fail(kState, "the turbulence model must be chosen before the fields are set");
    if (controls.segregated && cfg_.max_iterations != 1)
        fail(kArgument, "segregated turbulence requires one PISO momentum pass");
    if (controls.segregated && cfg.relaxation != 1.0)
        fail(kArgument, "single-pass transient turbulence requires turbulenceRelaxation 1");
    if (controls.max_iterations < 1) fail(kArgument, "turbulenceMaxIterations must be at least 1");
    if (controls.segregated && controls.correctors > 1)
        fail(kArgument, "segregated turbulence requires one transport correction");
    if (controls.correctors > controls.max_iterations)
        fail(kArgument, "turbulenceCorrectors must not exceed turbulenceMaxIterations");
    KOmegaConfig c = cfg;
    c.rho = cfg_.rho;
    c.mu = cfg_.mu;
    c.momentum_options = cfg_.momentum;
    turb_ = std::make_unique<KOmegaModel>(m_, c);
    turb_->setTransient(cfg_.time_method);
    tctl_ = controls;
    divStress_.resize(3 * static_cast<std::size_t>(m_.n_cells));
}

void PisoSolver::initializePotentialFlow(int initial_non_orthogonal_corrections) {
    if (started_) fail(kState, "the potential-flow start must be chosen before the fields are set");
    // negative: the key is absent and nonOrthogonalCorrections applies; otherwise the reference's
    // range, settings.integer(..., 0, 20) (piso/main.cpp:89-90)
    if (initial_non_orthogonal_corrections > 20) fail(kArgument, "initialNonOrthogonalCorrections must be at most 20");
    potential_start_ = true;
    initial_non_orth_ = initial_non_orthogonal_corrections;
}

void PisoSolver::potentialFlowStart() {
    // piso/main.cpp:123-146: pPrime = homogeneousLike(p); solves of laplacian(1) pPrime = div(phi);
    // U -= grad(pPrime); phi += faceFlux(potential equation, pPrime)
    const int N = m_.n_cells;
    DeviceField pP(m_, 0, 1);
    for (int patch = 0; patch < m_.n_patches; ++patch) {
        const int t = p_.bcs[patch].type;
        const double zero[3] = {0, 0, 0};
        pP.setBoundary(patch, t == 0 ? 0 : (t == 4 ? 4 : 2), zero);
    }
    divFlux(phi_, divPhiH_);
    const int corr = initial_non_orth_ >= 0 ? initial_non_orth_ : cfg_.non_orthogonal_corrections;
    const int solves = cfg_.pressure.diffusion == 0 ? 1 : corr + 1;
    DeviceEquation eq(pP, cfg_.pressure);
    for (int k = 0; k < solves; ++k) {
        eq.reset();
        addLaplacian(eq, nullptr, 1.0, -1.0, cfg_.pressure);
        addSource(eq, divPhiH_.data(), -1.0);
        referenceIfUnanchored(eq, 0.0, flags_.data());
        Dcsr<double> P{N, m_.cf_ptr.data(), m_.cf_col.data(), eq.diag.data(), eq.val.data(), 2LL * m_.n_interior};
        if (auto* jac = dynamic_cast<JacobiPreconditioner*>(ppc_.get())) { jac->diag = eq.diag.data(); jac->n = N; }
        if (auto* amg = dynamic_cast<AmgPreconditioner*>(ppc_.get())) amg->update(P, k == 0);
        if (k == 0) preuse_.force_rebuild = true;   // the first time step's matrix needs its own hierarchy
        const SolveOutcome o = krylov_.solveScalar(P, cfg_.pressure_solver, ppc_.get(), eq.src.data(), pP.v.data());
        if (o.status != 0) fail(kNumeric, "the initial potential-flow solve did not converge");
    }
    gradient(pP, cfg_.pressure.gradient, gradP_);
    launch(ctx_, kSubtract, 3LL * N, 3LL * N, (const double*)gradP_.data(), U_.v.data());
    faceFluxEquation(eq, pP.v.data(), pflux_);
    addArrays(ctx_, phi_.v.data(), phi_.v.data(), pflux_.data(), m_.n_faces);
    U_.setFluxContext(phi_);
}

void PisoSolver::start() {
    if (turb_) {
        // rans::load runs while phi is still the zero face field it was created as (piso/main.cpp:62, 98)
        phi_.v.zero(ctx_.stream);
        turb_->start(phi_);
    }
    faceFlux(U_, cfg_.pressure.interpolation, cfg_.pressure.gradient, phi_);  // piso/main.cpp:122
    const int pcType = cfg_.pressure_solver.preconditioner;
    if (pcType == 2 || pcType == 3) ppc_ = std::make_unique<AmgPreconditioner>(m_, cfg_.pressure_solver);
    else ppc_ = std::make_unique<JacobiPreconditioner>();
    if (potential_start_) potentialFlowStart();
    // time::history(U), time::history(phi): both levels start as copies (history.h:8)
    for (DeviceField* h : {&Uprev_lvl_, &Uolder_lvl_}) {
        copyAsync(ctx_, h->v.data(), U_.v.data(), 3LL * m_.n_cells);
        copyBoundaries(*h, U_);
        h->setFluxContext(phi_);
    }
    copyBoundaries(HbyA_, U_);
    copyAsync(ctx_, phi_prev_.data(), phi_.v.data(), m_.n_faces);
    copyAsync(ctx_, phi_older_.data(), phi_.v.data(), m_.n_faces);
    levels_ = 0;
    dt_ = prev_dt_ = 0.0;
    time_ = cfg_.start_time;
    step_ = 0;
    report_ = PisoReport{};
    report_.time = time_;
    started_ = true;
    ctx_.sync();
}

void PisoSolver::saveHistory(double dt) {
    // History::save (history.h:10-15): older = previous; previous = field
    copyAsync(ctx_, Uolder_lvl_.v.data(), Uprev_lvl_.v.data(), 3LL * m_.n_cells);
    copyAsync(ctx_, Uprev_lvl_.v.data(), U_.v.data(), 3LL * m_.n_cells);
    copyAsync(ctx_, phi_older_.data(), phi_prev_.data(), m_.n_faces);
    copyAsync(ctx_, phi_prev_.data(), phi_.v.data(), m_.n_faces);
    prev_dt_ = dt_;
    dt_ = dt;
    ++levels_;
}

PisoReport PisoSolver::advance(int steps) {
    if (!started_) start();
    for (int k = 0; k < steps; ++k) {
        if (time_ >= cfg_.end_time) break;
        if (!step()) break;
    }
    report_.time = time_;
    report_.steps = step_;
    if (report_.status != 2 && report_.accepted) report_.status = time_ >= cfg_.end_time ? 0 : 1;
    return report_;
}

bool PisoSolver::step() {
    const int N = m_.n_cells;
    const MeshView mv = view(m_);
    // TimeStepper::advance (src/io/case.cpp:391-403)
    const double tol = 32 * std::numeric_limits<double>::epsilon() *
                       std::max({std::fabs(cfg_.start_time), std::fabs(cfg_.end_time), cfg_.delta_t});
    double next = static_cast<double>(static_cast<long double>(cfg_.start_time) +
                                      static_cast<long double>(step_ + 1) * cfg_.delta_t);
    if (next >= cfg_.end_time - tol) next = cfg_.end_time;
    const double dt = next - time_;
    if (!(dt > 0)) fail(kState, "time step is below representable time precision");
    time_ = next;
    ++step_;
    saveHistory(dt);
    if (turb_) turb_->saveOld(dt);
    // rho * temporalFluxCorrection(U_old, phi_old) (piso/main.cpp:164-165)
    {
        BSG_PROFILE(ctx_, "piso_temporal_flux");
        double w1 = 1.0 / dt, w2 = 0.0;
        if (cfg_.time_method == 2 && levels_ >= 2) {
            const double ratio = dt / prev_dt_;
            w1 = (1.0 + ratio) / dt;
            w2 = -ratio * ratio / ((1.0 + ratio) * dt);
        }
        faceFlux(Uprev_lvl_, cfg_.pressure.interpolation, cfg_.pressure.gradient, flux_field_);
        if (w2 != 0.0) {
            flux_tmp_.resize(m_.n_faces);
            copyAsync(ctx_, flux_tmp_.data(), flux_field_.v.data(), m_.n_faces);
            faceFlux(Uolder_lvl_, cfg_.pressure.interpolation, cfg_.pressure.gradient, flux_field_);
            launch(ctx_, kTemporalFlux, m_.n_faces, m_.n_interior, m_.n_faces, cfg_.rho, w1, w2,
                   (const double*)phi_prev_.data(), (const double*)flux_tmp_.data(),
                   (const double*)phi_older_.data(), (const double*)flux_field_.v.data(), temporal_.data());
        } else {
            launch(ctx_, kTemporalFlux, m_.n_faces, m_.n_interior, m_.n_faces, cfg_.rho, w1, w2,
                   (const double*)phi_prev_.data(), (const double*)flux_field_.v.data(),
                   (const double*)phi_older_.data(), (const double*)flux_field_.v.data(), temporal_.data());
        }
    }
    // BDF2 falls back to Euler until two levels exist (procedural_equation.cpp:225-231)
    const int method = (cfg_.time_method == 2 && levels_ < 2) ? 1 : cfg_.time_method;
    const TimeWeights tw = timeWeights(method, dt_, prev_dt_, true);
    const int pressure_solves = cfg_.pressure.diffusion == 0 ? 1 : cfg_.non_orthogonal_corrections + 1;
    double* h = ctx_.pinned;
    bool converged = false;
    for (int iter = 0; iter < cfg_.max_iterations; ++iter) {
        copyAsync(ctx_, Uiter_.data(), U_.v.data(), 3LL * N);
        DeviceEquation& mom = *mom_;
        {
            BSG_PROFILE(ctx_, "momentum_assembly");
            mom.reset();
            addTimeTerm(mom, nullptr, cfg_.rho, Uprev_lvl_.v.data(), Uolder_lvl_.v.data(), tw);
            addConvection(mom, phi_, cfg_.rho, cfg_.momentum);
            addLaplacian(mom, turb_ ? &turb_->effectiveViscosity() : &muEff_, 0.0, -1.0, cfg_.momentum);
            gradient(p_, cfg_.pressure.gradient, gradP_);
            addSource(mom, gradP_.data(), -1.0);
            if (turb_) {
                // explicit remainder of the eddy-viscosity stress (piso/main.cpp:178-180)
                turb_->stressRemainderDivergence(U_, divStress_.data());
                addSource(mom, divStress_.data(), 1.0);
            }
        }
        relativeResidualNorms(mom, U_.v.data(), redR_);
        relax(mom, Uiter_.data(), cfg_.alpha_u);
        ratioVolume(m_, mom.diag.data(), rAU_.v.data());
        launch(ctx_, kOwnerTraceP, m_.n_boundary, mv, (const double*)rAU_.v.data(), rAU_.trace.data());
        rAU_.bcs_dirty = true;
        interpolate(rAU_, cfg_.pressure.coefInterp(), cfg_.pressure.coefGrad(), rAUf_.v);
        launch(ctx_, kNonPressureRhs, N, N, (const double*)mom.src.data(), (const double*)m_.V.data(),
               (const double*)gradP_.data(), npr_.data());
        Dcsr<double> A{N, m_.cf_ptr.data(), m_.cf_col.data(), mom.diag.data(), mom.val.data(), 2LL * m_.n_interior};
        SolveOutcome uo[3];
        krylov_.solveVector3(A, cfg_.momentum_solver, mom.src.data(), U_.v.data(), uo);
        int mom_iters = 0;
        bool mom_ok = true;
        for (const auto& o : uo) {
            mom_iters += o.iterations;
            mom_ok = mom_ok && o.status == 0;
            if (o.status == 2 || !std::isfinite(o.final_)) { report_.status = 2; return false; }
        }
        report_.momentum_iterations = mom_iters;
        bool p_ok = true;
        int p_iters = 0;
        double dP = 0.0, coupling = 0.0;
        int used = 0;
        bool first_matrix = true;
        DeviceEquation& peq = *peq_;
        for (int corrector = 0; corrector < cfg_.max_correctors; ++corrector) {
            {
                BSG_PROFILE(ctx_, "piso_hbya_flux");
                applyEquation(mom, U_.v.data(), AU_.data());
                launch(ctx_, kHbyA, N, N, (const double*)mom.diag.data(), (const double*)npr_.data(),
                       (const double*)AU_.data(), (const double*)U_.v.data(), HbyA_.v.data());
                HbyA_.setFluxContext(phi_);
                copyAsync(ctx_, pprev_.data(), p_.v.data(), N);
                faceFlux(HbyA_, cfg_.pressure.interpolation, cfg_.pressure.gradient, phiH_);
                launch(ctx_, kAddInteriorProduct, m_.n_interior, m_.n_interior, (const double*)rAUf_.v.data(),
                       (const double*)temporal_.data(), phiH_.v.data());
                divFlux(phiH_, divPhiH_);
            }
            for (int corr = 0; corr < pressure_solves; ++corr) {
                {
                    BSG_PROFILE(ctx_, "pressure_assembly");
                    peq.reset();
                    addLaplacian(peq, &rAUf_, 0.0, -1.0, cfg_.pressure);
                    addSource(peq, divPhiH_.data(), -1.0);
                    referenceIfUnanchored(peq, 0.0, flags_.data());
                }
                Dcsr<double> P{N, m_.cf_ptr.data(), m_.cf_col.data(), peq.diag.data(), peq.val.data(),
                               2LL * m_.n_interior};
                if (auto* jac = dynamic_cast<JacobiPreconditioner*>(ppc_.get())) { jac->diag = peq.diag.data(); jac->n = N; }
                auto* amg = dynamic_cast<AmgPreconditioner*>(ppc_.get());
                bool lagged = false;
                if (amg) {
                    BSG_PROFILE(ctx_, "amg_numeric_setup");
                    // one matrix per time step (rAUf is frozen), lagged across steps like the reference
                    amg->update(P, preuse_.needRebuild(first_matrix, cfg_.pressure_solver));
                    lagged = preuse_.lagged();
                }
                first_matrix = false;
                SolveOutcome po = krylov_.solveScalar(P, cfg_.pressure_solver, ppc_.get(), peq.src.data(), p_.v.data());
                int attempt = po.iterations;
                if (amg && lagged && po.status != 0) {
                    {
                        BSG_PROFILE(ctx_, "amg_numeric_setup");
                        amg->update(P, true);
                    }
                    preuse_.rebuilt();
                    const int first = po.iterations;
                    po = krylov_.solveScalar(P, cfg_.pressure_solver, ppc_.get(), peq.src.data(), p_.v.data());
                    attempt = po.iterations;
                    po.iterations += first;
                }
                if (amg) preuse_.afterSolve(po.status, attempt, po.iterations, cfg_.pressure_solver);
                if (po.status == 2 || !std::isfinite(po.final_)) { report_.status = 2; return false; }
                p_ok = p_ok && po.status == 0;
                p_iters += po.iterations;
            }
            BSG_PROFILE(ctx_, "piso_corrector_updates");
            // phi = phiH + faceFlux(p); U = HbyA - rAU grad(p) (piso/main.cpp:231-237)
            faceFluxEquation(peq, p_.v.data(), pflux_);
            addArrays(ctx_, phi_.v.data(), phiH_.v.data(), pflux_.data(), m_.n_faces);
            gradient(p_, cfg_.pressure.gradient, gradP_);
            copyAsync(ctx_, U_.v.data(), HbyA_.v.data(), 3LL * N);
            subtractScaledGradient(m_, U_.v.data(), rAU_.v.data(), gradP_.data());
            U_.setFluxContext(phi_);
            relativeChangeNorms(ctx_, p_.v.data(), pprev_.data(), N, redP_);
            applyEquation(mom, U_.v.data(), AU_.data());
            const int blocks = static_cast<int>(gridFor(N, kBlock));
            redC_.ensure(blocks, 4);
            launch(ctx_, kCouplingNorms, N, N, (const double*)npr_.data(), (const double*)AU_.data(),
                   (const double*)m_.V.data(), (const double*)gradP_.data(), redC_.partial.data());
            kFinish<<<1, 32 * 4, 0, ctx_.stream>>>(blocks, 4, 0u, redC_.partial.data(), redC_.result.data());
            BSG_CUDA(cudaGetLastError());
            ctx_.launched();
            BSG_CUDA(cudaMemcpyAsync(h + 0, redP_.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
            BSG_CUDA(cudaMemcpyAsync(h + 2, redC_.result.data(), 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
            ctx_.sync();
            dP = std::max(dP, std::sqrt(h[0]) / std::max(std::sqrt(h[1]), 1e-30));
            const double n0 = std::sqrt(h[2]), n1 = std::sqrt(h[3]), n2 = std::sqrt(h[4]), n3 = std::sqrt(h[5]);
            const double scale = n0 + n1 + n2;
            coupling = scale > 0.0 ? n3 / scale : n3;
            used = corrector + 1;
            if (used >= cfg_.correctors && coupling <= cfg_.coupling_tolerance) break;
        }
        report_.pressure_iterations = p_iters;
        report_.correctors = used;
        // turbulence correctors at this time level (piso/main.cpp:239-254)
        bool turb_converged = true, turb_linear = true;
        report_.turbulence_corrections = 0;
        if (turb_) {
            const int corrections = tctl_.correctors > 0 ? tctl_.correctors
                                    : (cfg_.max_iterations == 1 && !tctl_.segregated ? tctl_.max_iterations : 1);
            for (int c = 0; c < corrections; ++c) {
                const TransportResult tr = turb_->solveTransport(U_, phi_);
                ++report_.turbulence_corrections;
                report_.turbulence_change = tr.change;
                report_.turbulence_residual = tr.residual;
                if (!(tr.healthy && std::isfinite(tr.change) && std::isfinite(tr.residual))) {
                    report_.status = 2;
                    return false;
                }
                turb_linear = tr.linear_converged;
                turb_converged = turb_linear && tr.change <= turb_->config().tolerance &&
                                 tr.residual <= turb_->config().tolerance;
                if (!turb_linear || turb_converged) break;
            }
        }
        // diagnostics (piso/main.cpp:266-281)
        relativeChangeNorms(ctx_, U_.v.data(), Uiter_.data(), 3LL * N, redU_);
        fluxBalance(m_, phi_.v.data(), redM_);
        {
            const int blocks = static_cast<int>(gridFor(N, kBlock));
            redCo_.ensure(blocks, 3);
            launch(ctx_, kCourant, N, mv, (const double*)phi_.v.data(), dt_, redCo_.partial.data());
            kFinish<<<1, 32 * 3, 0, ctx_.stream>>>(blocks, 3, 0x4u, redCo_.partial.data(), redCo_.result.data());
            BSG_CUDA(cudaGetLastError());
            ctx_.launched();
        }
        BSG_CUDA(cudaMemcpyAsync(h + 0, redR_.result.data(), 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
        BSG_CUDA(cudaMemcpyAsync(h + 4, redU_.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
        BSG_CUDA(cudaMemcpyAsync(h + 6, redM_.result.data(), 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
        BSG_CUDA(cudaMemcpyAsync(h + 10, redCo_.result.data(), 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
        ctx_.sync();
        const double rU = std::sqrt(h[0]) / std::max(std::sqrt(h[1]) + std::sqrt(h[2]), 1e-30);
        const double dU = std::sqrt(h[4]) / std::max(std::sqrt(h[5]), 1e-30);
        const double mass = h[6] / std::max(h[8], 1e-30);
        report_.rU = rU;
        report_.dU = dU;
        report_.dP = dP;
        report_.mass = mass;
        report_.coupling = coupling;
        report_.courant_mean = h[10] / h[11];
        report_.courant_max = h[12];
        if (!(std::isfinite(rU) && std::isfinite(dU) && std::isfinite(dP) && std::isfinite(coupling) &&
              std::isfinite(mass))) {
            report_.status = 2;
            return false;
        }
        const bool linear_ok = mom_ok && p_ok && turb_linear;
        const bool accepted = linear_ok && mass <= cfg_.mass_tolerance && coupling <= cfg_.coupling_tolerance;
        const bool settled = rU <= cfg_.momentum_tolerance && dU <= cfg_.velocity_tolerance &&
                             dP <= cfg_.pressure_tolerance && turb_converged;
        converged = accepted && (cfg_.max_iterations == 1 ? (tctl_.segregated || turb_converged) : settled);
        report_.accepted = accepted;
        if (!accepted) { report_.status = 1; return false; }
        if (converged) break;
    }
    if (!converged) { report_.status = 1; report_.accepted = false; return false; }
    return true;
}

}  // namespace bsg
