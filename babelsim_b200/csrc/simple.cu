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

// Per case of a batch: cleared when one of its faces is non-orthogonal by Mesh::polyhedral's
// test (|k| > 1e-12 |Sf|, or for an interior face |skew| > 1e-12 |d|; the host geometry's
// criterion), so each case gets the orthogonal flag its own mesh would have.
__global__ void kCaseOrthogonal(MeshView m, const int* __restrict__ case_of, int* __restrict__ orth) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < m.n_interior) {
        const double k0 = m.kvec[3 * f], k1 = m.kvec[3 * f + 1], k2 = m.kvec[3 * f + 2];
        bool ortho = !(sqrt(k0 * k0 + k1 * k1 + k2 * k2) > 1e-12 * m.area[f]);
        const int o = m.own[f], n = m.nbr[f];
        const double d0 = m.xc[3 * n] - m.xc[3 * o], d1 = m.xc[3 * n + 1] - m.xc[3 * o + 1],
                     d2 = m.xc[3 * n + 2] - m.xc[3 * o + 2];
        const double s0 = m.skew[3 * f], s1 = m.skew[3 * f + 1], s2 = m.skew[3 * f + 2];
        if (sqrt(s0 * s0 + s1 * s1 + s2 * s2) > 1e-12 * sqrt(d0 * d0 + d1 * d1 + d2 * d2)) ortho = false;
        if (!ortho) atomicAnd(orth + case_of[o], 0);
    } else if (f < m.n_interior + m.n_boundary) {
        const int fb = f - m.n_interior;
        const double k0 = m.bk[3 * fb], k1 = m.bk[3 * fb + 1], k2 = m.bk[3 * fb + 2];
        if (sqrt(k0 * k0 + k1 * k1 + k2 * k2) > 1e-12 * m.barea[fb]) atomicAnd(orth + case_of[m.bown[fb]], 0);
    }
}

__global__ void kCellOrthogonal(int n, const int* __restrict__ case_of, const int* __restrict__ orth,
                                unsigned char* __restrict__ cell) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) cell[i] = orth[case_of[i]] ? 1 : 0;
}

// Traces of a calculated cell field whose constraints are the default
// zeroGradient ones: the owner value (geometry.cpp values(), field.h:264-272).
__global__ void kOwnerTrace(MeshView m, const double* __restrict__ x, double* __restrict__ trace) {
    const int fb = blockIdx.x * blockDim.x + threadIdx.x;
    if (fb < m.n_boundary) trace[fb] = x[m.bown[fb]];
}

}  // namespace

// One case of a batch (see SimpleSolver::setSegments).
struct SimpleSegment {
    int c0 = 0, n = 0;           // cells [c0, c0 + n)
    int fi0 = 0, nfi = 0;        // interior faces in the device order (sorted by owner)
    int fb0 = 0, nfb = 0;        // boundary faces in the device order (sorted by owner)
    long long slot0 = 0, nslot = 0;  // off-diagonal matrix slots [slot0, slot0 + nslot)
    DeviceArray<int> ptr, col;   // the case's cell->face pattern with local numbering
    std::unique_ptr<KrylovSolver> mom, pres;
    std::unique_ptr<AmgPreconditioner> amg;
    PcReusePolicy preuse;
    Reducer red, redU, redPP, redP, redM;
    SimpleReport report;
    bool frozen = false;         // converged: its state is kept while the others continue
    DeviceArray<double> keepU, keepP, keepPhi;
    // the case's rows of a matrix assembled on the whole mesh, in local numbering
    Dcsr<double> view(const double* diag, const double* val) const {
        return Dcsr<double>{n, ptr.data(), col.data(), diag + c0, val + slot0, nslot};
    }
};

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

SimpleSolver::~SimpleSolver() {
    if (seg_pinned_) cudaFreeHost(seg_pinned_);
}

void SimpleSolver::setSegments(const std::vector<int>& off, const std::vector<double>& viscosity) {
    if (started_) fail(kState, "segments must be set before the fields");
    if (turb_) fail(kArgument, "batched cases are laminar");
    const int K = static_cast<int>(off.size()) - 1;
    if (K < 1 || static_cast<int>(viscosity.size()) != K || off.front() != 0 || off.back() != m_.n_cells)
        fail(kArgument, "segment offsets must run from 0 to the cell count, one viscosity per segment");
    if (K > 4096) fail(kArgument, "at most 4096 segments");
    for (int k = 0; k < K; ++k) {
        if (off[k + 1] <= off[k]) fail(kArgument, "every segment needs at least one cell");
        if (!(viscosity[k] > 0.0) || !std::isfinite(viscosity[k])) fail(kArgument, "segment viscosity must be positive");
    }
    std::vector<int> seg_of(m_.n_cells);
    for (int k = 0; k < K; ++k)
        for (int i = off[k]; i < off[k + 1]; ++i) seg_of[i] = k;
    for (int f = 0; f < m_.n_interior; ++f)
        if (seg_of[m_.h_own[f]] != seg_of[m_.h_nbr[f]])
            fail(kArgument, "an interior face connects two segments: segments must be independent meshes");
    std::vector<double> mu(m_.n_cells);
    segs_.clear();
    int fi = 0, fb = 0;
    for (int k = 0; k < K; ++k) {
        auto sg = std::make_unique<SimpleSegment>();
        sg->c0 = off[k];
        sg->n = off[k + 1] - off[k];
        sg->fi0 = fi;
        while (fi < m_.n_interior && m_.h_own[fi] < off[k + 1]) ++fi;  // interior faces are sorted by owner
        sg->nfi = fi - sg->fi0;
        sg->fb0 = fb;
        while (fb < m_.n_boundary && m_.h_bown[fb] < off[k + 1]) ++fb;
        sg->nfb = fb - sg->fb0;
        sg->slot0 = m_.h_cf_ptr[off[k]];
        sg->nslot = m_.h_cf_ptr[off[k + 1]] - sg->slot0;
        std::vector<int> ptr(sg->n + 1), col(std::max<long long>(sg->nslot, 1));
        for (int i = 0; i <= sg->n; ++i) ptr[i] = static_cast<int>(m_.h_cf_ptr[off[k] + i] - sg->slot0);
        for (long long q = 0; q < sg->nslot; ++q) col[q] = m_.h_cf_col[sg->slot0 + q] - off[k];
        sg->ptr.upload(ptr, ctx_.stream);
        sg->col.upload(col, ctx_.stream);
        sg->mom = std::make_unique<KrylovSolver>(ctx_);
        sg->pres = std::make_unique<KrylovSolver>(ctx_);
        for (int i = off[k]; i < off[k + 1]; ++i) mu[i] = viscosity[k];
        segs_.push_back(std::move(sg));
    }
    muEff_.v.upload(mu, ctx_.stream);
    if (!seg_pinned_) BSG_CUDA(cudaMallocHost(reinterpret_cast<void**>(&seg_pinned_), sizeof(double) * 16 * 4096));
    // the second Green-Gauss pass follows each case's own orthogonality, not the batch mesh's
    if (!m_.h_cell_perm.empty())
        for (int k = 0; k < K; ++k)
            for (int i = off[k]; i < off[k + 1]; ++i)
                if (m_.h_cell_perm[i] < off[k] || m_.h_cell_perm[i] >= off[k + 1])
                    fail(kArgument, "segments must keep their cell ranges: each case must be one connected mesh");
    m_.cell_orth.release();
    if (!m_.orthogonal) {
        DeviceArray<int> d_case, d_orth;
        d_case.upload(seg_of, ctx_.stream);
        std::vector<int> ones(K, 1);
        d_orth.upload(ones, ctx_.stream);
        kCaseOrthogonal<<<gridFor(static_cast<long long>(m_.n_interior) + m_.n_boundary, kBlock), kBlock, 0,
                          ctx_.stream>>>(view(m_), d_case.data(), d_orth.data());
        m_.cell_orth.resize(m_.n_cells);
        kCellOrthogonal<<<gridFor(m_.n_cells, kBlock), kBlock, 0, ctx_.stream>>>(m_.n_cells, d_case.data(),
                                                                                 d_orth.data(), m_.cell_orth.data());
        BSG_CUDA(cudaGetLastError());
        ctx_.launches += 2;
        ctx_.sync();
    }
    ctx_.sync();
}

const SimpleReport& SimpleSolver::segmentReport(int k) const {
    if (k < 0 || k >= static_cast<int>(segs_.size())) fail(kArgument, "segment index out of range");
    return segs_[k]->report;
}

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
    U_.uploadExternal(U);
    p_.uploadExternal(p);
    // phi arrives in the caller's face numbering; the device keeps interior faces first.
    phi_.uploadExternal(phi);
}

SimpleReport SimpleSolver::iterate(int max_iterations) {
    if (!started_) start();
    for (int k = 0; k < max_iterations; ++k) {
        if (segs_.empty()) outerIteration();
        else outerIterationSegments();
        if (report_.converged || report_.status == 2) break;
    }
    return report_;
}

// outerIteration for a mesh of several independent cases: the same steps in the same order,
// with the per-case parts (momentum solve, gauge, pressure solves, diagnostics, convergence)
// done per segment and the pressure solves of all segments batched in one launch per attempt.
void SimpleSolver::outerIterationSegments() {
    const int N = m_.n_cells;
    const int K = static_cast<int>(segs_.size());
    const MeshView mv = view(m_);
    copyAsync(ctx_, Uprev_.data(), U_.v.data(), 3LL * N);
    DeviceEquation& mom = *mom_;
    {
        BSG_PROFILE(ctx_, "momentum_assembly");
        mom.reset();
        addConvection(mom, phi_, cfg_.rho, cfg_.momentum);
        addLaplacian(mom, &muEff_, 0.0, -1.0, cfg_.momentum);
        gradient(p_, cfg_.pressure.gradient, gradP_);
        addSource(mom, gradP_.data(), -1.0);
    }
    for (auto& sg : segs_) relativeResidualNorms(mom, U_.v.data(), sg->red, sg->c0, sg->n);
    relax(mom, Uprev_.data(), cfg_.alpha_u);
    scale(mom, cfg_.alpha_u);
    ratioVolume(m_, mom.diag.data(), rAU_.v.data());
    kOwnerTrace<<<gridFor(m_.n_boundary, kBlock), kBlock, 0, ctx_.stream>>>(mv, rAU_.v.data(), rAU_.trace.data());
    ctx_.launched();
    // momentum: each active case on its own rows
    std::vector<int> mom_ok(K, 1), p_ok(K, 1), mom_its(K, 0), p_its(K, 0);
    std::vector<double> linP(K, 0.0);
    bool failed = false;
    {
        // BiCGStab (kspType bcgs) in FP64: every active case's momentum system in one persistent
        // launch per attempt; other Krylov types, and FP32 inner iterations with FP64 refinement
        // (precision 1), solve case by case
        std::vector<BicgItem> items;
        std::vector<int> which;
        for (int k = 0; k < K; ++k) {
            SimpleSegment& sg = *segs_[k];
            if (sg.frozen) continue;
            const Dcsr<double> A = sg.view(mom.diag.data(), mom.val.data());
            if (cfg_.momentum_solver.solver == 1 && cfg_.momentum_solver.precision != 1) {
                BicgItem it;
                it.solver = sg.mom.get();
                it.A = A;
                it.b = mom.src.data() + 3LL * sg.c0;
                it.x = U_.v.data() + 3LL * sg.c0;
                it.cfg = cfg_.momentum_solver;
                items.push_back(it);
                which.push_back(k);
                continue;
            }
            SolveOutcome uo[3];
            sg.mom->solveVector3(A, cfg_.momentum_solver, mom.src.data() + 3LL * sg.c0, U_.v.data() + 3LL * sg.c0, uo);
            for (const auto& o : uo) {
                mom_its[k] += o.iterations;
                mom_ok[k] = mom_ok[k] && o.status == 0;
                if (o.status == 2 || !std::isfinite(o.final_)) failed = true;
            }
        }
        KrylovSolver::solveVector3Batch(ctx_, items, true);
        for (std::size_t q = 0; q < items.size(); ++q)
            for (const auto& o : items[q].out) {
                const int k = which[q];
                mom_its[k] += o.iterations;
                mom_ok[k] = mom_ok[k] && o.status == 0;
                if (o.status == 2 || !std::isfinite(o.final_)) failed = true;
            }
    }
    if (failed) { report_.status = 2; return; }
    {
        BSG_PROFILE(ctx_, "rhie_chow_flux");
        faceFlux(U_, cfg_.momentum.interpolation, cfg_.momentum.gradient, phiH_);
        kRhieChow<<<gridFor(m_.n_interior, kBlock), kBlock, 0, ctx_.stream>>>(
            mv, p_.bcView(), rAU_.v.data(), gradP_.data(), p_.v.data(), cfg_.pressure.diffusion, phiH_.v.data());
        ctx_.launched();
        divFlux(phiH_, divPhiH_);
    }
    BSG_CUDA(cudaMemsetAsync(pP_.v.data(), 0, sizeof(double) * N, ctx_.stream));
    const int pressure_solves = cfg_.pressure.diffusion == 0 ? 1 : cfg_.non_orthogonal_corrections + 1;
    DeviceEquation& peq = *peq_;
    const int pcType = cfg_.pressure_solver.preconditioner;
    if (!(pcType == 2 || pcType == 3) || cfg_.pressure_solver.solver != 0 || cfg_.pressure_solver.precision == 1)
        fail(kArgument, "batched cases solve the pressure with CG and the AMG preconditioner (FP64 or FP32 V-cycle)");
    if (flags_.size() < static_cast<std::size_t>(2 * K)) flags_.resize(2 * K);
    for (int corr = 0; corr < pressure_solves; ++corr) {
        {
            BSG_PROFILE(ctx_, "pressure_assembly");
            peq.reset();
            addLaplacian(peq, &rAU_, 0.0, -1.0, cfg_.pressure);
            addSource(peq, divPhiH_.data(), -1.0);
            for (int k = 0; k < K; ++k)
                referenceIfUnanchored(peq, 0.0, flags_.data() + 2 * k, segs_[k]->c0, segs_[k]->n);
        }
        std::vector<BatchSolve> items;
        std::vector<int> which;
        std::vector<bool> lagged(K, false);
        {
            BSG_PROFILE(ctx_, "amg_numeric_setup");
            for (int k = 0; k < K; ++k) {
                SimpleSegment& sg = *segs_[k];
                if (sg.frozen) continue;
                const Dcsr<double> P = sg.view(peq.diag.data(), peq.val.data());
                if (!sg.amg) sg.amg = std::make_unique<AmgPreconditioner>(m_, cfg_.pressure_solver);
                sg.amg->update(P, sg.preuse.needRebuild(corr == 0, cfg_.pressure_solver));
                lagged[k] = sg.preuse.lagged();
                BatchSolve b;
                b.solver = sg.pres.get();
                b.amg = sg.amg.get();
                b.A = P;
                b.b = peq.src.data() + sg.c0;
                b.x = pP_.v.data() + sg.c0;
                b.cfg = cfg_.pressure_solver;
                items.push_back(b);
                which.push_back(k);
            }
        }
        KrylovSolver::solveBatch(ctx_, items);
        for (std::size_t q = 0; q < items.size(); ++q) {
            const int k = which[q];
            SimpleSegment& sg = *segs_[k];
            SolveOutcome po = items[q].out;
            int attempt = po.iterations;
            if (lagged[k] && po.status != 0) {
                // a failed lagged solve is retried once with a fresh preconditioner
                const Dcsr<double> P = sg.view(peq.diag.data(), peq.val.data());
                sg.amg->update(P, true);
                sg.preuse.rebuilt();
                const int first = po.iterations;
                po = sg.pres->solveScalar(P, cfg_.pressure_solver, sg.amg.get(), peq.src.data() + sg.c0,
                                          pP_.v.data() + sg.c0);
                attempt = po.iterations;
                po.iterations += first;
            }
            sg.preuse.afterSolve(po.status, attempt, po.iterations, cfg_.pressure_solver);
            if (po.status == 2 || !std::isfinite(po.final_)) failed = true;
            p_ok[k] = p_ok[k] && po.status == 0;
            p_its[k] += po.iterations;
            linP[k] = po.relative;
        }
        if (failed) { report_.status = 2; return; }
    }
    axpyCell(ctx_, p_.v.data(), cfg_.alpha_p, pP_.v.data(), N);
    BSG_PROFILE(ctx_, "field_updates_diagnostics");
    faceFluxEquation(peq, pP_.v.data(), pflux_);
    gradient(pP_, cfg_.pressure.gradient, gradPP_);
    subtractScaledGradient(m_, U_.v.data(), rAU_.v.data(), gradPP_.data());
    addArrays(ctx_, phi_.v.data(), phiH_.v.data(), pflux_.data(), m_.n_faces);
    for (auto& sg : segs_) {
        relativeChangeNorms(ctx_, U_.v.data() + 3LL * sg->c0, Uprev_.data() + 3LL * sg->c0, 3LL * sg->n, sg->redU);
        relativeChangeNorms(ctx_, pP_.v.data() + sg->c0, nullptr, sg->n, sg->redPP);
        relativeChangeNorms(ctx_, p_.v.data() + sg->c0, nullptr, sg->n, sg->redP);
        fluxBalance(m_, phi_.v.data(), sg->redM, sg->c0, sg->n);
    }
    double* h = seg_pinned_;
    for (int k = 0; k < K; ++k) {
        SimpleSegment& sg = *segs_[k];
        double* hk = h + 16 * k;
        BSG_CUDA(cudaMemcpyAsync(hk + 0, sg.red.result.data(), 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
        BSG_CUDA(cudaMemcpyAsync(hk + 4, sg.redU.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
        BSG_CUDA(cudaMemcpyAsync(hk + 6, sg.redPP.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
        BSG_CUDA(cudaMemcpyAsync(hk + 8, sg.redP.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
        BSG_CUDA(cudaMemcpyAsync(hk + 10, sg.redM.result.data(), 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
    }
    ctx_.sync();
    bool bad = false;
    int total_mom = 0, total_p = 0;
    const std::size_t Fi = m_.n_interior;
    for (int k = 0; k < K; ++k) {
        SimpleSegment& sg = *segs_[k];
        if (sg.frozen) {
            // keep the converged state: the batch's update touched these cells and faces too
            copyAsync(ctx_, U_.v.data() + 3LL * sg.c0, sg.keepU.data(), 3LL * sg.n);
            copyAsync(ctx_, p_.v.data() + sg.c0, sg.keepP.data(), sg.n);
            copyAsync(ctx_, phi_.v.data() + sg.fi0, sg.keepPhi.data(), sg.nfi);
            copyAsync(ctx_, phi_.v.data() + Fi + sg.fb0, sg.keepPhi.data() + sg.nfi, sg.nfb);
            continue;
        }
        const double* hk = h + 16 * k;
        SimpleReport& r = sg.report;
        r.momentum_iterations = mom_its[k];
        r.pressure_iterations = p_its[k];
        r.linP = linP[k];
        r.rU = std::sqrt(hk[0]) / std::max(std::sqrt(hk[1]) + std::sqrt(hk[2]), 1e-30);
        r.dU = std::sqrt(hk[4]) / std::max(std::sqrt(hk[5]), 1e-30);
        r.dP = std::sqrt(hk[6]) / std::max(std::sqrt(hk[9]), 1e-30);
        r.mass = hk[10] / std::max(hk[12], 1e-30);
        r.iterations += 1;
        total_mom += mom_its[k];
        total_p += p_its[k];
        if (!(std::isfinite(r.rU) && std::isfinite(r.dU) && std::isfinite(r.dP) && std::isfinite(r.mass))) {
            r.status = 2;
            bad = true;
            continue;
        }
        r.converged = mom_ok[k] && p_ok[k] && r.rU <= cfg_.momentum_tolerance && r.dU <= cfg_.velocity_tolerance &&
                      r.dP <= cfg_.pressure_tolerance && r.mass <= cfg_.mass_tolerance;
        r.status = r.converged ? 0 : 1;
        if (r.converged) {
            sg.frozen = true;
            sg.keepU.resize(3 * static_cast<std::size_t>(sg.n));
            sg.keepP.resize(sg.n);
            sg.keepPhi.resize(std::max<std::size_t>(static_cast<std::size_t>(sg.nfi) + sg.nfb, 1));
            copyAsync(ctx_, sg.keepU.data(), U_.v.data() + 3LL * sg.c0, 3LL * sg.n);
            copyAsync(ctx_, sg.keepP.data(), p_.v.data() + sg.c0, sg.n);
            copyAsync(ctx_, sg.keepPhi.data(), phi_.v.data() + sg.fi0, sg.nfi);
            copyAsync(ctx_, sg.keepPhi.data() + sg.nfi, phi_.v.data() + Fi + sg.fb0, sg.nfb);
        }
    }
    bool all = true;
    for (auto& sg : segs_) all = all && sg->frozen;
    report_.iterations += 1;
    report_.momentum_iterations = total_mom;
    report_.pressure_iterations = total_p;
    report_.converged = all;
    report_.status = bad ? 2 : (all ? 0 : 1);
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
