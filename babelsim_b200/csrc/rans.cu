// Eddy-viscosity model transport on the device: k-omega, k-epsilon, Spalart-Allmaras (see rans.h).
#include "bsg_device.cuh"
#include "rans.h"

#include <cmath>

namespace bsg {
namespace {
constexpr int kBlock = 256;

template <class K, class... A>
void launch(Context& ctx, K kernel, long long n, A... args) {
    kernel<<<gridFor(n, kBlock), kBlock, 0, ctx.stream>>>(args...);
    BSG_CUDA(cudaGetLastError());
    ctx.launched();
}

__global__ void kBoundK(int n, double k_min, double* __restrict__ k) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) k[i] = fmax(k[i], k_min);
}

// omega = max(omega, omegaMin, rho k / (ratioMax mu)) (k_omega.cpp:140-150)
__global__ void kBoundOmega(int n, double omega_min, double rho, double ratio_mu, const double* __restrict__ k,
                            double* __restrict__ w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) w[i] = fmax(w[i], fmax(omega_min, rho * k[i] / ratio_mu));
}

// mut = rho k / max(omega, omegaMin), muEff = mu + mut on cells (k_omega.cpp:153-156)
__global__ void kViscosity(int n, double rho, double mu, double omega_min, const double* __restrict__ k,
                           const double* __restrict__ w, double* __restrict__ mut, double* __restrict__ mueff) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = (rho * k[i]) / fmax(w[i], omega_min);
    mut[i] = v;
    mueff[i] = v + mu;
}

// the same expressions on the boundary traces of k and omega (field.h:302-320)
__global__ void kViscosityTrace(MeshView m, BcView bk, BcView bw, const double* __restrict__ k,
                                const double* __restrict__ w, double rho, double mu, double omega_min,
                                double* __restrict__ mut_tr, double* __restrict__ mueff_tr) {
    const int fb = blockIdx.x * blockDim.x + threadIdx.x;
    if (fb >= m.n_boundary) return;
    double kt[1], wt[1];
    boundaryTrace<1>(m, bk, k, fb, NAN, kt);
    boundaryTrace<1>(m, bw, w, fb, NAN, wt);
    const double v = (rho * kt[0]) / fmax(wt[0], omega_min);
    mut_tr[fb] = v;
    mueff_tr[fb] = v + mu;
}

// 2 dev(symm G) : dev(symm G) (k_omega.cpp:11-23); G row c = gradient of component c
__device__ __forceinline__ double strainSquared(const double* G) {
    const double div = G[0] + G[4] + G[8];
    double sum = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double s = 0.5 * (G[3 * i + j] + G[3 * j + i]) - (i == j ? div / 3.0 : 0.0);
            sum += s * s;
        }
    return 2.0 * sum;
}

// Frozen transport coefficients of one solveTransport (k_omega.cpp:75-81).
__global__ void kTransportCoefficients(int n, double rho, double mu, double beta, double gamma, double sigma_k,
                                       double sigma_w, double k_min, const double* __restrict__ G,
                                       const double* __restrict__ mut, const double* __restrict__ k,
                                       const double* __restrict__ w, double* __restrict__ production,
                                       double* __restrict__ kdiff, double* __restrict__ wdiff,
                                       double* __restrict__ wdestruction, double* __restrict__ wproduction) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double p = mut[i] * strainSquared(G + 9 * i);
    production[i] = p;
    kdiff[i] = sigma_k * mut[i] + mu;
    wdiff[i] = sigma_w * mut[i] + mu;
    wdestruction[i] = (beta * rho) * w[i];
    wproduction[i] = ((gamma * p) * w[i]) / fmax(k[i], k_min);
}

// k-epsilon: mut = Cmu rho k k / max(epsilon, epsilonMin) on cells and boundary traces (k_epsilon.cpp:122-125)
__global__ void kViscosityKE(int n, double crho, double mu, double eps_min, const double* __restrict__ k,
                             const double* __restrict__ e, double* __restrict__ mut, double* __restrict__ mueff) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = ((crho * k[i]) * k[i]) / fmax(e[i], eps_min);
    mut[i] = v;
    mueff[i] = v + mu;
}

__global__ void kViscosityTraceKE(MeshView m, BcView bk, BcView be, const double* __restrict__ k,
                                  const double* __restrict__ e, double crho, double mu, double eps_min,
                                  double* __restrict__ mut_tr, double* __restrict__ mueff_tr) {
    const int fb = blockIdx.x * blockDim.x + threadIdx.x;
    if (fb >= m.n_boundary) return;
    double kt[1], et[1];
    boundaryTrace<1>(m, bk, k, fb, NAN, kt);
    boundaryTrace<1>(m, be, e, fb, NAN, et);
    const double v = ((crho * kt[0]) * kt[0]) / fmax(et[0], eps_min);
    mut_tr[fb] = v;
    mueff_tr[fb] = v + mu;
}

// Frozen k-epsilon coefficients (k_epsilon.cpp:70-77): production, diffusivities mu + mut/sigma,
// k sink rho eps/k, epsilon sink C2 rho eps/k, epsilon source C1 P eps/k.
__global__ void kTransportCoefficientsKE(int n, double rho, double mu, double c1, double c2, double inv_sk,
                                         double inv_se, double k_min, const double* __restrict__ G,
                                         const double* __restrict__ mut, const double* __restrict__ k,
                                         const double* __restrict__ e, double* __restrict__ production,
                                         double* __restrict__ kdiff, double* __restrict__ ediff,
                                         double* __restrict__ ksink, double* __restrict__ esink,
                                         double* __restrict__ eproduction) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double p = mut[i] * strainSquared(G + 9 * i);
    production[i] = p;
    kdiff[i] = inv_sk * mut[i] + mu;
    ediff[i] = inv_se * mut[i] + mu;
    const double eok = e[i] / fmax(k[i], k_min);
    ksink[i] = rho * eok;
    esink[i] = (c2 * rho) * eok;
    eproduction[i] = (c1 * p) * eok;
}

__global__ void kBoundMin(int n, double lo, double* __restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = fmax(x[i], lo);
}

__global__ void kDiffusivityTrace(int nb, double mu, double sigma_k, double sigma_w, const double* __restrict__ mut_tr,
                                  double* __restrict__ kdiff_tr, double* __restrict__ wdiff_tr) {
    const int fb = blockIdx.x * blockDim.x + threadIdx.x;
    if (fb >= nb) return;
    kdiff_tr[fb] = sigma_k * mut_tr[fb] + mu;
    wdiff_tr[fb] = sigma_w * mut_tr[fb] + mu;
}

// ---- Spalart-Allmaras (spalart_allmaras.cpp)
struct SaConstants {
    double rho, mu, nu, cb1, cb2, sigma, kappa2, cw1, cw2, cw3_6, cv1, ct3, ct4, dmin;
};

// fv1 = chi^3 / (chi^3 + cv1^3) (spalart_allmaras.cpp:125-130)
__device__ __forceinline__ double saFv1(double chi, double cv1) {
    const double c3 = (chi * chi) * chi;
    return c3 / (c3 + (cv1 * cv1) * cv1);
}

// mut = rho nuTilda fv1(nuTilda / nu), muEff = mu + mut on cells (:137-140)
__global__ void kViscositySA(int n, SaConstants c, const double* __restrict__ nt, double* __restrict__ mut,
                             double* __restrict__ mueff) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = (c.rho * nt[i]) * saFv1(nt[i] / c.nu, c.cv1);
    mut[i] = v;
    mueff[i] = v + c.mu;
}

// the same on the boundary trace of nuTilda (mut_tr, mueff_tr), and/or the transport diffusivity
// (mu + rho nuTilda) / sigma there (diff_tr); a null output is skipped
__global__ void kTraceSA(MeshView m, BcView bn, const double* __restrict__ nt, SaConstants c,
                         double* __restrict__ mut_tr, double* __restrict__ mueff_tr, double* __restrict__ diff_tr) {
    const int fb = blockIdx.x * blockDim.x + threadIdx.x;
    if (fb >= m.n_boundary) return;
    double t[1];
    boundaryTrace<1>(m, bn, nt, fb, NAN, t);
    if (mut_tr) {
        const double v = (c.rho * t[0]) * saFv1(t[0] / c.nu, c.cv1);
        mut_tr[fb] = v;
        mueff_tr[fb] = v + c.mu;
    }
    if (diff_tr) diff_tr[fb] = (c.mu + c.rho * t[0]) / c.sigma;
}

// Closure functions at the current iterate and the frozen coefficients of the nuTilda equation
// (:69-103): implicit destruction rho max(-a, 0), explicit source rho max(a, 0) nuTilda + rho cb2 /
// sigma |grad nuTilda|^2 with a = production - destruction rate, diffusivity (mu + rho nuTilda) / sigma.
// G row c = gradient of velocity component c; gn = gradient of nuTilda.
__global__ void kCoefficientsSA(int n, SaConstants c, const double* __restrict__ G, const double* __restrict__ gn,
                                const double* __restrict__ ntv, const double* __restrict__ dist,
                                double* __restrict__ implicit, double* __restrict__ explicit_src,
                                double* __restrict__ diff) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double nt = ntv[i];
    const double chi = nt / c.nu;
    const double fv1 = saFv1(chi, c.cv1);
    const double fv2 = 1.0 - chi / (1.0 + chi * fv1);
    const double ft2 = c.ct3 * exp(((-c.ct4) * chi) * chi);
    const double d = fmax(dist[i], c.dmin);
    const double inv_d2 = 1.0 / (d * d);
    const double* g = G + 9 * i;
    double sum = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const double rot = 0.5 * (g[3 * a + b] - g[3 * b + a]);
            sum += rot * rot;
        }
    const double rotation = sqrt(2.0 * sum);
    const double mod_rot = fmax(rotation + ((nt * fv2) * inv_d2) / c.kappa2, 1e-30);
    double r = (nt * inv_d2) / (c.kappa2 * mod_rot);
    r = r < 0.0 ? 0.0 : (10.0 < r ? 10.0 : r);
    const double gg = r + c.cw2 * (pow(r, 6.0) - r);
    const double fw = gg * pow((1.0 + c.cw3_6) / (pow(gg, 6.0) + c.cw3_6), 1.0 / 6.0);
    const double production = (c.cb1 * (1.0 - ft2)) * mod_rot;
    const double destruction = ((c.cw1 * fw - (c.cb1 / c.kappa2) * ft2) * nt) * inv_d2;
    const double net = production - destruction;
    implicit[i] = c.rho * fmax(-net, 0.0);
    const double* q = gn + 3 * i;
    const double grad_source = ((c.rho * c.cb2) / c.sigma) * (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    explicit_src[i] = (c.rho * fmax(net, 0.0)) * nt + grad_source;
    diff[i] = (c.mu + c.rho * nt) / c.sigma;
}

__global__ void kScaled(int n, double a, const double* __restrict__ x, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a * x[i];
}

// Boundary traces of grad(U) (fvm_execution.cpp:240-262): symmetry reflects the
// tensor, otherwise each component's normal derivative takes its constraint.
__global__ void kVectorGradientTrace(MeshView m, BcView bu, const double* __restrict__ U,
                                     const double* __restrict__ G, double* __restrict__ Gtr) {
    const int fb = blockIdx.x * blockDim.x + threadIdx.x;
    if (fb >= m.n_boundary) return;
    const int o = m.bown[fb];
    const double n[3] = {m.bn[3 * fb], m.bn[3 * fb + 1], m.bn[3 * fb + 2]};
    const double d[3] = {m.bxf[3 * fb] - m.xc[3 * o], m.bxf[3 * fb + 1] - m.xc[3 * o + 1],
                         m.bxf[3 * fb + 2] - m.xc[3 * o + 2]};
    double g[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) g[e] = G[9 * o + e];
    double val[3];
    const int t = faceCondition<3>(m, bu, fb, NAN, val);
    if (t == SY) {
        // 0.5 (g + R g R), R = I - 2 n n^T (include/babelsim/vector.h:107-116)
        double R[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) R[3 * i + j] = (i == j ? 1.0 : 0.0) - 2 * n[i] * n[j];
        double r[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) s += R[3 * i + kk] * g[3 * kk + l] * R[3 * l + j];
                r[3 * i + j] = s;
            }
#pragma unroll
        for (int e = 0; e < 9; ++e) g[e] = 0.5 * (g[e] + r[e]);
    } else {
        const double dn = d[0] * n[0] + d[1] * n[1] + d[2] * n[2];
        const double tg[3] = {d[0] - dn * n[0], d[1] - dn * n[1], d[2] - dn * n[2]};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double* gc = g + 3 * c;
            double sn = 0.0;
            if (t == FV) sn = (val[c] - U[3 * o + c] - (gc[0] * tg[0] + gc[1] * tg[1] + gc[2] * tg[2])) / dn;
            else if (t == FG) sn = val[c];
            const double k = sn - (gc[0] * n[0] + gc[1] * n[1] + gc[2] * n[2]);
            gc[0] += k * n[0];
            gc[1] += k * n[1];
            gc[2] += k * n[2];
        }
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) Gtr[9 * fb + e] = g[e];
}

// muEff (G^T - 2/3 tr(G) I) (model.cpp:65-69); `count` tensors, one mu each.
__global__ void kStressRemainder(int count, const double* __restrict__ G, const double* __restrict__ mueff,
                                 double* __restrict__ T) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const double* g = G + 9 * i;
    const double tr = g[0] + g[4] + g[8];
    const double m = mueff[i];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) T[9 * i + 3 * c + d] = m * (g[3 * d + c] - (c == d ? (2.0 / 3.0) * tr : 0.0));
}

// divergence(TensorField) with linear row reconstruction (operators.cpp:1568-1591), gathered per cell.
__global__ void kTensorDivergence(MeshView m, const double* __restrict__ T, const double* __restrict__ Ttr,
                                  double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n_cells) return;
    const double V = m.V[i];
    double acc[3] = {0.0, 0.0, 0.0};
    for (int s = m.cf_ptr[i]; s < m.cf_ptr[i + 1]; ++s) {
        const int f = m.cf_face[s];
        const int o = m.own[f], nb = m.nbr[f];
        const double w = m.w[f];
        const double* S = m.Sf + 3 * f;
        const bool owner = o == i;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double fv[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) fv[d] = w * T[9 * o + 3 * c + d] + (1.0 - w) * T[9 * nb + 3 * c + d];
            const double q = (fv[0] * S[0] + fv[1] * S[1] + fv[2] * S[2]) / V;
            acc[c] = owner ? acc[c] + q : acc[c] - q;
        }
    }
    for (int fb = m.cb_ptr[i]; fb < m.cb_ptr[i + 1]; ++fb) {
        const double* S = m.bSf + 3 * fb;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double* t = Ttr + 9 * fb + 3 * c;
            acc[c] += (t[0] * S[0] + t[1] * S[1] + t[2] * S[2]) / V;
        }
    }
    out[3 * i] = acc[0];
    out[3 * i + 1] = acc[1];
    out[3 * i + 2] = acc[2];
}

void makeCalculated(DeviceField& f, int n_boundary) {
    f.calculated = true;
    f.trace.resize(static_cast<std::size_t>(n_boundary) * f.comps);
}

SaConstants saConstants(const KOmegaConfig& k) {
    SaConstants c;
    c.rho = k.rho;
    c.mu = k.mu;
    c.nu = k.mu / k.rho;
    c.cb1 = k.sa_cb1;
    c.cb2 = k.sa_cb2;
    c.sigma = k.sa_sigma;
    c.kappa2 = k.sa_kappa * k.sa_kappa;
    c.cw1 = k.sa_cw1 > 0.0 ? k.sa_cw1 : k.sa_cb1 / (k.sa_kappa * k.sa_kappa) + (1.0 + k.sa_cb2) / k.sa_sigma;
    c.cw2 = k.sa_cw2;
    c.cw3_6 = std::pow(k.sa_cw3, 6.0);
    c.cv1 = k.sa_cv1;
    c.ct3 = k.sa_ct3;
    c.ct4 = k.sa_ct4;
    c.dmin = k.wall_distance_min;
    return c;
}

}  // namespace

KOmegaModel::KOmegaModel(DeviceMesh& mesh, const KOmegaConfig& cfg)
    : m_(mesh), ctx_(*mesh.ctx), cfg_(cfg), k_(mesh, 0, 1), omega_(mesh, 0, 1), mut_(mesh, 0, 1), muEff_(mesh, 0, 1),
      kDiff_(mesh, 0, 1), wDiff_(mesh, 0, 1), krylov_(*mesh.ctx) {
    if (!(cfg.rho > 0) || !(cfg.mu > 0)) fail(kArgument, "density and dynamicViscosity must be positive");
    if (cfg.kind < 0 || cfg.kind > 2) fail(kArgument, "unknown turbulence model");
    if (cfg.kind == 2)
        for (double v : {cfg.sa_cb1, cfg.sa_cb2, cfg.sa_sigma, cfg.sa_kappa, cfg.sa_cw2, cfg.sa_cw3, cfg.sa_cv1,
                         cfg.sa_ct3, cfg.sa_ct4, cfg.wall_distance_min})
            if (!(v > 0) || !std::isfinite(v)) fail(kArgument, "Spalart-Allmaras constants and bounds must be positive and finite");
    for (double v : {cfg.beta_star, cfg.beta, cfg.gamma, cfg.sigma_k, cfg.sigma_omega, cfg.k_min, cfg.omega_min,
                     cfg.viscosity_ratio_max, cfg.tolerance, cfg.c_mu, cfg.c1, cfg.c2})
        if (!(v > 0) || !std::isfinite(v)) fail(kArgument, "turbulence model constants and bounds must be positive and finite");
    if (!(cfg.relaxation > 0 && cfg.relaxation <= 1)) fail(kArgument, "turbulenceRelaxation must be in (0,1]");
    if (cfg.momentum_options.interpolation != 0)
        fail(kArgument, "the device stress-remainder divergence reconstructs the tensor rows linearly");
    const int nb = mesh.n_boundary;
    for (DeviceField* f : {&mut_, &muEff_, &kDiff_, &wDiff_}) makeCalculated(*f, nb);
    const std::size_t N = mesh.n_cells;
    G_.resize(9 * N);
    T_.resize(9 * N);
    Gtr_.resize(9 * static_cast<std::size_t>(std::max(nb, 1)));
    Ttr_.resize(9 * static_cast<std::size_t>(std::max(nb, 1)));
    for (DeviceArray<double>* a : {&production_, &wDestruction_, &wProduction_, &kSink_, &prevK_, &prevW_}) a->resize(N);
    keq_ = std::make_unique<DeviceEquation>(k_, cfg.k_options);
    weq_ = std::make_unique<DeviceEquation>(omega_, cfg.omega_options);
    if (cfg.kind == 2) {
        wallDist_.resize(N);
        gradNt_.resize(3 * N);
    }
}

void KOmegaModel::setTransient(int method) {
    if (method != 1 && method != 2) fail(kArgument, "transient turbulence needs the Euler or BDF2 time scheme");
    time_method_ = method;
    const std::size_t N = m_.n_cells;
    for (DeviceArray<double>* a : {&wPrevLvl_, &wOlderLvl_}) { a->resize(N); a->zero(ctx_.stream); }
    if (cfg_.kind != 2)
        for (DeviceArray<double>* a : {&kPrevLvl_, &kOlderLvl_}) { a->resize(N); a->zero(ctx_.stream); }
    tdt_ = tprev_dt_ = 0.0;
    tlevels_ = 0;
}

void KOmegaModel::saveOld(double dt) {
    // History::save for each transported field (k_omega.cpp:58-62, k_epsilon.cpp:57-60, spalart_allmaras.cpp:61-63)
    const int N = m_.n_cells;
    copyAsync(ctx_, wOlderLvl_.data(), wPrevLvl_.data(), N);
    copyAsync(ctx_, wPrevLvl_.data(), omega_.v.data(), N);
    if (cfg_.kind != 2) {
        copyAsync(ctx_, kOlderLvl_.data(), kPrevLvl_.data(), N);
        copyAsync(ctx_, kPrevLvl_.data(), k_.v.data(), N);
    }
    tprev_dt_ = tdt_;
    tdt_ = dt;
    ++tlevels_;
}

void KOmegaModel::timeTerm(DeviceEquation& eq, const DeviceArray<double>& previous, const DeviceArray<double>& older) {
    if (!time_method_) return;
    // BDF2 starts as Euler until two levels exist (procedural_equation.cpp:225-231)
    const int method = (time_method_ == 2 && tlevels_ < 2) ? 1 : time_method_;
    addTimeTerm(eq, nullptr, cfg_.rho, previous.data(), older.data(), timeWeights(method, tdt_, tprev_dt_, true));
}

void KOmegaModel::setWallDistance(const double* host) {
    if (cfg_.kind != 2) fail(kState, "a wall distance belongs to the Spalart-Allmaras model");
    for (int i = 0; i < m_.n_cells; ++i)
        if (!std::isfinite(host[i])) fail(kNumeric, "wall distance must be finite");
    wallDist_.resize(m_.n_cells);
    uploadCells(m_, wallDist_.data(), host, 1);
    wall_set_ = true;
}

KOmegaModel::~KOmegaModel() = default;

void KOmegaModel::boundOmega() {
    const int N = m_.n_cells;
    if (cfg_.kind >= 1) {  // epsilon = max(epsilon, epsilonMin) (k_epsilon.cpp:118), nuTilda likewise (:132-135)
        launch(ctx_, kBoundMin, N, N, cfg_.omega_min, omega_.v.data());
        return;
    }
    launch(ctx_, kBoundOmega, N, N, cfg_.omega_min, cfg_.rho, cfg_.viscosity_ratio_max * cfg_.mu,
           (const double*)k_.v.data(), omega_.v.data());
}

void KOmegaModel::updateViscosity() {
    const int N = m_.n_cells;
    if (cfg_.kind == 2) {
        const SaConstants c = saConstants(cfg_);
        launch(ctx_, kViscositySA, N, N, c, (const double*)omega_.v.data(), mut_.v.data(), muEff_.v.data());
        if (m_.n_boundary)
            launch(ctx_, kTraceSA, m_.n_boundary, view(m_), omega_.bcView(), (const double*)omega_.v.data(), c,
                   mut_.trace.data(), muEff_.trace.data(), (double*)nullptr);
        return;
    }
    if (cfg_.kind == 1) {
        const double crho = cfg_.c_mu * cfg_.rho;
        launch(ctx_, kViscosityKE, N, N, crho, cfg_.mu, cfg_.omega_min, (const double*)k_.v.data(),
               (const double*)omega_.v.data(), mut_.v.data(), muEff_.v.data());
        if (m_.n_boundary)
            launch(ctx_, kViscosityTraceKE, m_.n_boundary, view(m_), k_.bcView(), omega_.bcView(),
                   (const double*)k_.v.data(), (const double*)omega_.v.data(), crho, cfg_.mu, cfg_.omega_min,
                   mut_.trace.data(), muEff_.trace.data());
        return;
    }
    launch(ctx_, kViscosity, N, N, cfg_.rho, cfg_.mu, cfg_.omega_min, (const double*)k_.v.data(),
           (const double*)omega_.v.data(), mut_.v.data(), muEff_.v.data());
    if (m_.n_boundary)
        launch(ctx_, kViscosityTrace, m_.n_boundary, view(m_), k_.bcView(), omega_.bcView(),
               (const double*)k_.v.data(), (const double*)omega_.v.data(), cfg_.rho, cfg_.mu, cfg_.omega_min,
               mut_.trace.data(), muEff_.trace.data());
}

void KOmegaModel::start(const DeviceField& phi) {
    if (cfg_.kind == 2) {
        // boundTransportField(); updateViscosity() (spalart_allmaras.cpp:50-56)
        if (!wall_set_) fail(kState, "the Spalart-Allmaras model needs the wall distance before the fields are set");
        omega_.setFluxContext(phi);
        boundOmega();
        updateViscosity();
        return;
    }
    // boundTransportFields() then updateViscosity() (k_omega.cpp:51-56, 130-136)
    k_.setFluxContext(phi);
    omega_.setFluxContext(phi);
    launch(ctx_, kBoundK, m_.n_cells, m_.n_cells, cfg_.k_min, k_.v.data());
    boundOmega();
    updateViscosity();
}

void KOmegaModel::gradientWithTraces(DeviceField& U) {
    gradient(U, cfg_.momentum_options.gradient, G_);
    if (m_.n_boundary)
        launch(ctx_, kVectorGradientTrace, m_.n_boundary, view(m_), U.bcView(), (const double*)U.v.data(),
               (const double*)G_.data(), Gtr_.data());
}

void KOmegaModel::stressRemainderDivergence(DeviceField& U, double* out) {
    gradientWithTraces(U);
    const int N = m_.n_cells, nb = m_.n_boundary;
    launch(ctx_, kStressRemainder, N, N, (const double*)G_.data(), (const double*)muEff_.v.data(), T_.data());
    if (nb) launch(ctx_, kStressRemainder, nb, nb, (const double*)Gtr_.data(), (const double*)muEff_.trace.data(), Ttr_.data());
    launch(ctx_, kTensorDivergence, N, view(m_), (const double*)T_.data(), (const double*)Ttr_.data(), out);
}

TransportResult KOmegaModel::solveTransport(DeviceField& U, DeviceField& phi) {
    if (cfg_.kind == 2) return solveSpalartAllmaras(U, phi);
    BSG_PROFILE(ctx_, "komega_transport");
    const int N = m_.n_cells, nb = m_.n_boundary;
    TransportResult res;
    copyAsync(ctx_, prevK_.data(), k_.v.data(), N);
    copyAsync(ctx_, prevW_.data(), omega_.v.data(), N);
    U.setFluxContext(phi);
    updateViscosity();
    gradient(U, cfg_.momentum_options.gradient, G_);
    const bool ke = cfg_.kind == 1;
    if (ke) {
        launch(ctx_, kTransportCoefficientsKE, N, N, cfg_.rho, cfg_.mu, cfg_.c1, cfg_.c2, 1.0 / cfg_.sigma_k,
               1.0 / cfg_.sigma_omega, cfg_.k_min, (const double*)G_.data(), (const double*)mut_.v.data(),
               (const double*)k_.v.data(), (const double*)omega_.v.data(), production_.data(), kDiff_.v.data(),
               wDiff_.v.data(), kSink_.data(), wDestruction_.data(), wProduction_.data());
        if (nb) launch(ctx_, kDiffusivityTrace, nb, nb, cfg_.mu, 1.0 / cfg_.sigma_k, 1.0 / cfg_.sigma_omega,
                       (const double*)mut_.trace.data(), kDiff_.trace.data(), wDiff_.trace.data());
    } else {
        launch(ctx_, kTransportCoefficients, N, N, cfg_.rho, cfg_.mu, cfg_.beta, cfg_.gamma, cfg_.sigma_k,
               cfg_.sigma_omega, cfg_.k_min, (const double*)G_.data(), (const double*)mut_.v.data(),
               (const double*)k_.v.data(), (const double*)omega_.v.data(), production_.data(), kDiff_.v.data(),
               wDiff_.v.data(), wDestruction_.data(), wProduction_.data());
        if (nb) launch(ctx_, kDiffusivityTrace, nb, nb, cfg_.mu, cfg_.sigma_k, cfg_.sigma_omega,
                       (const double*)mut_.trace.data(), kDiff_.trace.data(), wDiff_.trace.data());
    }
    double* h = ctx_.pinned;
    auto solveOne = [&](DeviceEquation& eq, DeviceField& x, DeviceField& diff, const double* sink, const double* src,
                        const double* previous, const SolverConfig& scfg, Reducer& red, double& r0,
                        const DeviceArray<double>& hprev, const DeviceArray<double>& holder) {
        eq.reset();
        timeTerm(eq, hprev, holder);
        addConvection(eq, phi, cfg_.rho, eq.options);
        addLaplacian(eq, &diff, 0.0, -1.0, eq.options);
        addReaction(eq, sink, 0.0, 1.0);
        addSource(eq, src, 1.0);
        relativeResidualNorms(eq, x.v.data(), red);
        BSG_CUDA(cudaMemcpyAsync(h, red.result.data(), 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
        ctx_.sync();
        r0 = std::sqrt(h[0]) / std::max(std::sqrt(h[1]) + std::sqrt(h[2]), 1e-30);
        relax(eq, previous, cfg_.relaxation);
        Dcsr<double> A{N, m_.cf_ptr.data(), m_.cf_col.data(), eq.diag.data(), eq.val.data(), 2LL * m_.n_interior};
        JacobiPreconditioner jac;
        jac.diag = eq.diag.data();
        jac.n = N;
        const SolveOutcome o = krylov_.solveScalar(A, scfg, &jac, eq.src.data(), x.v.data());
        res.iterations += o.iterations;
        res.linear_converged = res.linear_converged && o.status == 0;
        res.healthy = res.healthy && o.status != 2 && std::isfinite(o.final_) && std::isfinite(r0);
    };
    double rW = 0.0, rK = 0.0;
    if (ke) {
        // k first, then epsilon, one frozen closure state (k_epsilon.cpp:79-103)
        solveOne(*keq_, k_, kDiff_, kSink_.data(), production_.data(), prevK_.data(), cfg_.k_solver, redK_, rK,
                 kPrevLvl_, kOlderLvl_);
        if (!res.healthy) return res;
        solveOne(*weq_, omega_, wDiff_, wDestruction_.data(), wProduction_.data(), prevW_.data(), cfg_.omega_solver,
                 redW_, rW, wPrevLvl_, wOlderLvl_);
        if (!res.healthy) return res;
    } else {
        // omega first, then k with the new omega in its sink (k_omega.cpp:83-110)
        solveOne(*weq_, omega_, wDiff_, wDestruction_.data(), wProduction_.data(), prevW_.data(), cfg_.omega_solver,
                 redW_, rW, wPrevLvl_, wOlderLvl_);
        if (!res.healthy) return res;
        boundOmega();
        launch(ctx_, kScaled, N, N, cfg_.beta_star * cfg_.rho, (const double*)omega_.v.data(), kSink_.data());
        solveOne(*keq_, k_, kDiff_, kSink_.data(), production_.data(), prevK_.data(), cfg_.k_solver, redK_, rK,
                 kPrevLvl_, kOlderLvl_);
        if (!res.healthy) return res;
    }
    // boundTransportFields(); updateViscosity() (k_omega.cpp:114-116)
    k_.setFluxContext(phi);
    omega_.setFluxContext(phi);
    launch(ctx_, kBoundK, N, N, cfg_.k_min, k_.v.data());
    boundOmega();
    updateViscosity();
    relativeChangeNorms(ctx_, omega_.v.data(), prevW_.data(), N, redDW_);
    relativeChangeNorms(ctx_, k_.v.data(), prevK_.data(), N, redDK_);
    BSG_CUDA(cudaMemcpyAsync(h, redDW_.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
    BSG_CUDA(cudaMemcpyAsync(h + 2, redDK_.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
    ctx_.sync();
    const double dW = std::sqrt(h[0]) / std::max(std::sqrt(h[1]), 1e-30);
    const double dK = std::sqrt(h[2]) / std::max(std::sqrt(h[3]), 1e-30);
    res.change = std::max(dW, dK);
    res.residual = std::max(rW, rK);
    res.healthy = res.healthy && std::isfinite(res.change);
    return res;
}

// SpalartAllmaras::solveTransport, steady (spalart_allmaras.cpp:65-122): closure functions at the
// current iterate, one nuTilda equation (convection, diffusion, implicit destruction, explicit
// source), relaxation, solve, bounding, viscosity update.
TransportResult KOmegaModel::solveSpalartAllmaras(DeviceField& U, DeviceField& phi) {
    BSG_PROFILE(ctx_, "sa_transport");
    const int N = m_.n_cells, nb = m_.n_boundary;
    TransportResult res;
    copyAsync(ctx_, prevW_.data(), omega_.v.data(), N);
    U.setFluxContext(phi);
    const SaConstants c = saConstants(cfg_);
    gradient(U, cfg_.momentum_options.gradient, G_);
    gradient(omega_, cfg_.omega_options.gradient, gradNt_);
    launch(ctx_, kCoefficientsSA, N, N, c, (const double*)G_.data(), (const double*)gradNt_.data(),
           (const double*)omega_.v.data(), (const double*)wallDist_.data(), wDestruction_.data(),
           wProduction_.data(), wDiff_.v.data());
    if (nb)
        launch(ctx_, kTraceSA, nb, view(m_), omega_.bcView(), (const double*)omega_.v.data(), c, (double*)nullptr,
               (double*)nullptr, wDiff_.trace.data());
    DeviceEquation& eq = *weq_;
    eq.reset();
    timeTerm(eq, wPrevLvl_, wOlderLvl_);
    addConvection(eq, phi, cfg_.rho, eq.options);
    addLaplacian(eq, &wDiff_, 0.0, -1.0, eq.options);
    addReaction(eq, wDestruction_.data(), 0.0, 1.0);
    addSource(eq, wProduction_.data(), 1.0);
    relativeResidualNorms(eq, omega_.v.data(), redW_);
    double* h = ctx_.pinned;
    BSG_CUDA(cudaMemcpyAsync(h, redW_.result.data(), 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
    ctx_.sync();
    const double r0 = std::sqrt(h[0]) / std::max(std::sqrt(h[1]) + std::sqrt(h[2]), 1e-30);
    relax(eq, prevW_.data(), cfg_.relaxation);
    Dcsr<double> A{N, m_.cf_ptr.data(), m_.cf_col.data(), eq.diag.data(), eq.val.data(), 2LL * m_.n_interior};
    JacobiPreconditioner jac;
    jac.diag = eq.diag.data();
    jac.n = N;
    const SolverConfig& scfg = cfg_.omega_solver;
    const SolveOutcome o = krylov_.solveScalar(A, scfg, &jac, eq.src.data(), omega_.v.data());
    res.iterations = o.iterations;
    res.linear_converged = o.status == 0;
    res.residual = r0;
    res.healthy = o.status != 2 && std::isfinite(o.final_) && std::isfinite(r0);
    if (!res.healthy) return res;
    omega_.setFluxContext(phi);
    boundOmega();
    updateViscosity();
    relativeChangeNorms(ctx_, omega_.v.data(), prevW_.data(), N, redDW_);
    BSG_CUDA(cudaMemcpyAsync(h, redDW_.result.data(), 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx_.stream));
    ctx_.sync();
    res.change = std::sqrt(h[0]) / std::max(std::sqrt(h[1]), 1e-30);
    res.healthy = std::isfinite(res.change);
    return res;
}

}  // namespace bsg
