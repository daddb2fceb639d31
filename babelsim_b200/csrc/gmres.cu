// Restarted GMRES(m) and FGMRES(m) on sm_100a, right-preconditioned, for the
// reference's kspType gmres / fgmres (KSPGMRES / KSPFGMRES,
// src/backend/petsc_linear_system.cpp:43-50).
//
// Arnoldi with classical Gram-Schmidt applied twice (CGS2): every projection is
// one multi-vector dot kernel (each block reads w once against up to eight basis
// vectors, fixed-order two-stage sums) and one multi-vector update kernel, so a
// basis of m = 30 vectors costs O(m) full-vector passes per step and no host
// loop over vectors.  The (m+1) x m Hessenberg matrix and its Givens rotations
// live on the host: each Arnoldi step reads back its column (a few dozen
// doubles), which also gives the residual estimate |g_{j+1}| of the right-
// preconditioned residual, i.e. the true unpreconditioned residual in exact
// arithmetic.  FGMRES keeps the preconditioned directions z_j = M^-1 v_j and
// updates x with them, so a preconditioner that changes between applications
// (an AMG V-cycle in lower precision) stays correct.
//
// Acceptance is the reference's contract: the true residual ||b - A x|| is
// checked after the Krylov loop; if it misses max(atol, rtol max(||r0||, ||b||))
// the loop continues from x with a halved internal target, at most three times
// (petsc_linear_system.cpp:355-481).
#include "bsg_device.cuh"
#include "linalg.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace bsg {
namespace {

constexpr int kBlock = 256;
constexpr int kDots = 8;  // basis vectors per dot launch

// partial[b * kDots + j] = block b's share of dot(V_j, w), j < k.
__global__ void kMultiDot(int n, const double* __restrict__ V, long long ldv, int k, const double* __restrict__ w,
                          double* __restrict__ partial) {
    double acc[kDots];
#pragma unroll
    for (int j = 0; j < kDots; ++j) acc[j] = 0.0;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        const double wi = w[i];
#pragma unroll
        for (int j = 0; j < kDots; ++j)
            if (j < k) acc[j] += V[j * ldv + i] * wi;
    }
    blockSum<kDots, kBlock>(acc);
    if (threadIdx.x == 0)
        for (int j = 0; j < kDots; ++j) partial[kDots * blockIdx.x + j] = acc[j];
}

// out[j] = sum over blocks of partial[.][j], one warp, fixed order.
__global__ void kFinishDots(int blocks, int k, const double* __restrict__ partial, double* __restrict__ out) {
    const int lane = threadIdx.x;
    for (int j = 0; j < k; ++j) {
        double x = 0.0;
        for (int b = lane; b < blocks; b += 32) x += partial[kDots * b + j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) out[j] = x;
    }
}

// out += sign * sum_j c[j] V_j over k vectors (c in device memory).
__global__ void kMultiAxpy(int n, const double* __restrict__ V, long long ldv, int k, const double* __restrict__ c,
                           double sign, double* __restrict__ out) {
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        double s = 0.0;
        for (int j = 0; j < k; ++j) s += c[j] * V[j * ldv + i];
        out[i] += sign * s;
    }
}

__global__ void kAddTo(int n, const double* __restrict__ d, double* __restrict__ x) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < n) x[i] += d[i];
}

__global__ void kScaleInto(int n, const double* __restrict__ w, double scale, double* __restrict__ v) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < n) v[i] = w[i] * scale;
}

// Component c of an interleaved C-component vector <-> a contiguous vector.
__global__ void kComponent(int n, int C, int c, const double* __restrict__ in, double* __restrict__ out, int gather) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= n) return;
    if (gather) out[i] = in[C * i + c];
    else out[C * i + c] = in[i];
}

int dotGrid(Context& ctx, int n) {
    const long long g = (static_cast<long long>(n) + kBlock - 1) / kBlock;
    return static_cast<int>(std::max<long long>(1, std::min<long long>(g, 4LL * ctx.sm_count)));
}

// out[0..k) = V_j . w in device memory (chunks of kDots vectors per launch).
void multiDot(Context& ctx, GmresWorkspace& ws, int n, const double* V, long long ldv, int k, const double* w,
              double* out) {
    const int g = dotGrid(ctx, n);
    for (int j0 = 0; j0 < k; j0 += kDots) {
        const int kk = std::min(kDots, k - j0);
        kMultiDot<<<g, kBlock, 0, ctx.stream>>>(n, V + j0 * ldv, ldv, kk, w, ws.partial.data());
        kFinishDots<<<1, 32, 0, ctx.stream>>>(g, kk, ws.partial.data(), out + j0);
        ctx.launches += 2;
    }
    BSG_CUDA(cudaGetLastError());
}

}  // namespace

void GmresWorkspace::ensure(int n, int m, bool flexible) {
    const std::size_t need = static_cast<std::size_t>(m + 1) * n;
    if (V.size() < need) V.resize(need);
    if (flexible && Z.size() < static_cast<std::size_t>(m) * n) Z.resize(static_cast<std::size_t>(m) * n);
    for (DeviceArray<double>* a : {&w, &r, &zt, &bc, &xc})
        if (a->size() < static_cast<std::size_t>(n)) a->resize(n);
    if (partial.size() < static_cast<std::size_t>(kDots) * 4096) partial.resize(static_cast<std::size_t>(kDots) * 4096);
    if (coef.size() < static_cast<std::size_t>(m + 2)) coef.resize(m + 2);
}

SolveOutcome gmresSolve(Context& ctx, GmresWorkspace& ws, const Dcsr<double>& A, const SolverConfig& cfg,
                        Preconditioner* pc, const double* b, double* x) {
    const int n = A.n;
    const bool flexible = cfg.solver == 3;
    // the pinned read-back buffer (64 doubles) holds two projections of at most 31 coefficients
    const int m = std::max(1, std::min({ws.restart, cfg.max_iterations, 30}));
    ws.ensure(n, m, flexible);
    const long long ld = n;
    double* V = ws.V.data();
    double* hdev = ws.coef.data();
    double* hpin = ctx.pinned;
    const unsigned g = gridFor(n, kBlock);
    const int ag = dotGrid(ctx, n);
    BSG_PROFILE(ctx, "gmres");
    SolveOutcome out;
    multiDot(ctx, ws, n, b, 0, 1, b, hdev);
    BSG_CUDA(cudaMemcpyAsync(hpin, hdev, sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    const double bnorm = std::sqrt(hpin[0]);
    if (!cfg.warm_start) BSG_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, ctx.stream));
    const double r0 = cfg.warm_start ? trueResidualNorm(ctx, A, b, x, ws.r.data()) : bnorm;
    out.initial = r0;
    const double scale = std::max(r0, bnorm) > 0.0 ? std::max(r0, bnorm) : 1.0;
    const double target = std::max(cfg.atol, cfg.rtol * scale);
    out.checks = 1;
    if (std::isfinite(r0) && r0 <= target) {
        out.status = 0;
        out.final_ = r0;
        out.relative = r0 / scale;
        return out;
    }
    std::vector<double> H(static_cast<std::size_t>(m + 1) * m), cs(m), sn(m), gv(m + 1), y(m), hcol(m + 2);
    double inner = target, fin = r0;
    int used = 0;
    bool breakdown = false;
    for (int attempt = 0; attempt < 3 && used < cfg.max_iterations && !breakdown; ++attempt) {
        while (used < cfg.max_iterations) {
            // restart cycle: v_0 = r / ||r||
            const double beta = trueResidualNorm(ctx, A, b, x, ws.r.data());
            if (!std::isfinite(beta)) { breakdown = true; break; }
            if (beta <= inner) break;
            kScaleInto<<<g, kBlock, 0, ctx.stream>>>(n, ws.r.data(), 1.0 / beta, V);
            ctx.launched();
            std::fill(gv.begin(), gv.end(), 0.0);
            gv[0] = beta;
            int j = 0;
            bool reached = false;
            for (; j < m && used < cfg.max_iterations; ++j) {
                double* vj = V + j * ld;
                double* zj = flexible ? ws.Z.data() + j * ld : ws.zt.data();
                if (pc) pc->apply(ctx, vj, zj);
                else BSG_CUDA(cudaMemcpyAsync(zj, vj, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx.stream));
                spmv(ctx, A, zj, ws.w.data(), 1);
                // CGS2: two projections against v_0..v_j, then ||w||
                for (int pass = 0; pass < 2; ++pass) {
                    multiDot(ctx, ws, n, V, ld, j + 1, ws.w.data(), hdev);
                    kMultiAxpy<<<ag, kBlock, 0, ctx.stream>>>(n, V, ld, j + 1, hdev, -1.0, ws.w.data());
                    ctx.launched();
                    BSG_CUDA(cudaMemcpyAsync(hpin + (pass ? 32 : 0), hdev, sizeof(double) * (j + 1),
                                             cudaMemcpyDeviceToHost, ctx.stream));
                }
                multiDot(ctx, ws, n, ws.w.data(), 0, 1, ws.w.data(), hdev + m + 1);
                BSG_CUDA(cudaMemcpyAsync(hpin + 63, hdev + m + 1, sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
                ctx.sync();
                for (int i = 0; i <= j; ++i) hcol[i] = hpin[i] + hpin[32 + i];
                const double hn = std::sqrt(hpin[63]);
                hcol[j + 1] = hn;
                if (hn > 0.0 && std::isfinite(hn)) {
                    kScaleInto<<<g, kBlock, 0, ctx.stream>>>(n, ws.w.data(), 1.0 / hn, V + (j + 1) * ld);
                    ctx.launched();
                }
                // the previous rotations, then a new one that zeroes h_{j+1,j}
                for (int i = 0; i < j; ++i) {
                    const double a = hcol[i], c = hcol[i + 1];
                    hcol[i] = cs[i] * a + sn[i] * c;
                    hcol[i + 1] = -sn[i] * a + cs[i] * c;
                }
                const double d = std::hypot(hcol[j], hcol[j + 1]);
                cs[j] = d > 0.0 ? hcol[j] / d : 1.0;
                sn[j] = d > 0.0 ? hcol[j + 1] / d : 0.0;
                hcol[j] = d;
                for (int i = 0; i <= j; ++i) H[static_cast<std::size_t>(i) * m + j] = hcol[i];
                gv[j + 1] = -sn[j] * gv[j];
                gv[j] = cs[j] * gv[j];
                ++used;
                if (!std::isfinite(gv[j + 1])) { breakdown = true; ++j; break; }
                if (std::fabs(gv[j + 1]) <= inner || !(hn > 0.0) || d == 0.0) { reached = true; ++j; break; }
            }
            // x += M^-1 V y (GMRES) or Z y (FGMRES), y from the triangular system H y = g
            if (j > 0 && !breakdown) {
                for (int i = j - 1; i >= 0; --i) {
                    double s = gv[i];
                    for (int q = i + 1; q < j; ++q) s -= H[static_cast<std::size_t>(i) * m + q] * y[q];
                    const double hii = H[static_cast<std::size_t>(i) * m + i];
                    y[i] = hii != 0.0 ? s / hii : 0.0;
                }
                BSG_CUDA(cudaMemcpyAsync(hdev, y.data(), sizeof(double) * j, cudaMemcpyHostToDevice, ctx.stream));
                if (flexible) {
                    kMultiAxpy<<<ag, kBlock, 0, ctx.stream>>>(n, ws.Z.data(), ld, j, hdev, 1.0, x);
                    ctx.launched();
                } else {
                    BSG_CUDA(cudaMemsetAsync(ws.zt.data(), 0, sizeof(double) * n, ctx.stream));
                    kMultiAxpy<<<ag, kBlock, 0, ctx.stream>>>(n, V, ld, j, hdev, 1.0, ws.zt.data());
                    ctx.launched();
                    const double* corr = ws.zt.data();
                    if (pc) {
                        pc->apply(ctx, ws.zt.data(), ws.w.data());
                        corr = ws.w.data();
                    }
                    kAddTo<<<g, kBlock, 0, ctx.stream>>>(n, corr, x);
                    ctx.launched();
                }
                BSG_CUDA(cudaGetLastError());
                ctx.sync();  // y lives in host memory that the next cycle overwrites
            }
            if (reached || breakdown) break;
        }
        fin = trueResidualNorm(ctx, A, b, x, ws.r.data());
        ++out.checks;
        if (!std::isfinite(fin) || fin <= target) break;
        inner *= 0.5;
    }
    out.iterations = used;
    out.final_ = fin;
    out.relative = fin / scale;
    out.status = (std::isfinite(fin) && fin <= target) ? 0 : (std::isfinite(fin) && !breakdown ? 1 : 2);
    return out;
}

void componentCopy(Context& ctx, int n, int C, int c, const double* in, double* out, bool gather) {
    kComponent<<<gridFor(n, kBlock), kBlock, 0, ctx.stream>>>(n, C, c, in, out, gather ? 1 : 0);
    ctx.launched();
    BSG_CUDA(cudaGetLastError());
}

SolveOutcome gmresComponent(Context& ctx, GmresWorkspace& ws, const Dcsr<double>& A, const SolverConfig& cfg,
                            Preconditioner* pc, int C, int c, const double* b, double* x) {
    const int n = A.n;
    ws.ensure(n, std::max(1, std::min({ws.restart, cfg.max_iterations, 30})), cfg.solver == 3);
    componentCopy(ctx, n, C, c, b, ws.bc.data(), true);
    componentCopy(ctx, n, C, c, x, ws.xc.data(), true);
    const SolveOutcome o = gmresSolve(ctx, ws, A, cfg, pc, ws.bc.data(), ws.xc.data());
    componentCopy(ctx, n, C, c, ws.xc.data(), x, false);
    return o;
}

}  // namespace bsg
