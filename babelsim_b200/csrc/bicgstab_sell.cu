// Persistent cooperative BiCGStab on SELL-32 (see bicgstab_sell.cuh).
//
// The iteration is the one of the reference's PETSc KSPBCGS with a point-Jacobi
// (right) preconditioner, per component c with its own rho, alpha, omega, beta:
//   p  = r + beta (p - omega v),  ph = p / d
//   v  = A ph,                    alpha = rho / (r0 . v)
//   s  = r - alpha v,             sh = s / d      (||s|| <= target: x += alpha ph, done)
//   t  = A sh,                    omega = (t . s) / (t . t)
//   x += alpha ph + omega sh,     r = s - omega t, rho' = r0 . r, beta = (rho'/rho)(alpha/omega)
// Phases are separated by group barriers (grid-wide, or per system of a batch),
// and every CTA keeps identical copies of the scalars because every reduction
// gives all CTAs the same fixed-order total.
#include "bicgstab_sell.cuh"

#include <algorithm>
#include <cmath>

namespace bsg {
namespace {

constexpr int BB = 256;  // threads per block

// (A x)_i for the C components of row i of slice sl (lane = row within the slice).
template <int C, class T>
__device__ __forceinline__ void sellProduct(const SellMat<T>& S, int sl, int lane, const T* __restrict__ x, T acc[C]) {
    const int beg = S.sptr[sl], w = (S.sptr[sl + 1] - beg) >> 5;
    const int* __restrict__ cp = S.col + beg + lane;
    const T* __restrict__ vp = S.val + beg + lane;
    T a[C];
#pragma unroll
    for (int c = 0; c < C; ++c) a[c] = T(0);
    int k = 0;
    for (; k + 4 <= w; k += 4) {
        int cc[4];
        T vv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            cc[u] = __ldg(cp + 32 * (k + u));
            vv[u] = __ldg(vp + 32 * (k + u));
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int c = 0; c < C; ++c) a[c] += vv[u] * x[C * cc[u] + c];
    }
    for (; k < w; ++k) {
        const int j = __ldg(cp + 32 * k);
        const T v = __ldg(vp + 32 * k);
#pragma unroll
        for (int c = 0; c < C; ++c) a[c] += v * x[C * j + c];
    }
    const int i = 32 * sl + lane;
    const T d = i < S.n ? S.diag[i] : T(0);
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = (i < S.n ? d * x[C * i + c] : T(0)) + a[c];
}

// Products of vector entries are summed in FP64 whatever the vectors' type.
template <class T>
__device__ __forceinline__ double dd(T x) {
    return static_cast<double>(x);
}

template <int C, class T, class G>
__device__ void bicgBody(G& g, const BicgArgs<C, T>& a) {
    const Lanes ln = lanes<BB>(g);
    const SellMat<T>& A = a.A;
    const int n = A.n;
    BicgState& st = *a.st;
    int buf = 0;
    double rho[C], alpha[C], omega[C], beta[C], target2[C];
    int done[C], iters[C];
    double target2_in[C];
    const int max_iters = st.max_iters;
    // inputs are read before block 0 writes any result into the same struct
#pragma unroll
    for (int c = 0; c < C; ++c) {
        done[c] = st.done[c];
        iters[c] = st.iters[c];
        target2_in[c] = st.target2[c];
        alpha[c] = 1.0;
        omega[c] = 1.0;
        beta[c] = 0.0;
    }
    auto active = [&](int c) { return done[c] == 0 && iters[c] < max_iters; };
    // r = b - A x, r0 = r, p = v = 0; ||r||^2 and ||b||^2 per component
    double nb[2 * C];
#pragma unroll
    for (int j = 0; j < 2 * C; ++j) nb[j] = 0.0;
    for (int sl = ln.gwarp; sl < A.nslices; sl += ln.nwarps) {
        T acc[C];
        sellProduct<C, T>(A, sl, ln.lane, a.x, acc);
        const int i = 32 * sl + ln.lane;
        if (i < n) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const T bi = a.b[C * i + c], ri = bi - acc[c];
                a.r[C * i + c] = ri;
                a.r0[C * i + c] = ri;
                a.p[C * i + c] = T(0);
                a.v[C * i + c] = T(0);
                nb[c] += dd(ri) * dd(ri);
                nb[C + c] += dd(bi) * dd(bi);
            }
        }
    }
    gridSum<2 * C, BB>(g, nb, a.partial, buf);
#pragma unroll
    for (int c = 0; c < C; ++c) {
        rho[c] = nb[c];
        if (target2_in[c] < 0.0) {
            // the reference's contract: max(atol, rtol * max(||r0||, ||b||)) (solver_control.h:199-210)
            double scale = fmax(sqrt(nb[c]), sqrt(nb[C + c]));
            if (!(scale > 0.0)) scale = 1.0;
            const double tg = fmax(st.atol, st.rtol * scale);
            target2[c] = tg * tg;
        } else {
            target2[c] = target2_in[c];
        }
        if (done[c] == 0 && (!(nb[c] > 0.0) || nb[c] <= target2[c])) done[c] = 1;
    }
    if (g.rank() == 0 && threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
            st.rr0[c] = nb[c];
            st.bb[c] = nb[C + c];
            st.target2[c] = target2[c];
        }
    }
    for (;;) {
        bool any = false;
#pragma unroll
        for (int c = 0; c < C; ++c) any = any || active(c);
        if (!any || g.aborted()) break;
        // p = r + beta (p - omega v), ph = p / d
        for (int i = ln.gthread; i < n; i += ln.nthreads) {
            const T rd = T(1) / A.diag[i];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                if (!active(c)) continue;
                const T pi = a.r[C * i + c] +
                             static_cast<T>(beta[c]) * (a.p[C * i + c] - static_cast<T>(omega[c]) * a.v[C * i + c]);
                a.p[C * i + c] = pi;
                a.ph[C * i + c] = pi * rd;
            }
        }
        g.sync();
        // v = A ph, r0 . v
        double r0v[C];
#pragma unroll
        for (int c = 0; c < C; ++c) r0v[c] = 0.0;
        for (int sl = ln.gwarp; sl < A.nslices; sl += ln.nwarps) {
            T acc[C];
            sellProduct<C, T>(A, sl, ln.lane, a.ph, acc);
            const int i = 32 * sl + ln.lane;
            if (i < n) {
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    a.v[C * i + c] = acc[c];
                    r0v[c] += dd(a.r0[C * i + c]) * dd(acc[c]);
                }
            }
        }
        gridSum<C, BB>(g, r0v, a.partial, buf);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            if (!active(c)) continue;
            if (!(fabs(r0v[c]) > 0.0) || !isfinite(r0v[c])) { done[c] = 2; continue; }
            alpha[c] = rho[c] / r0v[c];
        }
        // s = r - alpha v (kept in r), sh = s / d, ||s||^2
        double ss[C];
#pragma unroll
        for (int c = 0; c < C; ++c) ss[c] = 0.0;
        for (int i = ln.gthread; i < n; i += ln.nthreads) {
            const T rd = T(1) / A.diag[i];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                if (!active(c)) continue;
                const T si = a.r[C * i + c] - static_cast<T>(alpha[c]) * a.v[C * i + c];
                a.r[C * i + c] = si;
                a.sh[C * i + c] = si * rd;
                ss[c] += dd(si) * dd(si);
            }
        }
        gridSum<C, BB>(g, ss, a.partial, buf);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            if (!active(c)) continue;
            if (!isfinite(ss[c])) done[c] = 2;
            else if (ss[c] <= target2[c]) done[c] = 3;  // the half step is accepted
        }
        // t = A sh, t . t and t . s
        double ts[2 * C];
#pragma unroll
        for (int j = 0; j < 2 * C; ++j) ts[j] = 0.0;
        for (int sl = ln.gwarp; sl < A.nslices; sl += ln.nwarps) {
            T acc[C];
            sellProduct<C, T>(A, sl, ln.lane, a.sh, acc);
            const int i = 32 * sl + ln.lane;
            if (i < n) {
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    a.t[C * i + c] = acc[c];
                    ts[2 * c] += dd(acc[c]) * dd(acc[c]);
                    ts[2 * c + 1] += dd(acc[c]) * dd(a.r[C * i + c]);
                }
            }
        }
        gridSum<2 * C, BB>(g, ts, a.partial, buf);
#pragma unroll
        for (int c = 0; c < C; ++c)
            if (active(c)) omega[c] = ts[2 * c] > 0.0 ? ts[2 * c + 1] / ts[2 * c] : 0.0;
        // x += alpha ph + omega sh, r = s - omega t; ||r||^2 and r0 . r (half step: x += alpha ph)
        int mode[C];
#pragma unroll
        for (int c = 0; c < C; ++c) mode[c] = done[c] == 3 ? 2 : (active(c) ? 1 : 0);
        double nr[2 * C];
#pragma unroll
        for (int j = 0; j < 2 * C; ++j) nr[j] = 0.0;
        for (int i = ln.gthread; i < n; i += ln.nthreads) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
                if (mode[c] == 0) continue;
                if (mode[c] == 2) {
                    a.x[C * i + c] += static_cast<T>(alpha[c]) * a.ph[C * i + c];
                    continue;
                }
                a.x[C * i + c] += static_cast<T>(alpha[c]) * a.ph[C * i + c] + static_cast<T>(omega[c]) * a.sh[C * i + c];
                const T ri = a.r[C * i + c] - static_cast<T>(omega[c]) * a.t[C * i + c];
                a.r[C * i + c] = ri;
                nr[2 * c] += dd(ri) * dd(ri);
                nr[2 * c + 1] += dd(a.r0[C * i + c]) * dd(ri);
            }
        }
        gridSum<2 * C, BB>(g, nr, a.partial, buf);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            if (done[c] == 3) { done[c] = 1; iters[c] += 1; continue; }
            if (!active(c)) continue;
            iters[c] += 1;
            const double rr = nr[2 * c], rho_new = nr[2 * c + 1];
            if (!isfinite(rr)) { done[c] = 2; continue; }
            if (rr <= target2[c]) { done[c] = 1; continue; }
            if (omega[c] == 0.0 || !(fabs(rho_new) > 0.0)) { done[c] = 2; continue; }
            beta[c] = (rho_new / rho[c]) * (alpha[c] / omega[c]);
            rho[c] = rho_new;
        }
    }
    // the true residual of every component (the acceptance test's norm)
    double fr[C];
#pragma unroll
    for (int c = 0; c < C; ++c) fr[c] = 0.0;
    g.sync();
    for (int sl = ln.gwarp; sl < A.nslices; sl += ln.nwarps) {
        T acc[C];
        sellProduct<C, T>(A, sl, ln.lane, a.x, acc);
        const int i = 32 * sl + ln.lane;
        if (i < n) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const T ri = a.b[C * i + c] - acc[c];
                fr[c] += dd(ri) * dd(ri);
            }
        }
    }
    gridSum<C, BB>(g, fr, a.partial, buf);
    if (g.rank() == 0 && threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
            st.done[c] = done[c];
            st.iters[c] = iters[c];
            st.fin2[c] = fr[c];
        }
        st.status = g.failed() ? 3 : 0;
    }
}

// Whole-grid kernel at 4 blocks per SM (64 registers, no spills); the batched kernel keeps
// 3 (80 registers).
#ifndef BSG_BICG_MIN_BLOCKS
#define BSG_BICG_MIN_BLOCKS 4
#endif
template <int C, class T>
__global__ void __launch_bounds__(BB, BSG_BICG_MIN_BLOCKS) kBicgSell(BicgArgs<C, T> a, SegmentBarrier* bar) {
    GridGroup g{bar};
    bicgBody<C, T>(g, a);
}

template <int C>
__global__ void __launch_bounds__(BB, 3)
    kBicgSellBatch(const BicgArgs<C>* __restrict__ segs, const int* __restrict__ cta_begin, int nsegs,
                   SegmentBarrier* bars) {
    int lo = 0, hi = nsegs - 1;  // the system whose CTA range holds this block
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cta_begin[mid] <= static_cast<int>(blockIdx.x)) lo = mid;
        else hi = mid - 1;
    }
    SegmentGroup g{cta_begin[lo], cta_begin[lo + 1] - cta_begin[lo], bars + lo};
    const BicgArgs<C> a = segs[lo];
    bicgBody<C, double>(g, a);
}

}  // namespace

int bicgstabGrid(Context& ctx) {
    static int per_sm = -1;
    if (per_sm < 0) {
        BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kBicgSell<3, double>, BB, 0));
        int b = 0;
        BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kBicgSellBatch<3>, BB, 0));
        per_sm = std::min(per_sm, b);
        if (per_sm <= 0) fail(kCuda, "persistent BiCGStab kernel cannot be resident");
    }
    return ctx.sm_count * std::min(per_sm, 4);
}

namespace {
// Resident CTAs of one whole-grid launch of kBicgSell<C, T>.
template <int C, class T>
int singleGrid(Context& ctx) {
    static int per_sm = -1;
    if (per_sm < 0) {
        BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kBicgSell<C, T>, BB, 0));
        if (per_sm <= 0) fail(kCuda, "persistent BiCGStab kernel cannot be resident");
    }
    return ctx.sm_count * std::min(per_sm, 4);
}
}  // namespace

template <int C, class T>
void launchBicgstab(Context& ctx, const BicgArgs<C, T>& in) {
    BicgArgs<C, T> args = in;
    SegmentBarrier* bar = ctx.grid_barrier;
    const int grid = singleGrid<C, T>(ctx);
    resetBarriers(ctx, bar, 1, grid);
    void* params[] = {&args, &bar};
    BSG_PROFILE(ctx, sizeof(T) == 4 ? "bicgstab3_persistent_fp32" : "bicgstab3_persistent");
    BSG_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kBicgSell<C, T>), grid, BB, params, 0, ctx.stream));
    ctx.launched();
}

template <int C>
void launchBicgstabBatch(Context& ctx, BicgBatch<C>& batch) {
    const int nsegs = static_cast<int>(batch.args.size());
    if (nsegs == 0) return;
    if (static_cast<int>(batch.cta_begin.size()) != nsegs + 1 || batch.cta_begin.front() != 0)
        fail(kArgument, "batched BiCGStab: CTA table does not match the systems");
    for (int k = 0; k < nsegs; ++k)
        if (batch.cta_begin[k + 1] <= batch.cta_begin[k]) fail(kArgument, "batched BiCGStab: a system without CTAs");
    const int total = batch.cta_begin.back();
    if (total > bicgstabGrid(ctx)) fail(kArgument, "batched BiCGStab: CTA allotment exceeds the resident grid");
    batch.d_args.upload(batch.args, ctx.stream);
    batch.d_cta.upload(batch.cta_begin, ctx.stream);
    batch.d_bars.resize(nsegs);
    resetBarriers(ctx, batch.d_bars.data(), nsegs, total, batch.cta_begin.data());
    const BicgArgs<C>* segs = batch.d_args.data();
    const int* cta = batch.d_cta.data();
    SegmentBarrier* bars = batch.d_bars.data();
    int ns = nsegs;
    void* params[] = {&segs, &cta, &ns, &bars};
    BSG_PROFILE(ctx, "bicgstab3_persistent_batch");
    BSG_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kBicgSellBatch<C>), total, BB, params, 0,
                                         ctx.stream));
    ctx.launched();
}

template void launchBicgstab<3, double>(Context&, const BicgArgs<3, double>&);
template void launchBicgstab<1, double>(Context&, const BicgArgs<1, double>&);
template void launchBicgstab<3, float>(Context&, const BicgArgs<3, float>&);
template void launchBicgstab<1, float>(Context&, const BicgArgs<1, float>&);
template void launchBicgstabBatch<3>(Context&, BicgBatch<3>&);

}  // namespace bsg
