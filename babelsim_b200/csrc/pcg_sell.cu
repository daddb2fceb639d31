// Persistent cooperative PCG + AMG V-cycle on SELL-32 levels (see pcg_sell.cuh).
#include "group.cuh"
#include "pcg_sell.cuh"

#include <algorithm>
#include <cmath>

namespace bsg {
namespace {

#ifndef BSG_SELL_SB
#define BSG_SELL_SB 256
#endif
constexpr int SB = BSG_SELL_SB;  // threads per block
// Minimum resident blocks per SM the register budget must allow.  The single-system
// kernels: 4 (64 registers) measured faster than 3 (80) on the 1M-cell cavity (FP64:
// 2 %; FP32 V-cycle: 42.4 -> 40.3 ms per outer iteration; FP32 inner PCG: 49.6 ->
// 45.5), 2 (128) slower.  The batched kernel keeps 3: at 64 registers it spills heavily.
#ifndef BSG_SELL_MIN_BLOCKS
#define BSG_SELL_MIN_BLOCKS 4
#endif
#ifndef BSG_SELL_BATCH_MIN_BLOCKS
#define BSG_SELL_BATCH_MIN_BLOCKS 3
#endif
// Levels of at most this many rows compute their residual and its restriction in one
// pass (coarse row by coarse row, kRowLanes lanes per member row), one barrier fewer.
// On the 1M-cell solve (us per CG iteration, residual + restriction): 16k rows 11.8 ->
// 9.0, 4k rows 9.3 -> 8.0, 1k rows 7.9 -> 7.5, but 62k rows 17.8 -> 22.0, where the
// row-by-row reads of the level's matrix no longer pay for the barrier they save.
#ifndef BSG_RESTRICT_ROWS
#define BSG_RESTRICT_ROWS 20000
#endif
constexpr int kRestrictRows = BSG_RESTRICT_ROWS;
#ifndef BSG_ROW_LANES
#define BSG_ROW_LANES 8
#endif
constexpr int kRowLanes = BSG_ROW_LANES;
template <class TK, class TV>
constexpr int kSellMinBlocks = BSG_SELL_MIN_BLOCKS;

__device__ __forceinline__ void mark(const PhaseLog& log, int id) {
    if (log.entries && blockIdx.x == 0 && threadIdx.x == 0) {
        const int k = *log.count;
        if (k < log.capacity) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            log.entries[2 * k] = id;
            log.entries[2 * k + 1] = static_cast<long long>(t);
            *log.count = k + 1;
        }
    }
}

// Final value v of row i on level l: level 0 writes z and returns r_i z_i;
// coarser levels push gamma v into their members' iterate on the finer level
// `fin` (level l - 1).
template <class TK, class TV>
__device__ __forceinline__ double emitRow(const VCycleView<TV>& V, const VLevel<TV>& fin, int l, int i, TV v,
                                          const TK* r, TK* z) {
    if (l == 0) {
        const TK zi = static_cast<TK>(v);
        z[i] = zi;
        return static_cast<double>(r[i]) * static_cast<double>(zi);
    }
    const TV* from = V.nu >= 2 ? fin.x : fin.w;
    const TV add = V.gamma * v;
    for (int m = fin.agg_ptr[i]; m < fin.agg_ptr[i + 1]; ++m) {
        const int ii = fin.agg_rows[m];
        fin.x[ii] = from[ii] + add;
    }
    return 0.0;
}

// z = M r with M the V-cycle; returns this thread's share of r.z.  Level 0's b
// and w were written by the phase that produced r.
// Lanes per row on a level: the largest power of two (at most 32) that still
// gives every (slice, lane-group) unit its own warp; 1 on the fine levels.
__device__ __forceinline__ int splitOf(int nslices, int nwarps) {
    int K = 1;
    while (K < 32 && static_cast<long long>(nslices) * K * 2 <= nwarps) K *= 2;
    return K;
}

// Unit u of a split sweep: slice s, the row r within it and this lane's part q.
struct SplitUnit {
    int s, r, q;
};
__device__ __forceinline__ SplitUnit splitUnit(int u, int K, int lane) {
    const int rows = 32 / K;
    return {u / K, (u % K) * rows + lane / K, lane % K};
}

template <class TK, class TV, class G>
__device__ double vcycle(G& g, const VCycleView<TV>& V, const TK* r, TK* z, const PhaseLog& log,
                         bool level0_residual_done = false) {
    const Lanes c = lanes<SB>(g);
    const int L = V.levels;
    // ---- down
    for (int l = 0; l < L - 1; ++l) {
        const VLevel<TV> f = V.lv[l];
        const bool residual_done = l == 0 && level0_residual_done;
        // a small level's residual is summed straight into the coarser right-hand side
        const bool restrict_rows = !residual_done && f.A.n <= kRestrictRows;
        // t of level 0 may have come with the Krylov update (fused sweep in pcgBody)
        if (!residual_done) {
            if (V.nu >= 2) {
                for (int s = c.gwarp; s < f.A.nslices; s += c.nwarps) {
                    const int i = 32 * s + c.lane;
                    const TV* w = f.w;
                    const TV aw = sellRow(f.A, s, c.lane, [&](int j) { return w[j]; });
                    if (i < f.A.n) {
                        const TV wi = w[i];
                        f.x[i] = wi + f.rd[i] * (f.b[i] - (f.A.diag[i] * wi + aw));
                    }
                }
                g.sync();
                mark(log, 10 + l);
            }
            const TV* xs = V.nu >= 2 ? f.x : f.w;
            const int K = splitOf(f.A.nslices, c.nwarps);
            if (restrict_rows) {
                // coarse row I on one warp: its members' residual rows b_i - A x_i, each on
                // kRowLanes lanes, summed over the members in a fixed butterfly order
                const VLevel<TV> cl = V.lv[l + 1];
                constexpr int groups = 32 / kRowLanes;
                const int grp = c.lane / kRowLanes, q = c.lane % kRowLanes;
                for (int I = c.gwarp; I < cl.A.n; I += c.nwarps) {
                    const int m0 = f.agg_ptr[I], m1 = f.agg_ptr[I + 1];
                    TV sum = TV(0);
                    for (int mb = m0; mb < m1; mb += groups) {
                        const int m = mb + grp;
                        const bool on = m < m1;
                        // every lane takes part in the butterfly; idle groups sweep the first member
                        const int i = f.agg_rows[on ? m : m0];
                        const TV ax = sellRowSplit(f.A, i >> 5, i & 31, q, kRowLanes, [&](int j) { return xs[j]; });
                        TV ti = on ? f.b[i] - (f.A.diag[i] * xs[i] + ax) : TV(0);
                        for (int o = kRowLanes; o < 32; o <<= 1) ti += __shfl_xor_sync(0xffffffffu, ti, o);
                        sum += ti;
                    }
                    if (c.lane == 0) {
                        cl.b[I] = sum;
                        cl.w[I] = cl.rd[I] * sum;
                    }
                }
            } else if (K == 1) {
                for (int s = c.gwarp; s < f.A.nslices; s += c.nwarps) {
                    const int i = 32 * s + c.lane;
                    const TV ax = sellRow(f.A, s, c.lane, [&](int j) { return xs[j]; });
                    if (i < f.A.n) f.t[i] = f.b[i] - (f.A.diag[i] * xs[i] + ax);
                }
            } else {
                for (int u = c.gwarp; u < f.A.nslices * K; u += c.nwarps) {
                    const SplitUnit su = splitUnit(u, K, c.lane);
                    const int i = 32 * su.s + su.r;
                    const TV ax = sellRowSplit(f.A, su.s, su.r, su.q, K, [&](int j) { return xs[j]; });
                    if (su.q == 0 && i < f.A.n) f.t[i] = f.b[i] - (f.A.diag[i] * xs[i] + ax);
                }
            }
            if (!restrict_rows) {
                g.sync();
                mark(log, 30 + l);
            }
        }
        if (!restrict_rows) {
            const VLevel<TV> cl = V.lv[l + 1];
            for (int I = c.gthread; I < cl.A.n; I += c.nthreads) {
                TV s = TV(0);
                for (int m = f.agg_ptr[I]; m < f.agg_ptr[I + 1]; ++m) s += f.t[f.agg_rows[m]];
                cl.b[I] = s;
                cl.w[I] = cl.rd[I] * s;
            }
        }
        g.sync();
        mark(log, 100 + l);
    }
    // ---- coarsest: dense inverse, one warp per row, pushed into the finer level
    double rz = 0.0;
    {
        const VLevel<TV> cl = V.lv[L - 1];
        const int n = cl.A.n;
        const TV* b = cl.b;
        for (int I = c.gwarp; I < n; I += c.nwarps) {
            const TV* row = V.dense_inv + static_cast<long long>(I) * n;
            TV s = TV(0);
            for (int J = c.lane; J < n; J += 32) s += row[J] * b[J];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (L == 1) {
                if (c.lane == 0) rz += emitRow<TK, TV>(V, cl, 0, I, s, r, z);
            } else {
                const VLevel<TV> f = V.lv[L - 2];
                const TV* from = V.nu >= 2 ? f.x : f.w;
                const TV add = V.gamma * s;
                for (int m = f.agg_ptr[I] + c.lane; m < f.agg_ptr[I + 1]; m += 32) {
                    const int ii = f.agg_rows[m];
                    f.x[ii] = from[ii] + add;
                }
            }
        }
        if (L > 1) {
            g.sync();
            mark(log, 50);
        }
    }
    // ---- up: the coarse levels, each pushing its smoothed values into the finer level
    const bool single = V.nu < 2;
    for (int l = L - 2; l >= 1; --l) {
        const VLevel<TV> f = V.lv[l];
        const VLevel<TV> fin = V.lv[l - 1];
        const TV* y = f.x;
        const int K = single ? splitOf(f.A.nslices, c.nwarps) : 1;
        if (K == 1) {
            for (int s = c.gwarp; s < f.A.nslices; s += c.nwarps) {
                const int i = 32 * s + c.lane;
                const TV ay = sellRow(f.A, s, c.lane, [&](int j) { return y[j]; });
                if (i < f.A.n) {
                    const TV yi = y[i];
                    const TV v = yi + f.rd[i] * (f.b[i] - (f.A.diag[i] * yi + ay));
                    if (single) emitRow<TK, TV>(V, fin, l, i, v, r, z);
                    else f.t[i] = v;
                }
            }
        } else {
            // one smoothing step: the K lanes of a row share its push into the finer level
            const TV* from = fin.w;
            for (int u = c.gwarp; u < f.A.nslices * K; u += c.nwarps) {
                const SplitUnit su = splitUnit(u, K, c.lane);
                const int i = 32 * su.s + su.r;
                const TV ay = sellRowSplit(f.A, su.s, su.r, su.q, K, [&](int j) { return y[j]; });
                if (i < f.A.n) {
                    const TV yi = y[i];
                    const TV add = V.gamma * (yi + f.rd[i] * (f.b[i] - (f.A.diag[i] * yi + ay)));
                    for (int m = fin.agg_ptr[i] + su.q; m < fin.agg_ptr[i + 1]; m += K) {
                        const int ii = fin.agg_rows[m];
                        fin.x[ii] = from[ii] + add;
                    }
                }
            }
        }
        if (!single) {
            g.sync();
            mark(log, 60 + l);
            const TV* t = f.t;
            for (int s = c.gwarp; s < f.A.nslices; s += c.nwarps) {
                const int i = 32 * s + c.lane;
                const TV at = sellRow(f.A, s, c.lane, [&](int j) { return t[j]; });
                if (i < f.A.n) {
                    const TV ti = t[i];
                    emitRow<TK, TV>(V, fin, l, i, ti + f.rd[i] * (f.b[i] - (f.A.diag[i] * ti + at)), r, z);
                }
            }
        }
        g.sync();
        mark(log, 80 + l);
    }
    // ---- up, level 0, in a block of its own: the last sweep writes z and this thread's
    // share of r.z.  Kept out of the coarse levels' loop, whose push into a finer level it
    // never takes: sharing that loop made this sweep (one level-0 product) 1.7x slower,
    // 117 against 68 us per CG iteration on the 1M-cell case.
    if (L >= 2) {
        const VLevel<TV> f = V.lv[0];
        const TV* y = f.x;
        if (!single) {
            for (int s = c.gwarp; s < f.A.nslices; s += c.nwarps) {
                const int i = 32 * s + c.lane;
                const TV ay = sellRow(f.A, s, c.lane, [&](int j) { return y[j]; });
                if (i < f.A.n) {
                    const TV yi = y[i];
                    f.t[i] = yi + f.rd[i] * (f.b[i] - (f.A.diag[i] * yi + ay));
                }
            }
            g.sync();
            mark(log, 60);
            y = f.t;
        }
        for (int s = c.gwarp; s < f.A.nslices; s += c.nwarps) {
            const int i = 32 * s + c.lane;
            const TV ay = sellRow(f.A, s, c.lane, [&](int j) { return y[j]; });
            if (i < f.A.n) {
                const TV yi = y[i];
                const TK zi = static_cast<TK>(yi + f.rd[i] * (f.b[i] - (f.A.diag[i] * yi + ay)));
                z[i] = zi;
                rz += static_cast<double>(r[i]) * static_cast<double>(zi);
            }
        }
    }
    return rz;
}

// Level-0 V-cycle inputs from the current residual value of row i.
template <class TK, class TV>
__device__ __forceinline__ void seedLevel0(const VLevel<TV>& f0, int i, TK ri) {
    const TV rv = static_cast<TV>(ri);
    f0.b[i] = rv;
    f0.w[i] = f0.rd[i] * rv;
}

template <class TK, class TV, class G>
__device__ void pcgBody(G& g, const SellPcgArgs<TK, TV>& a) {
    const Lanes c = lanes<SB>(g);
    const SellMat<TK>& A = a.A;
    const int n = A.n;
    int buf = 0;
    PcgState& st = *a.st;
    const int warm = st.warm;
    const int max_iterations = st.max_iterations;
    const double target2_in = st.target2, atol = st.atol, rtol = st.rtol;
    const VLevel<TV> f0 = a.V.lv[0];
    // r = b - A x (x = 0 unless warm), ||r0||^2, ||b||^2, level-0 V-cycle inputs
    double v[2] = {0.0, 0.0};
    for (int s = c.gwarp; s < A.nslices; s += c.nwarps) {
        const int i = 32 * s + c.lane;
        TK ri = TK(0);
        if (warm) {
            const TK* x = a.x;
            const TK ax = sellRow(A, s, c.lane, [&](int j) { return x[j]; });
            if (i < n) ri = a.b[i] - (A.diag[i] * x[i] + ax);
        } else if (i < n) {
            ri = a.b[i];
            a.x[i] = TK(0);
        }
        if (i < n) {
            a.r[i] = ri;
            seedLevel0<TK, TV>(f0, i, ri);
            v[0] += static_cast<double>(ri) * static_cast<double>(ri);
            v[1] += static_cast<double>(a.b[i]) * static_cast<double>(a.b[i]);
        }
    }
    gridSum<2, SB>(g, v, a.partial, buf);
    mark(a.log, 1);
    double target2 = target2_in;
    if (target2 < 0.0) {
        // the reference's contract: max(atol, rtol * max(||r0||, ||b||)) (solver_control.h:199-210)
        double scale = fmax(sqrt(v[0]), sqrt(v[1]));
        if (!(scale > 0.0)) scale = 1.0;
        const double t = fmax(atol, rtol * scale);
        target2 = t * t;
    }
    if (g.rank() == 0 && threadIdx.x == 0) {
        st.rr0 = v[0];
        st.bb = v[1];
        st.target2 = target2;
        st.rr = v[0];
        st.iterations = 0;
        st.status = 1;
    }
    if (isfinite(v[0]) && v[0] <= target2) {
        if (g.rank() == 0 && threadIdx.x == 0) st.status = 0;
        return;
    }
    double w[1] = {vcycle<TK, TV>(g, a.V, a.r, a.z, a.log)};
    if (g.aborted()) {
        if (g.rank() == 0 && threadIdx.x == 0) st.status = 3;
        return;
    }
    gridSum<1, SB>(g, w, a.partial, buf);
    mark(a.log, 4);
    double rz = w[0];
    double beta = 0.0;
    TK* pold = a.p0;
    TK* pnew = a.p1;
    const bool fuse = a.r2 != nullptr && a.V.nu < 2 && a.V.levels >= 2;
    TK* rcur = a.r;
    TK* rnext = a.r2;
    int it = 0;
    int status = 1;
    double rr = v[0];
    while (it < max_iterations) {
        if (g.aborted()) { status = 3; break; }
        if (!isfinite(rz) || rz == 0.0) { status = 2; break; }
        // p_new = z + beta p_old and q = A p_new in one sweep (neighbours' p_new formed on the fly)
        const TK bk = static_cast<TK>(beta);
        const TK* zz = a.z;
        const TK* po = pold;
        double pq[1] = {0.0};
        for (int s = c.gwarp; s < A.nslices; s += c.nwarps) {
            const int i = 32 * s + c.lane;
            const TK ap = beta == 0.0 ? sellRow(A, s, c.lane, [&](int j) { return zz[j]; })
                                      : sellRow(A, s, c.lane, [&](int j) { return zz[j] + bk * po[j]; });
            if (i < n) {
                const TK pi = beta == 0.0 ? zz[i] : zz[i] + bk * po[i];
                const TK qi = A.diag[i] * pi + ap;
                pnew[i] = pi;
                a.q[i] = qi;
                pq[0] += static_cast<double>(pi) * static_cast<double>(qi);
            }
        }
        gridSum<1, SB>(g, pq, a.partial, buf);
        mark(a.log, 2);
        if (!(fabs(pq[0]) > 0.0) || !isfinite(pq[0])) { status = 2; break; }
        const double alpha = rz / pq[0];
        const TK ak = static_cast<TK>(alpha);
        double nr[2] = {0.0, 0.0};
        if (fuse) {
            // x += alpha p, r_new = r - alpha q, the level-0 seeds b = r_new, w = rd b, and the
            // level-0 residual t = b - A w with the neighbours' w formed from their r and q
            const TK* rc = rcur;
            const TK* qq = a.q;
            const TV* rd0 = f0.rd;
            for (int s = c.gwarp; s < f0.A.nslices; s += c.nwarps) {
                const int i = 32 * s + c.lane;
                const TV aw = sellRow(f0.A, s, c.lane,
                                      [&](int j) { return rd0[j] * static_cast<TV>(rc[j] - ak * qq[j]); });
                if (i < n) {
                    a.x[i] += ak * pnew[i];
                    const TK ri = rc[i] - ak * qq[i];
                    rnext[i] = ri;
                    const TV rv = static_cast<TV>(ri);
                    const TV wi = rd0[i] * rv;
                    f0.b[i] = rv;
                    f0.w[i] = wi;
                    f0.t[i] = rv - (f0.A.diag[i] * wi + aw);
                    nr[0] += static_cast<double>(ri) * static_cast<double>(ri);
                    if (a.flexible) nr[1] += static_cast<double>(ri) * static_cast<double>(a.z[i]);
                }
            }
        } else {
            for (int i = c.gthread; i < n; i += c.nthreads) {
                a.x[i] += ak * pnew[i];
                const TK ri = a.r[i] - ak * a.q[i];
                a.r[i] = ri;
                seedLevel0<TK, TV>(f0, i, ri);
                nr[0] += static_cast<double>(ri) * static_cast<double>(ri);
                if (a.flexible) nr[1] += static_cast<double>(ri) * static_cast<double>(a.z[i]);  // r_new . z_old
            }
        }
        gridSum<2, SB>(g, nr, a.partial, buf);
        mark(a.log, 3);
        rr = nr[0];
        const double rz_old_new = nr[1];
        ++it;
        if (!isfinite(rr)) { status = 2; break; }
        if (rr <= target2) { status = 0; break; }
        if (it >= max_iterations) break;
        double zr[1] = {vcycle<TK, TV>(g, a.V, fuse ? rnext : a.r, a.z, a.log, fuse)};
        gridSum<1, SB>(g, zr, a.partial, buf);
        mark(a.log, 4);
        beta = a.flexible ? (zr[0] - rz_old_new) / rz : zr[0] / rz;
        rz = zr[0];
        TK* tmp = pold;
        pold = pnew;
        pnew = tmp;
        if (fuse) {
            TK* t2 = rcur;
            rcur = rnext;
            rnext = t2;
        }
    }
    if (g.rank() == 0 && threadIdx.x == 0) {
        st.rr = rr;
        st.iterations = it;
        st.status = g.failed() ? 3 : status;
    }
}

template <class TK, class TV>
__global__ void __launch_bounds__(SB, (kSellMinBlocks<TK, TV>)) kPcgSell(SellPcgArgs<TK, TV> a, SegmentBarrier* bar) {
    GridGroup g{bar};
    pcgBody<TK, TV>(g, a);
}

// A batch: CTAs [cta_begin[s], cta_begin[s+1]) solve system s with its own
// arguments, barriers and reductions, independently of the other systems.
template <class TK, class TV>
__global__ void __launch_bounds__(SB, BSG_SELL_BATCH_MIN_BLOCKS)
    kPcgSellBatch(const SellPcgArgs<TK, TV>* __restrict__ segs, const int* __restrict__ cta_begin, int nsegs,
                  SegmentBarrier* bars) {
    int lo = 0, hi = nsegs - 1;  // the segment whose CTA range holds this block
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cta_begin[mid] <= static_cast<int>(blockIdx.x)) lo = mid;
        else hi = mid - 1;
    }
    SegmentGroup g{cta_begin[lo], cta_begin[lo + 1] - cta_begin[lo], bars + lo};
    const SellPcgArgs<TK, TV> a = segs[lo];
    pcgBody<TK, TV>(g, a);
}

template <class TK, class TV>
int sellGrid(Context& ctx) {
    static int per_sm = -1;
    if (per_sm < 0) {
        BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kPcgSell<TK, TV>, SB, 0));
        if (per_sm <= 0) fail(kCuda, "persistent SELL PCG kernel cannot be resident");
    }
    return ctx.sm_count * std::min(per_sm, 8);
}

// Resident CTAs of the batched kernels: the smaller of the two precisions' grids.
int batchGrid(Context& ctx) {
    static int per_sm = -1;
    if (per_sm < 0) {
        int a = 0, b = 0;
        BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, kPcgSellBatch<double, double>, SB, 0));
        BSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kPcgSellBatch<double, float>, SB, 0));
        per_sm = std::min(a, b);
        if (per_sm <= 0) fail(kCuda, "batched SELL PCG kernel cannot be resident");
    }
    return ctx.sm_count * std::min(per_sm, 8);
}

}  // namespace

template <class TK, class TV>
void launchSellPcg(Context& ctx, const SellPcgArgs<TK, TV>& in) {
    SellPcgArgs<TK, TV> args = in;
    args.log = PhaseLog{ctx.phase_entries, ctx.phase_capacity, ctx.phase_count};
    SegmentBarrier* bar = ctx.grid_barrier;
    const int grid = sellGrid<TK, TV>(ctx);
    resetBarriers(ctx, bar, 1, grid);
    void* params[] = {&args, &bar};
    BSG_PROFILE(ctx, "pcg_amg_persistent");
    BSG_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kPcgSell<TK, TV>), grid, SB, params, 0, ctx.stream));
    ctx.launched();
}

int sellBatchCapacity(Context& ctx) { return batchGrid(ctx); }

template <class TK, class TV>
void launchSellPcgBatch(Context& ctx, BatchLaunch<TK, TV>& batch) {
    const int nsegs = static_cast<int>(batch.args.size());
    if (nsegs == 0) return;
    if (static_cast<int>(batch.cta_begin.size()) != nsegs + 1 || batch.cta_begin.front() != 0)
        fail(kArgument, "batched PCG: CTA table does not match the systems");
    for (int k = 0; k < nsegs; ++k)
        if (batch.cta_begin[k + 1] <= batch.cta_begin[k]) fail(kArgument, "batched PCG: a system without CTAs");
    const int total = batch.cta_begin.back();
    if (total > batchGrid(ctx)) fail(kArgument, "batched PCG: CTA allotment exceeds the resident grid");
    batch.d_args.upload(batch.args, ctx.stream);
    batch.d_cta.upload(batch.cta_begin, ctx.stream);
    batch.d_bars.resize(nsegs);
    resetBarriers(ctx, batch.d_bars.data(), nsegs, total, batch.cta_begin.data());
    const SellPcgArgs<TK, TV>* segs = batch.d_args.data();
    const int* cta = batch.d_cta.data();
    SegmentBarrier* bars = batch.d_bars.data();
    int ns = nsegs;
    void* params[] = {&segs, &cta, &ns, &bars};
    BSG_PROFILE(ctx, "pcg_amg_persistent_batch");
    BSG_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kPcgSellBatch<TK, TV>), total, SB, params, 0,
                                         ctx.stream));
    ctx.launched();
}

template void launchSellPcgBatch<double, double>(Context&, BatchLaunch<double, double>&);
template void launchSellPcgBatch<double, float>(Context&, BatchLaunch<double, float>&);
template void launchSellPcg<double, double>(Context&, const SellPcgArgs<double, double>&);
template void launchSellPcg<double, float>(Context&, const SellPcgArgs<double, float>&);
template void launchSellPcg<float, float>(Context&, const SellPcgArgs<float, float>&);

}  // namespace bsg
