// Persistent cooperative PCG with an aggregation-AMG V-cycle on SELL-32 levels.
//
// One cooperative launch solves A x = b to the internal target (or the
// iteration budget).  Every matrix sweep is one thread per row over SELL-32
// slices (sell.cuh), so each warp streams its slice's column indices and values
// as contiguous transactions and keeps four gathers per thread in flight.
//
// V-cycle (levels 0..L-1, aggregates from pairwise matching, piecewise-constant
// transfer, damped Jacobi, dense inverse on the coarsest level), per level l on
// the way down:
//   D1  x = w + rd (b - A w)            (second Jacobi sweep; w = rd b is the first)
//   D2  t = b - A x                     (residual, one thread per fine row)
//   D3  b_c = P^T t, w_c = rd_c b_c     (coarse rows sum their members)
// coarsest: x_c = A_c^-1 b_c, pushed straight into the finer iterate
// (x_f[i] += gamma x_c[agg(i)], every fine row belongs to one aggregate), and on
// the way up:
//   U1  t = y + rd (b - A y)            (y = the prolongated iterate held in x)
//   U2  out = t + rd (b - A t)          (level 0: z; otherwise pushed into the
//                                        finer level's iterate as above)
// With one smoothing step D1 and U2 drop out (x = w, out = t).
//
// The Krylov vectors use TK and the V-cycle TV (FP64/FP64 for the plain path;
// FP32 V-cycle data for the mixed-precision path).  Reductions accumulate in
// FP64 and are deterministic (fixed-order two-stage sums), so runs repeat
// bit for bit.
#pragma once

#include "group.cuh"
#include "pcg_persistent.cuh"
#include "sell.cuh"

#include <vector>

namespace bsg {

template <class TV>
struct VLevel {
    SellMat<TV> A;
    const TV* rd = nullptr;        // omega / diag
    const int* agg_ptr = nullptr;  // next-coarser row -> its members on this level (nullptr on the coarsest)
    const int* agg_rows = nullptr;
    TV* b = nullptr;  // right-hand side
    TV* w = nullptr;  // first Jacobi sweep rd b
    TV* x = nullptr;  // pre-smoothed, then prolongated iterate
    TV* t = nullptr;  // residual on the way down, first post sweep on the way up
};

template <class TV>
struct VCycleView {
    int levels = 0;
    int nu = 2;
    TV gamma = TV(1);
    const VLevel<TV>* lv = nullptr;  // device array of `levels` views
    const TV* dense_inv = nullptr;   // coarsest inverse, n x n row-major
};

template <class TK, class TV>
struct SellPcgArgs {
    SellMat<TK> A;   // level-0 matrix in the Krylov precision
    VCycleView<TV> V;
    const TK* b;
    TK* x;
    TK* r;
    TK* z;
    TK* p0;
    TK* p1;
    TK* q;
    double* partial;
    PcgState* st;
    PhaseLog log;
    // 1: flexible (Polak-Ribiere) beta = r_new.(z_new - z_old) / r_old.z_old, for a
    // preconditioner that is not exactly the same linear operator every iteration
    // (an FP32 V-cycle); 0: beta = r_new.z_new / r_old.z_old.
    int flexible = 0;
    // Second residual buffer.  When given (and the V-cycle has one smoothing step and at
    // least two levels) the Krylov update of x and r is fused with the level-0 residual
    // sweep of the next V-cycle: neighbours' r are read from one buffer while the new r
    // goes to the other, saving one grid-wide phase and one pass over the vectors per
    // CG iteration.
    TK* r2 = nullptr;
};

// Launch (pcg_sell.cu); the grid is sized for co-residency.
template <class TK, class TV>
void launchSellPcg(Context& ctx, const SellPcgArgs<TK, TV>& args);

// Several independent systems (each with its own matrix, V-cycle, vectors, partials
// and PcgState, anywhere in device memory) solved by one cooperative launch: system s
// runs on CTAs [cta_begin[s], cta_begin[s+1]) with barriers of its own, so the systems
// neither wait for nor perturb one another, and each runs the kernel a single solve on
// that many CTAs would run.  The host fills args and cta_begin; the launch uploads them.
template <class TK, class TV>
struct BatchLaunch {
    std::vector<SellPcgArgs<TK, TV>> args;
    std::vector<int> cta_begin;  // args.size() + 1 entries, first 0, last = total CTAs
    DeviceArray<SellPcgArgs<TK, TV>> d_args;
    DeviceArray<int> d_cta;
    DeviceArray<SegmentBarrier> d_bars;
};

// CTAs one batched launch may use (the co-resident grid of the persistent kernel).
int sellBatchCapacity(Context& ctx);
template <class TK, class TV>
void launchSellPcgBatch(Context& ctx, BatchLaunch<TK, TV>& batch);

}  // namespace bsg
