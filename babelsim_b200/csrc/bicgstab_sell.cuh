// Persistent cooperative BiCGStab for C right-hand sides sharing one matrix
// (the momentum equation's three velocity components, the reference's
// kspType bcgs: KSPBCGS, src/backend/petsc_linear_system.cpp:43-50, solved per
// component by PetscBackend, petsc_backend.cpp:156-198).
//
// One cooperative launch runs the whole Jacobi-preconditioned BiCGStab
// iteration for every component in lockstep, each component with its own
// scalars and stopping test, and ends with the true residual b - A x of every
// component, so a solve costs one launch per acceptance attempt and no host
// round trip per iteration.  Products read the SELL-32 copy of the matrix (one
// warp per slice of 32 rows, one read of each entry for all components).
// Reductions are deterministic fixed-order grid sums.  A batch runs several
// independent systems in one launch, each on its own CTA range (group.cuh).
#pragma once

#include "group.cuh"
#include "sell.cuh"

#include <vector>

namespace bsg {

// Per-component state of one persistent BiCGStab launch (host-visible).
struct BicgState {
    double target2[3];  // squared internal target; < 0: max(atol, rtol max(||r0||, ||b||))^2 from this launch
    double atol, rtol;
    int done[3];        // in: 1 for a component that takes no part; out: 1 converged, 2 breakdown, 0 budget spent
    int iters[3];       // in: iterations already used; out: total
    int max_iters;
    double rr0[3];      // out: ||b - A x||^2 at the start of this launch
    double bb[3];       // out: ||b||^2
    double fin2[3];     // out: true residual ||b - A x||^2 at the end
    int status;         // out: 0 ok, 3 a barrier wait ran past its bound
};

// T: the type of the matrix copy, the vectors and their arithmetic (double, or float for
// the inner iterations of a mixed-precision solve); reductions are summed in FP64.
template <int C, class T = double>
struct BicgArgs {
    SellMat<T> A;            // SELL-32 copy of the matrix (diag included)
    const T* b;              // C-interleaved right-hand sides
    T* x;                    // C-interleaved initial guess / solution
    T *r, *r0, *p, *v, *ph, *sh, *t;  // C * n each
    double* partial;         // 2 * ctas * 2C doubles
    BicgState* st;
};

template <int C>
struct BicgBatch {
    std::vector<BicgArgs<C>> args;
    std::vector<int> cta_begin;
    DeviceArray<BicgArgs<C>> d_args;
    DeviceArray<int> d_cta;
    DeviceArray<SegmentBarrier> d_bars;
};

// Resident CTAs of the persistent BiCGStab kernel (the grid of one solve).
int bicgstabGrid(Context& ctx);
template <int C, class T>
void launchBicgstab(Context& ctx, const BicgArgs<C, T>& args);
template <int C>
void launchBicgstabBatch(Context& ctx, BicgBatch<C>& batch);

}  // namespace bsg
