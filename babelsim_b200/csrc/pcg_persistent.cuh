// Persistent cooperative PCG with the aggregation-AMG V-cycle inside one kernel.
//
// One launch solves A x = b to the internal target (or the iteration budget):
// every phase (SpMV, vector updates, each V-cycle level's smoothing,
// restriction, prolongation, the coarsest dense solve) is a grid-stride loop
// over rows, separated by cooperative-groups grid barriers (about 1.2 us on
// B200) instead of kernel launches.  Row operations use groups of 4 lanes per
// row (rows carry ~15 off-diagonals on every level), so the small coarse levels
// still spread over the whole GPU.  Grid reductions are deterministic: every
// block writes one partial, and after the barrier every block sums all partials
// in the same order, so all blocks take identical scalar decisions.
#pragma once

#include "bsg_internal.h"

namespace bsg {

constexpr int kMaxAmgLevels = 16;

template <class T>
struct AmgLevelView {
    int n;
    const int* ptr;
    const int* col;
    const T* diag;
    const T* val;
    const T* rd;          // omega / diag
    const int* agg;       // fine row -> next-level row (nullptr on the coarsest level)
    const int* agg_ptr;   // next-level row -> members (stored on this level)
    const int* agg_rows;
    T* x;                 // level iterate
    T* b;                 // level right-hand side (unused on level 0)
    T* t;                 // scratch
};

template <class T>
struct AmgView {
    int levels = 0;
    int nu = 2;                           // smoothing sweeps (1 or 2, fused into one pass each way)
    const AmgLevelView<T>* lv = nullptr;  // device array of `levels` views
    const T* dense_inv = nullptr;         // coarsest inverse, row i at dense_inv + i*dense_ld
    int dense_ld = 0;
    double gamma = 1.0;                   // coarse-correction scale: x += gamma * P x_c
};

// Optional phase timeline of a persistent solve: block 0 / thread 0 appends
// (phase id, %globaltimer ns) after every grid barrier, up to `capacity` entries.
struct PhaseLog {
    long long* entries = nullptr;  // 2 * capacity
    int capacity = 0;
    int* count = nullptr;
};

// Scalars of one persistent solve (host-visible results at the end).
struct PcgState {
    double target2;        // squared internal target on the recursive residual
    double rr;             // last squared recursive residual norm
    double rr0, bb;        // squared initial residual and rhs norms
    int iterations;        // iterations done in this launch
    int status;            // 0 converged (recursive), 1 budget spent, 2 breakdown
    int max_iterations;
    int warm;              // 1: x is the initial guess, 0: start from x = 0
    double atol, rtol;     // acceptance contract (target computed in the kernel when target2 < 0)
};

}  // namespace bsg
