// CTA groups of the persistent solver kernels (device code, sm_100a).
//
// A persistent kernel runs one cooperative launch per solve and separates its
// phases by barriers instead of kernel launches.  GridGroup is the whole
// cooperative grid; SegmentGroup is a contiguous range of its CTAs that owns one
// system of a batch, so one launch can solve several independent systems side by
// side.  Both synchronise through groupBarrier, whose every wait is bounded, and
// gridSum is the deterministic reduction both use.
#pragma once

#include "bsg_internal.h"

namespace bsg {

#ifdef __CUDACC__
constexpr long long kBarrierCycles = 4000000000LL;  // about 2 s at the B200's clock

// Barrier of n CTAs on one word.  Every CTA adds to `count` once per phase: the
// leader adds 2^31 - (n - 1), the others 1, so the n arrivals add exactly 2^31 and
// the top bit flips when the last one lands, while the low 31 bits come back to
// where they were (zero: the word is reset before each launch).  A CTA leaves
// when the top bit differs from the value its own add returned.  The add is a
// gpu-scope release (after __syncthreads, so it covers the whole CTA's writes);
// the poll uses relaxed loads and one acquire fence follows the flip.  All CTAs
// of a cooperative launch are resident, so the flip always comes unless a CTA
// skipped the barrier; the wait is bounded all the same: past kBarrierCycles the
// CTA records an abort (and, first of all, where it was and what it saw) and
// returns, and later barriers of the group stop waiting, so the launch ends and
// the host reports status 3 instead of hanging the GPU.
__device__ __forceinline__ unsigned arriveRelease(unsigned* word, unsigned add) {
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(word), "r"(add) : "memory");
    return old;
}
__device__ __forceinline__ unsigned loadRelaxed(const unsigned* word) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(word) : "memory");
    return v;
}

// Thread 0's barrier bookkeeping lives in shared memory, out of the registers of
// the kernels' hot loops: the number of this CTA's latest barrier and where the
// launch records it.
struct BarrierBook {
    unsigned seq;
    unsigned* progress;
};
__device__ __forceinline__ BarrierBook& barrierBook() {
    __shared__ BarrierBook book;
    return book;
}
__device__ __forceinline__ void openBarrierBook(const SegmentBarrier* bar) {
    if (threadIdx.x == 0) barrierBook() = BarrierBook{0u, bar->progress};
}

// Thread 0's part of a barrier: arrive, wait for the flip (bounded), acquire.
// Returns 1 when it left on the group's abort (its own timeout or another CTA's).
__device__ __forceinline__ int arriveAndWait(SegmentBarrier* bar, bool leader, int n) {
    const unsigned add = leader ? 0x80000000u - static_cast<unsigned>(n - 1) : 1u;
    const unsigned old = arriveRelease(&bar->count, add);
    BarrierBook& book = barrierBook();
    const unsigned seq = ++book.seq;
    // recorded after the arrival, so the release above never waits on this store
    if (book.progress) book.progress[blockIdx.x] = seq;
    long long t0 = 0;
    int stop = 0;
    for (unsigned spins = 1;; ++spins) {
        const unsigned cur = loadRelaxed(&bar->count);
        if ((cur ^ old) & 0x80000000u) break;
        if ((spins & 255u) != 0u) continue;
        if (*reinterpret_cast<volatile int*>(&bar->abort)) {
            stop = 1;
            break;
        }
        const long long now = clock64();
        if (spins == 256u) {
            t0 = now;
        } else if (now - t0 > kBarrierCycles) {
            if (atomicCAS(&bar->who, 0, static_cast<int>(blockIdx.x) + 1) == 0) {
                bar->where = seq;
                bar->seen = cur;
            }
            __threadfence();
            atomicExch(&bar->abort, 1);
            stop = 1;
            break;
        }
    }
    asm volatile("fence.acq_rel.gpu;" ::: "memory");  // the acquire that pairs with the last arrival
    return stop;
}

// Returns thread 0's result of arriveAndWait: the same value for every thread of
// the CTA, so a loop that stops on it stops in all of them.  Out of line: on the
// 1M-cell pressure solves every inlined copy slowed the sweeps between barriers
// (52.4 against 47.3 ms per SIMPLE iteration), while the call costs nothing visible.
__device__ static __noinline__ int groupBarrier(SegmentBarrier* bar, bool leader, int n) {
    __shared__ int aborted;
    __syncthreads();
    if (threadIdx.x == 0) aborted = arriveAndWait(bar, leader, n);
    __syncthreads();
    // the next write to `aborted` comes after the next barrier's first __syncthreads,
    // which every thread reaches only after this read
    return aborted;
}

// aborted(): this CTA has left a wait on the group's abort (sticky, uniform within
// the CTA; for stopping loops).  failed(): the group's flag in memory, read once
// at the end for the launch's status, since a CTA may pass every barrier it
// reaches after another CTA gave up.
struct GridGroup {
    SegmentBarrier* bar;
    int stop = 0;
    __device__ explicit GridGroup(SegmentBarrier* b) : bar(b) { openBarrierBook(b); }
    __device__ __forceinline__ int rank() const { return blockIdx.x; }
    __device__ __forceinline__ int size() const { return gridDim.x; }
    __device__ __forceinline__ bool aborted() const { return stop != 0; }
    __device__ __forceinline__ bool failed() const { return *reinterpret_cast<volatile int*>(&bar->abort) != 0; }
    __device__ __forceinline__ void sync() { stop |= groupBarrier(bar, blockIdx.x == 0, gridDim.x); }
};

struct SegmentGroup {
    int cta0, ncta;
    SegmentBarrier* bar;
    int stop = 0;
    __device__ SegmentGroup(int c0, int n, SegmentBarrier* b) : cta0(c0), ncta(n), bar(b) { openBarrierBook(b); }
    __device__ __forceinline__ int rank() const { return blockIdx.x - cta0; }
    __device__ __forceinline__ int size() const { return ncta; }
    __device__ __forceinline__ bool aborted() const { return stop != 0; }
    __device__ __forceinline__ bool failed() const { return *reinterpret_cast<volatile int*>(&bar->abort) != 0; }
    __device__ __forceinline__ void sync() { stop |= groupBarrier(bar, rank() == 0, ncta); }
};

struct Lanes {
    int lane, gwarp, nwarps, gthread, nthreads;
};

template <int BS, class G>
__device__ __forceinline__ Lanes lanes(const G& g) {
    Lanes c;
    c.gthread = g.rank() * BS + threadIdx.x;
    c.nthreads = g.size() * BS;
    c.lane = threadIdx.x & 31;
    c.gwarp = c.gthread >> 5;
    c.nwarps = c.nthreads >> 5;
    return c;
}

// Deterministic grid sum of NV values (FP64); every block returns the same
// totals.  `buf` alternates between two halves of `partial` so a fast block's
// next write never overtakes a slow block's read of the previous sum.
template <int NV, int BS, class G>
__device__ void gridSum(G& g, double v[NV], double* partial, int& buf) {
    __shared__ double sh[NV][BS / 32];
    __shared__ double tot[NV];
    double* part = partial + static_cast<long long>(buf) * g.size() * NV;
    buf ^= 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double x = v[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[j][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double s = 0.0;
            for (int w = 0; w < BS / 32; ++w) s += sh[j][w];
            part[g.rank() * NV + j] = s;
        }
    }
    g.sync();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double x = 0.0;
        // read at L2 (ld.global.cg): every CTA must see exactly the totals the others see,
        // whatever its SM's L1 still holds of the previous sum on this half
        for (int b = threadIdx.x; b < g.size(); b += BS) x += __ldcg(part + b * NV + j);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[j][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double s = 0.0;
            for (int w = 0; w < BS / 32; ++w) s += sh[j][w];
            tot[j] = s;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = tot[j];
    __syncthreads();
}

#endif

}  // namespace bsg
