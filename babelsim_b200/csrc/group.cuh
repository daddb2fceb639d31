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
// where they were (zero: the word is zeroed before each launch).  A CTA leaves
// when the top bit differs from the value its own add returned.  All CTAs of a
// cooperative launch are resident, so the flip always comes unless a CTA skipped
// the barrier; the wait is bounded all the same: past kBarrierCycles the CTA
// records an abort and returns, and later barriers of the group stop waiting, so
// the launch ends and the host reports status 3 instead of hanging the GPU.
__device__ __forceinline__ void groupBarrier(SegmentBarrier* bar, bool leader, int n) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned add = leader ? 0x80000000u - static_cast<unsigned>(n - 1) : 1u;
        __threadfence();  // this CTA's writes before its arrival
        const unsigned old = atomicAdd(&bar->count, add);
        volatile unsigned* word = &bar->count;
        volatile int* abort = &bar->abort;
        long long t0 = 0;
        for (unsigned spins = 1; ((*word ^ old) & 0x80000000u) == 0u; ++spins) {
            if ((spins & 255u) != 0u) continue;
            if (*abort) break;
            const long long now = clock64();
            if (spins == 256u) t0 = now;
            else if (now - t0 > kBarrierCycles) {
                atomicExch(&bar->abort, 1);
                break;
            }
        }
        __threadfence();  // the other CTAs' writes before this CTA reads them
    }
    __syncthreads();
}

// The CTAs that cooperate on one solve.  GridGroup: the whole cooperative grid.
// SegmentGroup: a contiguous range of the grid's CTAs that owns one system of a
// batch.  Each has its own zeroed SegmentBarrier.
struct GridGroup {
    SegmentBarrier* bar;
    __device__ __forceinline__ int rank() const { return blockIdx.x; }
    __device__ __forceinline__ int size() const { return gridDim.x; }
    __device__ __forceinline__ bool aborted() const { return *reinterpret_cast<volatile int*>(&bar->abort) != 0; }
    __device__ __forceinline__ void sync() { groupBarrier(bar, blockIdx.x == 0, gridDim.x); }
};

struct SegmentGroup {
    int cta0, ncta;
    SegmentBarrier* bar;
    __device__ __forceinline__ int rank() const { return blockIdx.x - cta0; }
    __device__ __forceinline__ int size() const { return ncta; }
    __device__ __forceinline__ bool aborted() const { return *reinterpret_cast<volatile int*>(&bar->abort) != 0; }
    __device__ __forceinline__ void sync() { groupBarrier(bar, rank() == 0, ncta); }
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
        for (int b = threadIdx.x; b < g.size(); b += BS) x += part[b * NV + j];
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
