// CTA groups of the persistent solver kernels (device code, sm_100a).
//
// A persistent kernel runs one cooperative launch per solve and separates its
// phases by barriers instead of kernel launches.  GridGroup is the whole
// cooperative grid; SegmentGroup is a contiguous range of its CTAs that owns one
// system of a batch, so one launch can solve several independent systems side by
// side.  gridSum is the deterministic reduction both use.
#pragma once

#include <cooperative_groups.h>

#include "bsg_internal.h"

namespace bsg {

// Barrier state of one system of a batch (zeroed before every launch).
struct SegmentBarrier {
    unsigned count;
    unsigned generation;
    int abort;   // set when a wait ran past its bound; the system then reports status 3
    int pad;
};

#ifdef __CUDACC__
namespace cgx = cooperative_groups;

// The CTAs that cooperate on one solve.  GridGroup: the whole cooperative grid,
// synchronised by cooperative groups.  SegmentGroup: a contiguous range of the
// grid's CTAs that owns one system of a batch; its barrier is a counter and a
// generation word in global memory (all CTAs of a cooperative launch are
// resident, so the spin always ends), and every wait is bounded: past
// kBarrierCycles the group records an abort and its barriers stop waiting, so
// the launch ends and the host reports the failure instead of hanging.
struct GridGroup {
    cgx::grid_group g;
    __device__ GridGroup() : g(cgx::this_grid()) {}
    __device__ __forceinline__ int rank() const { return blockIdx.x; }
    __device__ __forceinline__ int size() const { return gridDim.x; }
    __device__ __forceinline__ void sync() { g.sync(); }
    __device__ __forceinline__ bool aborted() const { return false; }
};

constexpr long long kBarrierCycles = 4000000000LL;  // about 2 s at the B200's clock

struct SegmentGroup {
    int cta0, ncta;
    SegmentBarrier* bar;
    __device__ __forceinline__ int rank() const { return blockIdx.x - cta0; }
    __device__ __forceinline__ int size() const { return ncta; }
    __device__ __forceinline__ bool aborted() const { return *reinterpret_cast<volatile int*>(&bar->abort) != 0; }
    __device__ void sync() {
        __syncthreads();
        if (threadIdx.x == 0) {
            volatile unsigned* gen = &bar->generation;
            const unsigned g0 = *gen;
            __threadfence();
            if (atomicAdd(&bar->count, 1u) == static_cast<unsigned>(ncta) - 1u) {
                atomicExch(&bar->count, 0u);
                __threadfence();
                atomicAdd(&bar->generation, 1u);
            } else {
                const long long t0 = clock64();
                while (*gen == g0) {
                    if (aborted()) break;
                    if (clock64() - t0 > kBarrierCycles) {
                        atomicExch(&bar->abort, 1);
                        break;
                    }
                    __nanosleep(32);
                }
            }
            __threadfence();
        }
        __syncthreads();
    }
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
