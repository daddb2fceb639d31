// Sliced-ELL ("SELL-32") storage of the off-diagonal part of a sparse matrix.
//
// Rows are grouped in slices of 32 (one warp).  Inside slice s every row is
// padded to the slice's widest row w_s and the slice is stored column-major:
// entry k of row 32 s + l sits at sptr[s] + 32 k + l.  A warp sweeping its
// slice therefore reads each column-index and value step as one contiguous
// 128-byte (int32) / 256-byte (FP64) or 128-byte (FP32) transaction, one thread
// per row, and issues its gathers four entries at a time.  Padding entries are
// (column = own row, value = 0), so they gather an already cached value and add
// nothing.  Rows past n in the last slice carry (column 0, value 0).
#pragma once

#include "bsg_internal.h"

#include <algorithm>
#include <vector>

namespace bsg {

constexpr int kSellC = 32;
// Entries each thread loads before it gathers (memory-level parallelism of a row sweep).
// 8 against 4: 39.5 against 40.5 ms per outer iteration on the 1M-cell cavity (6: 39.8).
#ifndef BSG_SELL_BATCH
#define BSG_SELL_BATCH 8
#endif
constexpr int kSellBatch = BSG_SELL_BATCH;

template <class T>
struct SellMat {
    int n = 0;
    int nslices = 0;
    const int* sptr = nullptr;  // nslices + 1 entry offsets
    const int* col = nullptr;
    const T* val = nullptr;
    const T* diag = nullptr;    // n
};

// Host-side pattern: slice offsets and padded column indices of a CSR pattern.
struct SellPattern {
    int n = 0, nslices = 0;
    long long entries = 0;
    std::vector<int> sptr, col;
    void build(int rows, const int* ptr, const int* colidx) {
        n = rows;
        nslices = (rows + kSellC - 1) / kSellC;
        sptr.assign(nslices + 1, 0);
        for (int s = 0; s < nslices; ++s) {
            int w = 0;
            for (int l = 0; l < kSellC; ++l) {
                const int i = kSellC * s + l;
                if (i < rows) w = std::max(w, ptr[i + 1] - ptr[i]);
            }
            sptr[s + 1] = sptr[s] + kSellC * w;
        }
        entries = sptr[nslices];
        col.assign(static_cast<std::size_t>(entries), 0);
        for (int s = 0; s < nslices; ++s) {
            const int w = (sptr[s + 1] - sptr[s]) / kSellC;
            for (int l = 0; l < kSellC; ++l) {
                const int i = kSellC * s + l;
                for (int k = 0; k < w; ++k) {
                    int c = i < rows ? i : 0;
                    if (i < rows && k < ptr[i + 1] - ptr[i]) c = colidx[ptr[i] + k];
                    col[static_cast<std::size_t>(sptr[s]) + kSellC * k + l] = c;
                }
            }
        }
    }
};

#ifdef __CUDACC__
// sum_k a_ik y(col_ik) over this lane's row of slice s (lane = row within the slice).
// Entries go in batches of kSellBatch: all index and value loads of a batch first, then
// all its gathers; the entries past the last full batch follow one at a time.  (A
// predicated last batch, which would shorten a row's chain of dependent load rounds,
// measured slower on the 1M-cell pressure solves: 36.8 against 31.0 ms per outer
// iteration.)
template <class T, class Y>
__device__ __forceinline__ T sellRow(const SellMat<T>& A, int s, int lane, Y y) {
    const int beg = A.sptr[s];
    const int w = (A.sptr[s + 1] - beg) >> 5;
    const int* __restrict__ c = A.col + beg + lane;
    const T* __restrict__ v = A.val + beg + lane;
    T a0 = T(0), a1 = T(0);
    int k = 0;
    for (; k + kSellBatch <= w; k += kSellBatch) {
        int cc[kSellBatch];
        T vv[kSellBatch];
#pragma unroll
        for (int u = 0; u < kSellBatch; ++u) {
            cc[u] = __ldg(c + 32 * (k + u));
            vv[u] = __ldg(v + 32 * (k + u));
        }
        T yy[kSellBatch];
#pragma unroll
        for (int u = 0; u < kSellBatch; ++u) yy[u] = y(cc[u]);
#pragma unroll
        for (int u = 0; u < kSellBatch; u += 2) {
            a0 += vv[u] * yy[u];
            if (u + 1 < kSellBatch) a1 += vv[u + 1] * yy[u + 1];
        }
    }
    for (; k < w; ++k) a0 += __ldg(v + 32 * k) * y(__ldg(c + 32 * k));
    return a0 + a1;
}

// The same row sum split over K consecutive lanes (K a power of two, 2..32): lane q
// of the group takes entries q, q + K, ... of row r of slice s, and the group's
// partial sums are combined in a fixed butterfly order, so every lane of the
// group returns the same, deterministic total.  For levels whose slices leave
// warps idle: the dependent index -> gather chain of a wide row gets K times
// shorter.  Every lane of the warp must call it (the butterfly uses the full mask).
template <class T, class Y>
__device__ __forceinline__ T sellRowSplit(const SellMat<T>& A, int s, int r, int q, int K, Y y) {
    const int beg = A.sptr[s];
    const int w = (A.sptr[s + 1] - beg) >> 5;
    const int* __restrict__ c = A.col + beg + r;
    const T* __restrict__ v = A.val + beg + r;
    T a0 = T(0), a1 = T(0);
    int k = q;
    for (; k + K < w; k += 2 * K) {
        const int c0 = __ldg(c + 32 * k), c1 = __ldg(c + 32 * (k + K));
        const T v0 = __ldg(v + 32 * k), v1 = __ldg(v + 32 * (k + K));
        const T y0 = y(c0), y1 = y(c1);
        a0 += v0 * y0;
        a1 += v1 * y1;
    }
    if (k < w) a0 += __ldg(v + 32 * k) * y(__ldg(c + 32 * k));
    T a = a0 + a1;
    for (int o = K >> 1; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    return a;
}

// Values of a CSR matrix (FP64) scattered into SELL positions, converted to T;
// diag and omega/diag converted alongside.  Padding entries are never written.
template <class T>
__global__ void kCsrToSell(int n, const int* __restrict__ ptr, const double* __restrict__ val,
                           const double* __restrict__ diag, const int* __restrict__ sptr, double omega,
                           T* __restrict__ sval, T* __restrict__ sdiag, T* __restrict__ rd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int base = sptr[i >> 5] + (i & 31);
    const int k0 = ptr[i], len = ptr[i + 1] - k0;
    for (int j = 0; j < len; ++j) sval[base + 32 * j] = static_cast<T>(val[k0 + j]);
    if (sdiag) sdiag[i] = static_cast<T>(diag[i]);
    if (rd) rd[i] = static_cast<T>(omega / diag[i]);
}
#endif

}  // namespace bsg
