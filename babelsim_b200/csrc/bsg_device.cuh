// Device-side views and boundary evaluation shared by the finite-volume kernels.
#pragma once

#include "bsg_internal.h"

#include <math.h>

namespace bsg {

// Raw pointers of a DeviceMesh, passed to kernels by value.
struct MeshView {
    int n_cells, n_interior, n_boundary;
    const double *V, *rV, *xc;
    const int *own, *nbr;
    const double *w, *dcoef, *area, *Sf, *xf, *kvec, *skew;
    const int *bown, *bpatch;
    const double *bdcoef, *barea, *bdist, *bSf, *bxf, *bn, *bk;
    const int *cf_ptr, *cf_face, *cf_col, *cb_ptr;
    const int *slot_own, *slot_nbr;  // the owner-row and neighbour-row matrix slots of each interior face
};

inline MeshView view(const DeviceMesh& m) {
    return MeshView{m.n_cells, m.n_interior, m.n_boundary, m.V.data(), m.rV.data(), m.xc.data(),
                    m.own.data(), m.nbr.data(), m.w.data(), m.dcoef.data(), m.area.data(), m.Sf.data(),
                    m.xf.data(), m.kvec.data(), m.skew.data(), m.bown.data(), m.bpatch.data(),
                    m.bdcoef.data(), m.barea.data(), m.bdist.data(), m.bSf.data(), m.bxf.data(),
                    m.bn.data(), m.bk.data(), m.cf_ptr.data(), m.cf_face.data(), m.cf_col.data(),
                    m.cb_ptr.data(), m.slot_own.data(), m.slot_nbr.data()};
}

// Boundary constraints of one cell field.  A calculated field has `trace`
// (fixed value per boundary face); otherwise `bc` per patch, with the saved
// boundary-flux context `flux` (per boundary face) for inletOutlet.
struct BcView {
    const PatchBC* bc;
    const double* trace;
    const double* flux;
};

constexpr int FV = 0, FG = 1, ZG = 2, IO = 3, SY = 4;

// Field::faceCondition (include/babelsim/field.h:285-301).  `outward` is the
// explicit flux argument or NaN to use the saved context.
template <int C>
__device__ __forceinline__ int faceCondition(const MeshView& m, const BcView& b, int fb, double outward,
                                             double val[C]) {
    if (b.trace) {
#pragma unroll
        for (int c = 0; c < C; ++c) val[c] = b.trace[C * fb + c];
        return FV;
    }
    const PatchBC p = b.bc[m.bpatch[fb]];
    int t = p.type;
#pragma unroll
    for (int c = 0; c < C; ++c) val[c] = p.value[c];
    if (t == IO) {
        double fl = outward;
        if (isnan(fl)) fl = b.flux ? b.flux[fb] : 0.0;
        if (fl < 0.0) t = FV;
        else {
            t = ZG;
#pragma unroll
            for (int c = 0; c < C; ++c) val[c] = 0.0;
        }
    }
    return t;
}

// Field::boundaryTrace (field.h:302-313).
template <int C>
__device__ __forceinline__ void boundaryTrace(const MeshView& m, const BcView& b, const double* x, int fb,
                                              double outward, double out[C]) {
    double val[C];
    const int t = faceCondition<C>(m, b, fb, outward, val);
    const int o = m.bown[fb];
#pragma unroll
    for (int c = 0; c < C; ++c) out[c] = x[C * o + c];
    if (t == FV) {
#pragma unroll
        for (int c = 0; c < C; ++c) out[c] = val[c];
    } else if (t == FG) {
        const double d = m.bdist[fb];
#pragma unroll
        for (int c = 0; c < C; ++c) out[c] += d * val[c];
    } else if (t == SY && C == 3) {
        const double* n = m.bn + 3 * fb;
        const double un = out[0] * n[0] + out[1] * n[1] + out[2] * n[2];
#pragma unroll
        for (int c = 0; c < C; ++c) out[c] -= un * n[c];
    }
}

// reconstructedBoundaryValue (src/discretization/operators.cpp:110-164).
// g holds 3*C gradient entries per cell (row c = gradient of component c).
template <int C>
__device__ __forceinline__ void reconstructedBoundary(const MeshView& m, const BcView& b, const double* x,
                                                      const double* g, int fb, double outward, double out[C]) {
    double val[C];
    const int t = faceCondition<C>(m, b, fb, outward, val);
    if (t == FV) {
#pragma unroll
        for (int c = 0; c < C; ++c) out[c] = val[c];
        return;
    }
    const int o = m.bown[fb];
    const double* n = m.bn + 3 * fb;
    const double off0 = m.bxf[3 * fb] - m.xc[3 * o], off1 = m.bxf[3 * fb + 1] - m.xc[3 * o + 1],
                 off2 = m.bxf[3 * fb + 2] - m.xc[3 * o + 2];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const double* gc = g + 3 * (C * o + c);
        const double pres = t == FG ? val[c] : 0.0;
        const double gn = gc[0] * n[0] + gc[1] * n[1] + gc[2] * n[2];
        const double k = pres - gn;
        out[c] = x[C * o + c] + (gc[0] + k * n[0]) * off0 + (gc[1] + k * n[1]) * off1 + (gc[2] + k * n[2]) * off2;
    }
    if (t == SY && C == 3) {
        const double un = out[0] * n[0] + out[1] * n[1] + out[2] * n[2];
#pragma unroll
        for (int c = 0; c < C; ++c) out[c] -= un * n[c];
    }
}

// limitNonOrthogonalCorrection (operators.cpp:499-513); method 1 corrected, 2 limited.
__device__ __forceinline__ double limitCorrection(double orth, double corr, int method) {
    if (method == 1) return corr;
    if (method == 2) {
        const double bnd = fabs(orth);
        return fmin(fmax(corr, -bnd), bnd);
    }
    return 0.0;
}

// Deterministic block reduction of NV doubles (sum); result valid in thread 0.
template <int NV, int BLOCK>
__device__ __forceinline__ void blockSum(double v[NV]) {
    __shared__ double sh[NV][BLOCK / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double x = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[i][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double x = lane < BLOCK / 32 ? sh[i][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[i] = x;
        }
    }
    __syncthreads();
}

}  // namespace bsg
