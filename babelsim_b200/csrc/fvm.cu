// Finite-volume operators and atomic-free LDU assembly on sm_100a.
//
// Every cell-producing kernel is a row gather over the cell->face CSR: thread i
// walks the interior faces of cell i (cf_ptr/cf_face) and then its boundary
// faces (cb_ptr), so there are no atomics and the summation order is fixed.
// Face-producing kernels run one thread per face.  Kernels cite the reference
// functions they restate (paths inside the BabelSim project).
#include "bsg_device.cuh"
#include "fvm.h"

#include <cmath>

namespace bsg {

namespace {
constexpr int kBlock = 256;
constexpr double kEps = 2.220446049250313e-16;

// ---------------------------------------------------------------- gradients
// greenGaussGradient (operators.cpp:275-316 scalar, 365-405 vector); PASS2 is
// the skew-corrected second pass that uses the first-pass gradient g1.
// orth_cells (second pass only, may be nullptr): cells whose case of a batch has orthogonal
// geometry keep the first-pass gradient.
template <int C, bool PASS2>
__global__ void kGradGauss(MeshView m, BcView b, const double* __restrict__ x, const double* __restrict__ g1,
                           double* __restrict__ out, const unsigned char* __restrict__ orth_cells) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n_cells) return;
    if (PASS2 && orth_cells && orth_cells[i]) {
#pragma unroll
        for (int j = 0; j < 3 * C; ++j) out[3 * C * i + j] = g1[3 * C * i + j];
        return;
    }
    double acc[3 * C];
#pragma unroll
    for (int j = 0; j < 3 * C; ++j) acc[j] = 0.0;
    const double rv = m.rV[i];
    for (int k = m.cf_ptr[i]; k < m.cf_ptr[i + 1]; ++k) {
        const int f = m.cf_face[k];
        const int o = m.own[f], n = m.nbr[f];
        const double sgn = o == i ? 1.0 : -1.0;
        const double w = m.w[f];
        const double s0 = m.Sf[3 * f], s1 = m.Sf[3 * f + 1], s2 = m.Sf[3 * f + 2];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            double val = w * x[C * o + c] + (1.0 - w) * x[C * n + c];
            if (PASS2) {
                const double* go = g1 + 3 * (C * o + c);
                const double* gn = g1 + 3 * (C * n + c);
                val += (w * go[0] + (1.0 - w) * gn[0]) * m.skew[3 * f] +
                       (w * go[1] + (1.0 - w) * gn[1]) * m.skew[3 * f + 1] +
                       (w * go[2] + (1.0 - w) * gn[2]) * m.skew[3 * f + 2];
            }
            acc[3 * c] += sgn * ((val * s0) * rv);
            acc[3 * c + 1] += sgn * ((val * s1) * rv);
            acc[3 * c + 2] += sgn * ((val * s2) * rv);
        }
    }
    for (int fb = m.cb_ptr[i]; fb < m.cb_ptr[i + 1]; ++fb) {
        double val[C];
        if (PASS2) reconstructedBoundary<C>(m, b, x, g1, fb, NAN, val);
        else boundaryTrace<C>(m, b, x, fb, NAN, val);
        const double s0 = m.bSf[3 * fb], s1 = m.bSf[3 * fb + 1], s2 = m.bSf[3 * fb + 2];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            acc[3 * c] += (val[c] * s0) * rv;
            acc[3 * c + 1] += (val[c] * s1) * rv;
            acc[3 * c + 2] += (val[c] * s2) * rv;
        }
    }
#pragma unroll
    for (int j = 0; j < 3 * C; ++j) out[3 * C * i + j] = acc[j];
}

// leastSquaresGradient (operators.cpp:318-363 scalar, 407-458 vector): inverse
// squared-distance weighted normal equations per cell, boundary mirror points,
// solved by an unpivoted 3x3 LDL^T.
template <int C>
__global__ void kGradLeastSquares(MeshView m, BcView b, const double* __restrict__ x, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n_cells) return;
    double a00 = 0, a01 = 0, a02 = 0, a11 = 0, a12 = 0, a22 = 0;
    double r[3 * C];
#pragma unroll
    for (int j = 0; j < 3 * C; ++j) r[j] = 0.0;
    const double xi0 = m.xc[3 * i], xi1 = m.xc[3 * i + 1], xi2 = m.xc[3 * i + 2];
    for (int k = m.cf_ptr[i]; k < m.cf_ptr[i + 1]; ++k) {
        const int other = m.cf_col[k];
        const double d0 = m.xc[3 * other] - xi0, d1 = m.xc[3 * other + 1] - xi1, d2 = m.xc[3 * other + 2] - xi2;
        const double wgt = 1.0 / (d0 * d0 + d1 * d1 + d2 * d2);
        a00 += wgt * d0 * d0; a01 += wgt * d0 * d1; a02 += wgt * d0 * d2;
        a11 += wgt * d1 * d1; a12 += wgt * d1 * d2; a22 += wgt * d2 * d2;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const double diff = x[C * other + c] - x[C * i + c];
            r[3 * c] += wgt * d0 * diff; r[3 * c + 1] += wgt * d1 * diff; r[3 * c + 2] += wgt * d2 * diff;
        }
    }
    for (int fb = m.cb_ptr[i]; fb < m.cb_ptr[i + 1]; ++fb) {
        double cv[C];
        const int t = faceCondition<C>(m, b, fb, NAN, cv);
        double d0, d1, d2;
        if (t == FV) {
            d0 = 2.0 * (m.bxf[3 * fb] - xi0); d1 = 2.0 * (m.bxf[3 * fb + 1] - xi1); d2 = 2.0 * (m.bxf[3 * fb + 2] - xi2);
        } else {
            const double s = 2.0 * m.bdist[fb];
            d0 = s * m.bn[3 * fb]; d1 = s * m.bn[3 * fb + 1]; d2 = s * m.bn[3 * fb + 2];
        }
        double tr[C];
        boundaryTrace<C>(m, b, x, fb, NAN, tr);
        const double wgt = 1.0 / (d0 * d0 + d1 * d1 + d2 * d2);
        a00 += wgt * d0 * d0; a01 += wgt * d0 * d1; a02 += wgt * d0 * d2;
        a11 += wgt * d1 * d1; a12 += wgt * d1 * d2; a22 += wgt * d2 * d2;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const double diff = 2.0 * (tr[c] - x[C * i + c]);
            r[3 * c] += wgt * d0 * diff; r[3 * c + 1] += wgt * d1 * diff; r[3 * c + 2] += wgt * d2 * diff;
        }
    }
    const double D0 = a00, l10 = a01 / D0, l20 = a02 / D0;
    const double D1 = a11 - l10 * l10 * D0, l21 = (a12 - l20 * l10 * D0) / D1;
    const double D2 = a22 - l20 * l20 * D0 - l21 * l21 * D1;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const double y0 = r[3 * c], y1 = r[3 * c + 1] - l10 * y0, y2 = r[3 * c + 2] - l20 * y0 - l21 * y1;
        const double z0 = y0 / D0, z1 = y1 / D1, z2 = y2 / D2;
        const double g2 = z2, g1 = z1 - l21 * g2, g0 = z0 - l10 * g1 - l20 * g2;
        out[3 * C * i + 3 * c] = g0; out[3 * C * i + 3 * c + 1] = g1; out[3 * C * i + 3 * c + 2] = g2;
    }
}

// Boundary traces of a computed scalar gradient (fvm_execution.cpp:213-237).
__global__ void kGradientTrace(MeshView m, BcView b, const double* __restrict__ x, const double* __restrict__ g,
                               double* __restrict__ trace) {
    const int fb = blockIdx.x * blockDim.x + threadIdx.x;
    if (fb >= m.n_boundary) return;
    const int o = m.bown[fb];
    const double n0 = m.bn[3 * fb], n1 = m.bn[3 * fb + 1], n2 = m.bn[3 * fb + 2];
    const double d0 = m.bxf[3 * fb] - m.xc[3 * o], d1 = m.bxf[3 * fb + 1] - m.xc[3 * o + 1],
                 d2 = m.bxf[3 * fb + 2] - m.xc[3 * o + 2];
    double g0 = g[3 * o], g1 = g[3 * o + 1], g2 = g[3 * o + 2];
    double cv[1];
    const int t = faceCondition<1>(m, b, fb, NAN, cv);
    const double dn = d0 * n0 + d1 * n1 + d2 * n2;
    double sn = 0.0;
    if (t == FV) {
        const double t0 = d0 - dn * n0, t1 = d1 - dn * n1, t2 = d2 - dn * n2;
        sn = (cv[0] - x[o] - (g0 * t0 + g1 * t1 + g2 * t2)) / dn;
    } else if (t == FG) {
        sn = cv[0];
    }
    const double k = sn - (g0 * n0 + g1 * n1 + g2 * n2);
    trace[3 * fb] = g0 + k * n0; trace[3 * fb + 1] = g1 + k * n1; trace[3 * fb + 2] = g2 + k * n2;
}

// ------------------------------------------------------------ interpolation
// interpolatedFaceValue / correctedFaceValue over all faces (operators.cpp:34-81,
// 166-186, 231-237); internal face order: interior, then boundary.
template <int C, bool CORRECTED>
__global__ void kInterpolate(MeshView m, BcView b, const double* __restrict__ x, const double* __restrict__ g,
                             double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m.n_interior) {
        const int o = m.own[t], n = m.nbr[t];
        const double w = m.w[t];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            double val = w * x[C * o + c] + (1.0 - w) * x[C * n + c];
            if (CORRECTED) {
                const double* go = g + 3 * (C * o + c);
                const double* gn = g + 3 * (C * n + c);
                val += (w * go[0] + (1.0 - w) * gn[0]) * m.skew[3 * t] +
                       (w * go[1] + (1.0 - w) * gn[1]) * m.skew[3 * t + 1] +
                       (w * go[2] + (1.0 - w) * gn[2]) * m.skew[3 * t + 2];
            }
            out[C * t + c] = val;
        }
    } else if (t < m.n_interior + m.n_boundary) {
        const int fb = t - m.n_interior;
        double val[C];
        if (CORRECTED) reconstructedBoundary<C>(m, b, x, g, fb, NAN, val);
        else boundaryTrace<C>(m, b, x, fb, NAN, val);
#pragma unroll
        for (int c = 0; c < C; ++c) out[C * t + c] = val[c];
    }
}

// flux of a cell vector: face value . Sf (operators.cpp:957-1002).
template <bool CORRECTED>
__global__ void kFlux(MeshView m, BcView b, const double* __restrict__ U, const double* __restrict__ g,
                      double* __restrict__ phi) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m.n_interior) {
        const int o = m.own[t], n = m.nbr[t];
        const double w = m.w[t];
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double val = w * U[3 * o + c] + (1.0 - w) * U[3 * n + c];
            if (CORRECTED) {
                const double* go = g + 3 * (3 * o + c);
                const double* gn = g + 3 * (3 * n + c);
                val += (w * go[0] + (1.0 - w) * gn[0]) * m.skew[3 * t] +
                       (w * go[1] + (1.0 - w) * gn[1]) * m.skew[3 * t + 1] +
                       (w * go[2] + (1.0 - w) * gn[2]) * m.skew[3 * t + 2];
            }
            s += val * m.Sf[3 * t + c];
        }
        phi[t] = s;
    } else if (t < m.n_interior + m.n_boundary) {
        const int fb = t - m.n_interior;
        double val[3];
        if (CORRECTED) reconstructedBoundary<3>(m, b, U, g, fb, NAN, val);
        else boundaryTrace<3>(m, b, U, fb, NAN, val);
        phi[t] = val[0] * m.bSf[3 * fb] + val[1] * m.bSf[3 * fb + 1] + val[2] * m.bSf[3 * fb + 2];
    }
}

// Initial inletOutlet direction: owner velocity . Sf (operators.cpp:978-986).
__global__ void kSeedFlux(MeshView m, const double* __restrict__ U, double* __restrict__ bflux) {
    const int fb = blockIdx.x * blockDim.x + threadIdx.x;
    if (fb >= m.n_boundary) return;
    const int o = m.bown[fb];
    bflux[fb] = U[3 * o] * m.bSf[3 * fb] + U[3 * o + 1] * m.bSf[3 * fb + 1] + U[3 * o + 2] * m.bSf[3 * fb + 2];
}

// divergence of an integrated face flux (operators.cpp:1055-1063).
__global__ void kDivFlux(MeshView m, const double* __restrict__ phi, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n_cells) return;
    const double rv = m.rV[i];
    double acc = 0.0;
    for (int k = m.cf_ptr[i]; k < m.cf_ptr[i + 1]; ++k) {
        const int f = m.cf_face[k];
        acc += (m.own[f] == i ? 1.0 : -1.0) * (phi[f] * rv);
    }
    for (int fb = m.cb_ptr[i]; fb < m.cb_ptr[i + 1]; ++fb) acc += phi[m.n_interior + fb] * rv;
    out[i] = acc;
}

// integratedNormalGradient (operators.cpp:857-902) / |Sf| for every face.
__global__ void kNormalGradient(MeshView m, BcView b, const double* __restrict__ x, const double* __restrict__ g,
                                int method, double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m.n_interior) {
        const int o = m.own[t], n = m.nbr[t];
        const double orth = m.dcoef[t] * (x[n] - x[o]);
        double v = orth;
        if (method != 0) {
            const double w = m.w[t];
            const double fg0 = w * g[3 * o] + (1.0 - w) * g[3 * n], fg1 = w * g[3 * o + 1] + (1.0 - w) * g[3 * n + 1],
                         fg2 = w * g[3 * o + 2] + (1.0 - w) * g[3 * n + 2];
            v = orth + limitCorrection(orth, m.kvec[3 * t] * fg0 + m.kvec[3 * t + 1] * fg1 + m.kvec[3 * t + 2] * fg2,
                                       method);
        }
        out[t] = v / m.area[t];
    } else if (t < m.n_interior + m.n_boundary) {
        const int fb = t - m.n_interior, o = m.bown[fb];
        double cv[1];
        const int ty = faceCondition<1>(m, b, fb, NAN, cv);
        double v = 0.0;
        if (ty == FG) v = cv[0] * m.barea[fb];
        else if (ty == FV) {
            const double orth = m.bdcoef[fb] * (cv[0] - x[o]);
            v = orth;
            if (method != 0)
                v = orth + limitCorrection(orth, m.bk[3 * fb] * g[3 * o] + m.bk[3 * fb + 1] * g[3 * o + 1] +
                                                     m.bk[3 * fb + 2] * g[3 * o + 2], method);
        }
        out[t] = v / m.barea[fb];
    }
}

// ---------------------------------------------------------------- assembly
// addConvectionImpl (operators.cpp:535-661) as a row gather: each interior face
// contributes to the slot of this row; method 0 upwind, 1 linearUpwind, 2 central.
template <int C>
__global__ void kAddConvection(MeshView m, BcView b, const double* __restrict__ x, const double* __restrict__ g,
                               const double* __restrict__ phi, int method, double scale, double* __restrict__ diag,
                               double* __restrict__ val, double* __restrict__ src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n_cells) return;
    double d = 0.0, s[C];
#pragma unroll
    for (int c = 0; c < C; ++c) s[c] = 0.0;
    for (int k = m.cf_ptr[i]; k < m.cf_ptr[i + 1]; ++k) {
        const int f = m.cf_face[k];
        const int o = m.own[f], n = m.nbr[f];
        const bool owner = o == i;
        const double F = scale * phi[f];
        if (method != 2) {
            if (owner) { d += fmax(F, 0.0); val[k] += fmin(F, 0.0); }
            else { d += fmax(-F, 0.0); val[k] += fmin(-F, 0.0); }
            if (method == 1) {
                const int up = F >= 0.0 ? o : n;
                const double off0 = m.xf[3 * f] - m.xc[3 * up], off1 = m.xf[3 * f + 1] - m.xc[3 * up + 1],
                             off2 = m.xf[3 * f + 2] - m.xc[3 * up + 2];
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const double* gu = g + 3 * (C * up + c);
                    const double corr = gu[0] * off0 + gu[1] * off1 + gu[2] * off2;
                    s[c] += owner ? -(F * corr) : F * corr;
                }
            }
        } else {
            const double w = m.w[f];
            if (owner) { d += F * w; val[k] += F * (1.0 - w); }
            else { d -= F * (1.0 - w); val[k] -= F * w; }
            if (g) {
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const double* go = g + 3 * (C * o + c);
                    const double* gn = g + 3 * (C * n + c);
                    const double corr = (w * go[0] + (1.0 - w) * gn[0]) * m.skew[3 * f] +
                                        (w * go[1] + (1.0 - w) * gn[1]) * m.skew[3 * f + 1] +
                                        (w * go[2] + (1.0 - w) * gn[2]) * m.skew[3 * f + 2];
                    s[c] += owner ? -(F * corr) : F * corr;
                }
            }
        }
    }
    for (int fb = m.cb_ptr[i]; fb < m.cb_ptr[i + 1]; ++fb) {
        const double F = scale * phi[m.n_interior + fb];
        double cv[C];
        const int t = faceCondition<C>(m, b, fb, F, cv);
        if (method != 2) {
            if (F >= 0.0) {
                d += F;
                if (method == 1) {
                    const double off0 = m.bxf[3 * fb] - m.xc[3 * i], off1 = m.bxf[3 * fb + 1] - m.xc[3 * i + 1],
                                 off2 = m.bxf[3 * fb + 2] - m.xc[3 * i + 2];
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        const double* gi = g + 3 * (C * i + c);
                        s[c] -= F * (gi[0] * off0 + gi[1] * off1 + gi[2] * off2);
                    }
                }
            } else {
                double bv[C];
                boundaryTrace<C>(m, b, x, fb, F, bv);
#pragma unroll
                for (int c = 0; c < C; ++c) s[c] -= F * bv[c];
            }
            continue;
        }
        if (t == FV) {
#pragma unroll
            for (int c = 0; c < C; ++c) s[c] -= F * cv[c];
        } else if (t == FG) {
            const double dist = m.bdist[fb];
            d += F;
#pragma unroll
            for (int c = 0; c < C; ++c) s[c] -= F * dist * cv[c];
        } else {
            d += F;
        }
        if (g) {
            double rb[C], tb[C];
            reconstructedBoundary<C>(m, b, x, g, fb, F, rb);
            boundaryTrace<C>(m, b, x, fb, F, tb);
#pragma unroll
            for (int c = 0; c < C; ++c) s[c] -= F * (rb[c] - tb[c]);
        }
    }
    diag[i] += d;
#pragma unroll
    for (int c = 0; c < C; ++c) src[C * i + c] += s[c];
}

// addScalarDiffusion / addVectorDiffusion (operators.cpp:1287-1438) as a row
// gather, every contribution multiplied by `mult` (accumulate(..., -factor),
// procedural_equation.cpp:62-70).  kf == nullptr means the constant kc.
// Interior faces of a diffusion term, once per face: the coefficient gamma*dcoef
// off both matrix slots, and per slot the record {coefficient, +-gamma*(corrected -
// orthogonal normal gradient)} (sign + on the owner's slot) that the cell pass sums
// (addScalarDiffusion / addVectorDiffusion, operators.cpp:1287-1438, with
// integratedNormalGradient 857-954 and limitNonOrthogonalCorrection 499-513).
template <int C>
__global__ void kDiffusionFaces(MeshView m, const double* __restrict__ x, const double* __restrict__ g,
                                const double* __restrict__ kf, double kc, int method, double mult,
                                double* __restrict__ val, double* __restrict__ slots) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.n_interior) return;
    const int so = m.slot_own[f], sn = m.slot_nbr[f];
    double* ro = slots + static_cast<long long>(1 + C) * so;
    double* rn = slots + static_cast<long long>(1 + C) * sn;
    const double gam = kf ? kf[f] : kc;
    if (gam == 0.0) {
#pragma unroll
        for (int c = 0; c <= C; ++c) { ro[c] = 0.0; rn[c] = 0.0; }
        return;
    }
    const double coef = gam * m.dcoef[f];
    val[so] -= mult * coef;
    val[sn] -= mult * coef;
    ro[0] = coef;
    rn[0] = coef;
    if (method == 0) return;
    const int o = m.own[f], n = m.nbr[f];
    const double w = m.w[f];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const double orth = m.dcoef[f] * (x[C * n + c] - x[C * o + c]);
        const double* go = g + 3 * (C * o + c);
        const double* gn = g + 3 * (C * n + c);
        const double corr = m.kvec[3 * f] * (w * go[0] + (1.0 - w) * gn[0]) +
                            m.kvec[3 * f + 1] * (w * go[1] + (1.0 - w) * gn[1]) +
                            m.kvec[3 * f + 2] * (w * go[2] + (1.0 - w) * gn[2]);
        const double ing = orth + limitCorrection(orth, corr, method);
        const double v = gam * (ing - orth);
        ro[1 + c] = v;
        rn[1 + c] = -v;
    }
}

// Cell pass of a diffusion term: the slot records of the cell's interior faces
// (in slot order) and its boundary faces, into diag and the explicit source.
template <int C>
__global__ void kAddDiffusion(MeshView m, BcView b, const double* __restrict__ x, const double* __restrict__ g,
                              const double* __restrict__ kf, double kc, int method, double mult,
                              const double* __restrict__ slots, double* __restrict__ diag,
                              double* __restrict__ src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n_cells) return;
    double d = 0.0, s[C];
#pragma unroll
    for (int c = 0; c < C; ++c) s[c] = 0.0;
    for (int k = m.cf_ptr[i]; k < m.cf_ptr[i + 1]; ++k) {
        const double* r = slots + static_cast<long long>(1 + C) * k;
        d += r[0];
        if (method != 0) {
#pragma unroll
            for (int c = 0; c < C; ++c) s[c] += r[1 + c];
        }
    }
    for (int fb = m.cb_ptr[i]; fb < m.cb_ptr[i + 1]; ++fb) {
        const double gam = kf ? kf[m.n_interior + fb] : kc;
        if (gam == 0.0) continue;
        double cv[C];
        const int t = faceCondition<C>(m, b, fb, NAN, cv);
        const double coef = gam * m.bdcoef[fb];
        if (t == FG) {
#pragma unroll
            for (int c = 0; c < C; ++c) s[c] += C == 1 ? gam * cv[c] * m.barea[fb] : gam * m.barea[fb] * cv[c];
            continue;
        }
        if (!(t == FV || (C == 3 && t == SY))) continue;
        double bv[C];
        if (C == 1) bv[0] = cv[0];
        else boundaryTrace<C>(m, b, x, fb, -1.0, bv);
        d += coef;
#pragma unroll
        for (int c = 0; c < C; ++c) s[c] += coef * bv[c];
        if (method != 0) {
            const double* nrm = m.bn + 3 * fb;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const double orth = m.bdcoef[fb] * (bv[c] - x[C * i + c]);
                const double* gi = g + 3 * (C * i + c);
                double g0 = gi[0], g1 = gi[1], g2 = gi[2];
                if (C == 3 && t == SY) {
                    const double gnn = g0 * nrm[0] + g1 * nrm[1] + g2 * nrm[2];
                    g0 -= gnn * nrm[0]; g1 -= gnn * nrm[1]; g2 -= gnn * nrm[2];
                }
                const double ing =
                    orth + limitCorrection(orth, m.bk[3 * fb] * g0 + m.bk[3 * fb + 1] * g1 + m.bk[3 * fb + 2] * g2, method);
                s[c] += gam * (ing - orth);
            }
        }
    }
    diag[i] += mult * d;
#pragma unroll
    for (int c = 0; c < C; ++c) src[C * i + c] += mult * s[c];
}

// Frozen explicit correction flux of one diffusion term:
// diffusionFlux(method) - diffusionFlux(orthogonal) (procedural_equation.cpp:77-87).
__global__ void kDiffusionCorrection(MeshView m, BcView b, const double* __restrict__ x, const double* __restrict__ g,
                                     const double* __restrict__ kf, int method, double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m.n_interior) {
        const int o = m.own[t], n = m.nbr[t];
        const double orth = m.dcoef[t] * (x[n] - x[o]);
        const double w = m.w[t];
        const double corr = m.kvec[3 * t] * (w * g[3 * o] + (1.0 - w) * g[3 * n]) +
                            m.kvec[3 * t + 1] * (w * g[3 * o + 1] + (1.0 - w) * g[3 * n + 1]) +
                            m.kvec[3 * t + 2] * (w * g[3 * o + 2] + (1.0 - w) * g[3 * n + 2]);
        out[t] = kf[t] * (orth + limitCorrection(orth, corr, method)) - kf[t] * orth;
    } else if (t < m.n_interior + m.n_boundary) {
        const int fb = t - m.n_interior, o = m.bown[fb];
        double cv[1];
        const int ty = faceCondition<1>(m, b, fb, NAN, cv);
        double full = 0.0, orth = 0.0;
        if (ty == FG) full = orth = cv[0] * m.barea[fb];
        else if (ty == FV) {
            orth = m.bdcoef[fb] * (cv[0] - x[o]);
            full = orth + limitCorrection(orth, m.bk[3 * fb] * g[3 * o] + m.bk[3 * fb + 1] * g[3 * o + 1] +
                                                    m.bk[3 * fb + 2] * g[3 * o + 2], method);
        }
        out[t] = kf[t] * full - kf[t] * orth;
    }
}

// equ::faceFlux term (procedural_equation.cpp:335-352): factor*(kf*orthogonal
// normal gradient of the solution under the frozen constraints + correction).
__global__ void kFaceFluxTerm(MeshView m, BcView b, const double* __restrict__ x, const double* __restrict__ kf,
                              const double* __restrict__ corr, double factor, int first, double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double v;
    if (t < m.n_interior) {
        v = kf[t] * (m.dcoef[t] * (x[m.nbr[t]] - x[m.own[t]]));
    } else if (t < m.n_interior + m.n_boundary) {
        const int fb = t - m.n_interior;
        double cv[1];
        const int ty = faceCondition<1>(m, b, fb, NAN, cv);
        double ing = 0.0;
        if (ty == FG) ing = cv[0] * m.barea[fb];
        else if (ty == FV) ing = m.bdcoef[fb] * (cv[0] - x[m.bown[fb]]);
        v = kf[t] * ing;
    } else {
        return;
    }
    const double inc = factor * (v + corr[t]);
    out[t] = first ? inc : out[t] + inc;
}

template <int C>
__global__ void kAddSource(int n, const double* __restrict__ V, const double* __restrict__ value, double factor,
                           double* __restrict__ src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < C; ++c) src[C * i + c] += factor * V[i] * value[C * i + c];
}

template <int C>
__global__ void kRelax(int n, double alpha, const double* __restrict__ prev, double* __restrict__ diag,
                       double* __restrict__ src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double extra = diag[i] * (1.0 / alpha - 1.0);
    diag[i] += extra;
#pragma unroll
    for (int c = 0; c < C; ++c) src[C * i + c] += extra * prev[C * i + c];
}

// Transient term (procedural_equation.cpp:198-223): with w = capacity * V,
// diag += w a0 and b += w a1 x_prev (+ w a2 x_older for variable-step BDF2).
template <int C>
__global__ void kTimeTerm(int n, const double* __restrict__ V, const double* __restrict__ cap, double c, double a0,
                          double a1, double a2, const double* __restrict__ prev, const double* __restrict__ older,
                          double* __restrict__ diag, double* __restrict__ src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double w = (cap ? cap[i] : c) * V[i];
    diag[i] += w * a0;
    const double w1 = w * a1, w2 = w * a2;
#pragma unroll
    for (int k = 0; k < C; ++k) {
        double s = src[C * i + k];
        s += w1 * prev[C * i + k];
        if (a2 != 0.0) s += w2 * older[C * i + k];
        src[C * i + k] = s;
    }
}

// Implicit reaction (procedural_equation.cpp:177-187): diag += factor c_i V_i.
__global__ void kReaction(int n, const double* __restrict__ V, const double* __restrict__ coef, double c,
                          double factor, double* __restrict__ diag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    diag[i] += coef ? factor * coef[i] * V[i] : c * V[i];
}

// flag[0] = 1 when any value is not positive and finite (flag[1]: any non-finite).
__global__ void kFill(int n, double v, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = v;
}

__global__ void kCheckValues(int n, const double* __restrict__ a, int* __restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = a[i];
    if (!(v > 0.0) || !isfinite(v)) flag[0] = 1;
    if (!isfinite(v)) flag[1] = 1;
}

__global__ void kScaleArray(long long n, double f, double* __restrict__ a) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i < n) a[i] *= f;
}

// reference(Equation, value) row-sum test (procedural_equation.cpp:316-333).
__global__ void kReferenceCheck(int row0, int n, const int* __restrict__ ptr, const double* __restrict__ diag,
                                const double* __restrict__ val, int* __restrict__ all_constant) {
    const int i = row0 + blockIdx.x * blockDim.x + threadIdx.x;
    int ok = 1;
    if (i < row0 + n) {
        double row = diag[i], mag = fabs(diag[i]);
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) { row += val[k]; mag += fabs(val[k]); }
        ok = isfinite(row) && fabs(row) <= 64.0 * kEps * mag;
    }
    const int warp_ok = __all_sync(0xffffffffu, ok);
    if ((threadIdx.x & 31) == 0 && !warp_ok) atomicAnd(all_constant, 0);
}

// reference(Equation, cell 0, value) (procedural_equation.cpp:306-315) on row `ref`: the
// caller's cell 0 (or first cell of a segment, when the mesh holds several independent
// cases) in the internal numbering.
__global__ void kApplyReference(int ref, const int* __restrict__ flag, double value, double* __restrict__ diag,
                                double* __restrict__ src, int* __restrict__ error) {
    if (*flag) {
        if (!(diag[ref] > 0.0)) { *error = 1; return; }
        src[ref] += diag[ref] * value;
        diag[ref] *= 2.0;
    }
}

template <int C>
__global__ void kApply(int n, const int* __restrict__ ptr, const int* __restrict__ col, const double* __restrict__ diag,
                       const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc[C];
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = diag[i] * x[C * i + c];
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
        const double a = val[k];
        const int j = col[k];
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] += a * x[C * j + c];
    }
#pragma unroll
    for (int c = 0; c < C; ++c) y[C * i + c] = acc[c];
}

// Partial sums of ||b-Ax||^2, ||Ax||^2, ||b||^2 (relativeResidual, procedural_equation.cpp:429-433).
template <int C>
__global__ void kResidualNorms(int row0, int n, const int* __restrict__ ptr, const int* __restrict__ col,
                               const double* __restrict__ diag, const double* __restrict__ val,
                               const double* __restrict__ src, const double* __restrict__ x,
                               double* __restrict__ partial) {
    const int i = row0 + blockIdx.x * kBlock + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    if (i < row0 + n) {
        double acc[C];
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] = diag[i] * x[C * i + c];
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
            const double a = val[k];
            const int j = col[k];
#pragma unroll
            for (int c = 0; c < C; ++c) acc[c] += a * x[C * j + c];
        }
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const double bb = src[C * i + c], r = bb - acc[c];
            v[0] += r * r; v[1] += acc[c] * acc[c]; v[2] += bb * bb;
        }
    }
    blockSum<3, kBlock>(v);
    if (threadIdx.x == 0) for (int j = 0; j < 3; ++j) partial[3 * blockIdx.x + j] = v[j];
}

// Flux balance per cell (fvm_execution.cpp:149-177): partial l1, l2^2, scale, and max.
__global__ void kFluxBalance(int row0, int n, MeshView m, const double* __restrict__ phi, double* __restrict__ partial) {
    const int i = row0 + blockIdx.x * kBlock + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    double mx = 0.0;
    if (i < row0 + n) {
        double imb = 0.0, sc = 0.0;
        for (int k = m.cf_ptr[i]; k < m.cf_ptr[i + 1]; ++k) {
            const int f = m.cf_face[k];
            const double o = m.own[f] == i ? phi[f] : -phi[f];
            imb += o; sc += fabs(o);
        }
        for (int fb = m.cb_ptr[i]; fb < m.cb_ptr[i + 1]; ++fb) {
            const double o = phi[m.n_interior + fb];
            imb += o; sc += fabs(o);
        }
        v[0] = fabs(imb); v[1] = imb * imb; v[2] = sc; mx = fabs(imb);
    }
    blockSum<3, kBlock>(v);
    __shared__ double smax[kBlock / 32];
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int j = 0; j < kBlock / 32; ++j) r = fmax(r, smax[j]);
        for (int j = 0; j < 3; ++j) partial[4 * blockIdx.x + j] = v[j];
        partial[4 * blockIdx.x + 3] = r;
    }
}

__global__ void kRelChange(long long n, const double* __restrict__ a, const double* __restrict__ b,
                           double* __restrict__ partial) {
    double v[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * static_cast<long long>(kBlock) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * kBlock) {
        const double d = a[i] - (b ? b[i] : 0.0);
        v[0] += d * d; v[1] += a[i] * a[i];
    }
    blockSum<2, kBlock>(v);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = v[0]; partial[2 * blockIdx.x + 1] = v[1]; }
}

// Sums per-block partials of NV quantities (max for entries flagged in max_mask).
// Second stage of a reduction: warp j combines value j of every block's partial
// (lanes stride over blocks, then a fixed shuffle tree), sum or max per max_mask.
__global__ void kFinishReduce(int blocks, int nv, unsigned max_mask, const double* __restrict__ partial,
                              double* __restrict__ result) {
    const int j = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (j >= nv) return;
    const bool is_max = (max_mask >> j) & 1u;
    double r = 0.0;
    for (int bidx = lane; bidx < blocks; bidx += 32) {
        const double p = partial[nv * bidx + j];
        r = is_max ? fmax(r, p) : r + p;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double q = __shfl_down_sync(0xffffffffu, r, o);
        r = is_max ? fmax(r, q) : r + q;
    }
    if (lane == 0) result[j] = r;
}

__global__ void kAxpy(long long n, double* __restrict__ y, double a, const double* __restrict__ x) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i < n) y[i] += a * x[i];
}
__global__ void kAdd(long long n, double* __restrict__ out, const double* __restrict__ a, const double* __restrict__ b) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i < n) out[i] = a[i] + b[i];
}
// Face reordering between the caller's numbering and the internal one:
// to_internal: out[perm[f]] = in[f]; otherwise out[f] = in[perm[f]] (C values per face).
__global__ void kPermuteFaces(int nf, int C, const int* __restrict__ perm, const double* __restrict__ in,
                              double* __restrict__ out, int to_internal) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const long long t = perm[f];
    for (int c = 0; c < C; ++c) {
        if (to_internal) out[C * t + c] = in[static_cast<long long>(C) * f + c];
        else out[static_cast<long long>(C) * f + c] = in[C * t + c];
    }
}

// out = b - out (residual after out = A x)
__global__ void kResidualFrom(long long n, const double* __restrict__ b, double* __restrict__ out) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i < n) out[i] = b[i] - out[i];
}
__global__ void kSubScaledGrad(int n, double* __restrict__ U, const double* __restrict__ r, const double* __restrict__ g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) U[3 * i + c] += -1.0 * r[i] * g[3 * i + c];
}
__global__ void kRatioVolume(int n, const double* __restrict__ V, const double* __restrict__ d, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = V[i] / d[i];
}

template <class K, class... A>
void launch(Context& ctx, K kernel, long long n, A... args) {
    kernel<<<gridFor(n, kBlock), kBlock, 0, ctx.stream>>>(args...);
    BSG_CUDA(cudaGetLastError());
    ctx.launched();
}

}  // namespace

// ----------------------------------------------------------------- fields
DeviceField::DeviceField(DeviceMesh& m, int loc, int c) : mesh(&m), location(loc), comps(c) {
    if (!(c == 1 || c == 3 || (c == 9 && loc == 0))) fail(kArgument, "field components must be 1, 3 or 9");
    v.resize(count() * c);
    v.zero(m.ctx->stream);
    bcs.assign(m.n_patches, PatchBC{ZG, {0.0, 0.0, 0.0}});
}

void DeviceField::setBoundary(int patch, int type, const double* value) {
    if (location != 0) fail(kState, "only cell fields have boundary conditions");
    if (calculated) fail(kState, "calculated field has boundary traces, not equation constraints");
    if (patch < 0 || patch >= mesh->n_patches) fail(kArgument, "field boundary patch is invalid");
    if (type < 0 || type > 4) fail(kArgument, "unknown boundary type");
    PatchBC p{type, {0.0, 0.0, 0.0}};
    if (value)
        for (int c = 0; c < std::min(comps, 3); ++c) p.value[c] = value[c];
    bcs[patch] = p;
    bcs_dirty = true;
}

BcView DeviceField::bcView() {
    if (bcs_dirty) {
        d_bcs.upload(bcs, mesh->ctx->stream);
        bcs_dirty = false;
    }
    return BcView{d_bcs.data(), calculated ? trace.data() : nullptr, has_flux ? bflux.data() : nullptr};
}

void uploadCells(DeviceMesh& m, double* device, const double* host, int C) {
    Context& ctx = *m.ctx;
    const std::size_t n = static_cast<std::size_t>(m.n_cells) * C;
    if (m.cell_perm.size() == 0) {
        if (n) BSG_CUDA(cudaMemcpyAsync(device, host, n * sizeof(double), cudaMemcpyHostToDevice, ctx.stream));
        ctx.sync();
        return;
    }
    if (m.cell_stage.size() < n) m.cell_stage.resize(n);
    if (n) BSG_CUDA(cudaMemcpyAsync(m.cell_stage.data(), host, n * sizeof(double), cudaMemcpyHostToDevice, ctx.stream));
    launch(ctx, kPermuteFaces, m.n_cells, m.n_cells, C, (const int*)m.cell_perm.data(),
           (const double*)m.cell_stage.data(), device, 1);
    ctx.sync();
}

void downloadCells(DeviceMesh& m, const double* device, double* host, int C) {
    Context& ctx = *m.ctx;
    const std::size_t n = static_cast<std::size_t>(m.n_cells) * C;
    if (m.cell_perm.size() == 0) {
        if (n) BSG_CUDA(cudaMemcpyAsync(host, device, n * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        return;
    }
    if (m.cell_stage.size() < n) m.cell_stage.resize(n);
    launch(ctx, kPermuteFaces, m.n_cells, m.n_cells, C, (const int*)m.cell_perm.data(), device,
           m.cell_stage.data(), 0);
    if (n) BSG_CUDA(cudaMemcpyAsync(host, m.cell_stage.data(), n * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
}

void DeviceField::uploadExternal(const double* host) {
    const int C = comps;
    Context& ctx = *mesh->ctx;
    if (location == 0) {
        v.resize(static_cast<std::size_t>(mesh->n_cells) * C);
        uploadCells(*mesh, v.data(), host, C);
        return;
    }
    // copy in caller order, then scatter to the internal face order on the device
    const std::size_t n = static_cast<std::size_t>(mesh->n_faces) * C;
    if (mesh->face_stage.size() < n) mesh->face_stage.resize(n);
    if (n) BSG_CUDA(cudaMemcpyAsync(mesh->face_stage.data(), host, n * sizeof(double), cudaMemcpyHostToDevice, ctx.stream));
    launch(ctx, kPermuteFaces, mesh->n_faces, mesh->n_faces, C, (const int*)mesh->face_perm.data(),
           (const double*)mesh->face_stage.data(), v.data(), 1);
    ctx.sync();
}

void DeviceField::downloadExternal(double* host) const {
    const int C = comps;
    Context& ctx = *mesh->ctx;
    if (location == 0) {
        downloadCells(*mesh, v.data(), host, C);
        return;
    }
    const std::size_t n = static_cast<std::size_t>(mesh->n_faces) * C;
    if (mesh->face_stage.size() < n) mesh->face_stage.resize(n);
    launch(ctx, kPermuteFaces, mesh->n_faces, mesh->n_faces, C, (const int*)mesh->face_perm.data(),
           (const double*)v.data(), mesh->face_stage.data(), 0);
    if (n) BSG_CUDA(cudaMemcpyAsync(host, mesh->face_stage.data(), n * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
}

void DeviceField::setFluxContext(const DeviceField& face_flux) {
    if (location != 0 || face_flux.location != 1 || face_flux.comps != 1 || face_flux.mesh != mesh)
        fail(kArgument, "boundary flux must be a scalar face field on the same mesh");
    bflux.resize(mesh->n_boundary);
    if (mesh->n_boundary)
        BSG_CUDA(cudaMemcpyAsync(bflux.data(), face_flux.v.data() + mesh->n_interior,
                                 sizeof(double) * mesh->n_boundary, cudaMemcpyDeviceToDevice, mesh->ctx->stream));
    has_flux = true;
}

DeviceEquation::DeviceEquation(DeviceField& unknown, const Options& o) : x(&unknown), options(o) {
    if (unknown.location != 0 || (unknown.comps != 1 && unknown.comps != 3))
        fail(kArgument, "equ requires a scalar or vector cell field");
    if (unknown.calculated) fail(kArgument, "equ unknown requires physical boundaries");
    DeviceMesh& m = *unknown.mesh;
    diag.resize(m.n_cells);
    val.resize(2 * static_cast<std::size_t>(m.n_interior));
    src.resize(static_cast<std::size_t>(m.n_cells) * unknown.comps);
    reset();
}

void DeviceEquation::reset() {
    cudaStream_t s = x->mesh->ctx->stream;
    diag.zero(s);
    val.zero(s);
    src.zero(s);
    for (auto& d : diffusion) spare.push_back(std::move(d));
    diffusion.clear();
    boundary_flux = nullptr;
    grad_method = -1;
}

std::unique_ptr<DiffusionSnapshot> DeviceEquation::takeSnapshot() {
    if (spare.empty()) return std::make_unique<DiffusionSnapshot>();
    auto s = std::move(spare.back());
    spare.pop_back();
    return s;
}

const double* DeviceEquation::unknownGradient(int method) {
    if (grad_method != method) {
        gradient(*x, method, grad_ws);
        grad_method = method;
    }
    return grad_ws.data();
}

void Reducer::ensure(int blocks, int nv) {
    if (partial.size() < static_cast<std::size_t>(blocks) * nv) partial.resize(static_cast<std::size_t>(blocks) * nv);
    if (result.size() < 16) result.resize(16);
}

// ----------------------------------------------------------------- operators
void gradient(DeviceField& x, int method, DeviceArray<double>& out) {
    DeviceMesh& m = *x.mesh;
    Context& ctx = *m.ctx;
    if (x.location != 0) fail(kArgument, "gradient input must be a cell field");
    const int C = x.comps;
    if (C != 1 && C != 3) fail(kArgument, "gradient of a scalar or vector field only");
    out.resize(static_cast<std::size_t>(m.n_cells) * 3 * C);
    const MeshView mv = view(m);
    const BcView b = x.bcView();
    if (method == 1) {
        if (C == 1) launch(ctx, kGradLeastSquares<1>, m.n_cells, mv, b, (const double*)x.v.data(), out.data());
        else launch(ctx, kGradLeastSquares<3>, m.n_cells, mv, b, (const double*)x.v.data(), out.data());
        return;
    }
    if (method != 0) fail(kArgument, "unsupported gradient method");
    const unsigned char* none = nullptr;
    if (m.orthogonal) {
        if (C == 1) launch(ctx, kGradGauss<1, false>, m.n_cells, mv, b, (const double*)x.v.data(), (const double*)nullptr, out.data(), none);
        else launch(ctx, kGradGauss<3, false>, m.n_cells, mv, b, (const double*)x.v.data(), (const double*)nullptr, out.data(), none);
        return;
    }
    DeviceArray<double>& first = m.ws_grad_pass1;  // persistent scratch: no allocation per call
    if (first.size() < out.size()) first.resize(out.size());
    const unsigned char* oc = m.cell_orth.size() ? m.cell_orth.data() : nullptr;
    if (C == 1) {
        launch(ctx, kGradGauss<1, false>, m.n_cells, mv, b, (const double*)x.v.data(), (const double*)nullptr, first.data(), none);
        launch(ctx, kGradGauss<1, true>, m.n_cells, mv, b, (const double*)x.v.data(), (const double*)first.data(), out.data(), oc);
    } else {
        launch(ctx, kGradGauss<3, false>, m.n_cells, mv, b, (const double*)x.v.data(), (const double*)nullptr, first.data(), none);
        launch(ctx, kGradGauss<3, true>, m.n_cells, mv, b, (const double*)x.v.data(), (const double*)first.data(), out.data(), oc);
    }
}

void gradientTrace(DeviceField& x, const double* g, DeviceArray<double>& trace_out) {
    DeviceMesh& m = *x.mesh;
    trace_out.resize(3 * static_cast<std::size_t>(m.n_boundary));
    launch(*m.ctx, kGradientTrace, m.n_boundary, view(m), x.bcView(), (const double*)x.v.data(), g, trace_out.data());
}

void interpolate(DeviceField& x, int interp, int grad, DeviceArray<double>& out, DeviceArray<double>* grad_ws) {
    DeviceMesh& m = *x.mesh;
    Context& ctx = *m.ctx;
    const int C = x.comps;
    out.resize(static_cast<std::size_t>(m.n_faces) * C);
    const MeshView mv = view(m);
    const BcView b = x.bcView();
    if (interp == 0) {
        if (C == 1) launch(ctx, kInterpolate<1, false>, m.n_faces, mv, b, (const double*)x.v.data(), (const double*)nullptr, out.data());
        else launch(ctx, kInterpolate<3, false>, m.n_faces, mv, b, (const double*)x.v.data(), (const double*)nullptr, out.data());
        return;
    }
    DeviceArray<double> local;
    DeviceArray<double>& g = grad_ws ? *grad_ws : local;
    gradient(x, grad, g);
    if (C == 1) launch(ctx, kInterpolate<1, true>, m.n_faces, mv, b, (const double*)x.v.data(), (const double*)g.data(), out.data());
    else launch(ctx, kInterpolate<3, true>, m.n_faces, mv, b, (const double*)x.v.data(), (const double*)g.data(), out.data());
    if (!grad_ws) ctx.sync();
}

void faceFlux(DeviceField& U, int interp, int grad, DeviceField& out) {
    DeviceMesh& m = *U.mesh;
    Context& ctx = *m.ctx;
    if (U.location != 0 || U.comps != 3 || out.location != 1 || out.comps != 1)
        fail(kArgument, "flux requires a cell vector and a scalar face result");
    if (!U.has_flux) {
        U.bflux.resize(m.n_boundary);
        launch(ctx, kSeedFlux, m.n_boundary, view(m), (const double*)U.v.data(), U.bflux.data());
        U.has_flux = true;
    }
    const BcView b = U.bcView();
    if (interp == 0) {
        launch(ctx, kFlux<false>, m.n_faces, view(m), b, (const double*)U.v.data(), (const double*)nullptr, out.v.data());
    } else {
        DeviceArray<double> g;
        gradient(U, grad, g);
        launch(ctx, kFlux<true>, m.n_faces, view(m), b, (const double*)U.v.data(), (const double*)g.data(), out.v.data());
        ctx.sync();
    }
    U.setFluxContext(out);  // FvmExecution::evaluate(FaceFlux), fvm_execution.cpp:269-280
}

void divFlux(const DeviceField& phi, DeviceArray<double>& out) {
    DeviceMesh& m = *phi.mesh;
    if (phi.location != 1 || phi.comps != 1) fail(kArgument, "div requires a scalar face flux");
    out.resize(m.n_cells);
    launch(*m.ctx, kDivFlux, m.n_cells, view(m), (const double*)phi.v.data(), out.data());
}

void normalGradient(DeviceField& x, const double* g, int diffusion, DeviceArray<double>& out) {
    DeviceMesh& m = *x.mesh;
    out.resize(m.n_faces);
    launch(*m.ctx, kNormalGradient, m.n_faces, view(m), x.bcView(), (const double*)x.v.data(), g, diffusion, out.data());
}

// ----------------------------------------------------------------- assembly
void addConvection(DeviceEquation& eq, DeviceField& phi, double scale, const Options& o) {
    DeviceField& x = *eq.x;
    DeviceMesh& m = *x.mesh;
    Context& ctx = *m.ctx;
    if (!std::isfinite(scale)) fail(kArgument, "nonfinite equ coefficient");
    if (phi.location != 1 || phi.comps != 1 || phi.mesh != &m) fail(kArgument, "equ::div requires a face flux");
    if (eq.boundary_flux && eq.boundary_flux != &phi)
        fail(kArgument, "one equation requires one boundary flux context");
    if (o.interpolation != 0 && o.interpolation != 1) fail(kArgument, "unsupported convection interpolation method");
    eq.boundary_flux = &phi;
    x.setFluxContext(phi);
    eq.grad_method = -1;  // the flux context feeds inletOutlet traces of the gradient
    const bool need_grad = o.convection == 1 || (o.convection == 2 && o.interpolation == 1);
    const double* g = need_grad ? eq.unknownGradient(o.gradient) : nullptr;
    const BcView b = x.bcView();
    if (x.comps == 1)
        launch(ctx, kAddConvection<1>, m.n_cells, view(m), b, (const double*)x.v.data(), g,
               (const double*)phi.v.data(), o.convection, scale, eq.diag.data(), eq.val.data(), eq.src.data());
    else
        launch(ctx, kAddConvection<3>, m.n_cells, view(m), b, (const double*)x.v.data(), g,
               (const double*)phi.v.data(), o.convection, scale, eq.diag.data(), eq.val.data(), eq.src.data());
}

void addLaplacian(DeviceEquation& eq, DeviceField* coef, double k, double factor, const Options& o) {
    DeviceField& x = *eq.x;
    DeviceMesh& m = *x.mesh;
    Context& ctx = *m.ctx;
    if (!std::isfinite(factor) || (!coef && !std::isfinite(k))) fail(kArgument, "nonfinite equ coefficient");
    auto snap = eq.takeSnapshot();
    snap->kf.resize(m.n_faces);
    if (coef) {
        if (coef->mesh != &m || coef->comps != 1) fail(kArgument, "equ diffusivity must be a compatible cell or face field");
        if (coef->location == 0) {
            // corrected coefficient interpolation needs the coefficient's own gradient
            if (o.coefInterp() != 0) interpolate(*coef, o.coefInterp(), o.coefGrad(), snap->kf, &snap->correction);
            else interpolate(*coef, 0, 0, snap->kf);
        } else {
            BSG_CUDA(cudaMemcpyAsync(snap->kf.data(), coef->v.data(), sizeof(double) * m.n_faces,
                                     cudaMemcpyDeviceToDevice, ctx.stream));
        }
    } else {
        if (k < 0.0) fail(kArgument, "diffusivity must be non-negative and finite");
        snap->kf.resize(m.n_faces);
        launch(ctx, kFill, m.n_faces, m.n_faces, k, snap->kf.data());
    }
    const double* g = o.diffusion != 0 ? eq.unknownGradient(o.gradient) : nullptr;
    const BcView b = x.bcView();
    const double mult = -factor;
    const std::size_t slot_doubles = static_cast<std::size_t>(1 + x.comps) * 2 * m.n_interior;
    if (m.ws_slots.size() < slot_doubles) m.ws_slots.resize(slot_doubles);
    const double* kfd = snap->kf.data();
    if (x.comps == 1) {
        launch(ctx, kDiffusionFaces<1>, m.n_interior, view(m), (const double*)x.v.data(), g, kfd, 0.0, o.diffusion,
               mult, eq.val.data(), m.ws_slots.data());
        launch(ctx, kAddDiffusion<1>, m.n_cells, view(m), b, (const double*)x.v.data(), g, kfd, 0.0, o.diffusion,
               mult, (const double*)m.ws_slots.data(), eq.diag.data(), eq.src.data());
    } else {
        launch(ctx, kDiffusionFaces<3>, m.n_interior, view(m), (const double*)x.v.data(), g, kfd, 0.0, o.diffusion,
               mult, eq.val.data(), m.ws_slots.data());
        launch(ctx, kAddDiffusion<3>, m.n_cells, view(m), b, (const double*)x.v.data(), g, kfd, 0.0, o.diffusion,
               mult, (const double*)m.ws_slots.data(), eq.diag.data(), eq.src.data());
    }
    if (x.comps == 1) {
        snap->correction.resize(m.n_faces);
        if (o.diffusion != 0)
            launch(ctx, kDiffusionCorrection, m.n_faces, view(m), b, (const double*)x.v.data(), g,
                   (const double*)snap->kf.data(), o.diffusion, snap->correction.data());
        else
            snap->correction.zero(ctx.stream);
        bool same = snap->bcs.size() == x.bcs.size();
        for (std::size_t i = 0; same && i < x.bcs.size(); ++i)
            same = snap->bcs[i].type == x.bcs[i].type && snap->bcs[i].value[0] == x.bcs[i].value[0] &&
                   snap->bcs[i].value[1] == x.bcs[i].value[1] && snap->bcs[i].value[2] == x.bcs[i].value[2];
        if (!same || snap->d_bcs.size() != x.bcs.size()) {
            snap->bcs = x.bcs;
            snap->d_bcs.upload(snap->bcs, ctx.stream);
        }
        snap->factor = factor;
        eq.diffusion.push_back(std::move(snap));
    } else {
        eq.spare.push_back(std::move(snap));
    }
}

void addSource(DeviceEquation& eq, const double* values, double factor) {
    DeviceMesh& m = *eq.x->mesh;
    if (!std::isfinite(factor)) fail(kArgument, "nonfinite equ coefficient");
    if (eq.x->comps == 1) launch(*m.ctx, kAddSource<1>, m.n_cells, m.n_cells, (const double*)m.V.data(), values, factor, eq.src.data());
    else launch(*m.ctx, kAddSource<3>, m.n_cells, m.n_cells, (const double*)m.V.data(), values, factor, eq.src.data());
}

void relax(DeviceEquation& eq, const double* previous, double alpha) {
    if (!(alpha > 0.0 && alpha <= 1.0)) fail(kArgument, "relaxation must be in (0,1]");
    DeviceMesh& m = *eq.x->mesh;
    if (eq.x->comps == 1) launch(*m.ctx, kRelax<1>, m.n_cells, m.n_cells, alpha, previous, eq.diag.data(), eq.src.data());
    else launch(*m.ctx, kRelax<3>, m.n_cells, m.n_cells, alpha, previous, eq.diag.data(), eq.src.data());
}

TimeWeights timeWeights(int method, double dt, double older_dt, bool have_older) {
    TimeWeights t;
    if (method == 0) return t;
    if (method != 1 && method != 2) fail(kArgument, "unsupported time method");
    if (!(dt > 0.0) || !std::isfinite(dt)) fail(kArgument, "equ::ddt requires positive finite dt");
    t.a0 = 1.0 / dt;
    t.a1 = 1.0 / dt;
    if (method == 2) {
        if (!have_older) fail(kArgument, "BDF2 requires explicit older field; use Euler to start");
        if (older_dt == 0.0) older_dt = dt;
        if (!(older_dt > 0.0) || !std::isfinite(older_dt)) fail(kArgument, "invalid previous dt");
        const double r = dt / older_dt;
        t.a0 = (1 + 2 * r) / ((1 + r) * dt);
        t.a1 = (1 + r) / dt;
        t.a2 = -r * r / ((1 + r) * dt);
    }
    t.active = true;
    return t;
}

void addTimeTerm(DeviceEquation& eq, const double* capacity, double c, const double* previous, const double* older,
                 const TimeWeights& t) {
    if (!t.active) return;
    if (!capacity && !(c > 0.0 && std::isfinite(c))) fail(kArgument, "time capacity must be positive and finite");
    DeviceMesh& m = *eq.x->mesh;
    if (eq.x->comps == 1)
        launch(*m.ctx, kTimeTerm<1>, m.n_cells, m.n_cells, (const double*)m.V.data(), capacity, c, t.a0, t.a1, t.a2,
               previous, older, eq.diag.data(), eq.src.data());
    else
        launch(*m.ctx, kTimeTerm<3>, m.n_cells, m.n_cells, (const double*)m.V.data(), capacity, c, t.a0, t.a1, t.a2,
               previous, older, eq.diag.data(), eq.src.data());
}

void addReaction(DeviceEquation& eq, const double* coefficient, double c, double factor) {
    if (!std::isfinite(c) || !std::isfinite(factor)) fail(kArgument, "nonfinite equ coefficient");
    DeviceMesh& m = *eq.x->mesh;
    launch(*m.ctx, kReaction, m.n_cells, m.n_cells, (const double*)m.V.data(), coefficient, c, factor, eq.diag.data());
}

void checkValues(Context& ctx, const double* a, long long n, int* flags_dev, int out[2]) {
    BSG_CUDA(cudaMemsetAsync(flags_dev, 0, 2 * sizeof(int), ctx.stream));
    if (n > 0) launch(ctx, kCheckValues, n, static_cast<int>(n), a, flags_dev);
    BSG_CUDA(cudaMemcpyAsync(out, flags_dev, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
}

void scale(DeviceEquation& eq, double f) {
    if (!std::isfinite(f)) fail(kArgument, "nonfinite equ coefficient");
    Context& ctx = *eq.x->mesh->ctx;
    launch(ctx, kScaleArray, (long long)eq.diag.size(), (long long)eq.diag.size(), f, eq.diag.data());
    launch(ctx, kScaleArray, (long long)eq.val.size(), (long long)eq.val.size(), f, eq.val.data());
    launch(ctx, kScaleArray, (long long)eq.src.size(), (long long)eq.src.size(), f, eq.src.data());
    for (auto& s : eq.diffusion) s->factor *= f;
}

void referenceIfUnanchored(DeviceEquation& eq, double value, int* flag_dev, int row0, int nrows) {
    if (eq.x->comps != 1) fail(kArgument, "reference requires a scalar equation");
    if (!std::isfinite(value)) fail(kArgument, "nonfinite equ coefficient");
    DeviceMesh& m = *eq.x->mesh;
    Context& ctx = *m.ctx;
    const int n = nrows < 0 ? m.n_cells : nrows;
    // flag_dev[0] = all-constant flag, flag_dev[1] = error flag
    const int init[2] = {1, 0};
    BSG_CUDA(cudaMemcpyAsync(flag_dev, init, sizeof(init), cudaMemcpyHostToDevice, ctx.stream));
    launch(ctx, kReferenceCheck, n, row0, n, (const int*)m.cf_ptr.data(), (const double*)eq.diag.data(),
           (const double*)eq.val.data(), flag_dev);
    // the anchored cell is the caller's first cell of the range, wherever renumbering put it
    // (a renumbered segment keeps its cell range)
    const int ref = m.h_cell_perm.empty() ? row0 : m.h_cell_perm[row0];
    if (ref < row0 || ref >= row0 + n) fail(kState, "reference cell outside its cell range");
    kApplyReference<<<1, 1, 0, ctx.stream>>>(ref, flag_dev, value, eq.diag.data(), eq.src.data(), flag_dev + 1);
    BSG_CUDA(cudaGetLastError());
    ctx.launched();
}

void applyEquation(const DeviceEquation& eq, const double* x, double* y) {
    DeviceMesh& m = *eq.x->mesh;
    if (eq.x->comps == 1)
        launch(*m.ctx, kApply<1>, m.n_cells, m.n_cells, (const int*)m.cf_ptr.data(), (const int*)m.cf_col.data(),
               eq.diag.data(), eq.val.data(), x, y);
    else
        launch(*m.ctx, kApply<3>, m.n_cells, m.n_cells, (const int*)m.cf_ptr.data(), (const int*)m.cf_col.data(),
               eq.diag.data(), eq.val.data(), x, y);
}

void residualEquation(const DeviceEquation& eq, const double* x, double* y) {
    applyEquation(eq, x, y);
    const long long n = static_cast<long long>(eq.x->mesh->n_cells) * eq.x->comps;
    launch(*eq.x->mesh->ctx, kResidualFrom, n, n, (const double*)eq.src.data(), y);
}

void faceFluxEquation(DeviceEquation& eq, const double* solution, DeviceArray<double>& out) {
    DeviceMesh& m = *eq.x->mesh;
    Context& ctx = *m.ctx;
    out.resize(m.n_faces);
    if (eq.diffusion.empty()) { out.zero(ctx.stream); return; }
    int first = 1;
    for (auto& s : eq.diffusion) {
        const BcView b{s->d_bcs.data(), nullptr, eq.x->has_flux ? eq.x->bflux.data() : nullptr};
        launch(ctx, kFaceFluxTerm, m.n_faces, view(m), b, solution, (const double*)s->kf.data(),
               (const double*)s->correction.data(), s->factor, first, out.data());
        first = 0;
    }
}

void relativeResidualNorms(const DeviceEquation& eq, const double* x, Reducer& red, int row0, int nrows) {
    DeviceMesh& m = *eq.x->mesh;
    Context& ctx = *m.ctx;
    const int n = nrows < 0 ? m.n_cells : nrows;
    const int blocks = static_cast<int>(gridFor(n, kBlock));
    red.ensure(blocks, 3);
    if (eq.x->comps == 1)
        launch(ctx, kResidualNorms<1>, n, row0, n, (const int*)m.cf_ptr.data(), (const int*)m.cf_col.data(),
               eq.diag.data(), eq.val.data(), eq.src.data(), x, red.partial.data());
    else
        launch(ctx, kResidualNorms<3>, n, row0, n, (const int*)m.cf_ptr.data(), (const int*)m.cf_col.data(),
               eq.diag.data(), eq.val.data(), eq.src.data(), x, red.partial.data());
    kFinishReduce<<<1, 32 * 3, 0, ctx.stream>>>(blocks, 3, 0u, red.partial.data(), red.result.data());
    BSG_CUDA(cudaGetLastError());
    ctx.launched();
}

void fluxBalance(DeviceMesh& m, const double* phi, Reducer& red, int row0, int nrows) {
    Context& ctx = *m.ctx;
    const int n = nrows < 0 ? m.n_cells : nrows;
    const int blocks = static_cast<int>(gridFor(n, kBlock));
    red.ensure(blocks, 4);
    launch(ctx, kFluxBalance, n, row0, n, view(m), phi, red.partial.data());
    kFinishReduce<<<1, 32 * 4, 0, ctx.stream>>>(blocks, 4, 0x8u, red.partial.data(), red.result.data());
    BSG_CUDA(cudaGetLastError());
    ctx.launched();
}

void relativeChangeNorms(Context& ctx, const double* a, const double* b, long long n, Reducer& red) {
    const int blocks = static_cast<int>(std::min<long long>(gridFor(n, kBlock), 4L * ctx.sm_count));
    red.ensure(blocks, 2);
    kRelChange<<<blocks, kBlock, 0, ctx.stream>>>(n, a, b, red.partial.data());
    BSG_CUDA(cudaGetLastError());
    ctx.launched();
    kFinishReduce<<<1, 32 * 2, 0, ctx.stream>>>(blocks, 2, 0u, red.partial.data(), red.result.data());
    BSG_CUDA(cudaGetLastError());
    ctx.launched();
}

void copyAsync(Context& ctx, double* dst, const double* src, long long n) {
    if (n) BSG_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx.stream));
}
void axpyCell(Context& ctx, double* y, double a, const double* x, long long n) { launch(ctx, kAxpy, n, n, y, a, x); }
void addArrays(Context& ctx, double* out, const double* a, const double* b, long long n) { launch(ctx, kAdd, n, n, out, a, b); }
void subtractScaledGradient(DeviceMesh& m, double* U, const double* rAU, const double* g) {
    launch(*m.ctx, kSubScaledGrad, m.n_cells, m.n_cells, U, rAU, g);
}
void ratioVolume(DeviceMesh& m, const double* diag, double* rAU) {
    launch(*m.ctx, kRatioVolume, m.n_cells, m.n_cells, (const double*)m.V.data(), diag, rAU);
}

}  // namespace bsg
