// Mesh::polyhedral geometry (src/core/mesh.cpp:321-564) on the device.
//
// The same algorithm as computePolyhedralGeometry in mesh.cpp, stage by stage:
//   kFaceClassify   per face: repeated vertices, the projection checks of the
//                   triangulation (mesh.cpp:60-161) for the ring and for its
//                   reversal, convexity, the sum of the ring's points
//   kCellReference  per cell: mean of its faces' points (mesh.cpp:361-377)
//   kFaceGeometry   per face: fan or ear-clipping triangles, area vector,
//                   outward orientation, centre, area, unit normal
//   kCellGeometry   per cell: vector areas close (Mesh::validate, mesh.cpp:709-730),
//                   volume and centroid from tetrahedra about the reference point
//                   (mesh.cpp:486-519)
//   kCellEdges      one warp per cell: every edge of the outward rings appears
//                   exactly twice, once in each direction (mesh.cpp:731-756)
//   kFaceCoefficients per face: orthogonal coefficient, non-orthogonal vector,
//                   interpolation weight, skewness (mesh.cpp:521-564)
// Every expression is evaluated in the host code's order and this unit is
// compiled without FMA contraction, so the device geometry is bit-identical to
// the host's.  A cell sums its faces in increasing face order (the host's
// loop order) through a cell->face list built on the host.  A stage that finds
// an invalid face or cell records the lowest index; the host then runs its own
// geometry, which raises the reference's message for the first failure.
#include "bsg_internal.h"

#include <cub/device/device_scan.cuh>

#include <climits>

namespace bsg {
namespace {

struct D3 { double x, y, z; };
__device__ inline D3 ld3(const double* v, long long i) { return {v[3 * i], v[3 * i + 1], v[3 * i + 2]}; }
__device__ inline void st3(double* v, long long i, D3 a) { v[3 * i] = a.x; v[3 * i + 1] = a.y; v[3 * i + 2] = a.z; }
__device__ inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ inline D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ inline D3 mul(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ inline D3 cross(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ inline double norm(D3 a) { return sqrt(dot(a, a)); }

// A face ring, optionally reversed about its first vertex (std::reverse(ring + 1, ring + n)).
struct Ring {
    const int* p;
    int n;
    bool flip;
    __device__ int operator[](int i) const { return flip ? (i == 0 ? p[0] : p[n - i]) : p[i]; }
};

// Projection of the ring on the plane that drops the dominant normal axis.
struct Projection {
    int drop;
    double tol, orient;
    bool convex;
};

__device__ inline void project2(const double* verts, int v, int drop, double& a, double& b) {
    const double* p = verts + 3LL * v;
    if (drop == 0) { a = p[1]; b = p[2]; }
    else if (drop == 1) { a = p[2]; b = p[0]; }
    else { a = p[0]; b = p[1]; }
}

struct Q { double a, b; };
__device__ inline Q qAt(const double* verts, const Ring& r, int i, int drop) {
    Q q;
    project2(verts, r[i], drop, q.a, q.b);
    return q;
}
__device__ inline double cross2(Q a, Q b, Q c) { return (b.a - a.a) * (c.b - a.b) - (b.b - a.b) * (c.a - a.a); }

// The checks and the convexity decision of the triangulation; false where it fails.
__device__ bool classify(const Ring& r, const double* verts, Projection& pj) {
    const int n = r.n;
    if (n < 3) return false;
    D3 nrm{0, 0, 0};
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; ++i) {
        const D3 c = ld3(verts, r[i]);
        const D3 d = ld3(verts, r[(i + 1) % n]);
        nrm = add(nrm, mul(0.5, cross(c, d)));
        const double cc[3] = {c.x, c.y, c.z};
        for (int k = 0; k < 3; ++k) {
            lo[k] = cc[k] < lo[k] ? cc[k] : lo[k];
            hi[k] = hi[k] < cc[k] ? cc[k] : hi[k];
        }
    }
    const double a0 = fabs(nrm.x), a1 = fabs(nrm.y), a2 = fabs(nrm.z);
    pj.drop = a1 > a0 ? (a2 > a1 ? 2 : 1) : (a2 > a0 ? 2 : 0);
    double scale = hi[0] - lo[0];                     // std::max over {dx, dy, dz, 1.0}
    const double rest[3] = {hi[1] - lo[1], hi[2] - lo[2], 1.0};
    for (int k = 0; k < 3; ++k) scale = scale < rest[k] ? rest[k] : scale;
    pj.tol = 1e-13 * scale * scale;
    double signed_area = 0.0;
    for (int i = 0; i < n; ++i) {
        const Q qi = qAt(verts, r, i, pj.drop), qj = qAt(verts, r, (i + 1) % n, pj.drop);
        signed_area += qi.a * qj.b - qj.a * qi.b;
    }
    if (fabs(signed_area) <= pj.tol) return false;
    pj.orient = signed_area > 0.0 ? 1.0 : -1.0;
    bool convex = true, saw = false;
    for (int i = 0; i < n; ++i) {
        const double t = pj.orient * cross2(qAt(verts, r, (i + n - 1) % n, pj.drop), qAt(verts, r, i, pj.drop),
                                            qAt(verts, r, (i + 1) % n, pj.drop));
        saw = saw || fabs(t) > pj.tol;
        if (t < -pj.tol) { convex = false; break; }
    }
    pj.convex = convex;
    return saw;
}

// Ear clipping of a non-convex ring into tri[3(n-2)], with rem[n] as the
// remaining-vertex list; false for a self-intersecting ring.
__device__ bool earClip(const Ring& r, const double* verts, const Projection& pj, int* tri, int* rem) {
    const int n = r.n;
    for (int i = 0; i < n; ++i) rem[i] = i;
    int m = n, k = 0;
    while (m > 3) {
        bool clipped = false;
        for (int pos = 0; pos < m; ++pos) {
            const int pv = rem[(pos + m - 1) % m], cu = rem[pos], nx = rem[(pos + 1) % m];
            const Q qp = qAt(verts, r, pv, pj.drop), qc = qAt(verts, r, cu, pj.drop), qn = qAt(verts, r, nx, pj.drop);
            if (pj.orient * cross2(qp, qc, qn) <= pj.tol) continue;
            bool inside = false;
            for (int t = 0; t < m; ++t) {
                const int c = rem[t];
                if (c == pv || c == cu || c == nx) continue;
                const Q qx = qAt(verts, r, c, pj.drop);
                const double ab = pj.orient * cross2(qp, qc, qx);
                const double bc = pj.orient * cross2(qc, qn, qx);
                const double ca = pj.orient * cross2(qn, qp, qx);
                if (ab >= -pj.tol && bc >= -pj.tol && ca >= -pj.tol) { inside = true; break; }
            }
            if (inside) continue;
            tri[3 * k] = r[pv];
            tri[3 * k + 1] = r[cu];
            tri[3 * k + 2] = r[nx];
            ++k;
            for (int t = pos; t + 1 < m; ++t) rem[t] = rem[t + 1];
            --m;
            clipped = true;
            break;
        }
        if (!clipped) return false;
    }
    tri[3 * k] = r[rem[0]];
    tri[3 * k + 1] = r[rem[1]];
    tri[3 * k + 2] = r[rem[2]];
    return true;
}

// Triangle t of a face: a fan from vertex 0 when convex, else the ear-clipped list.
__device__ inline void triangle(const Ring& r, bool convex, const int* tri, int t, int& a, int& b, int& c) {
    if (convex) { a = r[0]; b = r[t + 1]; c = r[t + 2]; }
    else { a = tri[3 * t]; b = tri[3 * t + 1]; c = tri[3 * t + 2]; }
}

__device__ inline void flag(int* err, int index) { atomicMin(err, index); }

// Flags per face: bit 0 ring convex, bit 1 reversed ring convex, bit 2 reversed (outward) orientation,
// bit 3 the reversed ring fails the triangulation checks (an error only if the face must be reversed).
constexpr unsigned char kConvex = 1, kConvexFlipped = 2, kFlipped = 4, kFlippedInvalid = 8;

__global__ void kFaceClassify(int F, const double* __restrict__ verts, const int* __restrict__ off,
                              const int* __restrict__ ids, double* __restrict__ fsum,
                              unsigned char* __restrict__ fflags, long long* __restrict__ scratch, int* err) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int b = off[f], n = off[f + 1] - b;
    const int* ring = ids + b;
    scratch[f] = 0;
    fflags[f] = 0;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
            if (ring[i] == ring[j]) { flag(err, f); return; }
    Projection p0, p1;
    if (!classify(Ring{ring, n, false}, verts, p0)) { flag(err, f); return; }
    const bool valid1 = classify(Ring{ring, n, true}, verts, p1);
    fflags[f] = (p0.convex ? kConvex : 0) | (valid1 && p1.convex ? kConvexFlipped : 0) |
                (valid1 ? 0 : kFlippedInvalid);
    // ear-clipping scratch: 3(n-2) triangle ids followed by n remaining-vertex slots
    if (!p0.convex || (valid1 && !p1.convex)) scratch[f] = 4LL * n - 6;
    D3 s{0, 0, 0};
    for (int i = 0; i < n; ++i) s = add(s, ld3(verts, ring[i]));
    st3(fsum, f, s);
}

// cface: faces of each cell in increasing face order, f for the owner side and -f-1 for the neighbour side.
__global__ void kCellReference(int N, const int* __restrict__ cptr, const int* __restrict__ cface,
                               const int* __restrict__ off, const double* __restrict__ fsum, double* __restrict__ ref) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    D3 s{0, 0, 0};
    double cnt = 0.0;
    for (int k = cptr[c]; k < cptr[c + 1]; ++k) {
        const int e = cface[k], f = e >= 0 ? e : -e - 1;
        s = add(s, ld3(fsum, f));
        cnt += static_cast<double>(off[f + 1] - off[f]);
    }
    st3(ref, c, mul(1.0 / (1.0 < cnt ? cnt : 1.0), s));
}

__device__ D3 areaVector(const Ring& r, bool convex, const int* tri, const double* verts) {
    D3 a{0, 0, 0};
    for (int t = 0; t + 2 < r.n; ++t) {
        int i, j, k;
        triangle(r, convex, tri, t, i, j, k);
        const D3 A = ld3(verts, i), B = ld3(verts, j), C = ld3(verts, k);
        a = add(a, mul(0.5, cross(sub(B, A), sub(C, A))));
    }
    return a;
}

__global__ void kFaceGeometry(int F, const double* __restrict__ verts, const int* __restrict__ off,
                              const int* __restrict__ ids, const int* __restrict__ owner,
                              const double* __restrict__ fsum, const double* __restrict__ ref,
                              unsigned char* __restrict__ fflags, const long long* __restrict__ scratch_off,
                              int* __restrict__ scratch, double* __restrict__ Sf, double* __restrict__ xf,
                              double* __restrict__ area, double* __restrict__ normal, int* err) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int b = off[f], n = off[f + 1] - b;
    Ring r{ids + b, n, false};
    const unsigned char fl = fflags[f];
    int* tri = scratch + scratch_off[f];
    int* rem = tri + 3 * (n - 2);
    Projection pj;
    bool convex = (fl & kConvex) != 0;
    if (!convex) {
        classify(r, verts, pj);
        if (!earClip(r, verts, pj, tri, rem)) { flag(err, f); return; }
    }
    D3 a = areaVector(r, convex, tri, verts);
    const D3 avg = mul(1.0 / static_cast<double>(n), ld3(fsum, f));
    bool flipped = false;
    if (dot(a, sub(avg, ld3(ref, owner[f]))) < 0.0) {
        if (fl & kFlippedInvalid) { flag(err, f); return; }
        flipped = true;
        r.flip = true;
        convex = (fl & kConvexFlipped) != 0;
        if (!convex) {
            classify(r, verts, pj);
            if (!earClip(r, verts, pj, tri, rem)) { flag(err, f); return; }
        }
        a = areaVector(r, convex, tri, verts);
    }
    const double na = norm(a);
    if (!(na > 0.0) || !isfinite(na)) { flag(err, f); return; }
    D3 centre{0, 0, 0};
    double total = 0.0;
    for (int t = 0; t + 2 < n; ++t) {
        int i, j, k;
        triangle(r, convex, tri, t, i, j, k);
        const D3 A = ld3(verts, i), B = ld3(verts, j), C = ld3(verts, k);
        const double wgt = norm(mul(0.5, cross(sub(B, A), sub(C, A))));
        if (!(wgt > 0.0)) { flag(err, f); return; }
        centre = add(centre, mul(wgt, mul(1.0 / 3.0, add(add(A, B), C))));
        total += wgt;
    }
    centre = mul(1.0 / total, centre);
    st3(Sf, f, a);
    st3(xf, f, centre);
    st3(normal, f, D3{a.x / total, a.y / total, a.z / total});
    area[f] = total;
    fflags[f] = fl | (flipped ? kFlipped : 0);
}

// Directed edge e of face f as seen from a cell (sign < 0 reverses the face).
__device__ inline void edgeOf(const Ring& r, int e, bool reverse, int& from, int& to) {
    from = r[e];
    to = r[(e + 1) % r.n];
    if (reverse) { const int t = from; from = to; to = t; }
}

__global__ void kCellGeometry(int N, const double* __restrict__ verts, const int* __restrict__ off,
                              const int* __restrict__ ids, const int* __restrict__ cptr,
                              const int* __restrict__ cface, const unsigned char* __restrict__ fflags,
                              const long long* __restrict__ scratch_off, const int* __restrict__ scratch,
                              const double* __restrict__ Sf, const double* __restrict__ area,
                              const double* __restrict__ ref, double* __restrict__ V, double* __restrict__ xc,
                              int* err) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int k0 = cptr[c], k1 = cptr[c + 1];
    // closed surface: vector areas sum to zero (mesh.cpp:709-730)
    double cx = 0, cy = 0, cz = 0, total = 0;
    for (int k = k0; k < k1; ++k) {
        const int e = cface[k], f = e >= 0 ? e : -e - 1;
        const double s = e >= 0 ? 1.0 : -1.0;
        cx += s * Sf[3LL * f]; cy += s * Sf[3LL * f + 1]; cz += s * Sf[3LL * f + 2];
        total += area[f];
    }
    if (!(isfinite(total) && sqrt(cx * cx + cy * cy + cz * cz) <= 1e-9 * (total < 1.0 ? 1.0 : total))) {
        flag(err, c);
        return;
    }
    // the edge check of Mesh::validate runs in kCellEdges
    // volume and centroid from tetrahedra about the reference point (mesh.cpp:486-519)
    const D3 rp = ld3(ref, c);
    double vol = 0.0;
    D3 mom{0, 0, 0};
    for (int k = k0; k < k1; ++k) {
        const int e = cface[k], f = e >= 0 ? e : -e - 1;
        const double sign = e >= 0 ? 1.0 : -1.0;
        const unsigned char fl = fflags[f];
        const bool flipped = (fl & kFlipped) != 0;
        const bool convex = (fl & (flipped ? kConvexFlipped : kConvex)) != 0;
        const Ring r{ids + off[f], off[f + 1] - off[f], flipped};
        const int* tri = scratch + scratch_off[f];
        for (int t = 0; t + 2 < r.n; ++t) {
            int i, j, l;
            triangle(r, convex, tri, t, i, j, l);
            const D3 A = ld3(verts, i), B = ld3(verts, j), D = ld3(verts, l);
            const double tet = sign * dot(sub(A, rp), cross(sub(B, rp), sub(D, rp))) / 6.0;
            vol += tet;
            mom = add(mom, mul(tet, mul(0.25, add(add(add(rp, A), B), D))));
        }
    }
    if (!(vol > 0.0) || !isfinite(vol)) { flag(err, c); return; }
    V[c] = vol;
    st3(xc, c, D3{mom.x / vol, mom.y / vol, mom.z / vol});
}

// Every edge of a cell's outward rings appears exactly twice, once in each direction
// (mesh.cpp:731-756), scanning the rings in global memory (cells with many edges).
__device__ bool edgesClosed(const int* __restrict__ off, const int* __restrict__ ids, const int* __restrict__ cface,
                            const unsigned char* __restrict__ fflags, int k0, int k1) {
    for (int k = k0; k < k1; ++k) {
        const int e = cface[k], f = e >= 0 ? e : -e - 1;
        const Ring r{ids + off[f], off[f + 1] - off[f], (fflags[f] & kFlipped) != 0};
        for (int i = 0; i < r.n; ++i) {
            int from, to;
            edgeOf(r, i, e < 0, from, to);
            int same = 0, opposite = 0;
            for (int kk = k0; kk < k1; ++kk) {
                const int e2 = cface[kk], f2 = e2 >= 0 ? e2 : -e2 - 1;
                const Ring r2{ids + off[f2], off[f2 + 1] - off[f2], (fflags[f2] & kFlipped) != 0};
                for (int j = 0; j < r2.n; ++j) {
                    int a, b;
                    edgeOf(r2, j, e2 < 0, a, b);
                    same += (a == from && b == to);
                    opposite += (a == to && b == from);
                }
            }
            if (same != 1 || opposite != 1) return false;
        }
    }
    return true;
}

// The same check with one warp per cell: the cell's directed edges (at most kEdgeCap) are staged in
// shared memory and each lane compares its share of them against all; larger cells take edgesClosed.
constexpr int kEdgeWarps = 8, kEdgeCap = 256;

__global__ void __launch_bounds__(32 * kEdgeWarps) kCellEdges(int N, const int* __restrict__ off,
                                                               const int* __restrict__ ids,
                                                               const int* __restrict__ cptr,
                                                               const int* __restrict__ cface,
                                                               const unsigned char* __restrict__ fflags, int* err) {
    __shared__ int2 edges[kEdgeWarps][kEdgeCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * kEdgeWarps + warp;
    if (c >= N) return;                       // whole warp
    const int k0 = cptr[c], k1 = cptr[c + 1];
    int total = 0;
    for (int k = k0; k < k1; ++k) {
        const int e = cface[k], f = e >= 0 ? e : -e - 1;
        total += off[f + 1] - off[f];
    }
    if (total > kEdgeCap) {
        if (lane == 0 && !edgesClosed(off, ids, cface, fflags, k0, k1)) flag(err, c);
        return;
    }
    int2* mine = edges[warp];
    int base = 0;
    for (int k = k0; k < k1; ++k) {
        const int e = cface[k], f = e >= 0 ? e : -e - 1;
        const Ring r{ids + off[f], off[f + 1] - off[f], (fflags[f] & kFlipped) != 0};
        for (int i = lane; i < r.n; i += 32) {
            int from, to;
            edgeOf(r, i, e < 0, from, to);
            mine[base + i] = make_int2(from, to);
        }
        base += r.n;
    }
    __syncwarp();
    bool ok = true;
    for (int q = lane; q < total; q += 32) {
        const int2 x = mine[q];
        int same = 0, opposite = 0;
        for (int t = 0; t < total; ++t) {
            const int2 y = mine[t];
            same += (y.x == x.x && y.y == x.y);
            opposite += (y.x == x.y && y.y == x.x);
        }
        ok = ok && same == 1 && opposite == 1;
    }
    if (!ok) flag(err, c);
}

__global__ void kFaceCoefficients(int F, const int* __restrict__ owner, const int* __restrict__ neighbour,
                                  const double* __restrict__ Sf, const double* __restrict__ xf,
                                  const double* __restrict__ area, const double* __restrict__ normal,
                                  const double* __restrict__ xc, double* __restrict__ weight,
                                  double* __restrict__ dcoef, double* __restrict__ kvec, double* __restrict__ skew,
                                  int* orthogonal, int* err) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int o = owner[f], n = neighbour[f];
    const D3 xfv = ld3(xf, f), xo = ld3(xc, o), S = ld3(Sf, f), nr = ld3(normal, f);
    D3 delta, xn{0, 0, 0};
    if (n < 0) delta = sub(xfv, xo);
    else { xn = ld3(xc, n); delta = sub(xn, xo); }
    const double d2 = dot(delta, delta), proj = dot(S, delta);
    if (!(d2 > 0.0) || !(proj > 0.0)) { flag(err, f); return; }
    const double dc = proj / d2;
    dcoef[f] = dc;
    const D3 k = sub(S, mul(dc, delta));
    st3(kvec, f, k);
    bool orth = !(norm(k) > 1e-12 * area[f]);
    double w = 1.0;
    D3 sk{0, 0, 0};
    if (n >= 0) {
        const double od = fabs(dot(sub(xfv, xo), nr)), nd = fabs(dot(sub(xn, xfv), nr));
        if (!(od + nd > 0.0)) { flag(err, f); return; }
        w = nd / (od + nd);
        const double den = dot(delta, nr);
        if (!(den > 0.0) || !isfinite(den)) { flag(err, f); return; }
        const double frac = dot(sub(xfv, xo), nr) / den;
        sk = sub(xfv, add(xo, mul(frac, delta)));
        if (norm(sk) > 1e-12 * sqrt(d2)) orth = false;
    }
    weight[f] = w;
    st3(skew, f, sk);
    if (!orth) atomicAnd(orthogonal, 0);
}

// Caller-numbered face and cell geometry -> the internal layout of DeviceMesh.
__global__ void kGatherInterior(int Fi, const int* __restrict__ ext, const double* __restrict__ weight,
                                const double* __restrict__ dcoef, const double* __restrict__ area,
                                const double* __restrict__ Sf, const double* __restrict__ xf,
                                const double* __restrict__ kvec, const double* __restrict__ skew, double* w_out,
                                double* dcoef_out, double* area_out, double* Sf_out, double* xf_out, double* k_out,
                                double* skew_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Fi) return;
    const int f = ext[i];
    w_out[i] = weight[f];
    dcoef_out[i] = dcoef[f];
    area_out[i] = area[f];
    st3(Sf_out, i, ld3(Sf, f));
    st3(xf_out, i, ld3(xf, f));
    st3(k_out, i, ld3(kvec, f));
    st3(skew_out, i, ld3(skew, f));
}

__global__ void kGatherBoundary(int Fb, const int* __restrict__ ext, const int* __restrict__ owner,
                                const double* __restrict__ dcoef, const double* __restrict__ area,
                                const double* __restrict__ Sf, const double* __restrict__ xf,
                                const double* __restrict__ normal, const double* __restrict__ kvec,
                                const double* __restrict__ xc, double* dcoef_out, double* area_out, double* dist_out,
                                double* Sf_out, double* xf_out, double* n_out, double* k_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Fb) return;
    const int f = ext[i], o = owner[f];
    dcoef_out[i] = dcoef[f];
    area_out[i] = area[f];
    double d = 0.0;
    for (int c = 0; c < 3; ++c) d += (xf[3LL * f + c] - xc[3LL * o + c]) * normal[3LL * f + c];
    dist_out[i] = d;
    st3(Sf_out, i, ld3(Sf, f));
    st3(xf_out, i, ld3(xf, f));
    st3(n_out, i, ld3(normal, f));
    st3(k_out, i, ld3(kvec, f));
}

__global__ void kReciprocal(int N, const double* __restrict__ V, double* __restrict__ rV) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < N) rV[c] = 1.0 / V[c];
}

// Lowest flagged index of a stage (INT_MAX when none), resetting the flag.
int readFlag(Context& ctx, DeviceArray<int>& err) {
    int h = INT_MAX;
    BSG_CUDA(cudaMemcpyAsync(&h, err.data(), sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    return h;
}

}  // namespace

std::unique_ptr<DeviceMesh> buildDeviceMeshPolyhedral(Context& ctx, int n_vertices, const double* vertices,
                                                      int n_faces, const int* offsets, const int* ids,
                                                      const int* owner, const int* neighbour, const int* patch,
                                                      int n_patches) {
    const int N = validatePolyhedralTopology(n_vertices, n_faces, offsets, ids, owner, neighbour, patch, n_patches);
    const int F = n_faces;
    cudaStream_t s = ctx.stream;
    // Any stage failure: the host geometry raises the first failure's own message.
    auto rejected = [&]() {
        computePolyhedralGeometry(n_vertices, vertices, n_faces, offsets, ids, owner, neighbour, patch, n_patches);
        fail(kState, "device geometry rejected a mesh that the host geometry accepts");
    };
    // cell -> faces in increasing face order (owner side f, neighbour side -f-1)
    std::vector<int> cptr(N + 1, 0);
    for (int f = 0; f < F; ++f) {
        ++cptr[owner[f] + 1];
        if (neighbour[f] >= 0) ++cptr[neighbour[f] + 1];
    }
    for (int c = 0; c < N; ++c) cptr[c + 1] += cptr[c];
    std::vector<int> cface(cptr[N]);
    {
        std::vector<int> fill(cptr.begin(), cptr.end() - 1);
        for (int f = 0; f < F; ++f) {
            cface[fill[owner[f]]++] = f;
            if (neighbour[f] >= 0) cface[fill[neighbour[f]]++] = -f - 1;
        }
    }
    DeviceArray<double> d_verts, fsum(3LL * F), ref(3LL * N), Sf(3LL * F), xf(3LL * F), area(F), normal(3LL * F);
    DeviceArray<int> d_off, d_ids, d_owner, d_nbr, d_cptr, d_cface, err(1), orth(1);
    DeviceArray<unsigned char> fflags(F);
    DeviceArray<long long> scratch_n(F), scratch_off(F);
    {
        BSG_PROFILE(ctx, "geometry_upload");
        d_verts.upload(vertices, 3LL * n_vertices, s);
        d_off.upload(offsets, F + 1LL, s);
        d_ids.upload(ids, static_cast<std::size_t>(offsets[F]), s);
        d_owner.upload(owner, F, s);
        d_nbr.upload(neighbour, F, s);
        d_cptr.upload(cptr, s);
        d_cface.upload(cface, s);
    }
    const int one = 1, none = INT_MAX;
    BSG_CUDA(cudaMemcpyAsync(err.data(), &none, sizeof(int), cudaMemcpyHostToDevice, s));
    BSG_CUDA(cudaMemcpyAsync(orth.data(), &one, sizeof(int), cudaMemcpyHostToDevice, s));
    constexpr int B = 128;
    {
        BSG_PROFILE(ctx, "kFaceClassify");
        kFaceClassify<<<gridFor(F, B), B, 0, s>>>(F, d_verts.data(), d_off.data(), d_ids.data(), fsum.data(),
                                                  fflags.data(), scratch_n.data(), err.data());
        ctx.launched();
    }
    if (readFlag(ctx, err) != INT_MAX) rejected();
    // ear-clipping scratch only for the faces that are not convex in some orientation
    long long scratch_total = 0;
    {
        std::size_t temp_bytes = 0;
        BSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, scratch_n.data(), scratch_off.data(), F, s));
        DeviceArray<unsigned char> temp(temp_bytes > 0 ? temp_bytes : 1);
        BSG_CUDA(cub::DeviceScan::ExclusiveSum(temp.data(), temp_bytes, scratch_n.data(), scratch_off.data(), F, s));
        ctx.launched();
        long long last[2] = {0, 0};
        BSG_CUDA(cudaMemcpyAsync(&last[0], scratch_off.data() + (F - 1), sizeof(long long), cudaMemcpyDeviceToHost, s));
        BSG_CUDA(cudaMemcpyAsync(&last[1], scratch_n.data() + (F - 1), sizeof(long long), cudaMemcpyDeviceToHost, s));
        ctx.sync();
        scratch_total = last[0] + last[1];
    }
    DeviceArray<int> scratch(scratch_total > 0 ? scratch_total : 1);
    {
        BSG_PROFILE(ctx, "kCellReference");
        kCellReference<<<gridFor(N, B), B, 0, s>>>(N, d_cptr.data(), d_cface.data(), d_off.data(), fsum.data(),
                                                   ref.data());
        ctx.launched();
    }
    {
        BSG_PROFILE(ctx, "kFaceGeometry");
        kFaceGeometry<<<gridFor(F, B), B, 0, s>>>(F, d_verts.data(), d_off.data(), d_ids.data(), d_owner.data(),
                                                  fsum.data(), ref.data(), fflags.data(), scratch_off.data(),
                                                  scratch.data(), Sf.data(), xf.data(), area.data(), normal.data(),
                                                  err.data());
        ctx.launched();
    }
    if (readFlag(ctx, err) != INT_MAX) rejected();
    fsum.release();
    auto m = std::make_unique<DeviceMesh>();
    m->V.resize(N);
    m->xc.resize(3LL * N);
    {
        BSG_PROFILE(ctx, "kCellGeometry");
        kCellGeometry<<<gridFor(N, B), B, 0, s>>>(N, d_verts.data(), d_off.data(), d_ids.data(), d_cptr.data(),
                                                  d_cface.data(), fflags.data(), scratch_off.data(), scratch.data(),
                                                  Sf.data(), area.data(), ref.data(), m->V.data(), m->xc.data(),
                                                  err.data());
        ctx.launched();
    }
    {
        BSG_PROFILE(ctx, "kCellEdges");
        kCellEdges<<<gridFor(N, kEdgeWarps), 32 * kEdgeWarps, 0, s>>>(N, d_off.data(), d_ids.data(), d_cptr.data(),
                                                                      d_cface.data(), fflags.data(), err.data());
        ctx.launched();
    }
    if (readFlag(ctx, err) != INT_MAX) rejected();
    d_verts.release(); d_ids.release(); d_off.release(); d_cptr.release(); d_cface.release();
    scratch.release(); scratch_off.release(); scratch_n.release(); fflags.release(); ref.release();
    DeviceArray<double> weight(F), dcoef(F), kvec(3LL * F), skew(3LL * F);
    {
        BSG_PROFILE(ctx, "kFaceCoefficients");
        kFaceCoefficients<<<gridFor(F, B), B, 0, s>>>(F, d_owner.data(), d_nbr.data(), Sf.data(), xf.data(),
                                                      area.data(), normal.data(), m->xc.data(), weight.data(),
                                                      dcoef.data(), kvec.data(), skew.data(), orth.data(),
                                                      err.data());
        ctx.launched();
    }
    if (readFlag(ctx, err) != INT_MAX) rejected();
    int orthogonal = 1;
    BSG_CUDA(cudaMemcpyAsync(&orthogonal, orth.data(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ctx.sync();
    // topology and the internal layout
    buildTopology(*m, ctx, N, F, n_patches, owner, neighbour, patch);
    m->orthogonal = orthogonal != 0;
    const int Fi = m->n_interior, Fb = m->n_boundary;
    DeviceArray<int> ext_i, ext_b;
    ext_i.upload(m->interior_ext, s);
    ext_b.upload(m->boundary_ext, s);
    m->w.resize(Fi); m->dcoef.resize(Fi); m->area.resize(Fi);
    m->Sf.resize(3LL * Fi); m->xf.resize(3LL * Fi); m->kvec.resize(3LL * Fi); m->skew.resize(3LL * Fi);
    m->bdcoef.resize(Fb); m->barea.resize(Fb); m->bdist.resize(Fb);
    m->bSf.resize(3LL * Fb); m->bxf.resize(3LL * Fb); m->bn.resize(3LL * Fb); m->bk.resize(3LL * Fb);
    m->rV.resize(N);
    {
        BSG_PROFILE(ctx, "kGatherGeometry");
        if (Fi > 0) {
            kGatherInterior<<<gridFor(Fi, 256), 256, 0, s>>>(Fi, ext_i.data(), weight.data(), dcoef.data(),
                                                             area.data(), Sf.data(), xf.data(), kvec.data(),
                                                             skew.data(), m->w.data(), m->dcoef.data(),
                                                             m->area.data(), m->Sf.data(), m->xf.data(),
                                                             m->kvec.data(), m->skew.data());
            ctx.launched();
        }
        if (Fb > 0) {
            kGatherBoundary<<<gridFor(Fb, 256), 256, 0, s>>>(Fb, ext_b.data(), d_owner.data(), dcoef.data(),
                                                             area.data(), Sf.data(), xf.data(), normal.data(),
                                                             kvec.data(), m->xc.data(), m->bdcoef.data(),
                                                             m->barea.data(), m->bdist.data(), m->bSf.data(),
                                                             m->bxf.data(), m->bn.data(), m->bk.data());
            ctx.launched();
        }
        kReciprocal<<<gridFor(N, 256), 256, 0, s>>>(N, m->V.data(), m->rV.data());
        ctx.launched();
    }
    BSG_CUDA(cudaGetLastError());
    ctx.sync();
    return m;
}

void ensureExternalGeometry(DeviceMesh& m) {
    if (!m.ext_V.empty()) return;
    Context& ctx = *m.ctx;
    const int N = m.n_cells, F = m.n_faces, Fi = m.n_interior, Fb = m.n_boundary;
    std::vector<double> w(Fi), dc(Fi), ar(Fi), S(3LL * Fi), x(3LL * Fi), k(3LL * Fi), sk(3LL * Fi);
    std::vector<double> bdc(Fb), bar(Fb), bS(3LL * Fb), bx(3LL * Fb), bn(3LL * Fb), bk(3LL * Fb);
    std::vector<double> V(N), xc(3LL * N);
    m.w.download(w.data(), ctx.stream); m.dcoef.download(dc.data(), ctx.stream); m.area.download(ar.data(), ctx.stream);
    m.Sf.download(S.data(), ctx.stream); m.xf.download(x.data(), ctx.stream); m.kvec.download(k.data(), ctx.stream);
    m.skew.download(sk.data(), ctx.stream);
    m.bdcoef.download(bdc.data(), ctx.stream); m.barea.download(bar.data(), ctx.stream);
    m.bSf.download(bS.data(), ctx.stream); m.bxf.download(bx.data(), ctx.stream); m.bn.download(bn.data(), ctx.stream);
    m.bk.download(bk.data(), ctx.stream);
    m.V.download(V.data(), ctx.stream); m.xc.download(xc.data(), ctx.stream);
    ctx.sync();
    m.ext_Sf.assign(3LL * F, 0.0); m.ext_xf.assign(3LL * F, 0.0); m.ext_n.assign(3LL * F, 0.0);
    m.ext_k.assign(3LL * F, 0.0); m.ext_skew.assign(3LL * F, 0.0);
    m.ext_area.assign(F, 0.0); m.ext_w.assign(F, 1.0); m.ext_dcoef.assign(F, 0.0);
    for (int i = 0; i < Fi; ++i) {
        const int f = m.interior_ext[i];
        m.ext_w[f] = w[i]; m.ext_dcoef[f] = dc[i]; m.ext_area[f] = ar[i];
        for (int c = 0; c < 3; ++c) {
            m.ext_Sf[3LL * f + c] = S[3LL * i + c];
            m.ext_xf[3LL * f + c] = x[3LL * i + c];
            m.ext_n[3LL * f + c] = S[3LL * i + c] / ar[i];   // the unit normal is Sf / |Sf| as computed
            m.ext_k[3LL * f + c] = k[3LL * i + c];
            m.ext_skew[3LL * f + c] = sk[3LL * i + c];
        }
    }
    for (int i = 0; i < Fb; ++i) {
        const int f = m.boundary_ext[i];
        m.ext_dcoef[f] = bdc[i]; m.ext_area[f] = bar[i];
        for (int c = 0; c < 3; ++c) {
            m.ext_Sf[3LL * f + c] = bS[3LL * i + c];
            m.ext_xf[3LL * f + c] = bx[3LL * i + c];
            m.ext_n[3LL * f + c] = bn[3LL * i + c];
            m.ext_k[3LL * f + c] = bk[3LL * i + c];
        }
    }
    if (!m.h_cell_perm.empty()) {  // renumbered cells: back to the caller's numbering
        std::vector<double> Vc(N), xcc(3LL * N);
        for (int c = 0; c < N; ++c) {
            const int i = m.h_cell_perm[c];
            Vc[c] = V[i];
            for (int q = 0; q < 3; ++q) xcc[3LL * c + q] = xc[3LL * i + q];
        }
        V.swap(Vc);
        xc.swap(xcc);
    }
    m.ext_V = std::move(V);
    m.ext_xc = std::move(xc);
}

}  // namespace bsg
