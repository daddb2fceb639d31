// Mesh ingest: polyhedral geometry on the host (FP64, once per mesh) and the
// device layout described in bsg_internal.h.
//
// computePolyhedralGeometry follows Mesh::polyhedral (src/core/mesh.cpp:321-564):
// outward ring orientation from the mean of the owner's face points, fan or
// ear-clipping triangulation (mesh.cpp:60-161), area vector = sum of triangle
// area vectors, face centre = triangle centroids weighted by |triangle area|,
// face area = sum of |triangle area|, cell volume/centroid from signed tetrahedra
// about the mean face point, and the face coefficients of mesh.cpp:521-564.
#include "bsg_internal.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <numeric>

namespace bsg {
namespace {

using V3 = std::array<double, 3>;
inline V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline V3 add(const V3& a, const V3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline V3 mul(double s, const V3& a) { return {s * a[0], s * a[1], s * a[2]}; }
inline double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline V3 cross(const V3& a, const V3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline double norm(const V3& a) { return std::sqrt(dot(a, a)); }

struct Tri { int a, b, c; };

double cross2(const double* a, const double* b, const double* c) {
    return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0]);
}

// Triangulation of one face ring (mesh.cpp:60-161).
void triangulate(const std::vector<int>& ring, const double* verts, std::vector<Tri>& out) {
    out.clear();
    const std::size_t n = ring.size();
    if (n < 3) fail(kArgument, "polyhedral face has fewer than three vertices");
    V3 nrm{0, 0, 0};
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (std::size_t i = 0; i < n; ++i) {
        const V3 c{verts[3 * ring[i]], verts[3 * ring[i] + 1], verts[3 * ring[i] + 2]};
        const int j = ring[(i + 1) % n];
        const V3 d{verts[3 * j], verts[3 * j + 1], verts[3 * j + 2]};
        nrm = add(nrm, mul(0.5, cross(c, d)));
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], c[k]); hi[k] = std::max(hi[k], c[k]); }
    }
    const double a0 = std::fabs(nrm[0]), a1 = std::fabs(nrm[1]), a2 = std::fabs(nrm[2]);
    const int drop = a1 > a0 ? (a2 > a1 ? 2 : 1) : (a2 > a0 ? 2 : 0);
    const double scale = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1.0});
    const double tol = 1e-13 * scale * scale;
    std::vector<double> q(2 * n);
    for (std::size_t i = 0; i < n; ++i) {
        const double* p = verts + 3 * ring[i];
        if (drop == 0) { q[2 * i] = p[1]; q[2 * i + 1] = p[2]; }
        else if (drop == 1) { q[2 * i] = p[2]; q[2 * i + 1] = p[0]; }
        else { q[2 * i] = p[0]; q[2 * i + 1] = p[1]; }
    }
    double signed_area = 0.0;
    for (std::size_t i = 0; i < n; ++i) {
        const std::size_t j = (i + 1) % n;
        signed_area += q[2 * i] * q[2 * j + 1] - q[2 * j] * q[2 * i + 1];
    }
    if (std::fabs(signed_area) <= tol) fail(kArgument, "polyhedral face projects to zero area");
    const double orient = signed_area > 0.0 ? 1.0 : -1.0;
    bool convex = true, saw = false;
    for (std::size_t i = 0; i < n; ++i) {
        const double t = orient * cross2(&q[2 * ((i + n - 1) % n)], &q[2 * i], &q[2 * ((i + 1) % n)]);
        saw = saw || std::fabs(t) > tol;
        if (t < -tol) { convex = false; break; }
    }
    if (!saw) fail(kArgument, "polyhedral face is collinear");
    if (convex) {
        for (std::size_t i = 1; i + 1 < n; ++i) out.push_back({ring[0], ring[i], ring[i + 1]});
        return;
    }
    std::vector<std::size_t> rem(n);
    std::iota(rem.begin(), rem.end(), 0);
    while (rem.size() > 3) {
        bool clipped = false;
        const std::size_t m = rem.size();
        for (std::size_t pos = 0; pos < m; ++pos) {
            const std::size_t pv = rem[(pos + m - 1) % m], cu = rem[pos], nx = rem[(pos + 1) % m];
            if (orient * cross2(&q[2 * pv], &q[2 * cu], &q[2 * nx]) <= tol) continue;
            bool inside = false;
            for (std::size_t c : rem) {
                if (c == pv || c == cu || c == nx) continue;
                const double ab = orient * cross2(&q[2 * pv], &q[2 * cu], &q[2 * c]);
                const double bc = orient * cross2(&q[2 * cu], &q[2 * nx], &q[2 * c]);
                const double ca = orient * cross2(&q[2 * nx], &q[2 * pv], &q[2 * c]);
                if (ab >= -tol && bc >= -tol && ca >= -tol) { inside = true; break; }
            }
            if (inside) continue;
            out.push_back({ring[pv], ring[cu], ring[nx]});
            rem.erase(rem.begin() + static_cast<std::ptrdiff_t>(pos));
            clipped = true;
            break;
        }
        if (!clipped) fail(kArgument, "polyhedral face is self-intersecting or not simple");
    }
    out.push_back({ring[rem[0]], ring[rem[1]], ring[rem[2]]});
}

V3 vtx(const double* verts, int i) { return {verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]}; }

}  // namespace

int validatePolyhedralTopology(int n_vertices, int n_faces, const int* offsets, const int* ids, const int* owner,
                               const int* neighbour, const int* patch, int n_patches) {
    if (n_vertices <= 0 || n_faces <= 0 || n_patches <= 0) fail(kArgument, "polyhedral mesh arrays are empty");
    if (offsets[0] != 0) fail(kArgument, "polyhedral face offsets must start at 0");
    int n_cells = 0;
    for (int f = 0; f < n_faces; ++f) {
        if (owner[f] < 0 || neighbour[f] < -1 || neighbour[f] == owner[f])
            fail(kArgument, "polyhedral face has invalid owner/neighbour");
        n_cells = std::max(n_cells, owner[f] + 1);
        if (neighbour[f] >= 0) n_cells = std::max(n_cells, neighbour[f] + 1);
        if (neighbour[f] >= 0 && patch[f] != -1)
            fail(kArgument, "internal polyhedral face cannot belong to a boundary patch");
        if (neighbour[f] < 0 && (patch[f] < 0 || patch[f] >= n_patches))
            fail(kArgument, "boundary polyhedral face " + std::to_string(f) + " has invalid patch");
        if (offsets[f + 1] < offsets[f]) fail(kArgument, "polyhedral face offsets decrease");
        for (int k = offsets[f]; k < offsets[f + 1]; ++k)
            if (ids[k] < 0 || ids[k] >= n_vertices) fail(kArgument, "face references an invalid vertex");
    }
    return n_cells;
}

HostGeometry computePolyhedralGeometry(int n_vertices, const double* verts, int n_faces,
                                       const int* offsets, const int* ids, const int* owner,
                                       const int* neighbour, const int* patch, int n_patches) {
    HostGeometry g;
    const int n_cells = validatePolyhedralTopology(n_vertices, n_faces, offsets, ids, owner, neighbour, patch,
                                                   n_patches);
    g.n_cells = n_cells;
    g.n_faces = n_faces;
    g.n_patches = n_patches;
    g.owner.assign(owner, owner + n_faces);
    g.nbr.assign(neighbour, neighbour + n_faces);
    g.patch.assign(patch, patch + n_faces);
    // Orientation reference: mean of all face points of each cell (mesh.cpp:361-377).
    std::vector<V3> psum(n_cells, V3{0, 0, 0});
    std::vector<double> pcnt(n_cells, 0.0);
    for (int f = 0; f < n_faces; ++f) {
        V3 s{0, 0, 0};
        for (int k = offsets[f]; k < offsets[f + 1]; ++k) s = add(s, vtx(verts, ids[k]));
        const double cnt = offsets[f + 1] - offsets[f];
        psum[owner[f]] = add(psum[owner[f]], s);
        pcnt[owner[f]] += cnt;
        if (neighbour[f] >= 0) { psum[neighbour[f]] = add(psum[neighbour[f]], s); pcnt[neighbour[f]] += cnt; }
    }
    std::vector<V3> ref(n_cells);
    for (int c = 0; c < n_cells; ++c) ref[c] = mul(1.0 / std::max(1.0, pcnt[c]), psum[c]);
    g.Sf.resize(3 * n_faces); g.xf.resize(3 * n_faces); g.area.resize(n_faces); g.normal.resize(3 * n_faces);
    std::vector<std::vector<Tri>> tris(n_faces);
    std::vector<int> oriented(ids, ids + offsets[n_faces]);  // rings after outward orientation
    std::vector<int> ring;
    for (int f = 0; f < n_faces; ++f) {
        ring.assign(ids + offsets[f], ids + offsets[f + 1]);
        {
            std::vector<int> sorted(ring);
            std::sort(sorted.begin(), sorted.end());
            if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
                fail(kArgument, "polyhedral face repeats a vertex");
        }
        V3 avg{0, 0, 0};
        for (int v : ring) avg = add(avg, vtx(verts, v));
        avg = mul(1.0 / ring.size(), avg);
        triangulate(ring, verts, tris[f]);
        auto areaOf = [&](const std::vector<Tri>& ts) {
            V3 a{0, 0, 0};
            for (const Tri& t : ts) {
                const V3 A = vtx(verts, t.a), B = vtx(verts, t.b), C = vtx(verts, t.c);
                a = add(a, mul(0.5, cross(sub(B, A), sub(C, A))));
            }
            return a;
        };
        V3 a = areaOf(tris[f]);
        if (dot(a, sub(avg, ref[owner[f]])) < 0.0) {
            std::reverse(ring.begin() + 1, ring.end());
            triangulate(ring, verts, tris[f]);
            a = areaOf(tris[f]);
        }
        if (!(norm(a) > 0.0) || !std::isfinite(norm(a))) fail(kArgument, "polyhedral face has zero area");
        V3 centre{0, 0, 0};
        double total = 0.0;
        for (const Tri& t : tris[f]) {
            const V3 A = vtx(verts, t.a), B = vtx(verts, t.b), C = vtx(verts, t.c);
            const double wgt = norm(mul(0.5, cross(sub(B, A), sub(C, A))));
            if (!(wgt > 0.0)) fail(kArgument, "polyhedral mesh contains a degenerate face triangle");
            centre = add(centre, mul(wgt, mul(1.0 / 3.0, add(add(A, B), C))));
            total += wgt;
        }
        centre = mul(1.0 / total, centre);
        for (int k = 0; k < 3; ++k) {
            g.Sf[3 * f + k] = a[k];
            g.xf[3 * f + k] = centre[k];
            g.normal[3 * f + k] = a[k] / total;
        }
        g.area[f] = total;
        std::copy(ring.begin(), ring.end(), oriented.begin() + offsets[f]);
    }
    // Every cell must be a closed, consistently oriented surface: vector areas
    // close and each edge of the outward-oriented rings appears exactly twice
    // with opposite directions (Mesh::validate, src/core/mesh.cpp:709-756).
    {
        std::vector<int> cptr(n_cells + 1, 0);
        for (int f = 0; f < n_faces; ++f) {
            ++cptr[owner[f] + 1];
            if (neighbour[f] >= 0) ++cptr[neighbour[f] + 1];
        }
        for (int c = 0; c < n_cells; ++c) cptr[c + 1] += cptr[c];
        std::vector<int> cface(cptr[n_cells]), fill(cptr.begin(), cptr.end() - 1);
        for (int f = 0; f < n_faces; ++f) {
            cface[fill[owner[f]]++] = f;
            if (neighbour[f] >= 0) cface[fill[neighbour[f]]++] = -f - 1;
        }
        std::vector<std::pair<long long, int>> edges;
        for (int c = 0; c < n_cells; ++c) {
            double cx = 0, cy = 0, cz = 0, total = 0;
            edges.clear();
            for (int k = cptr[c]; k < cptr[c + 1]; ++k) {
                const int f = cface[k] >= 0 ? cface[k] : -cface[k] - 1;
                const double s = cface[k] >= 0 ? 1.0 : -1.0;
                cx += s * g.Sf[3 * f]; cy += s * g.Sf[3 * f + 1]; cz += s * g.Sf[3 * f + 2];
                total += g.area[f];
                const int* ring = oriented.data() + offsets[f];
                const std::size_t m = static_cast<std::size_t>(offsets[f + 1] - offsets[f]);
                for (std::size_t e = 0; e < m; ++e) {
                    int from = ring[e], to = ring[(e + 1) % m];
                    if (s < 0) std::swap(from, to);
                    const int a = std::min(from, to), b = std::max(from, to);
                    edges.push_back({static_cast<long long>(a) * n_vertices + b, from == a ? 1 : -1});
                }
            }
            if (!(std::isfinite(total) && std::sqrt(cx * cx + cy * cy + cz * cz) <= 1e-9 * std::max(total, 1.0)))
                fail(kArgument, "polyhedral cell face area vectors do not close (cell " + std::to_string(c) + ")");
            std::sort(edges.begin(), edges.end());
            for (std::size_t e = 0; e < edges.size();) {
                std::size_t j = e;
                int orient = 0;
                while (j < edges.size() && edges[j].first == edges[e].first) orient += edges[j++].second;
                if (j - e != 2 || orient != 0)
                    fail(kArgument, "polyhedral cell surface has a non-manifold or inconsistently oriented edge " +
                                        std::to_string(edges[e].first / n_vertices) + "-" +
                                        std::to_string(edges[e].first % n_vertices));
                e = j;
            }
        }
    }
    // Cell volume and centroid (mesh.cpp:486-519).
    g.V.assign(n_cells, 0.0);
    g.xc.assign(3 * n_cells, 0.0);
    std::vector<V3> mom(n_cells, V3{0, 0, 0});
    for (int f = 0; f < n_faces; ++f) {
        for (int side = 0; side < 2; ++side) {
            const int cell = side == 0 ? owner[f] : neighbour[f];
            if (cell < 0) continue;
            const double sign = side == 0 ? 1.0 : -1.0;
            const V3& r = ref[cell];
            for (const Tri& t : tris[f]) {
                const V3 A = vtx(verts, t.a), B = vtx(verts, t.b), D = vtx(verts, t.c);
                const double tet = sign * dot(sub(A, r), cross(sub(B, r), sub(D, r))) / 6.0;
                g.V[cell] += tet;
                mom[cell] = add(mom[cell], mul(tet, mul(0.25, add(add(add(r, A), B), D))));
            }
        }
    }
    for (int c = 0; c < n_cells; ++c) {
        if (!(g.V[c] > 0.0) || !std::isfinite(g.V[c]))
            fail(kArgument, "polyhedral cell has non-positive signed volume");
        for (int k = 0; k < 3; ++k) g.xc[3 * c + k] = mom[c][k] / g.V[c];
    }
    // Face coefficients, interpolation weights and skewness (mesh.cpp:521-564).
    g.weight.assign(n_faces, 1.0);
    g.dcoef.assign(n_faces, 0.0);
    g.kvec.assign(3 * n_faces, 0.0);
    g.skew.assign(3 * n_faces, 0.0);
    g.orthogonal = true;
    for (int f = 0; f < n_faces; ++f) {
        const int o = owner[f], n = neighbour[f];
        const V3 xf{g.xf[3 * f], g.xf[3 * f + 1], g.xf[3 * f + 2]};
        const V3 xo{g.xc[3 * o], g.xc[3 * o + 1], g.xc[3 * o + 2]};
        const V3 Sf{g.Sf[3 * f], g.Sf[3 * f + 1], g.Sf[3 * f + 2]};
        const V3 nr{g.normal[3 * f], g.normal[3 * f + 1], g.normal[3 * f + 2]};
        V3 delta;
        V3 xn{0, 0, 0};
        if (n < 0) delta = sub(xf, xo);
        else { xn = V3{g.xc[3 * n], g.xc[3 * n + 1], g.xc[3 * n + 2]}; delta = sub(xn, xo); }
        const double d2 = dot(delta, delta), proj = dot(Sf, delta);
        if (!(d2 > 0.0) || !(proj > 0.0))
            fail(kArgument, "polyhedral face geometry has invalid owner/neighbour direction");
        g.dcoef[f] = proj / d2;
        const V3 k = sub(Sf, mul(g.dcoef[f], delta));
        for (int c = 0; c < 3; ++c) g.kvec[3 * f + c] = k[c];
        if (norm(k) > 1e-12 * g.area[f]) g.orthogonal = false;
        if (n >= 0) {
            const double od = std::fabs(dot(sub(xf, xo), nr)), nd = std::fabs(dot(sub(xn, xf), nr));
            if (!(od + nd > 0.0)) fail(kArgument, "polyhedral interpolation distance is invalid");
            g.weight[f] = nd / (od + nd);
            const double den = dot(delta, nr);
            if (!(den > 0.0) || !std::isfinite(den)) fail(kArgument, "polyhedral face interpolation direction is invalid");
            const double frac = dot(sub(xf, xo), nr) / den;
            const V3 sk = sub(xf, add(xo, mul(frac, delta)));
            for (int c = 0; c < 3; ++c) g.skew[3 * f + c] = sk[c];
            if (norm(sk) > 1e-12 * std::sqrt(d2)) g.orthogonal = false;
        }
    }
    return g;
}

void buildTopology(DeviceMesh& mesh, Context& ctx, int N, int F, int n_patches, const int* owner, const int* nbr,
                   const int* patch) {
    if (N <= 0 || F <= 0) fail(kArgument, "mesh has no cells or faces");
    DeviceMesh* m = &mesh;
    m->ctx = &ctx;
    m->n_cells = N;
    m->n_faces = F;
    m->n_patches = n_patches;
    // interior and boundary faces, each stably ordered by owner (a counting sort)
    std::vector<int> count_i(N + 1, 0), count_b(N + 1, 0);
    for (int f = 0; f < F; ++f) {
        if (owner[f] < 0 || owner[f] >= N || nbr[f] >= N || nbr[f] < -1)
            fail(kArgument, "face owner/neighbour out of range");
        if (nbr[f] < 0 && (patch[f] < 0 || patch[f] >= n_patches))
            fail(kArgument, "boundary face has an invalid patch");
        ++(nbr[f] >= 0 ? count_i : count_b)[owner[f] + 1];
    }
    for (int c = 0; c < N; ++c) { count_i[c + 1] += count_i[c]; count_b[c + 1] += count_b[c]; }
    const int Fi = count_i[N], Fb = count_b[N];
    m->interior_ext.assign(Fi, 0);
    m->boundary_ext.assign(Fb, 0);
    for (int f = 0; f < F; ++f) {
        if (nbr[f] >= 0) m->interior_ext[count_i[owner[f]]++] = f;
        else m->boundary_ext[count_b[owner[f]]++] = f;
    }
    m->n_interior = Fi;
    m->n_boundary = Fb;
    m->face_kind.assign(F, 0);
    m->face_slot.assign(F, 0);
    for (int i = 0; i < Fi; ++i) { m->face_kind[m->interior_ext[i]] = 0; m->face_slot[m->interior_ext[i]] = i; }
    for (int i = 0; i < Fb; ++i) { m->face_kind[m->boundary_ext[i]] = 1; m->face_slot[m->boundary_ext[i]] = i; }
    cudaStream_t s = ctx.stream;
    {
        // caller face -> internal face position (interior first), for device-side reordering
        std::vector<int> perm(F);
        for (int f = 0; f < F; ++f) perm[f] = m->face_kind[f] == 0 ? m->face_slot[f] : Fi + m->face_slot[f];
        m->face_perm.upload(perm, s);
    }
    m->h_own.resize(Fi);
    m->h_nbr.resize(Fi);
    for (int i = 0; i < Fi; ++i) { m->h_own[i] = owner[m->interior_ext[i]]; m->h_nbr[i] = nbr[m->interior_ext[i]]; }
    m->own.upload(m->h_own, s);
    m->nbr.upload(m->h_nbr, s);
    m->h_bown.resize(Fb);
    std::vector<int> bpatch(Fb);
    for (int i = 0; i < Fb; ++i) {
        m->h_bown[i] = owner[m->boundary_ext[i]];
        bpatch[i] = patch[m->boundary_ext[i]];
    }
    m->bown.upload(m->h_bown, s);
    m->bpatch.upload(bpatch, s);
    // cell -> interior face CSR, faces of a row in increasing internal face order
    m->h_cf_ptr.assign(N + 1, 0);
    for (int i = 0; i < Fi; ++i) { ++m->h_cf_ptr[m->h_own[i] + 1]; ++m->h_cf_ptr[m->h_nbr[i] + 1]; }
    for (int c = 0; c < N; ++c) m->h_cf_ptr[c + 1] += m->h_cf_ptr[c];
    m->h_cf_face.resize(2 * static_cast<std::size_t>(Fi));
    m->h_cf_col.resize(2 * static_cast<std::size_t>(Fi));
    {
        std::vector<int> fill(m->h_cf_ptr.begin(), m->h_cf_ptr.end() - 1);
        m->h_slot_own.resize(Fi);
        m->h_slot_nbr.resize(Fi);
        for (int i = 0; i < Fi; ++i) {
            const int o = m->h_own[i], n = m->h_nbr[i];
            m->h_slot_own[i] = fill[o];
            m->h_cf_face[fill[o]] = i; m->h_cf_col[fill[o]++] = n;
            m->h_slot_nbr[i] = fill[n];
            m->h_cf_face[fill[n]] = i; m->h_cf_col[fill[n]++] = o;
        }
    }
    m->slot_own.upload(m->h_slot_own, s);
    m->slot_nbr.upload(m->h_slot_nbr, s);
    m->cf_ptr.upload(m->h_cf_ptr, s);
    m->cf_face.upload(m->h_cf_face, s);
    m->cf_col.upload(m->h_cf_col, s);
    m->h_cb_ptr.assign(N + 1, 0);
    for (int i = 0; i < Fb; ++i) ++m->h_cb_ptr[m->h_bown[i] + 1];
    for (int c = 0; c < N; ++c) m->h_cb_ptr[c + 1] += m->h_cb_ptr[c];
    m->cb_ptr.upload(m->h_cb_ptr, s);
    m->ext_owner.assign(owner, owner + F);
    m->ext_nbr.assign(nbr, nbr + F);
    m->ext_patch.assign(patch, patch + F);
}

std::unique_ptr<DeviceMesh> buildDeviceMesh(Context& ctx, const HostGeometry& g) {
    if (g.n_cells <= 0 || g.n_faces <= 0) fail(kArgument, "mesh has no cells or faces");
    auto m = std::make_unique<DeviceMesh>();
    const int N = g.n_cells;
    buildTopology(*m, ctx, N, g.n_faces, g.n_patches, g.owner.data(), g.nbr.data(), g.patch.data());
    m->orthogonal = g.orthogonal;
    auto gather1 = [](const std::vector<double>& a, const std::vector<int>& idx) {
        std::vector<double> o(idx.size());
        for (std::size_t i = 0; i < idx.size(); ++i) o[i] = a[idx[i]];
        return o;
    };
    auto gather3 = [](const std::vector<double>& a, const std::vector<int>& idx) {
        std::vector<double> o(3 * idx.size());
        for (std::size_t i = 0; i < idx.size(); ++i)
            for (int c = 0; c < 3; ++c) o[3 * i + c] = a[3 * idx[i] + c];
        return o;
    };
    cudaStream_t s = ctx.stream;
    const int Fb = m->n_boundary;
    // interior faces
    m->w.upload(gather1(g.weight, m->interior_ext), s);
    m->dcoef.upload(gather1(g.dcoef, m->interior_ext), s);
    m->area.upload(gather1(g.area, m->interior_ext), s);
    m->Sf.upload(gather3(g.Sf, m->interior_ext), s);
    m->xf.upload(gather3(g.xf, m->interior_ext), s);
    m->kvec.upload(gather3(g.kvec, m->interior_ext), s);
    m->skew.upload(gather3(g.skew, m->interior_ext), s);
    // boundary faces
    std::vector<double> bdist(Fb);
    for (int i = 0; i < Fb; ++i) {
        const int f = m->boundary_ext[i], o = g.owner[f];
        double d = 0.0;
        for (int c = 0; c < 3; ++c) d += (g.xf[3 * f + c] - g.xc[3 * o + c]) * g.normal[3 * f + c];
        bdist[i] = d;
    }
    m->bdcoef.upload(gather1(g.dcoef, m->boundary_ext), s);
    m->barea.upload(gather1(g.area, m->boundary_ext), s);
    m->bdist.upload(bdist, s);
    m->bSf.upload(gather3(g.Sf, m->boundary_ext), s);
    m->bxf.upload(gather3(g.xf, m->boundary_ext), s);
    m->bn.upload(gather3(g.normal, m->boundary_ext), s);
    m->bk.upload(gather3(g.kvec, m->boundary_ext), s);
    // cells
    std::vector<double> rV(N);
    for (int c = 0; c < N; ++c) rV[c] = 1.0 / g.V[c];
    m->V.upload(g.V, s);
    m->rV.upload(rV, s);
    m->xc.upload(g.xc, s);
    // caller-numbered geometry for exports
    m->ext_Sf = g.Sf; m->ext_xf = g.xf; m->ext_area = g.area; m->ext_n = g.normal; m->ext_w = g.weight;
    m->ext_dcoef = g.dcoef; m->ext_k = g.kvec; m->ext_skew = g.skew; m->ext_xc = g.xc; m->ext_V = g.V;
    ctx.sync();
    return m;
}

}  // namespace bsg
