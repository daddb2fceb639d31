// CPU linear-system backend used to run the reference's own finite-volume
// sources as the oracle and as the timed CPU baseline.  Test infrastructure
// only, never the product.
//
// It replaces the PETSc/Hypre translation units at the reference's single
// link-time seam, `detail::makeComputeBackend` (src/internal/compute_backend.h:17-41),
// exactly as the reference's tests/backend_interface_test.cpp:72-80 does.  The
// acceptance contract is the reference's: unpreconditioned true residual
// ||b-Ax|| <= max(atol, rtol*max(||r0||,||b||)) (include/babelsim/solver_control.h:196-210),
// zero initial guess unless warm_start, true-residual restarts with a halved
// internal target (src/backend/petsc_linear_system.cpp:355-481).  Krylov
// iterates need not match PETSc's; only the converged solution is pinned.
//
// Like PetscBackend (src/backend/petsc_backend.cpp:201-213) it keeps one linear
// system per equation identity ("scalar:<equation>:<field>" / "vector:..."), and
// each system follows PetscLinearSystem's preconditioner lifecycle
// (petsc_linear_system.cpp:257-324, 446-470): an exactly unchanged matrix skips
// its update, a preconditioner is reused (lagged) until
// preconditioner_rebuild_interval matrix versions or right-hand-side solves have
// passed, a lagged solve that needs more than
// preconditioner_reuse_iteration_growth times the fresh iterations forces a
// rebuild before the next solve, and a lagged solve that fails is retried once
// with a fresh preconditioner.  Preconditioners: pcType hypre|gamg -> CPU
// aggregation AMG (stand-in for BoomerAMG / GAMG), bjacobi|asm|icc -> ILU(0) of
// the whole matrix (one process: PETSc's block Jacobi has a single block, ILU
// for non-symmetric Krylov methods, petsc_linear_system.cpp:326-353 makes it ICC
// for CG; ILU(0) of a symmetric matrix is its IC(0)), jacobi -> point Jacobi.
// Krylov: CG, BiCGStab, restarted GMRES(30) and FGMRES(30), right-preconditioned.
//
// With BABELSIM_ORACLE_DUMP=<dir> every assembled LDU system handed to solve()
// is written to <dir>/system_<seq>.bin together with the unknown before and
// after the solve, so the GPU assembly can be compared coefficient by
// coefficient against the reference's own discretisation.
#include "babelsim/field.h"
#include "babelsim/parallel.h"
#include "internal/compute_backend.h"
#include "internal/field_access.h"
#include "internal/mesh_access.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace babelsim::detail {

void ensurePetscSession() {}
void finalizePetscSession() {}

namespace {

using Clock = std::chrono::steady_clock;
double secondsSince(Clock::time_point t) { return std::chrono::duration<double>(Clock::now() - t).count(); }

struct Csr {
    int n = 0;
    std::vector<int> row, col, diag_pos;
    std::vector<double> val, inv_diag;
};

// Fixed CSR pattern of a mesh with rows in cell order (columns sorted), and for
// every LDU coefficient its CSR position: upper[f] sits at (owner, neighbour),
// lower[f] at (neighbour, owner), as in petsc_assembly_plan.cpp:62-87.
struct Pattern {
    Csr shape;
    std::vector<int> at_upper, at_lower;  // per face, -1 on boundary faces
    explicit Pattern(const Mesh& mesh) {
        const int n = mesh.cellCount();
        std::vector<std::vector<std::pair<int, int>>> rows(n);  // (column, face*2 + side) per row
        for (int i = 0; i < n; ++i) rows[i].push_back({i, -1});
        for (Index f = 0; f < mesh.faceCount(); ++f) {
            const Index nb = mesh.neighbour(f);
            if (nb == invalid_index) continue;
            rows[mesh.owner(f)].push_back({static_cast<int>(nb), 2 * static_cast<int>(f)});
            rows[nb].push_back({static_cast<int>(mesh.owner(f)), 2 * static_cast<int>(f) + 1});
        }
        shape.n = n;
        shape.row.assign(n + 1, 0);
        at_upper.assign(mesh.faceCount(), -1);
        at_lower.assign(mesh.faceCount(), -1);
        shape.diag_pos.resize(n);
        for (int i = 0; i < n; ++i) {
            auto& r = rows[i];
            std::stable_sort(r.begin(), r.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            for (const auto& e : r) {
                const int k = static_cast<int>(shape.col.size());
                shape.col.push_back(e.first);
                if (e.second < 0) shape.diag_pos[i] = k;
                else if (e.second % 2 == 0) at_upper[e.second / 2] = k;
                else at_lower[e.second / 2] = k;
            }
            shape.row[i + 1] = static_cast<int>(shape.col.size());
        }
        shape.val.assign(shape.col.size(), 0.0);
        shape.inv_diag.assign(n, 1.0);
    }
    // Values of an LDU system (repeated owner/neighbour pairs keep separate entries).
    void fill(Csr& a, const std::vector<double>& diag, const std::vector<double>& upper,
              const std::vector<double>& lower) const {
        if (a.n != shape.n) a = shape;
        for (int i = 0; i < a.n; ++i) a.val[a.diag_pos[i]] = diag[i];
        for (std::size_t f = 0; f < at_upper.size(); ++f) {
            if (at_upper[f] < 0) continue;
            a.val[at_upper[f]] = upper[f];
            a.val[at_lower[f]] = lower[f];
        }
        for (int i = 0; i < a.n; ++i) a.inv_diag[i] = diag[i] != 0.0 ? 1.0 / diag[i] : 1.0;
    }
};

void spmv(const Csr& a, const std::vector<double>& x, std::vector<double>& y) {
    for (int i = 0; i < a.n; ++i) {
        double s = 0.0;
        for (int k = a.row[i]; k < a.row[i + 1]; ++k) s += a.val[k] * x[a.col[k]];
        y[i] = s;
    }
}
double dotv(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (std::size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}
double trueResidual(const Csr& a, const std::vector<double>& b, const std::vector<double>& x,
                    std::vector<double>& r) {
    spmv(a, x, r);
    for (int i = 0; i < a.n; ++i) r[i] = b[i] - r[i];
    return std::sqrt(dotv(r, r));
}

struct Preconditioner {
    virtual ~Preconditioner() = default;
    virtual void apply(const std::vector<double>& r, std::vector<double>& z) = 0;
};

struct JacobiPc : Preconditioner {
    std::vector<double> inv_diag;
    explicit JacobiPc(const Csr& a) : inv_diag(a.inv_diag) {}
    void apply(const std::vector<double>& r, std::vector<double>& z) override {
        for (std::size_t i = 0; i < r.size(); ++i) z[i] = inv_diag[i] * r[i];
    }
};

// ILU(0): LU factors on the matrix's own pattern (columns sorted per row).
struct Ilu0Pc : Preconditioner {
    Csr lu;
    explicit Ilu0Pc(const Csr& a) : lu(a) {
        const int n = lu.n;
        std::vector<int> where(n, -1);
        for (int i = 0; i < n; ++i) {
            for (int k = lu.row[i]; k < lu.row[i + 1]; ++k) where[lu.col[k]] = k;
            for (int k = lu.row[i]; k < lu.row[i + 1]; ++k) {
                const int j = lu.col[k];
                if (j >= i) break;
                const double pivot = lu.val[lu.diag_pos[j]];
                const double f = pivot != 0.0 ? lu.val[k] / pivot : 0.0;
                lu.val[k] = f;
                for (int m = lu.diag_pos[j] + 1; m < lu.row[j + 1]; ++m) {
                    const int w = where[lu.col[m]];
                    if (w >= 0) lu.val[w] -= f * lu.val[m];
                }
            }
            for (int k = lu.row[i]; k < lu.row[i + 1]; ++k) where[lu.col[k]] = -1;
        }
    }
    void apply(const std::vector<double>& r, std::vector<double>& z) override {
        const int n = lu.n;
        for (int i = 0; i < n; ++i) {
            double s = r[i];
            for (int k = lu.row[i]; k < lu.diag_pos[i]; ++k) s -= lu.val[k] * z[lu.col[k]];
            z[i] = s;
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = z[i];
            for (int k = lu.diag_pos[i] + 1; k < lu.row[i + 1]; ++k) s -= lu.val[k] * z[lu.col[k]];
            const double d = lu.val[lu.diag_pos[i]];
            z[i] = d != 0.0 ? s / d : s;
        }
    }
};

// CPU aggregation AMG (stand-in for Hypre BoomerAMG behind pcType hypre|gamg):
// pairwise matching of strongest negative couplings applied twice per level,
// Galerkin coarse operators of piecewise-constant prolongation, V(2,2) cycle
// with damped Jacobi (omega 2/3) and a dense LU solve on the coarsest level.
struct CpuAmg : Preconditioner {
    struct Level {
        Csr a;
        std::vector<int> agg;  // to the next level
        std::vector<double> x, b, t;
    };
    std::vector<Level> levels;
    std::vector<double> lu;   // coarsest dense LU (row-major), partial pivoting
    std::vector<int> piv;

    static std::vector<int> pairwise(const Csr& a, int& nc) {
        std::vector<int> agg(a.n, -1);
        nc = 0;
        for (int i = 0; i < a.n; ++i) {
            if (agg[i] >= 0) continue;
            int best = -1;
            double bs = 0.0;
            for (int k = a.row[i]; k < a.row[i + 1]; ++k) {
                const int j = a.col[k];
                if (j == i || agg[j] >= 0) continue;
                if (-a.val[k] > bs) { bs = -a.val[k]; best = j; }
            }
            agg[i] = nc;
            if (best >= 0) agg[best] = nc;
            ++nc;
        }
        return agg;
    }
    // A_c = P^T A P for piecewise-constant P, with a sparse accumulator per coarse row.
    static Csr galerkin(const Csr& a, const std::vector<int>& agg, int nc) {
        std::vector<int> first(nc + 1, 0), members(a.n);
        for (int i = 0; i < a.n; ++i) ++first[agg[i] + 1];
        for (int I = 0; I < nc; ++I) first[I + 1] += first[I];
        std::vector<int> fill(first.begin(), first.end() - 1);
        for (int i = 0; i < a.n; ++i) members[fill[agg[i]]++] = i;
        Csr c;
        c.n = nc;
        c.row.assign(nc + 1, 0);
        c.diag_pos.assign(nc, -1);
        std::vector<int> where(nc, -1);
        std::vector<int> cols;
        for (int I = 0; I < nc; ++I) {
            cols.clear();
            const std::size_t base = c.col.size();
            for (int m = first[I]; m < first[I + 1]; ++m) {
                const int i = members[m];
                for (int k = a.row[i]; k < a.row[i + 1]; ++k) {
                    const int J = agg[a.col[k]];
                    if (where[J] < 0) { where[J] = static_cast<int>(cols.size()); cols.push_back(J); }
                }
            }
            std::sort(cols.begin(), cols.end());
            for (std::size_t q = 0; q < cols.size(); ++q) where[cols[q]] = static_cast<int>(base + q);
            c.col.insert(c.col.end(), cols.begin(), cols.end());
            c.val.resize(c.col.size(), 0.0);
            for (int m = first[I]; m < first[I + 1]; ++m) {
                const int i = members[m];
                for (int k = a.row[i]; k < a.row[i + 1]; ++k) c.val[where[agg[a.col[k]]]] += a.val[k];
            }
            for (int J : cols) {
                if (J == I) c.diag_pos[I] = where[J];
                where[J] = -1;
            }
            c.row[I + 1] = static_cast<int>(c.col.size());
        }
        c.inv_diag.assign(nc, 1.0);
        for (int I = 0; I < nc; ++I)
            if (c.diag_pos[I] >= 0 && c.val[c.diag_pos[I]] != 0.0) c.inv_diag[I] = 1.0 / c.val[c.diag_pos[I]];
        return c;
    }
    explicit CpuAmg(const Csr& fine) {
        levels.push_back({fine, {}, {}, {}, {}});
        while (levels.back().a.n > 64 && levels.size() < 12) {
            int n1 = 0, n2 = 0;
            const Csr& a = levels.back().a;
            const std::vector<int> a1 = pairwise(a, n1);
            const Csr c1 = galerkin(a, a1, n1);
            const std::vector<int> a2 = pairwise(c1, n2);
            if (n2 >= a.n) break;
            std::vector<int> agg(a.n);
            for (int i = 0; i < a.n; ++i) agg[i] = a2[a1[i]];
            Csr c = galerkin(a, agg, n2);
            levels.back().agg = std::move(agg);
            levels.push_back({std::move(c), {}, {}, {}, {}});
        }
        for (auto& l : levels) { l.x.resize(l.a.n); l.b.resize(l.a.n); l.t.resize(l.a.n); }
        const Csr& c = levels.back().a;
        const int n = c.n;
        lu.assign(static_cast<std::size_t>(n) * n, 0.0);
        for (int i = 0; i < n; ++i)
            for (int k = c.row[i]; k < c.row[i + 1]; ++k) lu[static_cast<std::size_t>(i) * n + c.col[k]] += c.val[k];
        piv.resize(n);
        for (int k = 0; k < n; ++k) {
            int p = k;
            for (int i = k + 1; i < n; ++i)
                if (std::fabs(lu[static_cast<std::size_t>(i) * n + k]) > std::fabs(lu[static_cast<std::size_t>(p) * n + k])) p = i;
            piv[k] = p;
            if (p != k)
                for (int j = 0; j < n; ++j) std::swap(lu[static_cast<std::size_t>(k) * n + j], lu[static_cast<std::size_t>(p) * n + j]);
            const double d = lu[static_cast<std::size_t>(k) * n + k];
            for (int i = k + 1; i < n; ++i) {
                const double f = (lu[static_cast<std::size_t>(i) * n + k] /= d);
                for (int j = k + 1; j < n; ++j) lu[static_cast<std::size_t>(i) * n + j] -= f * lu[static_cast<std::size_t>(k) * n + j];
            }
        }
    }
    void smooth(const Csr& a, const std::vector<double>& b, std::vector<double>& x, std::vector<double>& t) {
        for (int i = 0; i < a.n; ++i) {
            double ax = 0.0;
            for (int k = a.row[i]; k < a.row[i + 1]; ++k) ax += a.val[k] * x[a.col[k]];
            t[i] = x[i] + (2.0 / 3.0) * a.inv_diag[i] * (b[i] - ax);
        }
        x.swap(t);
    }
    void cycle(std::size_t l) {
        Level& L = levels[l];
        if (l + 1 == levels.size()) {
            const int n = L.a.n;
            std::vector<double> y(L.b);
            for (int k = 0; k < n; ++k) std::swap(y[k], y[piv[k]]);
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < i; ++j) y[i] -= lu[static_cast<std::size_t>(i) * n + j] * y[j];
            for (int i = n - 1; i >= 0; --i) {
                for (int j = i + 1; j < n; ++j) y[i] -= lu[static_cast<std::size_t>(i) * n + j] * y[j];
                y[i] /= lu[static_cast<std::size_t>(i) * n + i];
            }
            L.x = y;
            return;
        }
        std::fill(L.x.begin(), L.x.end(), 0.0);
        smooth(L.a, L.b, L.x, L.t);
        smooth(L.a, L.b, L.x, L.t);
        Level& C = levels[l + 1];
        std::fill(C.b.begin(), C.b.end(), 0.0);
        for (int i = 0; i < L.a.n; ++i) {
            double ax = 0.0;
            for (int k = L.a.row[i]; k < L.a.row[i + 1]; ++k) ax += L.a.val[k] * L.x[L.a.col[k]];
            C.b[L.agg[i]] += L.b[i] - ax;
        }
        cycle(l + 1);
        for (int i = 0; i < L.a.n; ++i) L.x[i] += C.x[L.agg[i]];
        smooth(L.a, L.b, L.x, L.t);
        smooth(L.a, L.b, L.x, L.t);
    }
    void apply(const std::vector<double>& r, std::vector<double>& z) override {
        levels[0].b = r;
        cycle(0);
        z = levels[0].x;
    }
};

// Preconditioned CG on the recursive residual; stops when the recursive norm
// reaches `inner` or the budget is spent.
int pcg(const Csr& a, const std::vector<double>& b, std::vector<double>& x, double inner, int budget,
        Preconditioner* pc) {
    const int n = a.n;
    std::vector<double> r(n), z(n), p(n), q(n);
    trueResidual(a, b, x, r);
    auto precondition = [&]() {
        if (pc) pc->apply(r, z);
        else z = r;
    };
    precondition();
    p = z;
    double rz = dotv(r, z);
    int it = 0;
    while (it < budget && std::sqrt(dotv(r, r)) > inner) {
        spmv(a, p, q);
        const double pq = dotv(p, q);
        if (!(std::fabs(pq) > 0.0) || !std::isfinite(pq)) break;
        const double alpha = rz / pq;
        for (int i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
        precondition();
        const double rz_new = dotv(r, z);
        const double beta = rz_new / rz;
        rz = rz_new;
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        ++it;
    }
    return it;
}

// Right-preconditioned BiCGStab.
int bicgstab(const Csr& a, const std::vector<double>& b, std::vector<double>& x, double inner, int budget,
             Preconditioner* pc) {
    const int n = a.n;
    std::vector<double> r(n), r0(n), p(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n);
    auto precondition = [&](const std::vector<double>& in, std::vector<double>& out) {
        if (pc) pc->apply(in, out);
        else out = in;
    };
    trueResidual(a, b, x, r);
    r0 = r;
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    int it = 0;
    while (it < budget && std::sqrt(dotv(r, r)) > inner) {
        const double rho_new = dotv(r0, r);
        if (!(std::fabs(rho_new) > 0.0) || !std::isfinite(rho_new)) break;
        const double beta = (rho_new / rho) * (alpha / omega);
        rho = rho_new;
        for (int i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        precondition(p, ph);
        spmv(a, ph, v);
        const double r0v = dotv(r0, v);
        if (!(std::fabs(r0v) > 0.0) || !std::isfinite(r0v)) break;
        alpha = rho / r0v;
        for (int i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        ++it;
        if (std::sqrt(dotv(s, s)) <= inner) {
            for (int i = 0; i < n; ++i) { x[i] += alpha * ph[i]; r[i] = s[i]; }
            break;
        }
        precondition(s, sh);
        spmv(a, sh, t);
        const double tt = dotv(t, t);
        omega = tt > 0.0 ? dotv(t, s) / tt : 0.0;
        for (int i = 0; i < n; ++i) {
            x[i] += alpha * ph[i] + omega * sh[i];
            r[i] = s[i] - omega * t[i];
        }
        if (omega == 0.0) break;
    }
    return it;
}

// Restarted right-preconditioned GMRES(m) (modified Gram-Schmidt, Givens
// rotations); `flexible` keeps the preconditioned directions (FGMRES), which is
// the same algorithm for a fixed preconditioner.
int gmres(const Csr& a, const std::vector<double>& b, std::vector<double>& x, double inner, int budget,
          Preconditioner* pc, bool flexible, int m = 30) {
    const int n = a.n;
    std::vector<double> r(n), w(n), zt(n);
    std::vector<std::vector<double>> V(m + 1, std::vector<double>(n)), Z(flexible ? m : 0, std::vector<double>(n));
    std::vector<double> H(static_cast<std::size_t>(m + 1) * m), cs(m), sn(m), g(m + 1);
    int it = 0;
    while (it < budget) {
        const double beta = trueResidual(a, b, x, r);
        if (!(beta > inner) || !std::isfinite(beta)) break;
        for (int i = 0; i < n; ++i) V[0][i] = r[i] / beta;
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        for (; j < m && it < budget; ++j) {
            std::vector<double>& z = flexible ? Z[j] : zt;
            if (pc) pc->apply(V[j], z);
            else z = V[j];
            spmv(a, z, w);
            for (int k = 0; k <= j; ++k) {
                const double h = dotv(w, V[k]);
                H[static_cast<std::size_t>(k) * m + j] = h;
                for (int i = 0; i < n; ++i) w[i] -= h * V[k][i];
            }
            const double hn = std::sqrt(dotv(w, w));
            H[static_cast<std::size_t>(j + 1) * m + j] = hn;
            if (hn > 0.0)
                for (int i = 0; i < n; ++i) V[j + 1][i] = w[i] / hn;
            for (int k = 0; k < j; ++k) {
                const double h0 = H[static_cast<std::size_t>(k) * m + j], h1 = H[static_cast<std::size_t>(k + 1) * m + j];
                H[static_cast<std::size_t>(k) * m + j] = cs[k] * h0 + sn[k] * h1;
                H[static_cast<std::size_t>(k + 1) * m + j] = -sn[k] * h0 + cs[k] * h1;
            }
            const double h0 = H[static_cast<std::size_t>(j) * m + j], h1 = H[static_cast<std::size_t>(j + 1) * m + j];
            const double d = std::hypot(h0, h1);
            cs[j] = d > 0.0 ? h0 / d : 1.0;
            sn[j] = d > 0.0 ? h1 / d : 0.0;
            H[static_cast<std::size_t>(j) * m + j] = d;
            H[static_cast<std::size_t>(j + 1) * m + j] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            ++it;
            if (std::fabs(g[j + 1]) <= inner || hn == 0.0) { ++j; break; }
        }
        std::vector<double> y(j);
        for (int k = j - 1; k >= 0; --k) {
            double s = g[k];
            for (int q = k + 1; q < j; ++q) s -= H[static_cast<std::size_t>(k) * m + q] * y[q];
            y[k] = s / H[static_cast<std::size_t>(k) * m + k];
        }
        if (flexible) {
            for (int k = 0; k < j; ++k)
                for (int i = 0; i < n; ++i) x[i] += y[k] * Z[k][i];
        } else {
            std::fill(w.begin(), w.end(), 0.0);
            for (int k = 0; k < j; ++k)
                for (int i = 0; i < n; ++i) w[i] += y[k] * V[k][i];
            if (pc) pc->apply(w, zt);
            else zt = w;
            for (int i = 0; i < n; ++i) x[i] += zt[i];
        }
        if (j > 0 && std::fabs(g[j]) <= inner) break;
    }
    return it;
}

// One equation's system with PetscLinearSystem's update / prepare / solveRhs
// lifecycle (petsc_linear_system.cpp:257-481).
class LinearSystem {
public:
    LinearSystem(const Pattern& pattern, std::size_t rhs) : m_pattern(pattern), m_fresh(rhs, 0) {}

    void updateMatrix(const std::vector<double>& diag, const std::vector<double>& upper,
                      const std::vector<double>& lower) {
        const bool same = m_ready && diag == m_diag && upper == m_upper && lower == m_lower;
        if (same) return;
        m_diag = diag;
        m_upper = upper;
        m_lower = lower;
        m_pattern.fill(m_a, diag, upper, lower);
        ++counters.updates;
        m_ready = true;
        m_setup_pending = true;
        ++m_matrix_updates;
    }

    void prepare(const LinearSolverConfig& config) {
        m_config = config;
        if (!m_setup_pending && !m_force_rebuild) return;
        const bool reuse = config.preconditioner != PreconditionerType::None && m_setups != 0 && !m_force_rebuild &&
                           m_matrix_updates - m_pc_matrix_update <
                               static_cast<unsigned long long>(config.preconditioner_rebuild_interval) &&
                           m_pc_rhs_solves < static_cast<unsigned long long>(config.preconditioner_rebuild_interval);
        setup(reuse);
    }

    SolveResult solveRhs(const std::vector<double>& b, std::vector<double>& x, std::size_t rhs = 0) {
        const LinearSolverConfig& config = m_config;
        std::vector<double> r(m_a.n);
        const std::vector<double> guess = x;
        const double bnorm = std::sqrt(dotv(b, b));
        const double r0 = config.warm_start ? trueResidual(m_a, b, x, r) : bnorm;
        auto reset = [&]() {
            if (config.warm_start) x = guess;
            else std::fill(x.begin(), x.end(), 0.0);
        };
        reset();
        const double scale = residualScale(r0, bnorm);
        const double target = residualTarget(config, scale);
        const bool reused = config.preconditioner != PreconditionerType::None && m_pc_matrix_update < m_matrix_updates;
        if (residualConverged(r0, target)) return SolveResult(SolveStatus::Converged, 0, r0, r0, r0 / scale);
        SolveResult result;
        int total = 0;
        const Clock::time_point t0 = Clock::now();
        if (reused) ++counters.reuses;
        for (int attempt = 0; attempt < 2; ++attempt) {
            int used = 0;
            double inner = target, final_residual = r0;
            for (int restart = 0; restart < 3 && used < config.max_iterations; ++restart) {
                const int budget = config.max_iterations - used;
                int its = 0;
                switch (config.solver) {
                case LinearSolverType::ConjugateGradient: its = pcg(m_a, b, x, inner, budget, m_pc.get()); break;
                case LinearSolverType::BiCGSTAB: its = bicgstab(m_a, b, x, inner, budget, m_pc.get()); break;
                case LinearSolverType::GMRES: its = gmres(m_a, b, x, inner, budget, m_pc.get(), false); break;
                case LinearSolverType::FGMRES: its = gmres(m_a, b, x, inner, budget, m_pc.get(), true); break;
                }
                used += its;
                total += its;
                final_residual = trueResidual(m_a, b, x, r);
                if (residualConverged(final_residual, target) || !std::isfinite(final_residual)) break;
                inner *= 0.5;
            }
            SolveStatus status = SolveStatus::NumericalFailure;
            if (residualConverged(final_residual, target)) status = SolveStatus::Converged;
            else if (std::isfinite(final_residual)) status = SolveStatus::MaxIterations;
            result = SolveResult(status, total, r0, final_residual, final_residual / scale);
            if (status != SolveStatus::Converged && attempt == 0 && reused) {
                ++counters.retries;
                setup(false);
                reset();
                continue;
            }
            if (status == SolveStatus::Converged) {
                int& fresh = m_fresh[rhs];
                if (m_pc_matrix_update == m_matrix_updates) fresh = std::max(fresh, used);
                else if (used > config.preconditioner_reuse_iteration_growth * static_cast<double>(std::max(fresh, 1)))
                    m_force_rebuild = true;
            }
            break;
        }
        if (total > 0) ++m_pc_rhs_solves;
        ++counters.solves;
        counters.iterations += static_cast<unsigned long long>(total);
        counters.solve_seconds += secondsSince(t0);
        return result;
    }

    const Csr& matrix() const { return m_a; }
    // Work and time of this system (the PerformanceCounters fields PetscBackend fills).
    struct Counters {
        unsigned long long solves = 0, iterations = 0, setups = 0, reuses = 0, retries = 0, updates = 0;
        double solve_seconds = 0.0, setup_seconds = 0.0;
    } counters;

private:
    void setup(bool reuse) {
        if (!reuse) {
            const Clock::time_point t0 = Clock::now();
            switch (m_config.preconditioner) {
            case PreconditionerType::None: m_pc.reset(); break;
            case PreconditionerType::Hypre:
            case PreconditionerType::GAMG: m_pc = std::make_unique<CpuAmg>(m_a); break;
            case PreconditionerType::Jacobi: m_pc = std::make_unique<JacobiPc>(m_a); break;
            default: m_pc = std::make_unique<Ilu0Pc>(m_a); break;
            }
            if (m_config.preconditioner != PreconditionerType::None) {
                ++m_setups;
                ++counters.setups;
            }
            counters.setup_seconds += secondsSince(t0);
            m_pc_matrix_update = m_matrix_updates;
            m_pc_rhs_solves = 0;
            std::fill(m_fresh.begin(), m_fresh.end(), 0);
        }
        m_setup_pending = false;
        m_force_rebuild = false;
    }

    const Pattern& m_pattern;
    Csr m_a;
    std::vector<double> m_diag, m_upper, m_lower;
    bool m_ready = false, m_setup_pending = false, m_force_rebuild = false;
    unsigned long long m_matrix_updates = 0, m_pc_matrix_update = 0, m_pc_rhs_solves = 0, m_setups = 0;
    std::vector<int> m_fresh;
    LinearSolverConfig m_config;
    std::unique_ptr<Preconditioner> m_pc;
};

class OracleBackend final : public ComputeBackend {
public:
    explicit OracleBackend(const Mesh& mesh) : m_mesh(&mesh), m_pattern(mesh) {
        if (const char* dir = std::getenv("BABELSIM_ORACLE_DUMP")) m_dump = dir;
    }
    void synchronize(ScalarField& f) override { markHaloValid(f); }
    void synchronize(VectorField& f) override { markHaloValid(f); }
    void synchronize(TensorField& f) override { markHaloValid(f); }
    void sum(const double* local, double* global, int count) const override {
        std::memmove(global, local, sizeof(double) * static_cast<std::size_t>(count));
    }
    void maximum(const double* local, double* global, int count) const override {
        std::memmove(global, local, sizeof(double) * static_cast<std::size_t>(count));
    }
    bool all(bool local_condition) const override { return local_condition; }

    PerformanceCounters performance() const override {
        PerformanceCounters p;
        for (const auto& entry : m_systems) {
            const auto& c = entry.second->counters;
            p.linear_solves += c.solves;
            p.krylov_iterations += c.iterations;
            p.preconditioner_setups += c.setups;
            p.preconditioner_reuses += c.reuses;
            p.preconditioner_retries += c.retries;
            p.matrix_value_updates += c.updates;
            p.linear_solve_seconds += c.solve_seconds;
            p.preconditioner_seconds += c.setup_seconds;
        }
        return p;
    }

    SolveResult solve(const ScalarDiscreteEquation& eq, ScalarField& x, const LinearSolverConfig& config) override {
        config.validate();
        LinearSystem& system = getSystem(identity(eq.numerical_identity, x.name(), false), 1);
        system.updateMatrix(eq.diagonal, eq.upper, eq.lower);
        system.prepare(config);
        std::vector<double> before(fieldValues(x));
        std::vector<double> sol(fieldValues(x));
        const SolveResult result = system.solveRhs(eq.source, sol);
        double* target = fieldData(x);
        for (std::size_t i = 0; i < sol.size(); ++i) target[i] = sol[i];
        markHaloValid(x);
        dump(eq.numerical_identity, x.name(), 1, eq, eq.source, before, sol, result);
        return result;
    }

    std::array<SolveResult, 3> solve(const VectorDiscreteEquation& eq, VectorField& x,
                                     const LinearSolverConfig& config) override {
        config.validate();
        LinearSystem& system = getSystem(identity(eq.numerical_identity, x.name(), true), 3);
        system.updateMatrix(eq.diagonal, eq.upper, eq.lower);
        system.prepare(config);
        const int n = static_cast<int>(eq.diagonal.size());
        std::vector<double> source(3 * n), before(3 * n), after(3 * n);
        Vec3* values = fieldData(x);
        for (int i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c) {
                source[3 * i + c] = eq.source[i][c];
                before[3 * i + c] = values[i][c];
            }
        std::array<SolveResult, 3> results;
        for (int c = 0; c < 3; ++c) {
            std::vector<double> b(n), sol(n);
            for (int i = 0; i < n; ++i) { b[i] = eq.source[i][c]; sol[i] = values[i][c]; }
            results[c] = system.solveRhs(b, sol, static_cast<std::size_t>(c));
            for (int i = 0; i < n; ++i) { values[i][c] = sol[i]; after[3 * i + c] = sol[i]; }
        }
        markHaloValid(x);
        dump(eq.numerical_identity, x.name(), 3, eq, source, before, after, results[0]);
        return results;
    }

private:
    // petsc_backend.cpp:201-205
    static std::string identity(const std::string& equation, const std::string& field, bool vector) {
        return std::string(vector ? "vector:" : "scalar:") + (equation.empty() ? field : equation) + ":" + field;
    }
    LinearSystem& getSystem(const std::string& key, std::size_t rhs) {
        auto found = m_systems.find(key);
        if (found == m_systems.end())
            found = m_systems.emplace(key, std::make_unique<LinearSystem>(m_pattern, rhs)).first;
        return *found->second;
    }

    template <class Eq>
    void dump(const std::string& identity, const std::string& field, int comps, const Eq& eq,
              const std::vector<double>& source, const std::vector<double>& before,
              const std::vector<double>& after, const SolveResult& result) {
        if (m_dump.empty()) return;
        char name[64];
        std::snprintf(name, sizeof(name), "/system_%05d.bin", m_sequence++);
        std::FILE* out = std::fopen((m_dump + name).c_str(), "wb");
        if (!out) throw std::runtime_error("cannot write oracle dump " + m_dump + name);
        // Header: 8 int64 {cells, faces, components, identity length, field length,
        // status, iterations, 0}, then identity and field names, then float64
        // {initial, final, relative} and the arrays diag, upper, lower, source,
        // unknown before, unknown after (components interleaved per cell).
        const long long header[8] = {static_cast<long long>(eq.diagonal.size()),
                                     static_cast<long long>(eq.upper.size()), comps,
                                     static_cast<long long>(identity.size()),
                                     static_cast<long long>(field.size()),
                                     static_cast<long long>(result.status), result.iterations, 0};
        std::fwrite(header, sizeof(header), 1, out);
        std::fwrite(identity.data(), 1, identity.size(), out);
        std::fwrite(field.data(), 1, field.size(), out);
        const double residuals[3] = {result.initial_residual, result.final_residual, result.relative_residual};
        std::fwrite(residuals, sizeof(residuals), 1, out);
        std::fwrite(eq.diagonal.data(), sizeof(double), eq.diagonal.size(), out);
        std::fwrite(eq.upper.data(), sizeof(double), eq.upper.size(), out);
        std::fwrite(eq.lower.data(), sizeof(double), eq.lower.size(), out);
        std::fwrite(source.data(), sizeof(double), source.size(), out);
        std::fwrite(before.data(), sizeof(double), before.size(), out);
        std::fwrite(after.data(), sizeof(double), after.size(), out);
        std::fclose(out);
    }

    const Mesh* m_mesh;
    Pattern m_pattern;
    std::map<std::string, std::unique_ptr<LinearSystem>> m_systems;
    std::string m_dump;
    int m_sequence = 0;
};

}  // namespace

std::unique_ptr<ComputeBackend> makeComputeBackend(const Mesh& mesh, ParallelContext) {
    return std::make_unique<OracleBackend>(mesh);
}

}  // namespace babelsim::detail
