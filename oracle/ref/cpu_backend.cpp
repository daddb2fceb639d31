// CPU linear-system backend used to run the reference's own finite-volume
// sources as the oracle.  Test infrastructure only, never the product.
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
// With BABELSIM_ORACLE_DUMP=<dir> every assembled LDU system handed to solve()
// is written to <dir>/system_<seq>.bin together with the unknown before and
// after the solve, so the GPU assembly can be compared coefficient by
// coefficient against the reference's own discretisation.
#include "babelsim/field.h"
#include "babelsim/parallel.h"
#include "internal/compute_backend.h"
#include "internal/field_access.h"
#include "internal/mesh_access.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace babelsim::detail {

void ensurePetscSession() {}
void finalizePetscSession() {}

namespace {

struct Csr {
    int n = 0;
    std::vector<int> row, col;
    std::vector<double> val, inv_diag;
};

// LDU -> CSR with rows in cell order.  upper[f] sits at (owner, neighbour),
// lower[f] at (neighbour, owner), as in petsc_assembly_plan.cpp:62-87.
Csr toCsr(const Mesh& mesh, const std::vector<double>& diag, const std::vector<double>& upper,
          const std::vector<double>& lower) {
    Csr a;
    a.n = mesh.cellCount();
    std::vector<int> count(a.n, 1);
    for (Index f = 0; f < mesh.faceCount(); ++f) {
        const Index n = mesh.neighbour(f);
        if (n == invalid_index) continue;
        ++count[mesh.owner(f)];
        ++count[n];
    }
    a.row.assign(a.n + 1, 0);
    for (int i = 0; i < a.n; ++i) a.row[i + 1] = a.row[i] + count[i];
    a.col.resize(a.row[a.n]);
    a.val.resize(a.row[a.n]);
    std::vector<int> fill(a.row.begin(), a.row.end() - 1);
    for (int i = 0; i < a.n; ++i) {
        a.col[fill[i]] = i;
        a.val[fill[i]++] = diag[i];
    }
    for (Index f = 0; f < mesh.faceCount(); ++f) {
        const Index o = mesh.owner(f), n = mesh.neighbour(f);
        if (n == invalid_index) continue;
        a.col[fill[o]] = n;
        a.val[fill[o]++] = upper[f];
        a.col[fill[n]] = o;
        a.val[fill[n]++] = lower[f];
    }
    a.inv_diag.resize(a.n);
    for (int i = 0; i < a.n; ++i) a.inv_diag[i] = diag[i] != 0.0 ? 1.0 / diag[i] : 1.0;
    return a;
}

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

// CPU aggregation AMG (stand-in for Hypre BoomerAMG behind pcType hypre|gamg):
// pairwise matching of strongest negative couplings applied twice per level,
// Galerkin coarse operators of piecewise-constant prolongation, V(2,2) cycle
// with damped Jacobi (omega 2/3) and a dense LU solve on the coarsest level.
struct CpuAmg {
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
    static Csr galerkin(const Csr& a, const std::vector<int>& agg, int nc) {
        std::vector<std::vector<std::pair<int, double>>> rows(nc);
        for (int i = 0; i < a.n; ++i)
            for (int k = a.row[i]; k < a.row[i + 1]; ++k) rows[agg[i]].push_back({agg[a.col[k]], a.val[k]});
        Csr c;
        c.n = nc;
        c.row.assign(nc + 1, 0);
        for (int I = 0; I < nc; ++I) {
            auto& r = rows[I];
            std::sort(r.begin(), r.end(), [](const auto& u, const auto& v) { return u.first < v.first; });
            int diag_pos = -1;
            for (std::size_t k = 0; k < r.size(); ++k) {
                if (!c.col.empty() && static_cast<int>(c.col.size()) > c.row[I] && c.col.back() == r[k].first) {
                    c.val.back() += r[k].second;
                } else {
                    c.col.push_back(r[k].first);
                    c.val.push_back(r[k].second);
                }
                if (r[k].first == I) diag_pos = static_cast<int>(c.col.size()) - 1;
            }
            (void)diag_pos;
            c.row[I + 1] = static_cast<int>(c.col.size());
        }
        c.inv_diag.assign(nc, 1.0);
        for (int I = 0; I < nc; ++I)
            for (int k = c.row[I]; k < c.row[I + 1]; ++k)
                if (c.col[k] == I && c.val[k] != 0.0) c.inv_diag[I] = 1.0 / c.val[k];
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
    void apply(const std::vector<double>& r, std::vector<double>& z) {
        levels[0].b = r;
        cycle(0);
        z = levels[0].x;
    }
};

// Preconditioned CG on the recursive residual (Jacobi, or the CPU AMG when
// given); stops when the recursive norm reaches `inner` or the budget is spent.
int pcg(const Csr& a, const std::vector<double>& b, std::vector<double>& x, double inner, int budget,
        CpuAmg* amg = nullptr) {
    const int n = a.n;
    std::vector<double> r(n), z(n), p(n), q(n);
    trueResidual(a, b, x, r);
    auto precondition = [&]() {
        if (amg) amg->apply(r, z);
        else for (int i = 0; i < n; ++i) z[i] = a.inv_diag[i] * r[i];
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

// Right-Jacobi-preconditioned BiCGStab.
int bicgstab(const Csr& a, const std::vector<double>& b, std::vector<double>& x, double inner, int budget) {
    const int n = a.n;
    std::vector<double> r(n), r0(n), p(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n);
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
        for (int i = 0; i < n; ++i) ph[i] = a.inv_diag[i] * p[i];
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
        for (int i = 0; i < n; ++i) sh[i] = a.inv_diag[i] * s[i];
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

// The reference's acceptance loop around one Krylov solve.
SolveResult acceptanceSolve(const Csr& a, const LinearSolverConfig& config, const std::vector<double>& b,
                            std::vector<double>& x) {
    std::vector<double> r(a.n);
    const double bnorm = std::sqrt(dotv(b, b));
    const double r0 = config.warm_start ? trueResidual(a, b, x, r) : bnorm;
    if (!config.warm_start) std::fill(x.begin(), x.end(), 0.0);
    const double scale = residualScale(r0, bnorm);
    const double target = residualTarget(config, scale);
    if (residualConverged(r0, target)) return SolveResult(SolveStatus::Converged, 0, r0, r0, r0 / scale);
    double inner = target;
    int used = 0;
    double final_residual = r0;
    std::unique_ptr<CpuAmg> amg;
    if (config.solver == LinearSolverType::ConjugateGradient &&
        (config.preconditioner == PreconditionerType::Hypre || config.preconditioner == PreconditionerType::GAMG))
        amg = std::make_unique<CpuAmg>(a);
    for (int restart = 0; restart < 3 && used < config.max_iterations; ++restart) {
        const int budget = config.max_iterations - used;
        used += config.solver == LinearSolverType::ConjugateGradient ? pcg(a, b, x, inner, budget, amg.get())
                                                                      : bicgstab(a, b, x, inner, budget);
        final_residual = trueResidual(a, b, x, r);
        if (residualConverged(final_residual, target) || !std::isfinite(final_residual)) break;
        inner *= 0.5;
    }
    SolveStatus status = SolveStatus::NumericalFailure;
    if (residualConverged(final_residual, target)) status = SolveStatus::Converged;
    else if (std::isfinite(final_residual)) status = SolveStatus::MaxIterations;
    return SolveResult(status, used, r0, final_residual, final_residual / scale);
}

class OracleBackend final : public ComputeBackend {
public:
    explicit OracleBackend(const Mesh& mesh) : m_mesh(&mesh) {
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

    SolveResult solve(const ScalarDiscreteEquation& eq, ScalarField& x, const LinearSolverConfig& config) override {
        config.validate();
        const Csr a = toCsr(*m_mesh, eq.diagonal, eq.upper, eq.lower);
        std::vector<double> before(fieldValues(x));
        std::vector<double> sol(fieldValues(x));
        const SolveResult result = acceptanceSolve(a, config, eq.source, sol);
        double* target = fieldData(x);
        for (int i = 0; i < a.n; ++i) target[i] = sol[i];
        markHaloValid(x);
        dump(eq.numerical_identity, x.name(), 1, eq, eq.source, before, sol, result);
        return result;
    }

    std::array<SolveResult, 3> solve(const VectorDiscreteEquation& eq, VectorField& x,
                                     const LinearSolverConfig& config) override {
        config.validate();
        const Csr a = toCsr(*m_mesh, eq.diagonal, eq.upper, eq.lower);
        const int n = a.n;
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
            results[c] = acceptanceSolve(a, config, b, sol);
            for (int i = 0; i < n; ++i) { values[i][c] = sol[i]; after[3 * i + c] = sol[i]; }
        }
        markHaloValid(x);
        dump(eq.numerical_identity, x.name(), 3, eq, source, before, after, results[0]);
        return results;
    }

private:
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
    std::string m_dump;
    int m_sequence = 0;
};

}  // namespace

std::unique_ptr<ComputeBackend> makeComputeBackend(const Mesh& mesh, ParallelContext) {
    return std::make_unique<OracleBackend>(mesh);
}

}  // namespace babelsim::detail
