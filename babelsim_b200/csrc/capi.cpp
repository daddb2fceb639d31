// extern "C" boundary: converts exceptions to status codes, host arrays in the
// caller's numbering to the device layout, and owns the opaque handles.
#include "../../include/babelsim_b200.h"
#include "amg.h"
#include "fvm.h"
#include "linalg.h"
#include "mesh_io.h"
#include "piso.h"
#include "renumber.h"
#include "results.h"
#include "simple.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>

struct bsg_context {
    std::unique_ptr<bsg::Context> ctx;
};
// One equation's persistent linear system (PetscLinearSystem's role): device
// buffers and the AMG structure live across solves, the matrix last uploaded is
// kept on the host for the exact-equality skip of petsc_linear_system.cpp:257-282.
struct bsg_system {
    bsg_mesh* mesh = nullptr;
    int comps = 1;
    std::unique_ptr<bsg::DeviceField> unknown;
    std::unique_ptr<bsg::DeviceEquation> eq;
    std::unique_ptr<bsg::KrylovSolver> krylov;
    std::unique_ptr<bsg::AmgPreconditioner> amg;
    bsg::JacobiPreconditioner jacobi;
    bsg::PcReusePolicy policy;
    std::vector<double> diag, upper, lower;  // matrix values of the last update (caller's face order)
    std::vector<double> slots;               // off-diagonal values in device slot order
    bool ready = false;
    bsg_system_counters counters{};
};
struct bsg_mesh {
    bsg_context* owner;
    std::unique_ptr<bsg::DeviceMesh> mesh;
    // systems of bsg_solve_ldu (1 and 3 components); destroyed before the mesh
    std::unique_ptr<bsg_system> ldu_system[2];
};
struct bsg_field {
    bsg_mesh* mesh;
    std::unique_ptr<bsg::DeviceField> field;
};
struct bsg_equation {
    bsg_field* unknown;
    std::unique_ptr<bsg::DeviceEquation> eq;
    std::unique_ptr<bsg::KrylovSolver> krylov;
    std::unique_ptr<bsg::AmgPreconditioner> amg;
    bsg::Reducer red;
    bsg::DeviceArray<int> flags;
};
struct bsg_simple {
    bsg_mesh* mesh;
    std::unique_ptr<bsg::SimpleSolver> solver;
};
struct bsg_piso {
    bsg_mesh* mesh;
    std::unique_ptr<bsg::PisoSolver> solver;
};

namespace bsg {

Context::Context(int dev) : device(dev) {
    int count = 0;
    checkCuda(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    if (dev < 0 || dev >= count) fail(kArgument, "CUDA device index out of range");
    checkCuda(cudaSetDevice(dev), "cudaSetDevice");
    cudaDeviceProp prop{};
    checkCuda(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
    if (prop.major < 10) fail(kState, "babelsim_b200 kernels are built for sm_100a (Blackwell); device is sm_" +
                                         std::to_string(prop.major) + std::to_string(prop.minor));
    sm_count = prop.multiProcessorCount;
    checkCuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    checkCuda(cudaMallocHost(reinterpret_cast<void**>(&pinned), 64 * sizeof(double)), "cudaMallocHost");
    checkCuda(cudaMalloc(reinterpret_cast<void**>(&grid_barrier), sizeof(SegmentBarrier)), "cudaMalloc");
    checkCuda(cudaMalloc(reinterpret_cast<void**>(&progress), sizeof(unsigned) * kMaxPersistentCtas), "cudaMalloc");
}

Context::~Context() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& r : records) { event_pool.push_back(r.start); event_pool.push_back(r.stop); }
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : user_events) if (e) cudaEventDestroy(e);
    if (phase_entries) cudaFree(phase_entries);
    if (phase_count) cudaFree(phase_count);
    if (pinned) cudaFreeHost(pinned);
    if (grid_barrier) cudaFree(grid_barrier);
    if (progress) cudaFree(progress);
    if (stream) cudaStreamDestroy(stream);
}

void resetBarriers(Context& ctx, SegmentBarrier* dev, int n, int ctas, const int* cta_begin) {
    if (ctas > kMaxPersistentCtas) fail(kArgument, "persistent launch larger than its progress record");
    std::vector<SegmentBarrier> h(static_cast<std::size_t>(n));
    for (int k = 0; k < n; ++k) {
        const int c0 = cta_begin ? cta_begin[k] : 0, c1 = cta_begin ? cta_begin[k + 1] : ctas;
        h[k] = SegmentBarrier{0u, 0, 0, 0u, 0u, c0, c1 - c0, 0, ctx.progress};
    }
    // pageable source: the call returns once the bytes are staged, so `h` may go
    BSG_CUDA(cudaMemcpyAsync(dev, h.data(), sizeof(SegmentBarrier) * h.size(), cudaMemcpyHostToDevice, ctx.stream));
    BSG_CUDA(cudaMemsetAsync(ctx.progress, 0, sizeof(unsigned) * ctas, ctx.stream));
}

std::string barrierReport(const SegmentBarrier* dev) {
    SegmentBarrier b{};
    if (cudaMemcpy(&b, dev, sizeof(b), cudaMemcpyDeviceToHost) != cudaSuccess) return "";
    std::string out = " (group of CTAs " + std::to_string(b.cta0) + ".." + std::to_string(b.cta0 + b.ncta - 1);
    if (b.who > 0)
        out += "; CTA " + std::to_string(b.who - 1) + " gave up at its barrier " + std::to_string(b.where) + " with " +
               std::to_string(b.seen & 0x7fffffffu) + " arrivals counted";
    if (b.progress && b.ncta > 0) {
        std::vector<unsigned> prog(static_cast<std::size_t>(b.ncta));
        if (cudaMemcpy(prog.data(), b.progress + b.cta0, sizeof(unsigned) * prog.size(), cudaMemcpyDeviceToHost) ==
            cudaSuccess) {
            const unsigned lo = *std::min_element(prog.begin(), prog.end());
            const unsigned hi = *std::max_element(prog.begin(), prog.end());
            int behind = 0, first = -1;
            for (int k = 0; k < b.ncta; ++k)
                if (prog[k] == lo) {
                    ++behind;
                    if (first < 0) first = b.cta0 + k;
                }
            out += "; barriers reached " + std::to_string(lo) + ".." + std::to_string(hi) + ", " +
                   std::to_string(behind) + " CTA(s) at " + std::to_string(lo) + " from CTA " + std::to_string(first);
        }
    }
    return out + ")";
}

std::string barrierReport(const SegmentBarrier* dev, int n) {
    std::vector<SegmentBarrier> h(static_cast<std::size_t>(std::max(n, 0)));
    if (n <= 0 || cudaMemcpy(h.data(), dev, sizeof(SegmentBarrier) * h.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return "";
    for (int k = 0; k < n; ++k)
        if (h[k].abort || h[k].who) return " in system " + std::to_string(k) + " of the launch" + barrierReport(dev + k);
    return "";
}

cudaEvent_t Context::takeEvent() {
    if (event_pool.empty()) {
        cudaEvent_t e;
        checkCuda(cudaEventCreate(&e), "cudaEventCreate");
        return e;
    }
    cudaEvent_t e = event_pool.back();
    event_pool.pop_back();
    return e;
}

std::string Context::profileReport() {
    sync();
    struct Acc { std::string name; long long launches = 0; double ms = 0.0, bytes = 0.0, units = 0.0; };
    std::vector<Acc> acc;
    auto slot = [&](const char* name) -> Acc& {
        auto it = std::find_if(acc.begin(), acc.end(), [&](const Acc& a) { return a.name == name; });
        if (it != acc.end()) return *it;
        acc.push_back(Acc{name});
        return acc.back();
    };
    for (auto& r : records) {
        float ms = 0.0f;
        checkCuda(cudaEventElapsedTime(&ms, r.start, r.stop), "cudaEventElapsedTime");
        Acc& a = slot(r.name);
        a.launches += 1;
        a.ms += ms;
        event_pool.push_back(r.start);
        event_pool.push_back(r.stop);
    }
    records.clear();
    for (const Note& n : notes) {
        Acc& a = slot(n.name);
        a.bytes += n.bytes;
        a.units += n.units;
    }
    notes.clear();
    std::string out = "{";
    for (std::size_t i = 0; i < acc.size(); ++i) {
        char buf[320];
        std::snprintf(buf, sizeof(buf), "%s\"%s\": [%lld, %.6f, %.17g, %.17g]", i ? ", " : "", acc[i].name.c_str(),
                      acc[i].launches, acc[i].ms, acc[i].bytes, acc[i].units);
        out += buf;
    }
    return out + "}";
}

}  // namespace bsg

namespace {

thread_local std::string g_error;

template <class F>
int guard(bsg_context* ctx, F&& body) {
    try {
        body();
        return bsg::kOk;
    } catch (const bsg::Error& e) {
        (ctx ? ctx->ctx->last_error : g_error) = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        (ctx ? ctx->ctx->last_error : g_error) = "host allocation failed";
        return bsg::kMemory;
    } catch (const std::exception& e) {
        (ctx ? ctx->ctx->last_error : g_error) = e.what();
        return bsg::kState;
    }
}

bsg_context* ctxOf(const bsg_mesh* m) { return m ? m->owner : nullptr; }
bsg_context* ctxOf(const bsg_field* f) { return f ? f->mesh->owner : nullptr; }

void require(bool ok, const char* message) {
    if (!ok) bsg::fail(bsg::kArgument, message);
}

bsg::Options options(const bsg_options* o) {
    bsg::Options r;
    if (!o) return r;
    r.interpolation = o->interpolation;
    r.gradient = o->gradient;
    r.convection = o->convection;
    r.diffusion = o->diffusion;
    r.coefficient_interpolation = o->coefficient_interpolation;
    r.coefficient_gradient = o->coefficient_gradient;
    require(r.interpolation == 0 || r.interpolation == 1, "unsupported interpolation method");
    require(r.gradient == 0 || r.gradient == 1, "unsupported gradient method");
    require(r.convection >= 0 && r.convection <= 2, "unsupported convection method");
    require(r.diffusion >= 0 && r.diffusion <= 2, "unsupported diffusion method");
    return r;
}

bsg::SolverConfig solverConfig(const bsg_solver_config* c) {
    bsg::SolverConfig r;
    if (!c) return r;
    r.solver = c->solver;
    r.preconditioner = c->preconditioner;
    r.atol = c->absolute_tolerance;
    r.rtol = c->relative_tolerance;
    r.max_iterations = c->max_iterations;
    r.warm_start = c->warm_start != 0;
    r.rebuild_interval = c->preconditioner_rebuild_interval;
    r.reuse_growth = c->preconditioner_reuse_iteration_growth;
    r.amg_max_levels = c->amg_max_levels;
    r.amg_coarse_size = c->amg_coarse_size;
    r.amg_smoothing_steps = c->amg_smoothing_steps;
    r.precision = c->precision;
    // LinearSolverConfig::validate (src/backend/solver_control.cpp:8-30)
    require(r.atol > 0 && std::isfinite(r.atol) && r.rtol > 0 && std::isfinite(r.rtol) && r.max_iterations > 0,
            "linear solver tolerances or iteration limit are invalid");
    require(r.solver >= 0 && r.solver <= 3, "unknown linear solver type");
    require(r.preconditioner >= 0 && r.preconditioner <= 6, "unknown preconditioner type");
    require(r.precision >= 0 && r.precision <= 2, "unknown precision mode");
    return r;
}

void toResult(const bsg::SolveOutcome& o, bsg_solve_result* r) {
    r->status = o.status;
    r->iterations = o.iterations;
    r->initial_residual = o.initial;
    r->final_residual = o.final_;
    r->relative_residual = o.relative;
}

// Solve an equation's device LDU system: 3 components through the lockstep
// BiCGStab, scalars through CG/BiCGStab with Jacobi or AMG.
void solveEquation(bsg_equation* e, const bsg::SolverConfig& cfg, bsg_solve_result* results) {
    bsg::DeviceEquation& eq = *e->eq;
    bsg::DeviceMesh& m = *eq.x->mesh;
    bsg::Context& ctx = *m.ctx;
    if (!e->krylov) e->krylov = std::make_unique<bsg::KrylovSolver>(ctx);
    bsg::Dcsr<double> A{m.n_cells, m.cf_ptr.data(), m.cf_col.data(), eq.diag.data(), eq.val.data(),
                        2LL * m.n_interior};
    if (eq.x->comps == 3) {
        bsg::SolveOutcome o[3];
        e->krylov->solveVector3(A, cfg, eq.src.data(), eq.x->v.data(), o);
        for (int c = 0; c < 3; ++c) toResult(o[c], results + c);
        return;
    }
    std::unique_ptr<bsg::Preconditioner> jac;
    bsg::Preconditioner* pc = nullptr;
    if (cfg.solver != 1 && (cfg.preconditioner == 2 || cfg.preconditioner == 3)) {
        if (!e->amg) e->amg = std::make_unique<bsg::AmgPreconditioner>(m, cfg);
        e->amg->update(A, true);
        pc = e->amg.get();
    } else if (cfg.preconditioner != 0) {
        auto j = std::make_unique<bsg::JacobiPreconditioner>();
        j->diag = eq.diag.data();
        j->n = m.n_cells;
        pc = j.get();
        jac = std::move(j);
    }
    const bsg::SolveOutcome o = e->krylov->solveScalar(A, cfg, pc, eq.src.data(), eq.x->v.data());
    toResult(o, results);
}

// The locality renumbering of a polyhedral description's cells (renumber.cpp): owner and
// neighbour in the internal numbering when it applies.
struct CellOrder {
    bool applied = false;
    std::vector<int> order, owner, neighbour;  // order[internal] = caller cell
};

CellOrder cellOrder(int n_vertices, int n_faces, const int* offsets, const int* ids, const int* owner,
                    const int* neighbour, const int* patch, int n_patches) {
    CellOrder r;
    const int N = bsg::validatePolyhedralTopology(n_vertices, n_faces, offsets, ids, owner, neighbour, patch, n_patches);
    r.order = bsg::localityOrder(N, n_faces, owner, neighbour, &r.applied);
    if (!r.applied) return r;
    std::vector<int> pos(N);
    for (int i = 0; i < N; ++i) pos[r.order[i]] = i;
    r.owner.resize(n_faces);
    r.neighbour.resize(n_faces);
    for (int f = 0; f < n_faces; ++f) {
        r.owner[f] = pos[owner[f]];
        r.neighbour[f] = neighbour[f] < 0 ? -1 : pos[neighbour[f]];
    }
    return r;
}

// A mesh built on renumbered cells: the caller-to-internal map for cell arrays crossing the
// ABI, and the exported topology and cell geometry back in the caller's numbering.
void applyCellOrder(bsg::DeviceMesh& m, const CellOrder& r) {
    if (!r.applied) return;
    const int N = m.n_cells;
    m.h_cell_perm.assign(N, 0);
    for (int i = 0; i < N; ++i) m.h_cell_perm[r.order[i]] = i;
    m.cell_perm.upload(m.h_cell_perm, m.ctx->stream);
    for (int& o : m.ext_owner) o = r.order[o];
    for (int& n : m.ext_nbr)
        if (n >= 0) n = r.order[n];
    if (!m.ext_V.empty()) {
        std::vector<double> V(N), xc(3LL * N);
        for (int i = 0; i < N; ++i) {
            V[r.order[i]] = m.ext_V[i];
            for (int c = 0; c < 3; ++c) xc[3LL * r.order[i] + c] = m.ext_xc[3LL * i + c];
        }
        m.ext_V = std::move(V);
        m.ext_xc = std::move(xc);
    }
    m.ctx->sync();
}

std::unique_ptr<bsg_system> makeSystem(bsg_mesh* mesh, int components) {
    require(components == 1 || components == 3, "components must be 1 or 3");
    bsg::DeviceMesh& m = *mesh->mesh;
    auto s = std::make_unique<bsg_system>();
    s->mesh = mesh;
    s->comps = components;
    s->unknown = std::make_unique<bsg::DeviceField>(m, 0, components);
    s->eq = std::make_unique<bsg::DeviceEquation>(*s->unknown, bsg::Options{});
    s->krylov = std::make_unique<bsg::KrylovSolver>(*m.ctx);
    s->slots.assign(2 * static_cast<std::size_t>(m.n_interior), 0.0);
    return s;
}

bool sameValues(const std::vector<double>& kept, const double* v, std::size_t n) {
    if (kept.size() != n) return false;
    for (std::size_t i = 0; i < n; ++i)
        if (kept[i] != v[i]) return false;  // exact equality; NaN always counts as changed
    return true;
}

double secondsSince(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}

// updateMatrix + prepare + solveRhs of PetscLinearSystem (petsc_linear_system.cpp:257-481)
// for one call of the seam, every right-hand side of the system at once.
void systemSolve(bsg_system* s, const bsg::SolverConfig& cfg, const double* diagonal, const double* upper,
                 const double* lower, const double* source, double* x, bsg_solve_result* results) {
    bsg::DeviceMesh& m = *s->mesh->mesh;
    bsg::Context& ctx = *m.ctx;
    const int N = m.n_cells, C = s->comps;
    const std::size_t F = m.n_faces;
    bsg_system_counters& k = s->counters;
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < N; ++i)
        if (!std::isfinite(diagonal[i])) bsg::fail(bsg::kNumeric, "nonfinite matrix diagonal");
    const bool changed = !s->ready || !sameValues(s->diag, diagonal, N) || !sameValues(s->upper, upper, F) ||
                         !sameValues(s->lower, lower, F);
    if (changed) {
        s->diag.assign(diagonal, diagonal + N);
        s->upper.assign(upper, upper + F);
        s->lower.assign(lower, lower + F);
        for (int i = 0; i < m.n_interior; ++i) {
            const int f = m.interior_ext[i];
            s->slots[m.h_slot_own[i]] = upper[f];
            s->slots[m.h_slot_nbr[i]] = lower[f];
        }
        s->eq->diag.resize(N);
        bsg::uploadCells(m, s->eq->diag.data(), diagonal, 1);
        s->eq->val.upload(s->slots, ctx.stream);
        s->ready = true;
        ++k.matrix_value_updates;
    } else {
        ++k.rhs_only_solves;
    }
    s->eq->src.resize(static_cast<std::size_t>(N) * C);
    bsg::uploadCells(m, s->eq->src.data(), source, C);
    s->unknown->v.resize(static_cast<std::size_t>(N) * C);
    bsg::uploadCells(m, s->unknown->v.data(), x, C);
    k.matrix_update_seconds += secondsSince(t0);
    const auto t1 = std::chrono::steady_clock::now();
    bsg::Dcsr<double> A{N, m.cf_ptr.data(), m.cf_col.data(), s->eq->diag.data(), s->eq->val.data(),
                        2LL * m.n_interior};
    const bool use_amg = C == 1 && cfg.solver != 1 && (cfg.preconditioner == 2 || cfg.preconditioner == 3);
    bool lagged = false;
    if (use_amg) {
        if (!s->amg) s->amg = std::make_unique<bsg::AmgPreconditioner>(m, cfg);
        const bool rebuild = s->policy.needRebuild(changed, cfg);
        if (rebuild || changed) s->amg->update(A, rebuild);
        if (rebuild) ++k.preconditioner_setups;
        lagged = s->policy.lagged();
        if (lagged) ++k.preconditioner_reuses;
        ctx.sync();
    } else if (cfg.preconditioner != 0 && changed) {
        ++k.preconditioner_setups;  // Jacobi-type: formed from the current diagonal
    }
    k.preconditioner_seconds += secondsSince(t1);
    const auto t2 = std::chrono::steady_clock::now();
    bsg::SolveOutcome o[3];
    double* dx = s->unknown->v.data();
    if (C == 3) {
        s->krylov->solveVector3(A, cfg, s->eq->src.data(), dx, o);
    } else {
        bsg::Preconditioner* pc = nullptr;
        if (use_amg) pc = s->amg.get();
        else if (cfg.preconditioner != 0) {
            s->jacobi.diag = s->eq->diag.data();
            s->jacobi.n = N;
            pc = &s->jacobi;
        }
        o[0] = s->krylov->solveScalar(A, cfg, pc, s->eq->src.data(), dx);
        int attempt = o[0].iterations;
        if (use_amg && lagged && o[0].status != 0) {
            // a failed lagged solve is retried once from the same guess with a fresh hierarchy
            const auto tr = std::chrono::steady_clock::now();
            s->amg->update(A, true);
            s->policy.rebuilt();
            ++k.preconditioner_retries;
            ++k.preconditioner_setups;
            bsg::uploadCells(m, s->unknown->v.data(), x, 1);
            k.preconditioner_seconds += secondsSince(tr);
            const bsg::SolveOutcome first = o[0];
            o[0] = s->krylov->solveScalar(A, cfg, pc, s->eq->src.data(), dx);
            attempt = o[0].iterations;
            o[0].iterations += first.iterations;
            o[0].checks += first.checks;
        }
        if (use_amg) s->policy.afterSolve(o[0].status, attempt, o[0].iterations, cfg);
    }
    bsg::downloadCells(m, s->unknown->v.data(), x, C);
    k.solve_seconds += secondsSince(t2);
    for (int c = 0; c < C; ++c) {
        toResult(o[c], results + c);
        ++k.linear_solves;
        k.krylov_iterations += static_cast<uint64_t>(std::max(o[c].iterations, 0));
        k.true_residual_checks += static_cast<uint64_t>(std::max(o[c].checks, 0));
        k.last_status = o[c].status;
        k.last_initial_residual = o[c].initial;
        k.last_final_residual = o[c].final_;
        k.last_relative_residual = o[c].relative;
    }
}

}  // namespace

extern "C" {

const char* bsg_global_error(void) { return g_error.c_str(); }

int bsg_context_create(int32_t device, bsg_context** out) {
    return guard(nullptr, [&] {
        require(out != nullptr, "null output handle");
        auto* c = new bsg_context();
        try {
            c->ctx = std::make_unique<bsg::Context>(device);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

int bsg_context_destroy(bsg_context* ctx) {
    delete ctx;
    return bsg::kOk;
}

const char* bsg_last_error(const bsg_context* ctx) { return ctx ? ctx->ctx->last_error.c_str() : g_error.c_str(); }

int bsg_context_launches(const bsg_context* ctx, int64_t* out) {
    if (!ctx || !out) return bsg::kArgument;
    *out = ctx->ctx->launches;
    return bsg::kOk;
}

int bsg_context_synchronize(bsg_context* ctx) {
    return guard(ctx, [&] { ctx->ctx->sync(); });
}

int bsg_context_profile(bsg_context* ctx, int32_t enable) {
    return guard(ctx, [&] {
        require(ctx != nullptr, "null context");
        ctx->ctx->profiling = enable != 0;
    });
}

int bsg_context_profile_report(bsg_context* ctx, char* buffer, int32_t capacity) {
    return guard(ctx, [&] {
        require(ctx && buffer && capacity > 0, "bad argument");
        const std::string r = ctx->ctx->profileReport();
        if (static_cast<int32_t>(r.size()) >= capacity) bsg::fail(bsg::kArgument, "profile report buffer too small");
        std::memcpy(buffer, r.c_str(), r.size() + 1);
    });
}

int bsg_context_phase_log(bsg_context* ctx, int32_t capacity) {
    return guard(ctx, [&] {
        require(ctx && capacity >= 0, "bad argument");
        bsg::Context& c = *ctx->ctx;
        c.sync();
        if (c.phase_entries) { cudaFree(c.phase_entries); c.phase_entries = nullptr; }
        if (c.phase_count) { cudaFree(c.phase_count); c.phase_count = nullptr; }
        c.phase_capacity = 0;
        if (capacity > 0) {
            BSG_CUDA(cudaMalloc(&c.phase_entries, sizeof(long long) * 2 * static_cast<std::size_t>(capacity)));
            BSG_CUDA(cudaMalloc(&c.phase_count, sizeof(int)));
            BSG_CUDA(cudaMemset(c.phase_count, 0, sizeof(int)));
            c.phase_capacity = capacity;
        }
    });
}

int bsg_context_phase_log_read(bsg_context* ctx, int64_t* pairs, int32_t capacity, int32_t* count) {
    return guard(ctx, [&] {
        require(ctx && pairs && count, "null argument");
        bsg::Context& c = *ctx->ctx;
        require(c.phase_capacity > 0, "phase log is not enabled");
        c.sync();
        int n = 0;
        BSG_CUDA(cudaMemcpy(&n, c.phase_count, sizeof(int), cudaMemcpyDeviceToHost));
        n = std::min(n, std::min(capacity, c.phase_capacity));
        if (n) BSG_CUDA(cudaMemcpy(pairs, c.phase_entries, sizeof(long long) * 2 * n, cudaMemcpyDeviceToHost));
        BSG_CUDA(cudaMemset(c.phase_count, 0, sizeof(int)));
        *count = n;
    });
}

int bsg_context_event_record(bsg_context* ctx, int32_t slot) {
    return guard(ctx, [&] {
        require(ctx && slot >= 0 && slot < 64, "event slot must be in [0,64)");
        auto& ev = ctx->ctx->user_events;
        if (ev.size() <= static_cast<std::size_t>(slot)) ev.resize(slot + 1, nullptr);
        if (!ev[slot]) BSG_CUDA(cudaEventCreate(&ev[slot]));
        BSG_CUDA(cudaEventRecord(ev[slot], ctx->ctx->stream));
    });
}

int bsg_context_event_elapsed(bsg_context* ctx, int32_t a, int32_t b, double* ms) {
    return guard(ctx, [&] {
        require(ctx && ms, "null argument");
        auto& ev = ctx->ctx->user_events;
        require(a >= 0 && b >= 0 && static_cast<std::size_t>(std::max(a, b)) < ev.size() && ev[a] && ev[b],
                "event slot was never recorded");
        BSG_CUDA(cudaEventSynchronize(ev[b]));
        float f = 0.0f;
        BSG_CUDA(cudaEventElapsedTime(&f, ev[a], ev[b]));
        *ms = f;
    });
}

int bsg_mesh_create(bsg_context* ctx, const bsg_mesh_geometry* g, bsg_mesh** out) {
    return guard(ctx, [&] {
        require(ctx && g && out, "null argument");
        require(g->n_cells > 0 && g->n_faces > 0 && g->n_patches > 0, "mesh sizes must be positive");
        bsg::HostGeometry h;
        h.n_cells = g->n_cells;
        h.n_faces = g->n_faces;
        h.n_patches = g->n_patches;
        const std::size_t F = g->n_faces, N = g->n_cells;
        h.owner.assign(g->face_owner, g->face_owner + F);
        h.nbr.assign(g->face_neighbour, g->face_neighbour + F);
        h.patch.assign(g->face_patch, g->face_patch + F);
        h.Sf.assign(g->face_area_vectors, g->face_area_vectors + 3 * F);
        h.xf.assign(g->face_centres, g->face_centres + 3 * F);
        h.area.assign(g->face_areas, g->face_areas + F);
        h.normal.assign(g->face_normals, g->face_normals + 3 * F);
        h.weight.assign(g->face_owner_weights, g->face_owner_weights + F);
        h.dcoef.assign(g->face_orthogonal_coefficients, g->face_orthogonal_coefficients + F);
        h.kvec.assign(g->face_non_orthogonal, g->face_non_orthogonal + 3 * F);
        h.skew.assign(g->face_skewness, g->face_skewness + 3 * F);
        h.xc.assign(g->cell_centres, g->cell_centres + 3 * N);
        h.V.assign(g->cell_volumes, g->cell_volumes + N);
        h.orthogonal = g->orthogonal_geometry != 0;
        auto* m = new bsg_mesh{ctx, nullptr};
        try {
            m->mesh = bsg::buildDeviceMesh(*ctx->ctx, h);
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
    });
}

int bsg_mesh_create_polyhedral(bsg_context* ctx, int32_t n_vertices, const double* vertices, int32_t n_faces,
                               const int32_t* offsets, const int32_t* ids, const int32_t* owner,
                               const int32_t* neighbour, const int32_t* patch, int32_t n_patches, bsg_mesh** out) {
    return guard(ctx, [&] {
        require(ctx && vertices && offsets && ids && owner && neighbour && patch && out, "null argument");
        const CellOrder r = cellOrder(n_vertices, n_faces, offsets, ids, owner, neighbour, patch, n_patches);
        auto* m = new bsg_mesh{ctx, nullptr};
        try {
            m->mesh = bsg::buildDeviceMeshPolyhedral(*ctx->ctx, n_vertices, vertices, n_faces, offsets, ids,
                                                     r.applied ? r.owner.data() : owner,
                                                     r.applied ? r.neighbour.data() : neighbour, patch, n_patches);
            applyCellOrder(*m->mesh, r);
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
    });
}

int bsg_mesh_create_polyhedral_host(bsg_context* ctx, int32_t n_vertices, const double* vertices, int32_t n_faces,
                                    const int32_t* offsets, const int32_t* ids, const int32_t* owner,
                                    const int32_t* neighbour, const int32_t* patch, int32_t n_patches,
                                    bsg_mesh** out) {
    return guard(ctx, [&] {
        require(ctx && vertices && offsets && ids && owner && neighbour && patch && out, "null argument");
        const CellOrder r = cellOrder(n_vertices, n_faces, offsets, ids, owner, neighbour, patch, n_patches);
        const bsg::HostGeometry h = bsg::computePolyhedralGeometry(
            n_vertices, vertices, n_faces, offsets, ids, r.applied ? r.owner.data() : owner,
            r.applied ? r.neighbour.data() : neighbour, patch, n_patches);
        auto* m = new bsg_mesh{ctx, nullptr};
        try {
            m->mesh = bsg::buildDeviceMesh(*ctx->ctx, h);
            applyCellOrder(*m->mesh, r);
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
    });
}

int bsg_mesh_create_from_file(bsg_context* ctx, const char* path, bsg_mesh** out) {
    return guard(ctx, [&] {
        require(ctx && path && out, "null argument");
        const bsg::PolyFile f = bsg::readPolyFile(path);
        auto m = std::make_unique<bsg_mesh>();
        m->owner = ctx;
        try {
            const int nv = static_cast<int>(f.vertices.size() / 3), nf = static_cast<int>(f.owner.size());
            const int np = static_cast<int>(f.patch_names.size());
            const CellOrder r = cellOrder(nv, nf, f.offsets.data(), f.ids.data(), f.owner.data(), f.neighbour.data(),
                                          f.patch.data(), np);
            m->mesh = bsg::buildDeviceMeshPolyhedral(*ctx->ctx, nv, f.vertices.data(), nf, f.offsets.data(),
                                                     f.ids.data(), r.applied ? r.owner.data() : f.owner.data(),
                                                     r.applied ? r.neighbour.data() : f.neighbour.data(),
                                                     f.patch.data(), np);
            applyCellOrder(*m->mesh, r);
        } catch (const bsg::Error& e) {
            if (e.code != bsg::kArgument) throw;
            bsg::fail(bsg::kArgument, std::string("invalid BabelSim mesh file ") + path + ": " + e.what());
        }
        *out = m.release();
    });
}

int bsg_mesh_file_info(const char* path, int64_t out[4], char* patches, int32_t capacity) {
    return guard(nullptr, [&] {
        require(path && out, "null argument");
        const bsg::PolyFile f = bsg::readPolyFile(path);
        out[0] = f.n_cells;
        out[1] = static_cast<int64_t>(f.owner.size());
        out[2] = static_cast<int64_t>(f.vertices.size() / 3);
        out[3] = static_cast<int64_t>(f.patch_names.size());
        if (patches && capacity > 0) {
            static const char* kinds[] = {"generic", "wall", "inlet", "outlet", "symmetry", "processor"};
            std::string text;
            for (std::size_t p = 0; p < f.patch_names.size(); ++p)
                text += f.patch_names[p] + " " + kinds[f.patch_kinds[p]] + "\n";
            require(static_cast<int32_t>(text.size()) < capacity, "patch list buffer too small");
            std::memcpy(patches, text.c_str(), text.size() + 1);
        }
    });
}

int bsg_mesh_locality_order(int32_t n_cells, int32_t n_faces, const int32_t* owner, const int32_t* neighbour,
                            int32_t* order, int32_t* applied) {
    return guard(nullptr, [&] {
        require(owner && neighbour && order && applied && n_cells > 0 && n_faces > 0, "bad argument");
        for (int f = 0; f < n_faces; ++f)
            require(owner[f] >= 0 && owner[f] < n_cells && neighbour[f] < n_cells, "owner or neighbour out of range");
        bool a = false;
        const std::vector<int> o = bsg::localityOrder(n_cells, n_faces, owner, neighbour, &a);
        std::memcpy(order, o.data(), sizeof(int) * o.size());
        *applied = a ? 1 : 0;
    });
}

int bsg_mesh_destroy(bsg_mesh* mesh) {
    delete mesh;
    return bsg::kOk;
}

int bsg_mesh_validate_polyhedral(int32_t n_vertices, const double* vertices, int32_t n_faces, const int32_t* offsets,
                                 const int32_t* ids, const int32_t* owner, const int32_t* neighbour,
                                 const int32_t* patch, int32_t n_patches, int32_t* n_cells_out,
                                 int32_t* orthogonal_out) {
    return guard(nullptr, [&] {
        require(vertices && offsets && ids && owner && neighbour && patch, "null argument");
        const bsg::HostGeometry h = bsg::computePolyhedralGeometry(n_vertices, vertices, n_faces, offsets, ids, owner,
                                                                    neighbour, patch, n_patches);
        if (n_cells_out) *n_cells_out = h.n_cells;
        if (orthogonal_out) *orthogonal_out = h.orthogonal ? 1 : 0;
    });
}

int bsg_write_results(const char* time_directory, const char* time_name, int32_t n_vertices, const double* vertices,
                      int32_t n_faces, const int32_t* offsets, const int32_t* ids, const int32_t* owner,
                      const int32_t* neighbour, const int32_t* patch, int32_t n_patches, int32_t n_fields,
                      const char* const* names, const int32_t* components, const double* const* values) {
    return guard(nullptr, [&] {
        require(time_directory && time_name && vertices && offsets && ids && owner && neighbour && patch && names &&
                    components && values && n_fields > 0,
                "null argument");
        std::vector<bsg::ResultField> fields(n_fields);
        for (int i = 0; i < n_fields; ++i) {
            require(names[i] != nullptr, "null field name");
            fields[i] = bsg::ResultField{names[i], components[i], values[i]};
        }
        bsg::writeResults(time_directory, time_name, n_vertices, vertices, n_faces, offsets, ids, owner, neighbour,
                          patch, n_patches, fields);
    });
}

int bsg_mesh_sizes(const bsg_mesh* mesh, int64_t out[5]) {
    if (!mesh || !out) return bsg::kArgument;
    const bsg::DeviceMesh& m = *mesh->mesh;
    out[0] = m.n_cells; out[1] = m.n_faces; out[2] = m.n_interior; out[3] = m.n_patches; out[4] = m.orthogonal;
    return bsg::kOk;
}

int bsg_mesh_export(const bsg_mesh* mesh, const char* name, void* host_out) {
    return guard(ctxOf(mesh), [&] {
        require(mesh && name && host_out, "null argument");
        bsg::DeviceMesh& m = *mesh->mesh;
        bsg::ensureExternalGeometry(m);
        const std::string n(name);
        auto put = [&](const auto& v) { std::memcpy(host_out, v.data(), v.size() * sizeof(v[0])); };
        if (n == "face_owner") put(m.ext_owner);
        else if (n == "face_neighbour") put(m.ext_nbr);
        else if (n == "face_patch") put(m.ext_patch);
        else if (n == "face_area_vectors") put(m.ext_Sf);
        else if (n == "face_centres") put(m.ext_xf);
        else if (n == "face_areas") put(m.ext_area);
        else if (n == "face_normals") put(m.ext_n);
        else if (n == "face_owner_weights") put(m.ext_w);
        else if (n == "face_orthogonal_coefficients") put(m.ext_dcoef);
        else if (n == "face_non_orthogonal") put(m.ext_k);
        else if (n == "face_skewness") put(m.ext_skew);
        else if (n == "cell_centres") put(m.ext_xc);
        else if (n == "cell_volumes") put(m.ext_V);
        else bsg::fail(bsg::kArgument, "unknown geometry array " + n);
    });
}

int bsg_field_create(bsg_mesh* mesh, int32_t location, int32_t components, bsg_field** out) {
    return guard(ctxOf(mesh), [&] {
        require(mesh && out, "null argument");
        require(location == 0 || location == 1, "field location must be cell or face");
        auto* f = new bsg_field{mesh, nullptr};
        try {
            f->field = std::make_unique<bsg::DeviceField>(*mesh->mesh, location, components);
        } catch (...) {
            delete f;
            throw;
        }
        *out = f;
    });
}

int bsg_field_destroy(bsg_field* field) {
    delete field;
    return bsg::kOk;
}

int bsg_field_set_boundary(bsg_field* field, int32_t patch, int32_t type, const double* value) {
    return guard(ctxOf(field), [&] {
        require(field != nullptr, "null field");
        field->field->setBoundary(patch, type, value);
    });
}

int bsg_field_upload(bsg_field* field, const double* host) {
    return guard(ctxOf(field), [&] {
        require(field && host, "null argument");
        field->field->uploadExternal(host);
    });
}

int bsg_field_download(const bsg_field* field, double* host) {
    return guard(ctxOf(field), [&] {
        require(field && host, "null argument");
        field->field->downloadExternal(host);
    });
}

int bsg_field_set_boundary_flux(bsg_field* field, const bsg_field* face_flux) {
    return guard(ctxOf(field), [&] {
        require(field && face_flux, "null argument");
        field->field->setFluxContext(*face_flux->field);
        field->mesh->owner->ctx->sync();
    });
}

int bsg_math_grad(const bsg_field* in, int32_t method, bsg_field* out) {
    return guard(ctxOf(in), [&] {
        require(in && out, "null argument");
        bsg::DeviceField& x = *in->field;
        require(out->field->location == 0 && out->field->comps == 3 * x.comps, "gradient result has the wrong shape");
        bsg::gradient(x, method, out->field->v);
        x.mesh->ctx->sync();
    });
}

int bsg_math_interpolate(const bsg_field* in, const bsg_options* o, bsg_field* out) {
    return guard(ctxOf(in), [&] {
        require(in && out, "null argument");
        const bsg::Options op = options(o);
        require(out->field->location == 1 && out->field->comps == in->field->comps, "interpolation result has the wrong shape");
        bsg::interpolate(*in->field, op.interpolation, op.gradient, out->field->v);
        in->field->mesh->ctx->sync();
    });
}

int bsg_math_flux(bsg_field* velocity, const bsg_options* o, bsg_field* out) {
    return guard(ctxOf(velocity), [&] {
        require(velocity && out, "null argument");
        const bsg::Options op = options(o);
        bsg::faceFlux(*velocity->field, op.interpolation, op.gradient, *out->field);
        velocity->field->mesh->ctx->sync();
    });
}

int bsg_math_div_flux(const bsg_field* phi, bsg_field* out) {
    return guard(ctxOf(phi), [&] {
        require(phi && out && out->field->location == 0 && out->field->comps == 1, "divergence result must be a scalar cell field");
        bsg::divFlux(*phi->field, out->field->v);
        phi->field->mesh->ctx->sync();
    });
}

int bsg_math_normal_gradient(const bsg_field* in, const bsg_field* gradient, const bsg_options* o, bsg_field* out) {
    return guard(ctxOf(in), [&] {
        require(in && out && in->field->comps == 1, "normal gradient of a scalar cell field");
        const bsg::Options op = options(o);
        bsg::DeviceArray<double> g;
        const double* gp = nullptr;
        if (gradient) gp = gradient->field->v.data();
        else {
            bsg::gradient(*in->field, op.gradient, g);
            gp = g.data();
        }
        bsg::normalGradient(*in->field, gp, op.diffusion, out->field->v);
        in->field->mesh->ctx->sync();
    });
}

int bsg_equation_create(bsg_field* unknown, const bsg_options* o, bsg_equation** out) {
    return guard(ctxOf(unknown), [&] {
        require(unknown && out, "null argument");
        auto* e = new bsg_equation();
        e->unknown = unknown;
        try {
            e->eq = std::make_unique<bsg::DeviceEquation>(*unknown->field, options(o));
            e->flags.resize(4);
        } catch (...) {
            delete e;
            throw;
        }
        *out = e;
    });
}

int bsg_equation_destroy(bsg_equation* eq) {
    delete eq;
    return bsg::kOk;
}

int bsg_equ_reset(bsg_equation* e) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] { e->eq->reset(); });
}

int bsg_equ_div(bsg_equation* e, const bsg_field* flux, double scale, const bsg_options* term) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e && flux, "null argument");
        const bsg::Options op = term ? options(term) : e->eq->options;
        bsg::addConvection(*e->eq, *flux->field, scale, op);
        e->eq->x->mesh->ctx->sync();
    });
}

int bsg_equ_laplacian(bsg_equation* e, const bsg_field* coefficient, double k, double factor, const bsg_options* term) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e != nullptr, "null equation");
        const bsg::Options op = term ? options(term) : e->eq->options;
        bsg::addLaplacian(*e->eq, coefficient ? coefficient->field.get() : nullptr, k, factor, op);
    });
}

int bsg_equ_source(bsg_equation* e, const bsg_field* value, double factor) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e && value && value->field->location == 0 && value->field->comps == e->eq->x->comps,
                "equ::source requires a compatible cell field");
        bsg::addSource(*e->eq, value->field->v.data(), factor);
        e->eq->x->mesh->ctx->sync();
    });
}

int bsg_equ_ddt(bsg_equation* e, const bsg_field* capacity, double c, const bsg_field* previous,
                const bsg_field* older, double dt, double older_dt, int32_t method) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e && previous, "null argument");
        const int C = e->eq->x->comps;
        auto cellOf = [&](const bsg_field* f, int comps) {
            return f && f->mesh == e->unknown->mesh && f->field->location == 0 && f->field->comps == comps;
        };
        require(cellOf(previous, C), "equ::ddt previous level must be a compatible cell field");
        require(!older || cellOf(older, C), "equ::ddt older level must be a compatible cell field");
        require(!capacity || cellOf(capacity, 1), "equ::ddt capacity must be a cell scalar field");
        const bsg::TimeWeights t = bsg::timeWeights(method, dt, older_dt, older != nullptr);
        if (!t.active) return;
        bsg::Context& ctx = *e->eq->x->mesh->ctx;
        if (capacity) {
            int bad[2];
            bsg::checkValues(ctx, capacity->field->v.data(), e->eq->x->mesh->n_cells, e->flags.data(), bad);
            if (bad[0]) bsg::fail(bsg::kArgument, "time capacity must be positive and finite");
        }
        bsg::addTimeTerm(*e->eq, capacity ? capacity->field->v.data() : nullptr, c, previous->field->v.data(),
                         older ? older->field->v.data() : nullptr, t);
        ctx.sync();
    });
}

int bsg_equ_reaction(bsg_equation* e, const bsg_field* coefficient, double c, double factor) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e != nullptr, "null equation");
        bsg::Context& ctx = *e->eq->x->mesh->ctx;
        if (coefficient) {
            require(coefficient->mesh == e->unknown->mesh && coefficient->field->location == 0 &&
                        coefficient->field->comps == 1,
                    "equ::reaction coefficient must be a cell scalar field");
            int bad[2];
            bsg::checkValues(ctx, coefficient->field->v.data(), e->eq->x->mesh->n_cells, e->flags.data(), bad);
            if (bad[1]) bsg::fail(bsg::kArgument, "nonfinite equ coefficient");
        }
        bsg::addReaction(*e->eq, coefficient ? coefficient->field->v.data() : nullptr, c, factor);
        ctx.sync();
    });
}

int bsg_equ_apply(const bsg_equation* e, const bsg_field* x, bsg_field* out) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e && x && out, "null argument");
        const int C = e->eq->x->comps;
        require(x->field->location == 0 && x->field->comps == C && out->field->location == 0 &&
                    out->field->comps == C && x->mesh == e->unknown->mesh && out->mesh == e->unknown->mesh,
                "equ::apply requires compatible cell fields");
        bsg::applyEquation(*e->eq, x->field->v.data(), out->field->v.data());
        e->eq->x->mesh->ctx->sync();
    });
}

int bsg_equ_residual(const bsg_equation* e, const bsg_field* x, bsg_field* out) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e && x && out, "null argument");
        const int C = e->eq->x->comps;
        require(x->field->location == 0 && x->field->comps == C && out->field->location == 0 &&
                    out->field->comps == C && x->mesh == e->unknown->mesh && out->mesh == e->unknown->mesh,
                "equ::residual requires compatible cell fields");
        require(x->field.get() != out->field.get(), "equ::residual output must differ from its input");
        bsg::residualEquation(*e->eq, x->field->v.data(), out->field->v.data());
        e->eq->x->mesh->ctx->sync();
    });
}

int bsg_equ_relax(bsg_equation* e, const bsg_field* previous, double alpha) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e && previous && previous->field->comps == e->eq->x->comps, "equ::relax requires a compatible cell field");
        bsg::relax(*e->eq, previous->field->v.data(), alpha);
        e->eq->x->mesh->ctx->sync();
    });
}

int bsg_equ_scale(bsg_equation* e, double factor) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        bsg::scale(*e->eq, factor);
        e->eq->x->mesh->ctx->sync();
    });
}

int bsg_equ_reference_if_unanchored(bsg_equation* e, double value, int32_t* anchored_out) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        bsg::referenceIfUnanchored(*e->eq, value, e->flags.data());
        bsg::Context& ctx = *e->eq->x->mesh->ctx;
        int h[2];
        BSG_CUDA(cudaMemcpyAsync(h, e->flags.data(), sizeof(h), cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        if (h[1]) bsg::fail(bsg::kArgument, "reference requires a positive diagonal");
        if (anchored_out) *anchored_out = h[0];
    });
}

int bsg_equ_face_flux(const bsg_equation* e, const bsg_field* solution, bsg_field* out) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e && solution && out && out->field->location == 1 && out->field->comps == 1, "bad face-flux arguments");
        bsg::faceFluxEquation(*e->eq, solution->field->v.data(), out->field->v);
        e->eq->x->mesh->ctx->sync();
    });
}

int bsg_equ_relative_residual(const bsg_equation* e, const bsg_field* x, double* out) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e && x && out, "null argument");
        auto* me = const_cast<bsg_equation*>(e);
        bsg::relativeResidualNorms(*me->eq, x->field->v.data(), me->red);
        bsg::Context& ctx = *e->eq->x->mesh->ctx;
        double h[3];
        BSG_CUDA(cudaMemcpyAsync(h, me->red.result.data(), sizeof(h), cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        *out = std::sqrt(h[0]) / std::max(std::sqrt(h[1]) + std::sqrt(h[2]), 1e-30);
    });
}

int bsg_equ_solve(bsg_equation* e, const bsg_solver_config* config, bsg_solve_result* results) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e && config && results, "null argument");
        solveEquation(e, solverConfig(config), results);
    });
}

int bsg_equ_download(const bsg_equation* e, double* diagonal, double* upper, double* lower, double* source) {
    return guard(e ? ctxOf(e->unknown) : nullptr, [&] {
        require(e != nullptr, "null equation");
        const bsg::DeviceEquation& eq = *e->eq;
        bsg::DeviceMesh& m = *eq.x->mesh;
        bsg::Context& ctx = *m.ctx;
        std::vector<double> val(eq.val.size());
        if (diagonal) bsg::downloadCells(m, eq.diag.data(), diagonal, 1);
        if (source) bsg::downloadCells(m, eq.src.data(), source, eq.x->comps);
        eq.val.download(val.data(), ctx.stream);
        ctx.sync();
        for (int f = 0; f < m.n_faces; ++f) {
            double u = 0.0, l = 0.0;
            if (m.face_kind[f] == 0) {
                const int i = m.face_slot[f];
                u = val[m.h_slot_own[i]];
                l = val[m.h_slot_nbr[i]];
            }
            if (upper) upper[f] = u;
            if (lower) lower[f] = l;
        }
    });
}

int bsg_solve_ldu(bsg_mesh* mesh, const bsg_solver_config* config, int32_t components, const double* diagonal,
                  const double* upper, const double* lower, const double* source, double* x,
                  bsg_solve_result* results) {
    return guard(ctxOf(mesh), [&] {
        require(mesh && config && diagonal && upper && lower && source && x && results, "null argument");
        require(components == 1 || components == 3, "components must be 1 or 3");
        const bsg::SolverConfig cfg = solverConfig(config);
        std::unique_ptr<bsg_system>& sys = mesh->ldu_system[components == 3 ? 1 : 0];
        if (!sys) sys = makeSystem(mesh, components);
        systemSolve(sys.get(), cfg, diagonal, upper, lower, source, x, results);
    });
}

int bsg_system_create(bsg_mesh* mesh, int32_t components, bsg_system** out) {
    return guard(ctxOf(mesh), [&] {
        require(mesh && out, "null argument");
        *out = makeSystem(mesh, components).release();
    });
}

int bsg_system_destroy(bsg_system* system) {
    delete system;
    return bsg::kOk;
}

int bsg_system_solve(bsg_system* system, const bsg_solver_config* config, const double* diagonal,
                     const double* upper, const double* lower, const double* source, double* x,
                     bsg_solve_result* results) {
    return guard(system ? ctxOf(system->mesh) : nullptr, [&] {
        require(system && config && diagonal && upper && lower && source && x && results, "null argument");
        systemSolve(system, solverConfig(config), diagonal, upper, lower, source, x, results);
    });
}

int bsg_system_counters_read(const bsg_system* system, bsg_system_counters* out) {
    return guard(system ? ctxOf(system->mesh) : nullptr, [&] {
        require(system && out, "null argument");
        *out = system->counters;
    });
}

int bsg_pcg_jacobi_static(int32_t n, const int32_t* row_ptr, const int32_t* cols, const double* diag,
                          const double* vals, const double* b, double* x, double absolute_tolerance,
                          double relative_tolerance, int32_t max_iterations, bsg_solve_result* result) {
    return guard(nullptr, [&] {
        require(result != nullptr, "null result");
        const bsg::SolveOutcome o = bsg::staticJacobiPcg(n, row_ptr, cols, diag, vals, b, x, absolute_tolerance,
                                                          relative_tolerance, max_iterations);
        toResult(o, result);
    });
}

int bsg_simple_create(bsg_mesh* mesh, const bsg_simple_config* c, bsg_simple** out) {
    return guard(ctxOf(mesh), [&] {
        require(mesh && c && out, "null argument");
        bsg::SimpleConfig cfg;
        cfg.rho = c->density;
        cfg.mu = c->viscosity;
        cfg.alpha_u = c->velocity_relaxation;
        cfg.alpha_p = c->pressure_relaxation;
        cfg.non_orthogonal_corrections = c->non_orthogonal_corrections;
        cfg.mass_tolerance = c->continuity_tolerance;
        cfg.velocity_tolerance = c->velocity_tolerance;
        cfg.momentum_tolerance = c->momentum_tolerance;
        cfg.pressure_tolerance = c->pressure_correction_tolerance;
        cfg.momentum = options(&c->momentum);
        cfg.pressure = options(&c->pressure);
        cfg.momentum_solver = solverConfig(&c->momentum_solver);
        cfg.pressure_solver = solverConfig(&c->pressure_solver);
        require(cfg.alpha_u > 0 && cfg.alpha_u <= 1 && cfg.alpha_p > 0 && cfg.alpha_p <= 1, "relaxation must be in (0,1]");
        require(cfg.non_orthogonal_corrections >= 0 && cfg.non_orthogonal_corrections <= 20,
                "nonOrthogonalCorrections must be in [0,20]");
        auto* s = new bsg_simple{mesh, nullptr};
        try {
            s->solver = std::make_unique<bsg::SimpleSolver>(*mesh->mesh, cfg);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

int bsg_simple_set_boundary(bsg_simple* s, const char* field, int32_t patch, int32_t type, const double* value) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && field, "null argument");
        const std::string n(field);
        bsg::KOmegaModel* t = s->solver->turbulence();
        if (n == "U") s->solver->U().setBoundary(patch, type, value);
        else if (n == "p") s->solver->p().setBoundary(patch, type, value);
        else if (n == "k" && t && t->config().kind != 2) t->k().setBoundary(patch, type, value);
        else if (n == "nuTilda" && t && t->config().kind == 2) t->omega().setBoundary(patch, type, value);
        else if (n == "omega" && t && t->config().kind == 0) t->omega().setBoundary(patch, type, value);
        else if (n == "epsilon" && t && t->config().kind == 1) t->omega().setBoundary(patch, type, value);
        else bsg::fail(bsg::kArgument,
                       "SIMPLE boundary field must be U or p (k and omega or epsilon with a two-equation model, "
                       "nuTilda with Spalart-Allmaras)");
    });
}

int bsg_simple_set_fields(bsg_simple* s, const double* U, const double* p) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && U && p, "null argument");
        s->solver->U().uploadExternal(U);
        s->solver->p().uploadExternal(p);
        s->solver->start();
    });
}

int bsg_simple_set_flux(bsg_simple* s, const double* phi) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && phi, "null argument");
        s->solver->phi().uploadExternal(phi);
    });
}

int bsg_simple_load_state(bsg_simple* s, const double* U, const double* p, const double* phi) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && U && p && phi, "null argument");
        s->solver->loadState(U, p, phi);
    });
}

void fillReport(const bsg::SimpleReport& r, bsg_simple_report* report) {
    report->iterations = r.iterations;
    report->converged = r.converged;
    report->status = r.status;
    report->mass = r.mass;
    report->dU = r.dU;
    report->rU = r.rU;
    report->dP = r.dP;
    report->linear_pressure_residual = r.linP;
    report->momentum_iterations = r.momentum_iterations;
    report->pressure_iterations = r.pressure_iterations;
    report->turbulence_change = r.turbulence_change;
    report->turbulence_residual = r.turbulence_residual;
}

int bsg_simple_iterate(bsg_simple* s, int32_t max_iterations, bsg_simple_report* report) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && max_iterations >= 0, "bad argument");
        const bsg::SimpleReport r = s->solver->iterate(max_iterations);
        if (report) fillReport(r, report);
    });
}

int bsg_simple_set_segments(bsg_simple* s, int32_t n_segments, const int32_t* cell_offsets, const double* viscosity) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && cell_offsets && viscosity && n_segments > 0, "bad argument");
        s->solver->setSegments(std::vector<int>(cell_offsets, cell_offsets + n_segments + 1),
                               std::vector<double>(viscosity, viscosity + n_segments));
    });
}

int bsg_simple_segment_report(const bsg_simple* s, int32_t segment, bsg_simple_report* report) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && report, "null argument");
        fillReport(s->solver->segmentReport(segment), report);
    });
}

namespace {
bsg::KOmegaConfig komegaConfigOf(const bsg_komega_config* c) {
    bsg::KOmegaConfig k;
    k.beta_star = c->beta_star;
    k.beta = c->beta;
    k.gamma = c->gamma;
    k.sigma_k = c->sigma_k;
    k.sigma_omega = c->sigma_omega;
    k.k_min = c->k_min;
    k.omega_min = c->omega_min;
    k.viscosity_ratio_max = c->max_viscosity_ratio;
    k.relaxation = c->relaxation;
    k.tolerance = c->tolerance;
    k.k_options = options(&c->k_transport);
    k.omega_options = options(&c->omega_transport);
    k.k_solver = solverConfig(&c->k_solver);
    k.omega_solver = solverConfig(&c->omega_solver);
    return k;
}

bsg::KOmegaConfig kepsilonConfigOf(const bsg_kepsilon_config* c) {
    bsg::KOmegaConfig k;
    k.kind = 1;
    k.c_mu = c->c_mu;
    k.c1 = c->c1;
    k.c2 = c->c2;
    k.sigma_k = c->sigma_k;
    k.sigma_omega = c->sigma_epsilon;
    k.k_min = c->k_min;
    k.omega_min = c->epsilon_min;
    k.relaxation = c->relaxation;
    k.tolerance = c->tolerance;
    k.k_options = options(&c->k_transport);
    k.omega_options = options(&c->epsilon_transport);
    k.k_solver = solverConfig(&c->k_solver);
    k.omega_solver = solverConfig(&c->epsilon_solver);
    return k;
}

bsg::KOmegaConfig saConfigOf(const bsg_sa_config* c) {
    bsg::KOmegaConfig k;
    k.kind = 2;
    k.sa_cb1 = c->cb1;
    k.sa_cb2 = c->cb2;
    k.sa_sigma = c->sigma;
    k.sa_kappa = c->kappa;
    k.sa_cw1 = c->cw1;
    k.sa_cw2 = c->cw2;
    k.sa_cw3 = c->cw3;
    k.sa_cv1 = c->cv1;
    k.sa_ct3 = c->ct3;
    k.sa_ct4 = c->ct4;
    k.omega_min = c->nu_tilda_min;
    k.wall_distance_min = c->wall_distance_min;
    k.relaxation = c->relaxation;
    k.tolerance = c->tolerance;
    k.omega_options = options(&c->nu_tilda_transport);
    k.omega_solver = solverConfig(&c->nu_tilda_solver);
    return k;
}
}  // namespace

int bsg_simple_enable_komega(bsg_simple* s, const bsg_komega_config* c) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && c, "null argument");
        s->solver->enableKOmega(komegaConfigOf(c));
    });
}

int bsg_simple_enable_kepsilon(bsg_simple* s, const bsg_kepsilon_config* c) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && c, "null argument");
        s->solver->enableKOmega(kepsilonConfigOf(c));
    });
}

int bsg_simple_enable_spalart_allmaras(bsg_simple* s, const bsg_sa_config* c) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && c, "null argument");
        s->solver->enableKOmega(saConfigOf(c));
    });
}

int bsg_simple_set_wall_distance(bsg_simple* s, const double* wall_distance) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && wall_distance, "null argument");
        bsg::KOmegaModel* t = s->solver->turbulence();
        if (!t) bsg::fail(bsg::kState, "no turbulence model is enabled");
        t->setWallDistance(wall_distance);
    });
}

int bsg_simple_set_turbulence_fields(bsg_simple* s, const double* k, const double* omega) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && omega, "null argument");
        bsg::KOmegaModel* t = s->solver->turbulence();
        if (!t) bsg::fail(bsg::kState, "no turbulence model is enabled");
        if (t->config().kind == 2) require(k == nullptr, "the Spalart-Allmaras model has no k");
        else require(k != nullptr, "null argument");
        if (k) t->k().uploadExternal(k);
        t->omega().uploadExternal(omega);
    });
}

int bsg_simple_get_turbulence_fields(const bsg_simple* s, double* k, double* omega, double* mut) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s != nullptr, "null argument");
        bsg::KOmegaModel* t = s->solver->turbulence();
        if (!t) bsg::fail(bsg::kState, "no turbulence model is enabled");
        if (k && t->config().kind == 2) bsg::fail(bsg::kArgument, "the Spalart-Allmaras model has no k");
        if (k) t->k().downloadExternal(k);
        if (omega) t->omega().downloadExternal(omega);
        if (mut) t->turbulentViscosity().downloadExternal(mut);
    });
}

int bsg_simple_get_fields(const bsg_simple* s, double* U, double* p, double* phi) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s != nullptr, "null argument");
        if (U) s->solver->U().downloadExternal(U);
        if (p) s->solver->p().downloadExternal(p);
        if (phi) s->solver->phi().downloadExternal(phi);
    });
}

int bsg_simple_destroy(bsg_simple* s) {
    delete s;
    return bsg::kOk;
}

int bsg_piso_create(bsg_mesh* mesh, const bsg_piso_config* c, bsg_piso** out) {
    return guard(ctxOf(mesh), [&] {
        require(mesh && c && out, "null argument");
        bsg::PisoConfig cfg;
        cfg.rho = c->density;
        cfg.mu = c->viscosity;
        cfg.alpha_u = c->velocity_relaxation;
        cfg.max_iterations = c->max_iterations;
        cfg.correctors = c->correctors;
        cfg.max_correctors = c->max_correctors > 0 ? c->max_correctors : c->correctors;
        cfg.coupling_tolerance = c->coupling_tolerance > 0 ? c->coupling_tolerance : 1.7976931348623157e308;
        cfg.non_orthogonal_corrections = c->non_orthogonal_corrections;
        cfg.mass_tolerance = c->continuity_tolerance;
        cfg.velocity_tolerance = c->velocity_tolerance;
        cfg.momentum_tolerance = c->momentum_tolerance;
        cfg.pressure_tolerance = c->pressure_correction_tolerance;
        cfg.time_method = c->time_method;
        cfg.start_time = c->start_time;
        cfg.end_time = c->end_time;
        cfg.delta_t = c->delta_t;
        cfg.momentum = options(&c->momentum);
        cfg.pressure = options(&c->pressure);
        cfg.momentum_solver = solverConfig(&c->momentum_solver);
        cfg.pressure_solver = solverConfig(&c->pressure_solver);
        auto* s = new bsg_piso{mesh, nullptr};
        try {
            s->solver = std::make_unique<bsg::PisoSolver>(*mesh->mesh, cfg);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

int bsg_piso_set_boundary(bsg_piso* s, const char* field, int32_t patch, int32_t type, const double* value) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && field, "null argument");
        const std::string n(field);
        bsg::KOmegaModel* t = s->solver->turbulence();
        const int kind = t ? t->config().kind : -1;
        if (n == "U") s->solver->U().setBoundary(patch, type, value);
        else if (n == "p") s->solver->p().setBoundary(patch, type, value);
        else if (n == "k" && t && kind != 2) t->k().setBoundary(patch, type, value);
        else if ((n == "omega" && kind == 0) || (n == "epsilon" && kind == 1) || (n == "nuTilda" && kind == 2))
            t->omega().setBoundary(patch, type, value);
        else bsg::fail(bsg::kArgument, "PISO boundary field must be U or p, or a field of the turbulence model");
    });
}

namespace {
void enablePisoTurbulence(bsg_piso* s, bsg::KOmegaConfig k, const bsg_piso_turbulence_controls* tc) {
    bsg::PisoTurbulenceControls c;
    if (tc) {
        c.segregated = tc->coupling != 0;
        c.max_iterations = tc->max_iterations > 0 ? tc->max_iterations : 1000;
        c.correctors = tc->correctors;
    }
    s->solver->enableTurbulence(k, c);
}
}  // namespace

int bsg_piso_enable_komega(bsg_piso* s, const bsg_komega_config* c, const bsg_piso_turbulence_controls* tc) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && c, "null argument");
        enablePisoTurbulence(s, komegaConfigOf(c), tc);
    });
}

int bsg_piso_enable_kepsilon(bsg_piso* s, const bsg_kepsilon_config* c, const bsg_piso_turbulence_controls* tc) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && c, "null argument");
        enablePisoTurbulence(s, kepsilonConfigOf(c), tc);
    });
}

int bsg_piso_enable_spalart_allmaras(bsg_piso* s, const bsg_sa_config* c, const bsg_piso_turbulence_controls* tc) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && c, "null argument");
        enablePisoTurbulence(s, saConfigOf(c), tc);
    });
}

int bsg_piso_set_wall_distance(bsg_piso* s, const double* wall_distance) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && wall_distance, "null argument");
        bsg::KOmegaModel* t = s->solver->turbulence();
        if (!t) bsg::fail(bsg::kState, "no turbulence model is enabled");
        t->setWallDistance(wall_distance);
    });
}

int bsg_piso_set_turbulence_fields(bsg_piso* s, const double* k, const double* second) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && second, "null argument");
        bsg::KOmegaModel* t = s->solver->turbulence();
        if (!t) bsg::fail(bsg::kState, "no turbulence model is enabled");
        if (t->config().kind == 2) require(k == nullptr, "the Spalart-Allmaras model has no k");
        else require(k != nullptr, "null argument");
        if (k) t->k().uploadExternal(k);
        t->omega().uploadExternal(second);
    });
}

int bsg_piso_get_turbulence_fields(const bsg_piso* s, double* k, double* second, double* mut) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s != nullptr, "null argument");
        bsg::KOmegaModel* t = s->solver->turbulence();
        if (!t) bsg::fail(bsg::kState, "no turbulence model is enabled");
        if (k && t->config().kind == 2) bsg::fail(bsg::kArgument, "the Spalart-Allmaras model has no k");
        if (k) t->k().downloadExternal(k);
        if (second) t->omega().downloadExternal(second);
        if (mut) t->turbulentViscosity().downloadExternal(mut);
    });
}

int bsg_piso_initialize_potential_flow(bsg_piso* s, int32_t initial_non_orthogonal_corrections) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s != nullptr, "null argument");
        s->solver->initializePotentialFlow(initial_non_orthogonal_corrections);
    });
}

int bsg_piso_set_fields(bsg_piso* s, const double* U, const double* p) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && U && p, "null argument");
        s->solver->U().uploadExternal(U);
        s->solver->p().uploadExternal(p);
        s->solver->start();
    });
}

int bsg_piso_advance(bsg_piso* s, int32_t steps, bsg_piso_report* report) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s && steps >= 0, "bad argument");
        const bsg::PisoReport r = s->solver->advance(steps);
        if (report) {
            report->steps = r.steps;
            report->time = r.time;
            report->status = r.status;
            report->accepted = r.accepted;
            report->mass = r.mass;
            report->dU = r.dU;
            report->rU = r.rU;
            report->dP = r.dP;
            report->coupling = r.coupling;
            report->courant_max = r.courant_max;
            report->courant_mean = r.courant_mean;
            report->correctors = r.correctors;
            report->momentum_iterations = r.momentum_iterations;
            report->pressure_iterations = r.pressure_iterations;
            report->turbulence_change = r.turbulence_change;
            report->turbulence_residual = r.turbulence_residual;
            report->turbulence_corrections = r.turbulence_corrections;
        }
    });
}

int bsg_piso_get_fields(const bsg_piso* s, double* U, double* p, double* phi) {
    return guard(s ? ctxOf(s->mesh) : nullptr, [&] {
        require(s != nullptr, "null argument");
        if (U) s->solver->U().downloadExternal(U);
        if (p) s->solver->p().downloadExternal(p);
        if (phi) s->solver->phi().downloadExternal(phi);
    });
}

int bsg_piso_destroy(bsg_piso* s) {
    delete s;
    return bsg::kOk;
}

}  // extern "C"
