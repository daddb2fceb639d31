// Aggregation AMG: host structure setup once per mesh, device numeric setup per
// matrix version, device V-cycle.  See amg.h for the design.
#include "amg.h"
#include "bsg_device.cuh"
#include "pcg_sell.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <numeric>

namespace bsg {

struct AmgPreconditioner::Level {
    int n = 0;
    long long nnz = 0;
    // matrix of this level (level 0 borrows the caller's arrays)
    DeviceArray<int> ptr, col;
    DeviceArray<double> diag, val;
    const int* dptr = nullptr;
    const int* dcol = nullptr;
    const double* ddiag = nullptr;
    const double* dval = nullptr;
    DeviceArray<double> rdiag;           // omega / diag for damped Jacobi
    // transfer to the next coarser level
    DeviceArray<int> agg;                // fine row -> coarse row
    DeviceArray<int> agg_ptr, agg_rows;  // coarse row -> fine rows
    DeviceArray<int> cslot_ptr, cslot_src, cintra_ptr, cintra_src;
    // work vectors
    DeviceArray<double> x, b, t;
    // coarsest level
    DeviceArray<double> dense;           // coarsest level: n x n inverse, row-major
    // SELL-32 copies for the persistent solver (pcg_sell.cuh)
    int nslices = 0;
    long long sell_entries = 0;
    DeviceArray<int> s_ptr, s_col;
    DeviceArray<double> s_val;           // FP64 values (FP64 V-cycle; on level 0 also the Krylov matrix)
    DeviceArray<double> w;               // first Jacobi sweep (FP64 V-cycle)
    DeviceArray<float> s_val32, diag32, rd32, x32, b32, w32, t32;
    void buildSell(const int* hptr, const int* hcol, cudaStream_t s) {
        SellPattern pat;
        pat.build(n, hptr, hcol);
        nslices = pat.nslices;
        sell_entries = pat.entries;
        s_ptr.upload(pat.sptr, s);
        if (pat.col.empty()) pat.col.push_back(0);
        s_col.upload(pat.col, s);
    }
};

namespace {
constexpr int kBlock = 256;
constexpr double kOmega = 2.0 / 3.0;

struct HostCsr {
    int n = 0;
    std::vector<int> ptr, col;
    std::vector<double> diag, val;
};

// Greedy pairwise matching on strongest negative couplings.
std::vector<int> pairwise(const HostCsr& a, int& n_coarse) {
    std::vector<int> mate(a.n, -1), agg(a.n, -1);
    int next = 0;
    for (int i = 0; i < a.n; ++i) {
        if (agg[i] >= 0) continue;
        int best = -1;
        double bs = 0.0;
        for (int k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
            const int j = a.col[k];
            if (j == i || agg[j] >= 0) continue;
            const double s = -a.val[k];
            if (s > bs) { bs = s; best = j; }
        }
        agg[i] = next;
        if (best >= 0) agg[best] = next;
        ++next;
    }
    n_coarse = next;
    return agg;
}

// Galerkin coarse graph of piecewise-constant aggregation (host, structure + values).
HostCsr coarsen(const HostCsr& a, const std::vector<int>& agg, int nc, std::vector<int>* slot_target) {
    HostCsr c;
    c.n = nc;
    c.ptr.assign(nc + 1, 0);
    c.diag.assign(nc, 0.0);
    std::vector<std::vector<int>> members(nc);
    for (int i = 0; i < a.n; ++i) members[agg[i]].push_back(i);
    std::vector<int> marker(nc, -1);
    std::vector<int> cols;
    if (slot_target) slot_target->assign(a.ptr[a.n], -1);
    for (int I = 0; I < nc; ++I) {
        cols.clear();
        for (int i : members[I]) {
            c.diag[I] += a.diag[i];
            for (int k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
                const int J = agg[a.col[k]];
                if (J == I) { c.diag[I] += a.val[k]; continue; }
                if (marker[J] != I) { marker[J] = I; cols.push_back(J); }
            }
        }
        std::sort(cols.begin(), cols.end());
        const int base = static_cast<int>(c.col.size());
        for (int J : cols) { c.col.push_back(J); c.val.push_back(0.0); }
        c.ptr[I + 1] = static_cast<int>(c.col.size());
        for (int i : members[I]) {
            for (int k = a.ptr[i]; k < a.ptr[i + 1]; ++k) {
                const int J = agg[a.col[k]];
                if (J == I) continue;
                const int pos = base + static_cast<int>(std::lower_bound(cols.begin(), cols.end(), J) - cols.begin());
                c.val[pos] += a.val[k];
                if (slot_target) (*slot_target)[k] = pos;
            }
        }
    }
    return c;
}

__global__ void kRdiag(int n, double omega, const double* __restrict__ d, double* __restrict__ rd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rd[i] = omega / d[i];
}

// Coarse Galerkin values: fixed-order gathers over precomputed fine contributions.
__global__ void kGalerkin(int nc, const int* __restrict__ agg_ptr, const int* __restrict__ agg_rows,
                          const int* __restrict__ cintra_ptr, const int* __restrict__ cintra_src,
                          const int* __restrict__ cptr, const int* __restrict__ cslot_ptr,
                          const int* __restrict__ cslot_src, const double* __restrict__ fdiag,
                          const double* __restrict__ fval, double* __restrict__ cdiag, double* __restrict__ cval) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= nc) return;
    double d = 0.0;
    for (int k = agg_ptr[I]; k < agg_ptr[I + 1]; ++k) d += fdiag[agg_rows[k]];
    for (int k = cintra_ptr[I]; k < cintra_ptr[I + 1]; ++k) d += fval[cintra_src[k]];
    cdiag[I] = d;
    for (int c = cptr[I]; c < cptr[I + 1]; ++c) {
        double v = 0.0;
        for (int k = cslot_ptr[c]; k < cslot_ptr[c + 1]; ++k) v += fval[cslot_src[k]];
        cval[c] = v;
    }
}

// In-place Gauss-Jordan inverse of the coarsest matrix (SPD, so no pivoting),
// one block; each step stages the pivot row and column in shared memory and
// every thread updates its share of the n x n entries.
__global__ void kDenseInverse(int n, const int* __restrict__ ptr, const int* __restrict__ col,
                              const double* __restrict__ diag, const double* __restrict__ val, double* __restrict__ M) {
    extern __shared__ double sh[];
    double* prow = sh;
    double* pcol = sh + n;
    const int nn = n * n;
    for (int e = threadIdx.x; e < nn; e += blockDim.x) M[e] = 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        M[static_cast<long long>(i) * n + i] = diag[i];
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) M[static_cast<long long>(i) * n + col[k]] += val[k];
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double p = 1.0 / M[static_cast<long long>(k) * n + k];
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            prow[j] = M[static_cast<long long>(k) * n + j];
            pcol[j] = M[static_cast<long long>(j) * n + k];
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nn; e += blockDim.x) {
            const int i = e / n, j = e - i * n;
            double v;
            if (i == k) v = j == k ? p : prow[j] * p;
            else if (j == k) v = -pcol[i] * p;
            else v = M[e] - pcol[i] * prow[j] * p;
            M[e] = v;
        }
        __syncthreads();
    }
}

// The same in-place Gauss-Jordan inverse on a cluster of kDenseCluster CTAs that
// keeps the matrix in distributed shared memory: CTA q owns rows [q*rows, (q+1)*rows).
// Step k: every CTA holds pivot row k in its own buffer pk[k & 1] (pushed there by
// the row's owner during step k - 1), saves its rows' column k, updates its rows
// exactly as kDenseInverse does, and the owner of row k + 1 pushes that row's new
// values into every CTA's other buffer; one cluster barrier ends the step.  The
// barrier orders the pushes of step k before their reads in step k + 1, and the
// reads of a buffer in step k - 1 before its overwrite in step k.
constexpr int kDenseCluster = 8;
// Largest coarsest level whose rows, pivot buffers and column copy fit 8 CTAs of 200 KB:
// ceil(n/8) n + 2n + ceil(n/8) doubles per CTA.
constexpr int kAmgCoarsestRows = 440;

__global__ void __cluster_dims__(kDenseCluster, 1, 1)
    kDenseInverseCluster(int n, int rows, const int* __restrict__ ptr, const int* __restrict__ col,
                         const double* __restrict__ diag, const double* __restrict__ val, double* __restrict__ M) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ double sh[];
    double* Ml = sh;                                   // rows x n, this CTA's rows
    double* pk = sh + static_cast<long long>(rows) * n;  // two pivot-row buffers of n
    double* pc = pk + 2 * n;                           // column k of this CTA's rows
    const int q = static_cast<int>(cluster.block_rank());
    const int r0 = q * rows, r1 = min(n, r0 + rows), nr = max(0, r1 - r0);
    for (int e = threadIdx.x; e < nr * n; e += blockDim.x) Ml[e] = 0.0;
    __syncthreads();
    for (int li = threadIdx.x; li < nr; li += blockDim.x) {
        const int i = r0 + li;
        Ml[static_cast<long long>(li) * n + i] = diag[i];
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) Ml[static_cast<long long>(li) * n + col[k]] += val[k];
    }
    __syncthreads();
    // row 0 into every CTA's buffer 0
    if (q == 0)
        for (int e = threadIdx.x; e < kDenseCluster * n; e += blockDim.x) {
            double* dst = cluster.map_shared_rank(pk, e / n);
            dst[e % n] = Ml[e % n];
        }
    cluster.sync();
    // each thread owns one column slot of `rpp` rows per pass (one division, outside the step loop)
    const int bd = static_cast<int>(blockDim.x);
    const int rpp = n >= bd ? 1 : bd / n;
    const int tj = n >= bd ? static_cast<int>(threadIdx.x) : static_cast<int>(threadIdx.x) % n;
    const int tr = n >= bd ? 0 : static_cast<int>(threadIdx.x) / n;
    const int jstep = n >= bd ? bd : n;
    for (int k = 0; k < n; ++k) {
        const double* prow = pk + (k & 1) * n;
        const double p = 1.0 / prow[k];
        for (int li = threadIdx.x; li < nr; li += blockDim.x) pc[li] = Ml[static_cast<long long>(li) * n + k];
        __syncthreads();
        if (tr < rpp)
            for (int li = tr; li < nr; li += rpp) {
                const int i = r0 + li;
                double* row = Ml + static_cast<long long>(li) * n;
                const double c = pc[li];
                for (int j = tj; j < n; j += jstep) {
                    double v;
                    if (i == k) v = j == k ? p : prow[j] * p;
                    else if (j == k) v = -c * p;
                    else v = row[j] - c * prow[j] * p;
                    row[j] = v;
                }
            }
        __syncthreads();
        const int next = k + 1;
        if (next < n && next >= r0 && next < r1) {
            const double* src = Ml + static_cast<long long>(next - r0) * n;
            for (int e = threadIdx.x; e < kDenseCluster * n; e += blockDim.x) {
                double* dst = cluster.map_shared_rank(pk + (next & 1) * n, e / n);
                dst[e % n] = src[e % n];
            }
        }
        cluster.sync();
    }
    for (int e = threadIdx.x; e < nr * n; e += blockDim.x) M[static_cast<long long>(r0) * n + e] = Ml[e];
}

__global__ void kDenseSolve(int n, const double* __restrict__ Minv, const double* __restrict__ b, double* __restrict__ x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) s += Minv[static_cast<long long>(i) * n + j] * b[j];
        x[i] = s;
    }
}

__global__ void kToFloat(long long n, const double* __restrict__ a, float* __restrict__ out) {
    const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (e < n) out[e] = static_cast<float>(a[e]);
}

// x = omega D^-1 b (first Jacobi sweep from a zero guess)
__global__ void kSmoothZero(int n, const double* __restrict__ rd, const double* __restrict__ b, double* __restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = rd[i] * b[i];
}

// x_out = x + omega D^-1 (b - A x)
__global__ void kSmooth(int n, const int* __restrict__ ptr, const int* __restrict__ col, const double* __restrict__ diag,
                        const double* __restrict__ val, const double* __restrict__ rd, const double* __restrict__ b,
                        const double* __restrict__ x, double* __restrict__ xo) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double ax = diag[i] * x[i];
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) ax += val[k] * x[col[k]];
    xo[i] = x[i] + rd[i] * (b[i] - ax);
}

// Post-smoothing sweep fused with prolongation: y = x + P xc, x_out = y + omega D^-1 (b - A y).
__global__ void kProlongSmooth(int n, const int* __restrict__ ptr, const int* __restrict__ col,
                               const double* __restrict__ diag, const double* __restrict__ val,
                               const double* __restrict__ rd, const int* __restrict__ agg,
                               const double* __restrict__ xc, const double* __restrict__ b,
                               const double* __restrict__ x, double* __restrict__ xo) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double yi = x[i] + xc[agg[i]];
    double ay = diag[i] * yi;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
        const int j = col[k];
        ay += val[k] * (x[j] + xc[agg[j]]);
    }
    xo[i] = yi + rd[i] * (b[i] - ay);
}

__global__ void kProlong(int n, const int* __restrict__ agg, const double* __restrict__ xc, double* __restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += xc[agg[i]];
}

// b_c[I] = sum over fine rows i of aggregate I of (b - A x)_i
__global__ void kResidualRestrict(int nc, const int* __restrict__ agg_ptr, const int* __restrict__ agg_rows,
                                  const int* __restrict__ ptr, const int* __restrict__ col,
                                  const double* __restrict__ diag, const double* __restrict__ val,
                                  const double* __restrict__ b, const double* __restrict__ x, double* __restrict__ bc) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= nc) return;
    double s = 0.0;
    for (int m = agg_ptr[I]; m < agg_ptr[I + 1]; ++m) {
        const int i = agg_rows[m];
        double ax = diag[i] * x[i];
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) ax += val[k] * x[col[k]];
        s += b[i] - ax;
    }
    bc[I] = s;
}

__global__ void kCopy(int n, const double* __restrict__ a, double* __restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

}  // namespace

namespace {
// Dynamic shared memory of one CTA of the cluster inverse (the rest of the SM's
// 228 KB stays for the driver's reserve).
constexpr std::size_t kDenseClusterSmem = 200 * 1024;

bool clusterReady() {
    static int ok = -1;
    if (ok < 0) {
        ok = cudaFuncSetAttribute(kDenseInverseCluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(kDenseClusterSmem)) == cudaSuccess;
        if (ok && std::getenv("BSG_DENSE_SINGLE_BLOCK")) ok = 0;
        cudaGetLastError();
    }
    return ok == 1;
}
}  // namespace

AmgPreconditioner::AmgPreconditioner(DeviceMesh& mesh, const SolverConfig& cfg)
    : mesh_(mesh), ctx_(*mesh.ctx), cfg_(cfg) {
    // Tuning overrides for experiments: Jacobi weight and coarse-correction scale.
    if (const char* w = std::getenv("BSG_AMG_OMEGA")) omega_ = std::atof(w);
    if (const char* g = std::getenv("BSG_AMG_GAMMA")) gamma_ = std::atof(g);
    if (!(omega_ > 0.0 && omega_ <= 1.0) || !(gamma_ > 0.0 && gamma_ <= 3.0))
        fail(kArgument, "AMG Jacobi weight must be in (0,1] and the correction scale in (0,3]");
    // FP32 V-cycle data on the mixed-precision path (FP64 Krylov vectors and true residual stay FP64)
    fp32_ = cfg.precision == 1 || cfg.precision == 2 || std::getenv("BSG_AMG_FP32") != nullptr;
    if (const char* p = std::getenv("BSG_AMG_PASSES0")) passes0_ = std::max(1, std::min(4, std::atoi(p)));
    if (const char* p = std::getenv("BSG_AMG_PASSES")) passes_ = std::max(1, std::min(4, std::atoi(p)));
}

AmgPreconditioner::~AmgPreconditioner() {
    for (Level* l : levels_) delete l;
}

int AmgPreconditioner::levels() const { return static_cast<int>(levels_.size()); }
long long AmgPreconditioner::coarseRows(int level) const { return levels_.at(level)->n; }

void AmgPreconditioner::buildStructure(const Dcsr<double>& A) {
    HostCsr cur;
    cur.n = A.n;
    cur.ptr.resize(A.n + 1);
    cur.col.resize(A.nnz_off);
    cur.diag.resize(A.n);
    cur.val.resize(A.nnz_off);
    BSG_CUDA(cudaMemcpyAsync(cur.ptr.data(), A.ptr, sizeof(int) * (A.n + 1), cudaMemcpyDeviceToHost, ctx_.stream));
    BSG_CUDA(cudaMemcpyAsync(cur.col.data(), A.col, sizeof(int) * A.nnz_off, cudaMemcpyDeviceToHost, ctx_.stream));
    BSG_CUDA(cudaMemcpyAsync(cur.diag.data(), A.diag, sizeof(double) * A.n, cudaMemcpyDeviceToHost, ctx_.stream));
    BSG_CUDA(cudaMemcpyAsync(cur.val.data(), A.val, sizeof(double) * A.nnz_off, cudaMemcpyDeviceToHost, ctx_.stream));
    ctx_.sync();
    // Coarsening stops at the configured size, at most kAmgCoarsestRows: a coarsest level that
    // size still fits the cluster inverse's distributed shared memory, and every level removed
    // saves the V-cycle its phases, whose cost is latency, not size, on small levels.
    const int coarse_target = std::max(std::min(cfg_.amg_coarse_size, kAmgCoarsestRows), 16);
    const int max_levels = std::max(2, cfg_.amg_max_levels);
    auto* l0 = new Level();
    l0->n = A.n;
    l0->nnz = A.nnz_off;
    l0->buildSell(cur.ptr.data(), cur.col.data(), ctx_.stream);
    levels_.push_back(l0);
    while (cur.n > coarse_target && static_cast<int>(levels_.size()) < max_levels) {
        // aggregates from `passes` rounds of pairwise matching (2 by default: up to 4 rows)
        const int passes = levels_.size() == 1 ? passes0_ : passes_;
        int n2 = cur.n;
        std::vector<int> agg(cur.n);
        for (int i = 0; i < cur.n; ++i) agg[i] = i;
        HostCsr work = cur;
        for (int pass = 0; pass < passes; ++pass) {
            int nn = 0;
            const std::vector<int> a = pairwise(pass == 0 ? cur : work, nn);
            if (pass + 1 < passes) work = coarsen(pass == 0 ? cur : work, a, nn, nullptr);
            for (int i = 0; i < cur.n; ++i) agg[i] = a[agg[i]];
            n2 = nn;
        }
        // stop when coarsening stalls (< 1.5x fewer rows): such levels cost a
        // V-cycle their barriers and gathers without shrinking the problem
        if (3 * static_cast<long long>(n2) > 2 * static_cast<long long>(cur.n) && cur.n <= 1024) break;
        if (n2 >= cur.n) break;  // no coarsening possible
        std::vector<int> target;
        HostCsr next = coarsen(cur, agg, n2, &target);
        Level* fine = levels_.back();
        // transfer maps
        std::vector<int> agg_ptr(n2 + 1, 0), agg_rows(cur.n);
        for (int i = 0; i < cur.n; ++i) ++agg_ptr[agg[i] + 1];
        for (int I = 0; I < n2; ++I) agg_ptr[I + 1] += agg_ptr[I];
        {
            std::vector<int> fill(agg_ptr.begin(), agg_ptr.end() - 1);
            for (int i = 0; i < cur.n; ++i) agg_rows[fill[agg[i]]++] = i;
        }
        const long long cnnz = static_cast<long long>(next.col.size());
        std::vector<int> cslot_ptr(cnnz + 1, 0), cslot_src(cur.ptr[cur.n]);
        std::vector<int> cintra_ptr(n2 + 1, 0), cintra_src;
        std::vector<int> counts(cnnz, 0);
        for (int k = 0; k < cur.ptr[cur.n]; ++k)
            if (target[k] >= 0) ++cslot_ptr[target[k] + 1];
        for (long long c = 0; c < cnnz; ++c) cslot_ptr[c + 1] += cslot_ptr[c];
        {
            std::vector<int> fill(cslot_ptr.begin(), cslot_ptr.end() - 1);
            for (int I = 0; I < n2; ++I)
                for (int mm = agg_ptr[I]; mm < agg_ptr[I + 1]; ++mm) {
                    const int i = agg_rows[mm];
                    for (int k = cur.ptr[i]; k < cur.ptr[i + 1]; ++k) {
                        if (target[k] >= 0) cslot_src[fill[target[k]]++] = k;
                        else cintra_src.push_back(k);
                    }
                    cintra_ptr[I + 1] = static_cast<int>(cintra_src.size());
                }
            for (int I = 0; I < n2; ++I) cintra_ptr[I + 1] = std::max(cintra_ptr[I + 1], cintra_ptr[I]);
        }
        cudaStream_t s = ctx_.stream;
        fine->agg.upload(agg, s);
        fine->agg_ptr.upload(agg_ptr, s);
        fine->agg_rows.upload(agg_rows, s);
        fine->cslot_ptr.upload(cslot_ptr, s);
        fine->cslot_src.upload(cslot_src, s);
        fine->cintra_ptr.upload(cintra_ptr, s);
        if (cintra_src.empty()) cintra_src.push_back(0);
        fine->cintra_src.upload(cintra_src, s);
        auto* lv = new Level();
        lv->n = n2;
        lv->nnz = cnnz;
        lv->ptr.upload(next.ptr, s);
        if (next.col.empty()) { next.col.push_back(0); next.val.push_back(0.0); }
        lv->col.upload(next.col, s);
        lv->diag.resize(n2);
        lv->val.resize(std::max<long long>(cnnz, 1));
        lv->dptr = lv->ptr.data();
        lv->dcol = lv->col.data();
        lv->ddiag = lv->diag.data();
        lv->dval = lv->val.data();
        lv->buildSell(next.ptr.data(), next.col.data(), s);
        levels_.push_back(lv);
        ctx_.sync();
        cur = std::move(next);
    }
    for (Level* l : levels_) {
        l->x.resize(l->n);
        l->b.resize(l->n);
        l->t.resize(l->n);
        l->rdiag.resize(l->n);
        const std::size_t e = std::max<long long>(l->sell_entries, 1);
        if (fp32_) {
            for (DeviceArray<float>* a : {&l->diag32, &l->rd32, &l->x32, &l->b32, &l->w32, &l->t32}) a->resize(l->n);
            l->s_val32.resize(e);
            l->s_val32.zero(ctx_.stream);  // padding entries stay zero
        } else {
            l->w.resize(l->n);
        }
        if (!fp32_ || l == levels_.front()) {  // FP64 V-cycle values, and the level-0 Krylov matrix
            l->s_val.resize(e);
            l->s_val.zero(ctx_.stream);
        }
    }
    Level* last = levels_.back();
    if (last->n > 2048)
        fail(kState, "AMG coarsening stalled at " + std::to_string(last->n) +
                         " rows, too many for the dense coarsest solve");
    const std::size_t nn = static_cast<std::size_t>(last->n) * last->n;
    last->dense.resize(nn);
    if (fp32_) dense32_.resize(nn);
    built_ = true;
    if (std::getenv("BSG_AMG_VERBOSE")) {
        long long total = 0;
        for (Level* l : levels_) total += l->nnz + l->n;
        for (std::size_t i = 0; i < levels_.size(); ++i)
            std::fprintf(stderr, "amg level %zu: rows %d, off-diagonal nnz %lld (%.1f per row)\n", i, levels_[i]->n,
                         levels_[i]->nnz, levels_[i]->n ? double(levels_[i]->nnz) / levels_[i]->n : 0.0);
        std::fprintf(stderr, "amg operator complexity %.3f\n", double(total) / double(levels_[0]->nnz + levels_[0]->n));
    }
}

void AmgPreconditioner::update(const Dcsr<double>& A, bool numeric) {
    if (!built_) buildStructure(A);
    fine_ = A;
    Level* l0 = levels_[0];
    l0->dptr = A.ptr; l0->dcol = A.col; l0->ddiag = A.diag; l0->dval = A.val;
    if (!numeric) {
        // coarse levels kept; the level-0 matrix and its Jacobi weights always follow the matrix being
        // solved, so a lagged V-cycle smooths the new matrix with its own diagonal (a fresh fine
        // smoother over a lagged coarse correction stays a symmetric positive definite cycle; old
        // weights on a new matrix can stop smoothing when the diagonal moves between versions)
        kRdiag<<<gridFor(l0->n, kBlock), kBlock, 0, ctx_.stream>>>(l0->n, omega_, l0->ddiag, l0->rdiag.data());
        ctx_.launched();
        kCsrToSell<double><<<gridFor(l0->n, kBlock), kBlock, 0, ctx_.stream>>>(
            l0->n, l0->dptr, l0->dval, l0->ddiag, l0->s_ptr.data(), omega_, l0->s_val.data(), nullptr, nullptr);
        ctx_.launched();
        if (fp32_) {
            kCsrToSell<float><<<gridFor(l0->n, kBlock), kBlock, 0, ctx_.stream>>>(
                l0->n, l0->dptr, l0->dval, l0->ddiag, l0->s_ptr.data(), omega_, l0->s_val32.data(), l0->diag32.data(),
                l0->rd32.data());
            ctx_.launched();
        }
        BSG_CUDA(cudaGetLastError());
        uploadViews();
        return;
    }
    for (std::size_t l = 0; l + 1 < levels_.size(); ++l) {
        Level* f = levels_[l];
        Level* c = levels_[l + 1];
        kGalerkin<<<gridFor(c->n, kBlock), kBlock, 0, ctx_.stream>>>(
            c->n, f->agg_ptr.data(), f->agg_rows.data(), f->cintra_ptr.data(), f->cintra_src.data(), c->dptr,
            f->cslot_ptr.data(), f->cslot_src.data(), f->ddiag, f->dval, c->diag.data(), c->val.data());
        ctx_.launched();
    }
    for (Level* l : levels_) {
        kRdiag<<<gridFor(l->n, kBlock), kBlock, 0, ctx_.stream>>>(l->n, omega_, l->ddiag, l->rdiag.data());
        ctx_.launched();
    }
    Level* last = levels_.back();
    const int crow = (last->n + kDenseCluster - 1) / kDenseCluster;
    const std::size_t csmem = sizeof(double) * (static_cast<std::size_t>(crow) * last->n + 2 * last->n + crow);
    if (csmem <= kDenseClusterSmem && clusterReady()) {
        kDenseInverseCluster<<<kDenseCluster, 1024, csmem, ctx_.stream>>>(last->n, crow, last->dptr, last->dcol,
                                                                         last->ddiag, last->dval, last->dense.data());
    } else
    kDenseInverse<<<1, 1024, 2 * sizeof(double) * last->n, ctx_.stream>>>(last->n, last->dptr, last->dcol, last->ddiag,
                                                                         last->dval, last->dense.data());
    ctx_.launched();
    BSG_CUDA(cudaGetLastError());
    // SELL-32 values for the persistent solver
    const int nn = last->n * last->n;
    if (fp32_) {
        kToFloat<<<gridFor(nn, kBlock), kBlock, 0, ctx_.stream>>>(nn, last->dense.data(), dense32_.data());
        ctx_.launched();
    }
    for (std::size_t li = 0; li < levels_.size(); ++li) {
        Level* l = levels_[li];
        const unsigned g = gridFor(l->n, kBlock);
        if (fp32_)
            kCsrToSell<float><<<g, kBlock, 0, ctx_.stream>>>(l->n, l->dptr, l->dval, l->ddiag, l->s_ptr.data(), omega_,
                                                              l->s_val32.data(), l->diag32.data(), l->rd32.data());
        if (!fp32_ || li == 0)
            kCsrToSell<double><<<g, kBlock, 0, ctx_.stream>>>(l->n, l->dptr, l->dval, l->ddiag, l->s_ptr.data(), omega_,
                                                               l->s_val.data(), nullptr, nullptr);
        ctx_.launches += (fp32_ && li == 0) ? 2 : 1;
    }
    BSG_CUDA(cudaGetLastError());
    uploadViews();
}

void AmgPreconditioner::uploadViews() {
    // level views for the persistent solver (level 0 borrows the caller's matrix arrays)
    std::vector<AmgLevelView<double>> views(levels_.size());
    for (std::size_t l = 0; l < levels_.size(); ++l) {
        Level* lv = levels_[l];
        const bool coarser = l + 1 < levels_.size();
        views[l] = AmgLevelView<double>{lv->n, lv->dptr, lv->dcol, lv->ddiag, lv->dval, lv->rdiag.data(),
                                        coarser ? lv->agg.data() : nullptr, coarser ? lv->agg_ptr.data() : nullptr,
                                        coarser ? lv->agg_rows.data() : nullptr, lv->x.data(), lv->b.data(),
                                        lv->t.data()};
    }
    d_views_.upload(views, ctx_.stream);
    const int L = static_cast<int>(levels_.size());
    if (fp32_) {
        std::vector<VLevel<float>> v(L);
        for (int l = 0; l < L; ++l) {
            Level* lv = levels_[l];
            const bool coarser = l + 1 < L;
            v[l].A = SellMat<float>{lv->n, lv->nslices, lv->s_ptr.data(), lv->s_col.data(), lv->s_val32.data(),
                                    lv->diag32.data()};
            v[l].rd = lv->rd32.data();
            v[l].agg_ptr = coarser ? lv->agg_ptr.data() : nullptr;
            v[l].agg_rows = coarser ? lv->agg_rows.data() : nullptr;
            v[l].b = lv->b32.data();
            v[l].w = lv->w32.data();
            v[l].x = lv->x32.data();
            v[l].t = lv->t32.data();
        }
        d_vl32_.upload(v, ctx_.stream);
    } else {
        std::vector<VLevel<double>> v(L);
        for (int l = 0; l < L; ++l) {
            Level* lv = levels_[l];
            const bool coarser = l + 1 < L;
            v[l].A = SellMat<double>{lv->n, lv->nslices, lv->s_ptr.data(), lv->s_col.data(), lv->s_val.data(),
                                     lv->ddiag};
            v[l].rd = lv->rdiag.data();
            v[l].agg_ptr = coarser ? lv->agg_ptr.data() : nullptr;
            v[l].agg_rows = coarser ? lv->agg_rows.data() : nullptr;
            v[l].b = lv->b.data();
            v[l].w = lv->w.data();
            v[l].x = lv->x.data();
            v[l].t = lv->t.data();
        }
        d_vl64_.upload(v, ctx_.stream);
    }
}

SellMat<double> AmgPreconditioner::krylovMatrix() const {
    const Level* l = levels_.front();
    return SellMat<double>{l->n, l->nslices, l->s_ptr.data(), l->s_col.data(), l->s_val.data(), l->ddiag};
}

SellMat<float> AmgPreconditioner::krylovMatrix32() const {
    const Level* l = levels_.front();
    return SellMat<float>{l->n, l->nslices, l->s_ptr.data(), l->s_col.data(), l->s_val32.data(), l->diag32.data()};
}

long long AmgPreconditioner::krylovEntries() const { return levels_.front()->sell_entries; }

VCycleView<double> AmgPreconditioner::sellView64() const {
    VCycleView<double> v;
    v.levels = static_cast<int>(levels_.size());
    v.nu = std::max(1, std::min(2, cfg_.amg_smoothing_steps));
    v.gamma = gamma_;
    v.lv = d_vl64_.data();
    v.dense_inv = levels_.back()->dense.data();
    return v;
}

VCycleView<float> AmgPreconditioner::sellView32() const {
    VCycleView<float> v;
    v.levels = static_cast<int>(levels_.size());
    v.nu = std::max(1, std::min(2, cfg_.amg_smoothing_steps));
    v.gamma = static_cast<float>(gamma_);
    v.lv = d_vl32_.data();
    v.dense_inv = dense32_.data();
    return v;
}

double AmgPreconditioner::sellVcycleBytes() const {
    // One V-cycle of the SELL persistent kernel, every array a phase touches counted once.
    const int L = static_cast<int>(levels_.size());
    const int nu = std::max(1, std::min(2, cfg_.amg_smoothing_steps));
    const double s = fp32_ ? 4.0 : 8.0;  // V-cycle value size
    double bytes = 0.0;
    for (int l = 0; l + 1 < L; ++l) {
        const Level* f = levels_[l];
        const double n = f->n, nc = levels_[l + 1]->n;
        const double sweep = (4.0 + s) * static_cast<double>(f->sell_entries) + 4.0 * (f->nslices + 1) + s * n;  // matrix + diag
        if (nu >= 2) bytes += sweep + 4.0 * s * n;                   // D1: w (gathered), rd, b read; x written
        bytes += sweep + 3.0 * s * n;                                // D2: x, b read; t written
        bytes += 4.0 * (nc + 1) + 4.0 * n + s * n + 3.0 * s * nc;    // D3: lists, t read; b_c, w_c written, rd_c read
        bytes += sweep + 4.0 * s * n;                                // U1: y, rd, b read; t (or output) written
        if (nu >= 2) bytes += sweep + 4.0 * s * n;                   // U2: t, rd, b read; output written
        bytes += 4.0 * n + 4.0 * (nc + 1) + 2.0 * s * n;             // pushes into the finer iterate (l > 0) / z
    }
    const double nc = levels_.back()->n;
    bytes += s * nc * nc + 2.0 * s * nc + 12.0 * (L > 1 ? levels_[L - 2]->n : 0);  // dense solve + push
    return bytes;
}

AmgView<double> AmgPreconditioner::deviceView() const {
    AmgView<double> v;
    v.levels = static_cast<int>(levels_.size());
    v.nu = std::max(1, std::min(2, cfg_.amg_smoothing_steps));
    v.gamma = gamma_;
    v.lv = d_views_.data();
    const Level* last = levels_.back();
    v.dense_inv = last->dense.data();
    v.dense_ld = last->n;
    return v;
}

double AmgPreconditioner::vcycleBytes() const {
    const int L = static_cast<int>(levels_.size());
    const int nu = std::max(1, std::min(2, cfg_.amg_smoothing_steps));
    double bytes = 0.0;
    for (int l = 0; l + 1 < L; ++l) {
        const double n = levels_[l]->n, nc = levels_[l + 1]->n;
        const double matrix = 8.0 * n + 4.0 * (n + 1) + 12.0 * static_cast<double>(levels_[l]->nnz);
        // pre-smoothing: nu == 2 reads the matrix once (first sweep formed on the fly)
        bytes += nu == 2 ? matrix + 24.0 * n : 24.0 * n;
        // residual + restriction: aggregate lists, matrix, x, b; coarse b written
        bytes += 4.0 * (nc + 1) + 4.0 * n + matrix + 16.0 * n + 8.0 * nc;
        // prolongation + first post sweep: matrix, x, agg, rd, b, coarse x; t (or z) written
        bytes += matrix + 36.0 * n + 8.0 * nc;
        if (nu == 2) bytes += matrix + 32.0 * n + (l == 0 ? 8.0 * n : 0.0);  // second sweep (+ r for r.z)
        else bytes += l == 0 ? 8.0 * n : 16.0 * n;                           // r.z, or the t -> x copy
    }
    const double nc = levels_.back()->n;
    bytes += 8.0 * nc * nc + 16.0 * nc;  // dense coarsest solve
    return bytes;
}

void AmgPreconditioner::apply(Context& ctx, const double* r, double* z) {
    const int L = static_cast<int>(levels_.size());
    const int nu = std::max(1, cfg_.amg_smoothing_steps);
    cudaStream_t s = ctx.stream;
    std::vector<double*> xs(L, nullptr);   // buffer holding each level's pre-smoothed iterate
    // Downward leg: damped-Jacobi pre-smoothing from a zero guess, then the
    // fused residual + aggregate restriction.
    for (int l = 0; l < L - 1; ++l) {
        Level* f = levels_[l];
        Level* c = levels_[l + 1];
        const double* b = l == 0 ? r : f->b.data();
        double* cur = f->x.data();
        double* other = f->t.data();
        const unsigned g = gridFor(f->n, kBlock);
        BSG_PROFILE(ctx, l == 0 ? "amg_pre_smooth_restrict_l0" : "amg_coarse_levels");
        kSmoothZero<<<g, kBlock, 0, s>>>(f->n, f->rdiag.data(), b, cur);
        ctx.launched();
        for (int it = 1; it < nu; ++it) {
            kSmooth<<<g, kBlock, 0, s>>>(f->n, f->dptr, f->dcol, f->ddiag, f->dval, f->rdiag.data(), b, cur, other);
            ctx.launched();
            std::swap(cur, other);
        }
        xs[l] = cur;
        kResidualRestrict<<<gridFor(c->n, kBlock), kBlock, 0, s>>>(c->n, f->agg_ptr.data(), f->agg_rows.data(), f->dptr,
                                                                    f->dcol, f->ddiag, f->dval, b, cur, c->b.data());
        ctx.launched();
    }
    Level* last = levels_.back();
    {
        BSG_PROFILE(ctx, "amg_coarse_levels");
        const double* b = L == 1 ? r : last->b.data();
        double* x = L == 1 ? z : last->x.data();
        kDenseSolve<<<gridFor(last->n, 128), 128, 0, s>>>(last->n, last->dense.data(), b, x);
        ctx.launched();
        xs[L - 1] = x;
    }
    // Upward leg: first post-smoothing sweep fused with the prolongation, then
    // further sweeps ping-pong; level 0 ends in z.
    for (int l = L - 2; l >= 0; --l) {
        Level* f = levels_[l];
        const double* b = l == 0 ? r : f->b.data();
        double* x = xs[l];
        double* other = x == f->x.data() ? f->t.data() : f->x.data();
        const unsigned g = gridFor(f->n, kBlock);
        BSG_PROFILE(ctx, l == 0 ? "amg_prolong_post_smooth_l0" : "amg_coarse_levels");
        double* out = (l == 0 && nu == 1) ? z : other;
        kProlongSmooth<<<g, kBlock, 0, s>>>(f->n, f->dptr, f->dcol, f->ddiag, f->dval, f->rdiag.data(), f->agg.data(),
                                            xs[l + 1], b, x, out);
        ctx.launched();
        double* cur = out;
        for (int it = 1; it < nu; ++it) {
            double* dst = (l == 0 && it == nu - 1) ? z : (cur == f->x.data() ? f->t.data() : f->x.data());
            kSmooth<<<g, kBlock, 0, s>>>(f->n, f->dptr, f->dcol, f->ddiag, f->dval, f->rdiag.data(), b, cur, dst);
            ctx.launched();
            cur = dst;
        }
        xs[l] = cur;
    }
    BSG_CUDA(cudaGetLastError());
}

}  // namespace bsg
