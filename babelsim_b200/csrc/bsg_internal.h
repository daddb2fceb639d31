// Internal structures shared by the host runtime and the sm_100a kernels.
//
// Device layout (all FP64 unless stated, all resident in HBM):
//   cells      : V[N], rV[N] = 1/V, xc[3N] (xyz interleaved)
//   interior   : faces [0, Fi) sorted by owner; own[Fi], nbr[Fi], w[Fi], dcoef[Fi],
//                area[Fi], Sf/xf/kvec/skew[3Fi]
//   boundary   : faces [0, Fb) sorted by owner; bown[Fb], bpatch[Fb], bdcoef[Fb],
//                barea[Fb], bdist[Fb] = (xf-xc).n, bSf/bxf/bn/bk[3Fb]
//   cell->face : cf_ptr[N+1], cf_face[2Fi] (interior face id), cf_col[2Fi]
//                (the other cell); cb_ptr[N+1] (boundary faces of a cell are the
//                contiguous range [cb_ptr[i], cb_ptr[i+1]))
// A matrix is "diagonal + off-diagonal CSR" on the cell->face pattern: diag[N]
// and val[2Fi] with val[k] the coefficient of cf_col[k] in row i.  Every
// interior face owns exactly two slots (one per side), so face-based and
// row-based assembly are both atomic-free and a repeated owner/neighbour pair
// (two faces between the same cells) simply keeps two slots.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace bsg {

enum Status { kOk = 0, kArgument = 1, kCuda = 2, kNumeric = 3, kState = 4, kMemory = 5 };

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& message) { throw Error(code, message); }

inline void checkCuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(kCuda, std::string(what) + ": " + cudaGetErrorString(e));
}
#define BSG_CUDA(call) ::bsg::checkCuda((call), #call)

// Owning device allocation.
template <class T>
class DeviceArray {
public:
    DeviceArray() = default;
    explicit DeviceArray(std::size_t n) { resize(n); }
    ~DeviceArray() { release(); }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    DeviceArray(DeviceArray&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DeviceArray& operator=(DeviceArray&& o) noexcept {
        if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    void resize(std::size_t n) {
        if (n == n_) return;
        release();
        if (n) {
            cudaError_t e = cudaMalloc(&p_, n * sizeof(T));
            if (e != cudaSuccess) {
                p_ = nullptr;
                fail(kMemory, "device allocation of " + std::to_string(n * sizeof(T)) + " bytes failed: " +
                                  cudaGetErrorString(e));
            }
        }
        n_ = n;
    }
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    T* data() { return p_; }
    const T* data() const { return p_; }
    std::size_t size() const { return n_; }
    void upload(const T* host, std::size_t n, cudaStream_t s) {
        resize(n);
        if (n) BSG_CUDA(cudaMemcpyAsync(p_, host, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& v, cudaStream_t s) { upload(v.data(), v.size(), s); }
    void download(T* host, cudaStream_t s) const {
        if (n_) BSG_CUDA(cudaMemcpyAsync(host, p_, n_ * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    void zero(cudaStream_t s) {
        if (n_) BSG_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
    }

private:
    T* p_ = nullptr;
    std::size_t n_ = 0;
};

// One device, one stream, a launch counter, pinned scratch for scalars read
// back by the host, and optional per-kernel CUDA-event timing.
// Barrier of one group of CTAs in a persistent solver launch (set by
// resetBarriers before the launch): the arrival count, whose top bit flips once
// per phase; the flag a wait that ran past its bound sets, with what that wait
// saw; and where each CTA of the launch last arrived.
struct SegmentBarrier {
    unsigned count;
    int abort;
    int who;              // 1 + grid rank of the first CTA whose wait ran out (0: none)
    unsigned where;       // that CTA's barrier number (1 = its first barrier)
    unsigned seen;        // the count word it last read
    int cta0, ncta;       // the group's CTAs (grid ranks)
    int pad;
    unsigned* progress;   // per CTA of the launch (grid rank): number of its latest barrier; may be null
};

constexpr int kMaxPersistentCtas = 8192;  // CTAs of one persistent launch, at most

struct Context;
// Sets `n` device barriers to their launch state (no arrivals, no abort, progress
// recorded in ctx.progress, whose first `ctas` entries are zeroed), in stream order.
// Barrier k covers CTAs [cta_begin[k], cta_begin[k+1]); without cta_begin, the one
// barrier covers all `ctas`.
void resetBarriers(Context& ctx, SegmentBarrier* dev, int n, int ctas, const int* cta_begin = nullptr);
// After a launch reported status 3 (the stream synchronised): which CTAs of the
// barrier's group stopped where, for the error message.
std::string barrierReport(const SegmentBarrier* dev);
// The same for the first of `n` barriers of a batched launch whose wait ran out.
std::string barrierReport(const SegmentBarrier* dev, int n);

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 148;
    long long launches = 0;
    std::string last_error;
    double* pinned = nullptr;            // 64 doubles of pinned host memory
    SegmentBarrier* grid_barrier = nullptr;  // device: the barrier of whole-grid persistent launches
    unsigned* progress = nullptr;            // device, kMaxPersistentCtas: barrier numbers per CTA
    // Per-kernel timing: while `profiling`, every instrumented launch is
    // bracketed by two events on `stream`; profileReport() resolves them.
    bool profiling = false;
    struct Record { const char* name; cudaEvent_t start, stop; };
    std::vector<Record> records;
    std::vector<cudaEvent_t> event_pool;
    std::vector<cudaEvent_t> user_events;  // bsg_context_event_record slots
    // Algorithmic bytes and work units (e.g. Krylov iterations) that instrumented
    // launches declare while profiling; reported beside their timings.
    struct Note { const char* name; double bytes, units; };
    std::vector<Note> notes;
    void profileNote(const char* name, double bytes, double units) {
        if (profiling) notes.push_back({name, bytes, units});
    }
    // Phase timeline of persistent kernels (device memory, enabled on request).
    long long* phase_entries = nullptr;
    int* phase_count = nullptr;
    int phase_capacity = 0;
    explicit Context(int dev);
    ~Context();
    void sync() { BSG_CUDA(cudaStreamSynchronize(stream)); }
    void launched() { ++launches; }
    cudaEvent_t takeEvent();
    // JSON {"name": [launches, total_ms, algorithmic_bytes, units], ...}; clears the records
    std::string profileReport();
};

// Brackets the launches issued in its scope with timing events when profiling.
class ProfileScope {
public:
    ProfileScope(Context& ctx, const char* name) : ctx_(ctx) {
        if (ctx.profiling) {
            rec_ = {name, ctx.takeEvent(), ctx.takeEvent()};
            checkCuda(cudaEventRecord(rec_.start, ctx.stream), "cudaEventRecord");
        }
    }
    ~ProfileScope() {
        if (ctx_.profiling && rec_.start) {
            cudaEventRecord(rec_.stop, ctx_.stream);
            ctx_.records.push_back(rec_);
        }
    }

private:
    Context& ctx_;
    Context::Record rec_{nullptr, nullptr, nullptr};
};
#define BSG_PROFILE(ctx, name) ::bsg::ProfileScope bsg_profile_scope_((ctx), (name))

// Per-patch boundary constraint as seen by the kernels.
struct PatchBC {
    int type;
    double value[3];
};

// Device geometry and connectivity (see the layout note at the top).
struct DeviceMesh {
    Context* ctx = nullptr;
    int n_cells = 0, n_faces = 0, n_interior = 0, n_boundary = 0, n_patches = 0;
    bool orthogonal = true;
    // caller numbering <-> internal numbering
    std::vector<int> face_kind;          // per external face: 0 interior, 1 boundary
    std::vector<int> face_slot;          // per external face: index in interior or boundary list
    std::vector<int> interior_ext, boundary_ext;
    DeviceArray<int> face_perm;          // caller face -> internal position (interior faces first)
    // caller cell -> internal cell when the cells were renumbered for locality (empty: the
    // caller's numbering is kept); cell arrays crossing the ABI go through cell_stage
    std::vector<int> h_cell_perm;
    DeviceArray<int> cell_perm;
    DeviceArray<double> cell_stage;
    DeviceArray<double> face_stage;      // staging for face fields crossing the ABI
    // host copies kept for setup work (AMG aggregation, exports)
    std::vector<int> h_own, h_nbr, h_cf_ptr, h_cf_col, h_cf_face, h_bown, h_cb_ptr;
    // device arrays
    DeviceArray<double> V, rV, xc;
    DeviceArray<int> own, nbr;
    DeviceArray<double> w, dcoef, area, Sf, xf, kvec, skew;
    DeviceArray<int> bown, bpatch;
    DeviceArray<double> bdcoef, barea, bdist, bSf, bxf, bn, bk;
    DeviceArray<int> cf_ptr, cf_face, cf_col, cb_ptr;
    // the two matrix slots of each interior face: owner row (upper) and neighbour row (lower)
    std::vector<int> h_slot_own, h_slot_nbr;
    DeviceArray<int> slot_own, slot_nbr;
    // scratch for the first Green-Gauss pass (3*9*n_cells doubles at most)
    DeviceArray<double> ws_grad_pass1;
    // per cell, for a mesh that holds several independent cases (a batch): 1 where the cell's
    // case has orthogonal geometry, so the second Green-Gauss pass leaves its cells alone as a
    // solo run of that case would; empty when the mesh's own flag applies to every cell
    DeviceArray<unsigned char> cell_orth;
    // per-slot records of the face pass of diffusion assembly ((1 + C) * 2 n_interior doubles)
    DeviceArray<double> ws_slots;
    // external geometry copy for bsg_mesh_export (host; filled on first export when the
    // geometry was computed on the device)
    std::vector<double> ext_Sf, ext_xf, ext_area, ext_n, ext_w, ext_dcoef, ext_k, ext_skew, ext_xc, ext_V;
    std::vector<int> ext_owner, ext_nbr, ext_patch;
};

// Mesh geometry as the caller supplies it (mirrors bsg_mesh_geometry).
struct HostGeometry {
    int n_cells = 0, n_faces = 0, n_patches = 0;
    std::vector<int> owner, nbr, patch;
    std::vector<double> Sf, xf, area, normal, weight, dcoef, kvec, skew, xc, V;
    bool orthogonal = true;
};

// Mesh::polyhedral geometry (src/core/mesh.cpp:321-564), computed on the host.
HostGeometry computePolyhedralGeometry(int n_vertices, const double* vertices, int n_faces,
                                       const int* face_point_offsets, const int* face_point_ids,
                                       const int* owner, const int* neighbour, const int* patch,
                                       int n_patches);
std::unique_ptr<DeviceMesh> buildDeviceMesh(Context& ctx, const HostGeometry& g);
// The integer checks of Mesh::polyhedral's input; returns the cell count.
int validatePolyhedralTopology(int n_vertices, int n_faces, const int* offsets, const int* ids, const int* owner,
                               const int* neighbour, const int* patch, int n_patches);
// Internal face order, cell->face lists and matrix slots (host counting passes, then uploaded).
void buildTopology(DeviceMesh& m, Context& ctx, int n_cells, int n_faces, int n_patches, const int* owner,
                   const int* neighbour, const int* patch);
// Mesh::polyhedral with the geometry computed on the device, bit-identical to
// computePolyhedralGeometry (geometry.cu).
std::unique_ptr<DeviceMesh> buildDeviceMeshPolyhedral(Context& ctx, int n_vertices, const double* vertices,
                                                      int n_faces, const int* offsets, const int* ids,
                                                      const int* owner, const int* neighbour, const int* patch,
                                                      int n_patches);
// Fills the caller-numbered host geometry (ext_*) from the device arrays if it is absent.
void ensureExternalGeometry(DeviceMesh& m);

// Launch helpers.
inline unsigned gridFor(long long n, int block) {
    long long g = (n + block - 1) / block;
    return static_cast<unsigned>(g < 1 ? 1 : g);
}

}  // namespace bsg
