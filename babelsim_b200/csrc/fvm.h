// Device-resident fields and equations, and the finite-volume operators on them.
#pragma once

#include "bsg_internal.h"

#include <memory>
#include <vector>

namespace bsg {

struct BcView;

// OperatorOptions (include/babelsim/methods.h:31-60); -1 = unset.
struct Options {
    int interpolation = 0, gradient = 0, convection = 0, diffusion = 0;
    int coefficient_interpolation = -1, coefficient_gradient = -1;
    int coefInterp() const { return coefficient_interpolation >= 0 ? coefficient_interpolation : interpolation; }
    int coefGrad() const { return coefficient_gradient >= 0 ? coefficient_gradient : gradient; }
};

// Field<T> (include/babelsim/field.h:57-374) on the device.  Cell values are
// C doubles per cell; face values are C doubles per face in internal order
// (interior faces, then boundary faces).
struct DeviceField {
    DeviceMesh* mesh = nullptr;
    int location = 0;   // 0 cell, 1 face
    int comps = 1;
    DeviceArray<double> v;
    std::vector<PatchBC> bcs;
    DeviceArray<PatchBC> d_bcs;
    bool bcs_dirty = true;
    bool calculated = false;
    DeviceArray<double> trace;   // n_boundary*C (calculated fields)
    DeviceArray<double> bflux;   // n_boundary (inletOutlet flux context)
    bool has_flux = false;

    DeviceField(DeviceMesh& m, int loc, int c);
    std::size_t count() const { return location == 0 ? mesh->n_cells : mesh->n_faces; }
    void setBoundary(int patch, int type, const double* value);
    BcView bcView();
    void uploadExternal(const double* host);
    void downloadExternal(double* host) const;
    void setFluxContext(const DeviceField& face_flux);
};

// One frozen diffusion contribution (procedural_equation.cpp:22-31).
struct DiffusionSnapshot {
    DeviceArray<double> kf;          // face diffusivity (n_faces)
    DeviceArray<double> correction;  // frozen explicit correction flux (n_faces)
    std::vector<PatchBC> bcs;        // boundary constraints of the unknown at assembly
    DeviceArray<PatchBC> d_bcs;
    double factor = 0.0;
};

// DiscreteEquation<T> + equ::Equation state (procedural_equation.cpp:15-34).
// Snapshot buffers and the gradient workspace persist across reset(), so an
// outer iteration allocates no device memory.
struct DeviceEquation {
    DeviceField* x = nullptr;
    Options options;
    DeviceArray<double> diag, val, src;
    std::vector<std::unique_ptr<DiffusionSnapshot>> diffusion;  // active contributions
    std::vector<std::unique_ptr<DiffusionSnapshot>> spare;      // recycled buffers
    const DeviceField* boundary_flux = nullptr;
    DeviceArray<double> grad_ws;     // gradient of the unknown, valid for grad_method while assembling
    int grad_method = -1;
    DeviceEquation(DeviceField& unknown, const Options& o);
    void reset();
    std::unique_ptr<DiffusionSnapshot> takeSnapshot();
    // Gradient of the unknown for this assembly (computed once per method).
    const double* unknownGradient(int method);
};

// Reduction workspace: per-block partials + final results in device memory.
struct Reducer {
    DeviceArray<double> partial, result;
    void ensure(int blocks, int nv);
};

// Cell arrays between the caller's numbering (host) and the device's (C values per cell):
// a plain copy, or through the mesh's locality renumbering when it has one.
void uploadCells(DeviceMesh& m, double* device, const double* host, int C);
void downloadCells(DeviceMesh& m, const double* device, double* host, int C);

// ---- explicit operators ---------------------------------------------------
void gradient(DeviceField& x, int method, DeviceArray<double>& out);
void interpolate(DeviceField& x, int interp, int grad, DeviceArray<double>& out_face,
                 DeviceArray<double>* grad_ws = nullptr);
void faceFlux(DeviceField& U, int interp, int grad, DeviceField& out);
void divFlux(const DeviceField& phi, DeviceArray<double>& out);
void normalGradient(DeviceField& x, const double* g, int diffusion, DeviceArray<double>& out_face);
// boundary traces of a computed scalar gradient (fvm_execution.cpp:213-237)
void gradientTrace(DeviceField& x, const double* g, DeviceArray<double>& trace_out);

// ---- implicit assembly -------------------------------------------------------
void addConvection(DeviceEquation& eq, DeviceField& phi, double scale, const Options& o);
void addLaplacian(DeviceEquation& eq, DeviceField* coef, double k, double factor, const Options& o);
void addSource(DeviceEquation& eq, const double* values, double factor);
void relax(DeviceEquation& eq, const double* previous, double alpha);
// Time-derivative weights of equ::ddt (procedural_equation.cpp:198-223); method
// follows TimeMethod (0 steady, 1 Euler, 2 BDF2 with variable step).
struct TimeWeights {
    bool active = false;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
};
TimeWeights timeWeights(int method, double dt, double older_dt, bool have_older);
// capacity: per-cell values (checked by the caller) or nullptr for the constant c.
void addTimeTerm(DeviceEquation& eq, const double* capacity, double c, const double* previous, const double* older,
                 const TimeWeights& t);
// diag += factor * coefficient_i * V_i, or c * V_i when coefficient is nullptr.
void addReaction(DeviceEquation& eq, const double* coefficient, double c, double factor);
// out[0] = any value not positive-finite, out[1] = any value non-finite (synchronises).
void checkValues(Context& ctx, const double* a, long long n, int* flags_dev, int out[2]);
void scale(DeviceEquation& eq, double f);
// Returns through *flag_dev (device int) whether the gauge was applied; host reads if asked.
// With nrows >= 0 only cells [row0, row0 + nrows) are checked and cell row0 is the anchor
// (one segment of a mesh that holds several independent cases).
void referenceIfUnanchored(DeviceEquation& eq, double value, int* flag_dev, int row0 = 0, int nrows = -1);
void applyEquation(const DeviceEquation& eq, const double* x, double* y);
// y = b - A x (procedural_equation.cpp:291-296)
void residualEquation(const DeviceEquation& eq, const double* x, double* y);
void faceFluxEquation(DeviceEquation& eq, const double* solution, DeviceArray<double>& out_face);
// ||b-Ax||, ||Ax||, ||b|| into red.result[0..2] (over cells [row0, row0 + nrows) when nrows >= 0)
void relativeResidualNorms(const DeviceEquation& eq, const double* x, Reducer& red, int row0 = 0, int nrows = -1);

// ---- device reductions and vector helpers ------------------------------------
// l1, l2^2, scale, max over cells [row0, row0 + nrows) (all cells when nrows < 0)
void fluxBalance(DeviceMesh& m, const double* phi, Reducer& red, int row0 = 0, int nrows = -1);
void relativeChangeNorms(Context& ctx, const double* a, const double* b, long long n, Reducer& red);  // |a-b|^2, |a|^2
void copyAsync(Context& ctx, double* dst, const double* src, long long n);
void axpyCell(Context& ctx, double* y, double a, const double* x, long long n);
void subtractScaledGradient(DeviceMesh& m, double* U, const double* rAU, const double* g);
void ratioVolume(DeviceMesh& m, const double* diag, double* rAU);  // rAU = V/diag
void addArrays(Context& ctx, double* out, const double* a, const double* b, long long n);

}  // namespace bsg
