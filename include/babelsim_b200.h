/*
 * babelsim_b200 - C ABI of the B200-native BabelSim finite-volume hot path.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes.  Every
 * entry point returns BSG_OK (0) or a positive error code and records a message
 * readable with bsg_last_error().  No entry point throws across the ABI.
 *
 * The ABI replaces two seams of the reference (midway-official/BabelSim):
 *
 *   1. the linear-system backend, detail::ComputeBackend
 *      (src/internal/compute_backend.h:17-41; PETSc implementation
 *      src/backend/petsc_backend.cpp:123-198) -> bsg_solve_ldu();
 *   2. the equ:: / math:: operator SDK whose face loops live in
 *      src/discretization/{operators,procedural_equation,fvm_execution}.cpp
 *      -> bsg_field_* / bsg_math_* / bsg_equ_* on device-resident fields and
 *      equations, plus the steady SIMPLE driver (src/physics/simple/main.cpp)
 *      -> bsg_simple_*.
 *
 * Numbering: every host array crossing the ABI uses the caller's (reference)
 * cell and face numbering.  Vec3 data are xyz-interleaved (MeshStorage<Vec3>
 * layout, include/babelsim/vector.h); Tensor3 data are 9 doubles per cell,
 * row c = gradient of component c (vector.h Tensor3::rows).
 */
#ifndef BABELSIM_B200_H
#define BABELSIM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
enum {
    BSG_OK = 0,
    BSG_ERR_ARGUMENT = 1,   /* std::invalid_argument in the reference */
    BSG_ERR_CUDA = 2,       /* CUDA runtime failure */
    BSG_ERR_NUMERIC = 3,    /* non-finite coefficient or value */
    BSG_ERR_STATE = 4,      /* std::logic_error in the reference */
    BSG_ERR_MEMORY = 5      /* device allocation or admission refused */
};

/* ---- enumerations: same order as the reference's enums ---------------- */
/* BoundaryType, include/babelsim/field.h:23-32 */
enum { BSG_FIXED_VALUE = 0, BSG_FIXED_GRADIENT = 1, BSG_ZERO_GRADIENT = 2,
       BSG_INLET_OUTLET = 3, BSG_SYMMETRY = 4 };
/* InterpolationMethod / GradientMethod / ConvectionMethod / DiffusionMethod,
 * include/babelsim/methods.h:7-27 */
enum { BSG_INTERP_LINEAR = 0, BSG_INTERP_CORRECTED = 1 };
enum { BSG_GRAD_GREEN_GAUSS = 0, BSG_GRAD_LEAST_SQUARES = 1 };
enum { BSG_CONV_UPWIND = 0, BSG_CONV_LINEAR_UPWIND = 1, BSG_CONV_CENTRAL = 2 };
enum { BSG_DIFF_ORTHOGONAL = 0, BSG_DIFF_CORRECTED = 1, BSG_DIFF_LIMITED_CORRECTED = 2 };
/* TimeMethod, include/babelsim/methods.h:33-37 */
enum { BSG_TIME_STEADY = 0, BSG_TIME_EULER = 1, BSG_TIME_BDF2 = 2 };
/* LinearSolverType / PreconditionerType / SolveStatus,
 * include/babelsim/solver_control.h:12-36 */
enum { BSG_KSP_CG = 0, BSG_KSP_BICGSTAB = 1, BSG_KSP_GMRES = 2, BSG_KSP_FGMRES = 3 };
enum { BSG_PC_NONE = 0, BSG_PC_ICC = 1, BSG_PC_HYPRE = 2, BSG_PC_GAMG = 3,
       BSG_PC_BJACOBI = 4, BSG_PC_ASM = 5, BSG_PC_JACOBI = 6 };
enum { BSG_CONVERGED = 0, BSG_MAX_ITERATIONS = 1, BSG_NUMERICAL_FAILURE = 2 };
/* Precision of the inner Krylov/AMG iterations: all FP64; FP32 CG and FP32
 * V-cycles inside FP64 iterative refinement; or FP64 (flexible) CG with FP32
 * V-cycles.  The acceptance test is the FP64 true residual in every case. */
enum { BSG_PRECISION_FP64 = 0, BSG_PRECISION_FP32_REFINED = 1, BSG_PRECISION_FP32_PRECONDITIONER = 2 };
/* Field locations, include/babelsim/field.h:17-21 */
enum { BSG_CELL = 0, BSG_FACE = 1 };

typedef struct bsg_context bsg_context;
typedef struct bsg_mesh bsg_mesh;
typedef struct bsg_field bsg_field;
typedef struct bsg_equation bsg_equation;
typedef struct bsg_simple bsg_simple;

/* OperatorOptions, include/babelsim/methods.h:31-60.  -1 in a coefficient
 * member means "not set" (std::nullopt). */
typedef struct {
    int32_t interpolation;
    int32_t gradient;
    int32_t convection;
    int32_t diffusion;
    int32_t coefficient_interpolation;
    int32_t coefficient_gradient;
} bsg_options;

/* LinearSolverConfig, include/babelsim/solver_control.h:165-184, plus the
 * precision of the inner iterations: 0 FP64; 1 FP32 inner iterations inside FP64
 * iterative refinement (CG + AMG pressure solves, and the Jacobi BiCGStab solves of
 * momentum and transport equations), the acceptance test always on the FP64
 * residual; 2 FP64 Krylov iterations around an FP32 AMG V-cycle (CG + AMG only;
 * other solvers run in FP64). */
typedef struct {
    int32_t solver;
    int32_t preconditioner;
    double absolute_tolerance;
    double relative_tolerance;
    int32_t max_iterations;
    int32_t warm_start;
    int32_t preconditioner_rebuild_interval;
    double preconditioner_reuse_iteration_growth;
    int32_t amg_max_levels;
    int32_t amg_coarse_size;
    int32_t amg_smoothing_steps;
    int32_t precision;
} bsg_solver_config;

/* SolveResult, include/babelsim/solver_control.h:227-258 */
typedef struct {
    int32_t status;
    int32_t iterations;
    double initial_residual;
    double final_residual;
    double relative_residual;
} bsg_solve_result;

/* Geometry of a mesh as the reference computes it (Mesh::Storage,
 * include/babelsim/mesh.h:138-177; src/core/mesh.cpp:321-564). */
typedef struct {
    int32_t n_cells;
    int32_t n_faces;
    int32_t n_patches;
    const int32_t* face_owner;                  /* n_faces */
    const int32_t* face_neighbour;              /* n_faces, -1 on boundary */
    const int32_t* face_patch;                  /* n_faces, -1 on interior */
    const double* face_area_vectors;            /* 3*n_faces */
    const double* face_centres;                 /* 3*n_faces */
    const double* face_areas;                   /* n_faces */
    const double* face_normals;                 /* 3*n_faces */
    const double* face_owner_weights;           /* n_faces */
    const double* face_orthogonal_coefficients; /* n_faces */
    const double* face_non_orthogonal;          /* 3*n_faces */
    const double* face_skewness;                /* 3*n_faces */
    const double* cell_centres;                 /* 3*n_cells */
    const double* cell_volumes;                 /* n_cells */
    int32_t orthogonal_geometry;
} bsg_mesh_geometry;

/* ---- context ---------------------------------------------------------- */
int bsg_context_create(int32_t device, bsg_context** out);
int bsg_context_destroy(bsg_context* ctx);
/* Message of the last failed call on this context (never NULL). */
const char* bsg_last_error(const bsg_context* ctx);
/* Message of the last failure of a call that had no context to report on. */
const char* bsg_global_error(void);
/* Number of kernels this context has launched so far. */
int bsg_context_launches(const bsg_context* ctx, int64_t* out);
/* Wait for all work of this context. */
int bsg_context_synchronize(bsg_context* ctx);
/* Per-kernel timing: while enabled, instrumented kernels are bracketed by CUDA
 * events on the context's stream.  The report is JSON
 * {"kernel": [launches, total_ms], ...} and clears the records. */
int bsg_context_profile(bsg_context* ctx, int32_t enable);
int bsg_context_profile_report(bsg_context* ctx, char* buffer, int32_t capacity);
/* Phase timeline of the persistent solver kernels: with capacity > 0, each grid
 * barrier appends (phase id, device nanoseconds) until `capacity` entries;
 * capacity 0 turns it off.  Reading returns the entries and clears the log.
 * Phase ids: 1 initial residual, 2 SpMV+dot, 3 update+norm, 4 r.z (and the
 * level-0 post sweep before it), 10+l pre-smoothing of level l, 30+l residual
 * of level l, 100+l restriction to level l+1, 50 coarsest solve, 60+l first
 * post sweep (when a second follows), 80+l last post sweep of level l > 0 with
 * its prolongation into level l-1. */
int bsg_context_phase_log(bsg_context* ctx, int32_t capacity);
int bsg_context_phase_log_read(bsg_context* ctx, int64_t* pairs, int32_t capacity, int32_t* count);
/* CUDA events on the context's stream, for timing a region of calls:
 * record into numbered slots, then read the elapsed milliseconds between two. */
int bsg_context_event_record(bsg_context* ctx, int32_t slot);
int bsg_context_event_elapsed(bsg_context* ctx, int32_t start_slot, int32_t stop_slot, double* ms);

/* ---- mesh --------------------------------------------------------------
 * bsg_mesh_create takes geometry already computed by the caller (the drop-in
 * for a reference Mesh: pass its MeshStorage arrays).
 * bsg_mesh_create_polyhedral computes the geometry itself from a polyhedral
 * description (Mesh::polyhedral, src/core/mesh.cpp:321-564; the
 * BABELSIM_MESH 3 face list, src/io/mesh_reader.cpp:44-111) on the device,
 * bit-identical to the host computation; bsg_mesh_create_polyhedral_host
 * computes the same geometry on the host and uploads it.  Both reject the
 * meshes Mesh::polyhedral rejects, with the same message. */
int bsg_mesh_create(bsg_context* ctx, const bsg_mesh_geometry* geometry, bsg_mesh** out);
int bsg_mesh_create_polyhedral(bsg_context* ctx, int32_t n_vertices, const double* vertices,
                               int32_t n_faces, const int32_t* face_point_offsets,
                               const int32_t* face_point_ids, const int32_t* owner,
                               const int32_t* neighbour, const int32_t* patch, int32_t n_patches,
                               bsg_mesh** out);
int bsg_mesh_create_polyhedral_host(bsg_context* ctx, int32_t n_vertices, const double* vertices,
                                    int32_t n_faces, const int32_t* face_point_offsets,
                                    const int32_t* face_point_ids, const int32_t* owner,
                                    const int32_t* neighbour, const int32_t* patch, int32_t n_patches,
                                    bsg_mesh** out);
/* The reference's mesh file (BABELSIM_MESH 3, readMeshFile, src/io/mesh_reader.cpp:44-111) read
 * natively on the host and built as bsg_mesh_create_polyhedral builds it (geometry on the device).
 * A bad file is rejected with the reference's message, "invalid BabelSim mesh file <path>: ...". */
int bsg_mesh_create_from_file(bsg_context* ctx, const char* path, bsg_mesh** out);
/* Host only: reads and checks a mesh file.  out = {cells, faces, vertices, patches}; when `patches`
 * is given, one "<name> <kind>" line per patch in file order. */
int bsg_mesh_file_info(const char* path, int64_t out[4], char* patches, int32_t capacity);
/* Locality renumbering (no counterpart in the reference, which keeps the file's numbering).
 * Every polyhedral mesh (bsg_mesh_create_polyhedral, _host, _from_file) is renumbered inside
 * the library when its cells are poorly ordered: reverse Cuthill-McKee on the cell graph per
 * connected component (components in the order of their lowest cell), applied when it cuts the
 * mean |i - j| over interior faces more than twofold.  Every array crossing the ABI stays in the
 * caller's numbering.  Host only: the order the library uses, order[internal] = caller cell,
 * and whether it applies (a mesh built from given geometry, bsg_mesh_create, is never
 * renumbered). */
int bsg_mesh_locality_order(int32_t n_cells, int32_t n_faces, const int32_t* owner, const int32_t* neighbour,
                            int32_t* order, int32_t* applied);
int bsg_mesh_destroy(bsg_mesh* mesh);
/* Host-only check of a polyhedral description: computes the geometry exactly as
 * bsg_mesh_create_polyhedral does (no device needed) and reports the first
 * problem the reference's Mesh::polyhedral would reject.  Outputs: cell count
 * and the orthogonal-geometry flag. */
int bsg_mesh_validate_polyhedral(int32_t n_vertices, const double* vertices, int32_t n_faces,
                                 const int32_t* face_point_offsets, const int32_t* face_point_ids,
                                 const int32_t* owner, const int32_t* neighbour, const int32_t* patch,
                                 int32_t n_patches, int32_t* n_cells_out, int32_t* orthogonal_out);
/* Write cell fields in the reference's result format (src/parallel/parallel_writer.cpp:42-171):
 * <time_directory>/rank-0000/<name>.csv, metadata.bs and mesh.geometry, one rank.  Host only:
 * the polyhedral description gives the cell centres and the cell vertex lists; values are in
 * the caller's cell numbering, `components[i]` doubles per cell (1, 3 or 9).  The reference's
 * restart reader (field file `internal file <time_directory>`) and tools read the result. */
int bsg_write_results(const char* time_directory, const char* time_name, int32_t n_vertices,
                      const double* vertices, int32_t n_faces, const int32_t* face_point_offsets,
                      const int32_t* face_point_ids, const int32_t* owner, const int32_t* neighbour,
                      const int32_t* patch, int32_t n_patches, int32_t n_fields, const char* const* names,
                      const int32_t* components, const double* const* values);
/* n_cells, n_faces, n_interior_faces, n_patches, orthogonal flag. */
int bsg_mesh_sizes(const bsg_mesh* mesh, int64_t out[5]);
/* Copy one geometry array (a bsg_mesh_geometry member name, e.g.
 * "face_area_vectors") back to host memory in the caller's numbering. */
int bsg_mesh_export(const bsg_mesh* mesh, const char* name, void* host_out);

/* ---- fields (Field<T>, include/babelsim/field.h:57-374) ----------------
 * components: 1 (scalar), 3 (vector) or 9 (tensor, cell only). */
int bsg_field_create(bsg_mesh* mesh, int32_t location, int32_t components, bsg_field** out);
int bsg_field_destroy(bsg_field* field);
int bsg_field_set_boundary(bsg_field* field, int32_t patch, int32_t type, const double* value);
int bsg_field_upload(bsg_field* field, const double* host_values);
int bsg_field_download(const bsg_field* field, double* host_values);
/* The inletOutlet flux context (Field::setBoundaryFlux, field.h:274-281). */
int bsg_field_set_boundary_flux(bsg_field* field, const bsg_field* face_flux);

/* ---- explicit operators (math::, include/babelsim/math.h:106-180) ------ */
int bsg_math_grad(const bsg_field* in, int32_t gradient_method, bsg_field* out);
int bsg_math_interpolate(const bsg_field* in, const bsg_options* options, bsg_field* out_face);
int bsg_math_flux(bsg_field* velocity, const bsg_options* options, bsg_field* out_face);
int bsg_math_div_flux(const bsg_field* face_flux, bsg_field* out_cell);
int bsg_math_normal_gradient(const bsg_field* in, const bsg_field* gradient,
                             const bsg_options* options, bsg_field* out_face);

/* ---- implicit assembly (equ::, include/babelsim/equ.h:16-101) -----------
 * An equation owns its LDU coefficients on the device; the unknown field
 * supplies layout, boundary constraints and the current iterate. */
int bsg_equation_create(bsg_field* unknown, const bsg_options* options, bsg_equation** out);
int bsg_equation_destroy(bsg_equation* eq);
int bsg_equ_reset(bsg_equation* eq);
int bsg_equ_div(bsg_equation* eq, const bsg_field* flux, double scale, const bsg_options* term);
/* coefficient: a cell or face scalar field, or NULL for the constant k. */
int bsg_equ_laplacian(bsg_equation* eq, const bsg_field* coefficient, double k, double factor,
                      const bsg_options* term);
int bsg_equ_source(bsg_equation* eq, const bsg_field* value, double factor);
/* equ::ddt with explicit time levels (include/babelsim/equ.h:63-70,
 * src/discretization/procedural_equation.cpp:198-223): capacity is a cell scalar
 * field or NULL for the constant c; older may be NULL for Euler; older_dt 0
 * means dt (variable-step BDF2 weights from r = dt/older_dt).  A steady method
 * adds nothing. */
int bsg_equ_ddt(bsg_equation* eq, const bsg_field* capacity, double c, const bsg_field* previous,
                const bsg_field* older, double dt, double older_dt, int32_t method);
/* equ::reaction (equ.h:56-57, procedural_equation.cpp:177-187): diagonal +=
 * factor*coefficient*V, or c*V when coefficient is NULL. */
int bsg_equ_reaction(bsg_equation* eq, const bsg_field* coefficient, double c, double factor);
/* equ::apply / equ::residual (equ.h:79-80, procedural_equation.cpp:281-297):
 * out = A x, or out = b - A x; x and out are cell fields shaped like the unknown. */
int bsg_equ_apply(const bsg_equation* eq, const bsg_field* x, bsg_field* out);
int bsg_equ_residual(const bsg_equation* eq, const bsg_field* x, bsg_field* out);
int bsg_equ_relax(bsg_equation* eq, const bsg_field* previous, double alpha);
int bsg_equ_scale(bsg_equation* eq, double factor);
int bsg_equ_reference_if_unanchored(bsg_equation* eq, double value, int32_t* anchored_out);
int bsg_equ_face_flux(const bsg_equation* eq, const bsg_field* solution, bsg_field* out_face);
/* ||b-Ax|| / max(||Ax||+||b||, 1e-30) (procedural_equation.cpp:429-433). */
int bsg_equ_relative_residual(const bsg_equation* eq, const bsg_field* x, double* out);
int bsg_equ_solve(bsg_equation* eq, const bsg_solver_config* config, bsg_solve_result* results);
/* LDU in the caller's face numbering (DiscreteEquation, discrete_equation.h:14-50). */
int bsg_equ_download(const bsg_equation* eq, double* diagonal, double* upper, double* lower,
                     double* source);

/* ---- linear-system seam (ComputeBackend::solve, compute_backend.h:31-32) --
 * Solves the LDU system given in host memory for 1 or 3 right-hand sides that
 * share one matrix.  x is the initial guess when warm_start and the solution
 * on return; source and x are xyz-interleaved for 3 components.  results gets
 * one entry per component.  The mesh keeps one persistent system per component
 * count for these calls (see bsg_system_solve); a caller with several
 * equations should keep one bsg_system per equation instead. */
int bsg_solve_ldu(bsg_mesh* mesh, const bsg_solver_config* config, int32_t components,
                  const double* diagonal, const double* upper, const double* lower,
                  const double* source, double* x, bsg_solve_result* results);

/* One equation's persistent linear system (PetscLinearSystem,
 * src/backend/petsc_linear_system.cpp; PetscBackend keeps one per equation
 * identity "scalar:<equation>:<field>" / "vector:...", petsc_backend.cpp:201-213).
 * Device buffers, the SELL copy and the AMG structure are made by the first
 * solve and reused by every later one.  Each solve follows updateMatrix /
 * prepare / solveRhs (petsc_linear_system.cpp:257-481): an exactly unchanged
 * matrix is not re-uploaded (a right-hand-side-only solve); an AMG hierarchy is
 * reused (lagged) until preconditioner_rebuild_interval matrix versions or
 * right-hand-side solves have passed since its setup, rebuilt before the next
 * solve after a lagged solve needed more than
 * preconditioner_reuse_iteration_growth times the fresh iterations, and a
 * lagged solve that fails is retried once from the same guess with a fresh
 * hierarchy.  Jacobi-type preconditioners are formed from the current diagonal
 * on every solve (free on the device), so only AMG setups are lagged.  Destroy
 * every system before its mesh. */
typedef struct bsg_system bsg_system;
int bsg_system_create(bsg_mesh* mesh, int32_t components, bsg_system** out);
int bsg_system_destroy(bsg_system* system);
int bsg_system_solve(bsg_system* system, const bsg_solver_config* config, const double* diagonal,
                     const double* upper, const double* lower, const double* source, double* x,
                     bsg_solve_result* results);
/* The EquationPerformanceCounters fields one system fills
 * (include/babelsim/solver_control.h:37-60; PetscBackend::record*,
 * petsc_backend.cpp:228-286); seconds are host wall time of each stage. */
typedef struct {
    uint64_t linear_solves;           /* one per right-hand side */
    uint64_t krylov_iterations;
    uint64_t matrix_value_updates;
    uint64_t rhs_only_solves;
    uint64_t preconditioner_setups;
    uint64_t preconditioner_reuses;
    uint64_t preconditioner_retries;
    uint64_t true_residual_checks;
    double matrix_update_seconds;
    double preconditioner_seconds;
    double solve_seconds;
    int32_t last_status;
    double last_initial_residual;
    double last_final_residual;
    double last_relative_residual;
} bsg_system_counters;
int bsg_system_counters_read(const bsg_system* system, bsg_system_counters* out);

/* ---- allocation-free solve ---------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory while running (an application that owns a fixed device-memory budget
 * or pool, a real-time loop that must not take cudaMalloc's implicit device
 * synchronisation, a host that forbids allocation after start-up): Jacobi-
 * preconditioned CG on a matrix, right-hand side and solution that live in the
 * caller's device memory, with all scratch in a fixed array compiled into the
 * library (each GPU that loads the library holds about 5.4 MB until exit).
 * It calls no cudaMalloc, cudaFree or allocating library routine.
 *
 * Matrix: n rows, diagonal `diag[n]` plus the off-diagonal entries in CSR
 * (`row_ptr[n+1]`, `cols`, `vals`), all device pointers; n <= 131072, larger
 * systems are rejected with BSG_ERR_ARGUMENT.  x (device, n) receives the
 * solution from a zero initial guess; the acceptance contract is the same as
 * bsg_solve_ldu.  Runs on the default stream of the current device and returns
 * when the result is in `result`.  Every call looks up the scratch's device
 * address and uses synchronous copies on the legacy default stream, so no call
 * may be made while a stream of the device is being captured, and data written
 * on other streams must be complete before the call.  All calls
 * share the scratch: calls that overlap on the GPU race, so issue one at a time. */
int bsg_pcg_jacobi_static(int32_t n, const int32_t* row_ptr, const int32_t* cols, const double* diag,
                          const double* vals, const double* b, double* x, double absolute_tolerance,
                          double relative_tolerance, int32_t max_iterations, bsg_solve_result* result);

/* ---- steady SIMPLE (src/physics/simple/main.cpp:11-131) ----------------- */
typedef struct {
    double density;
    double viscosity;                   /* dynamic viscosity (physics "dynamicViscosity") */
    double velocity_relaxation;
    double pressure_relaxation;
    int32_t non_orthogonal_corrections;
    double continuity_tolerance;
    double velocity_tolerance;
    double momentum_tolerance;
    double pressure_correction_tolerance;
    bsg_options momentum;               /* equation.momentum (terms identical) */
    bsg_options pressure;               /* equation.pressureCorrection diffusion term */
    bsg_solver_config momentum_solver;
    bsg_solver_config pressure_solver;
} bsg_simple_config;

typedef struct {
    int32_t iterations;                 /* outer iterations done so far */
    int32_t converged;
    int32_t status;                     /* BSG_CONVERGED / MAX_ITERATIONS / NUMERICAL_FAILURE */
    double mass;                        /* flux-balance relative imbalance */
    double dU, rU, dP;
    double linear_pressure_residual;
    int32_t momentum_iterations;        /* Krylov iterations in the last outer iteration */
    int32_t pressure_iterations;
    double turbulence_change;           /* max relative change of the transported turbulence fields */
    double turbulence_residual;         /* max initial normalised residual of their equations */
} bsg_simple_report;

/* Wilcox-1988m k-omega (src/physics/RANS/k_omega.cpp:25-160): physics keys
 * kOmegaBetaStar/Beta/Gamma/SigmaK/SigmaOmega, kMin, omegaMin,
 * maxTurbulentViscosityRatio; solution keys turbulenceRelaxation and
 * turbulenceTolerance; equation controls kTransport and omegaTransport. */
typedef struct {
    double beta_star, beta, gamma, sigma_k, sigma_omega;
    double k_min, omega_min, max_viscosity_ratio;
    double relaxation;
    double tolerance;
    bsg_options k_transport;
    bsg_options omega_transport;
    bsg_solver_config k_solver;
    bsg_solver_config omega_solver;
} bsg_komega_config;

/* standard k-epsilon (src/physics/RANS/k_epsilon.cpp:25-128): physics keys kEpsilonCmu/C1/C2/
 * SigmaK/SigmaEpsilon, kMin, epsilonMin; equation controls kTransport and epsilonTransport. */
typedef struct {
    double c_mu, c1, c2, sigma_k, sigma_epsilon;
    double k_min, epsilon_min;
    double relaxation;
    double tolerance;
    bsg_options k_transport;
    bsg_options epsilon_transport;
    bsg_solver_config k_solver;
    bsg_solver_config epsilon_solver;
} bsg_kepsilon_config;

/* Spalart-Allmaras (src/physics/RANS/spalart_allmaras.cpp:23-154): physics keys saCb1, saCb2,
 * saSigma, saKappa, saCw1 (<= 0: cb1/kappa^2 + (1 + cb2)/sigma), saCw2, saCw3, saCv1, saCt3, saCt4,
 * saNuTildaMin, saWallDistanceMin; equation control nuTildaTransport. */
typedef struct {
    double cb1, cb2, sigma, kappa, cw1, cw2, cw3, cv1, ct3, ct4;
    double nu_tilda_min, wall_distance_min;
    double relaxation;
    double tolerance;
    bsg_options nu_tilda_transport;
    bsg_solver_config nu_tilda_solver;
} bsg_sa_config;

int bsg_simple_create(bsg_mesh* mesh, const bsg_simple_config* config, bsg_simple** out);
/* Boundary constraint of "U" or "p" on one patch (the case's fields/initial). */
int bsg_simple_set_boundary(bsg_simple* s, const char* field, int32_t patch, int32_t type,
                            const double* value);
/* Initial U (3*n_cells) and p (n_cells); phi becomes flux(U) as in simple/main.cpp:40. */
int bsg_simple_set_fields(bsg_simple* s, const double* U, const double* p);
/* Resume from a saved face flux phi (n_faces) instead of flux(U). */
int bsg_simple_set_flux(bsg_simple* s, const double* phi);
/* Overwrite U, p and phi with host values between outer iterations, keeping
 * every other piece of solver state (the drop-in path whose fields live in
 * host memory copies them in and out around each iteration). */
int bsg_simple_load_state(bsg_simple* s, const double* U, const double* p, const double* phi);
/* Run outer iterations until converged or max_iterations more have been done. */
int bsg_simple_iterate(bsg_simple* s, int32_t max_iterations, bsg_simple_report* report);
/* Block-diagonal batching (no counterpart in the reference, whose unit of work is one case per
 * process, src/runtime/application.cpp:238-272): the mesh is several independent cases
 * concatenated, case k owning cells [cell_offsets[k], cell_offsets[k+1]) (n_segments + 1
 * offsets from 0 to the cell count; no interior face may join two cases; each case has its own
 * patches) with dynamic viscosity viscosity[k].  Every assembly, gradient, flux and update
 * kernel then runs once over all cases, each case's momentum system is solved on its own rows,
 * the pressure systems of all cases are solved in one persistent launch per attempt (each on
 * CTAs of its own, with its own AMG hierarchy and preconditioner lag), and the gauge,
 * diagnostics and convergence tests are per case.  A converged case keeps its converged U, p
 * and phi while the others continue; bsg_simple_iterate stops when every case has converged,
 * and its report's iterations count the batch's outer iterations.  Call after create and
 * before set_fields; laminar, with pressure CG + AMG (precision 0 or 2).  Up to 4096 cases. */
int bsg_simple_set_segments(bsg_simple* s, int32_t n_segments, const int32_t* cell_offsets,
                            const double* viscosity);
/* The report of one case of a batch (its own outer iterations, residuals and status). */
int bsg_simple_segment_report(const bsg_simple* s, int32_t segment, bsg_simple_report* report);
/* turbulenceModel kOmega (src/physics/RANS/model.cpp:24-53): call after create and
 * before set_fields; then "k" and "omega" take boundary conditions through
 * bsg_simple_set_boundary and initial values through set_turbulence_fields. */
int bsg_simple_enable_komega(bsg_simple* s, const bsg_komega_config* config);
/* turbulenceModel kEpsilon: as above, with "k" and "epsilon". */
int bsg_simple_enable_kepsilon(bsg_simple* s, const bsg_kepsilon_config* config);
/* turbulenceModel SA: "nuTilda" takes boundary conditions, set_turbulence_fields takes k = NULL and
 * the initial nuTilda, and the wall distance (n_cells, the reference's wallDistance input field, which
 * it reads and does not compute) must be given before set_fields. */
int bsg_simple_enable_spalart_allmaras(bsg_simple* s, const bsg_sa_config* config);
int bsg_simple_set_wall_distance(bsg_simple* s, const double* wall_distance);
/* initial k and the second transported field (omega, epsilon, or nuTilda with k = NULL) */
int bsg_simple_set_turbulence_fields(bsg_simple* s, const double* k, const double* second);
/* k, the second transported field and the turbulent viscosity mut (n_cells each; NULL skips;
 * k must be NULL for the one-equation model). */
int bsg_simple_get_turbulence_fields(const bsg_simple* s, double* k, double* second, double* mut);
int bsg_simple_get_fields(const bsg_simple* s, double* U, double* p, double* phi);
int bsg_simple_destroy(bsg_simple* s);

/* ---- transient PISO (src/physics/piso/main.cpp:60-301) -------------------
 * Time control follows TimeStepper (src/io/case.cpp:391-403): level k is at
 * start_time + k*delta_t, the last step shortened to end at end_time. */
typedef struct bsg_piso bsg_piso;

typedef struct {
    double density;
    double viscosity;                   /* dynamic viscosity */
    double velocity_relaxation;         /* momentum predictor relaxation (1: none) */
    int32_t max_iterations;             /* predictor-corrector passes per time step */
    int32_t correctors;                 /* nCorrectors */
    int32_t max_correctors;             /* maxCorrectors (>= correctors) */
    double coupling_tolerance;          /* DBL_MAX when unset */
    int32_t non_orthogonal_corrections;
    double continuity_tolerance;
    double velocity_tolerance;
    double momentum_tolerance;
    double pressure_correction_tolerance;
    int32_t time_method;                /* BSG_TIME_EULER or BSG_TIME_BDF2 */
    double start_time;
    double end_time;
    double delta_t;
    bsg_options momentum;
    bsg_options pressure;
    bsg_solver_config momentum_solver;
    bsg_solver_config pressure_solver;
} bsg_piso_config;

typedef struct {
    int32_t steps;                      /* time steps done so far */
    double time;
    int32_t status;                     /* 0 end time reached, 1 running or a step rejected, 2 numerical failure */
    int32_t accepted;                   /* the last step met the continuity and coupling tolerances */
    double mass, dU, rU, dP, coupling;
    double courant_max, courant_mean;
    int32_t correctors;
    int32_t momentum_iterations;
    int32_t pressure_iterations;
    double turbulence_change;           /* dTurb, rTurb of the last turbulence correction */
    double turbulence_residual;
    int32_t turbulence_corrections;     /* turbulence transport solves in the last pass */
} bsg_piso_report;

/* runPiso's turbulence controls (src/physics/piso/main.cpp:99-120). */
typedef struct {
    int32_t coupling;                   /* turbulenceCoupling: 0 iterated, 1 segregated */
    int32_t max_iterations;             /* turbulenceMaxIterations (<= 0: 1000) */
    int32_t correctors;                 /* turbulenceCorrectors (<= 0: the reference's default, max_iterations
                                           with one PISO pass and iterated coupling, else 1) */
} bsg_piso_turbulence_controls;

int bsg_piso_create(bsg_mesh* mesh, const bsg_piso_config* config, bsg_piso** out);
int bsg_piso_set_boundary(bsg_piso* s, const char* field, int32_t patch, int32_t type, const double* value);
/* solution key initializePotentialFlow 1 (src/physics/piso/main.cpp:123-146): call before set_fields;
 * the start then solves laplacian(1) pPrime = div(phi) (homogeneous pressure constraints,
 * initialNonOrthogonalCorrections + 1 solves with corrected diffusion; < 0 takes
 * nonOrthogonalCorrections) and corrects U -= grad(pPrime), phi += its face flux. */
int bsg_piso_initialize_potential_flow(bsg_piso* s, int32_t initial_non_orthogonal_corrections);
/* Initial U (3*n_cells) and p (n_cells); phi becomes flux(U) with the pressure options. */
int bsg_piso_set_fields(bsg_piso* s, const double* U, const double* p);
/* Advance up to `steps` time steps (fewer at end_time or when a step is rejected). */
int bsg_piso_advance(bsg_piso* s, int32_t steps, bsg_piso_report* report);
int bsg_piso_get_fields(const bsg_piso* s, double* U, double* p, double* phi);
/* rans::load in runPiso (piso/main.cpp:98-121): the model of turbulenceModel kOmega, kEpsilon or SA,
 * after create and before set_fields; its fields take boundary conditions through
 * bsg_piso_set_boundary ("k", "omega" / "epsilon" / "nuTilda") and initial values through
 * bsg_piso_set_turbulence_fields (k = NULL for SA); SA needs bsg_piso_set_wall_distance.  Each time
 * step saves the model's histories, the transport equations take the configured time term, and the
 * transport is corrected after the pressure correctors until turbulenceTolerance. */
int bsg_piso_enable_komega(bsg_piso* s, const bsg_komega_config* config, const bsg_piso_turbulence_controls* c);
int bsg_piso_enable_kepsilon(bsg_piso* s, const bsg_kepsilon_config* config, const bsg_piso_turbulence_controls* c);
int bsg_piso_enable_spalart_allmaras(bsg_piso* s, const bsg_sa_config* config,
                                     const bsg_piso_turbulence_controls* c);
int bsg_piso_set_wall_distance(bsg_piso* s, const double* wall_distance);
int bsg_piso_set_turbulence_fields(bsg_piso* s, const double* k, const double* second);
int bsg_piso_get_turbulence_fields(const bsg_piso* s, double* k, double* second, double* mut);
int bsg_piso_destroy(bsg_piso* s);

#ifdef __cplusplus
}
#endif
#endif
