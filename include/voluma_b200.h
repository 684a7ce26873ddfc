/* voluma_b200.h — C ABI of the B200-native pressure-equation hot path.
 *
 * One process per GPU; every call is synchronous with respect to the host unless its
 * name ends in _device (then it is ordered on the context's stream and reads/writes
 * device pointers).  No C++ types, no exceptions cross this boundary: every entry point
 * returns a vlm_status and leaves a message retrievable with vlm_last_error().
 *
 * Reference interfaces replaced (paths inside the Voluma project):
 *   vlm_mesh_register     <- the per-Mesh caches Mesh::cached("GAMG"/"precondFaces")
 *                            (src/fvm/mesh/Mesh.h:118-122, src/fvm/linalg/GAMG.cpp:204,
 *                             src/fvm/linalg/LinearSolver.cpp:52-54) and the Mesh arrays
 *                            owner/neighbour/magSf/nonOrthDeltaCoeffs (Mesh.h:62-73)
 *   vlm_ldu_solve         <- SolverPerformance solveLdu(const LduSystem&, std::vector<scalar>& x,
 *                            const SolverControls&)   (src/fvm/linalg/LinearSolver.h:42,
 *                            LinearSolver.cpp:135-284)
 *   vlm_amul              <- void amul(const LduSystem&, x, y)  (LinearSolver.h:45, .cpp:121-133)
 *   vlm_gamg_apply        <- GamgPreconditioner::apply           (src/fvm/linalg/GAMG.h:63, .cpp:445)
 *   vlm_flow_*            <- IncompressibleFlow::initialize / step (src/fvm/solvers/IncompressibleFlow.cpp)
 *   vlm_precond_apply     <- Preconditioner ctor + apply (none/diagonal/DIC/DILU/GAMG)
 *                            (src/fvm/linalg/LinearSolver.cpp:56-107)
 *   vlm_gamg_levels/_level<- buildHierarchy                      (GAMG.h:57, GAMG.cpp:206-261)
 *   vlm_laplacian         <- fvm::laplacian(gamma, psi, nonOrthCorr) (src/fvm/discretization/Fvm.h:141-182)
 *   vlm_grad              <- fvc::grad (Gauss linear / leastSquares) (src/fvm/discretization/Fvc.h:209-291)
 *   vlm_exact_sum         <- par::ExactSum::add/value            (src/fvm/parallel/Comm.h:42-93, Comm.cpp:107-164)
 *   vlm_div               <- fvc::div(mesh, F)                   (src/fvm/discretization/Fvc.h:294-304)
 *   vlm_pressure_solve    <- the pressure-corrector loop          (src/fvm/solvers/IncompressibleFlow.cpp:322-341)
 *                            = fvm::laplacian + FvMatrix::operator-= + setReference + FvMatrix::solve + flux
 *                            (Fvm.h:141-182, FvMatrix.h:93-97,134-175,210-222)
 */
#ifndef VOLUMA_B200_H
#define VOLUMA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    VLM_OK = 0,
    VLM_ERR_BAD_ARG = 1,      /* invalid pointer/size/name (reference: std::invalid_argument / runtime_error) */
    VLM_ERR_CUDA = 2,         /* CUDA runtime failure */
    VLM_ERR_OOM = 3,          /* device allocation failed / HBM budget exceeded */
    VLM_ERR_SINGULAR = 4,     /* zero pivot in the coarsest GAMG matrix (GAMG.cpp:336) */
    VLM_ERR_NONFINITE = 5,    /* Inf/NaN residual */
    VLM_ERR_TIMEOUT = 6,      /* a bounded device wait gave up */
    VLM_ERR_UNSUPPORTED = 7,  /* unknown solver / preconditioner, PCG on asymmetric (LinearSolver.cpp:76,177,280) */
    VLM_ERR_NO_DEVICE = 8     /* no CUDA device / extension unusable */
} vlm_status;

typedef struct vlm_ctx vlm_ctx;   /* one per host thread; owns a CUDA stream and scratch */
typedef struct vlm_mesh vlm_mesh; /* device-resident addressing, geometry and GAMG hierarchy */

/* Mesh description: the arrays of cfd::Mesh (src/fvm/mesh/Mesh.h:54-109), host pointers.
 * Faces [0, n_internal_faces) are internal (owner < neighbour not required), the rest are
 * boundary faces grouped by patch.  Geometry pointers may be NULL when only solving:
 * magSf and ndc are needed for the GAMG agglomeration weights (GAMG.cpp:215); the rest is
 * needed by vlm_laplacian / vlm_grad. */
typedef struct {
    int32_t n_cells;
    int32_t n_internal_faces;
    int32_t n_faces;
    const int32_t* owner;      /* n_faces */
    const int32_t* neighbour;  /* n_internal_faces */
    const double* magSf;       /* n_faces */
    const double* ndc;         /* n_faces, nonOrthDeltaCoeffs */
    const double* V;           /* n_cells */
    const double* Sf;          /* 3*n_faces */
    const double* d;           /* 3*n_faces, owner->neighbour (boundary: owner->face centre) */
    const double* w;           /* n_faces, linear interpolation weight of the owner */
    const double* corrVecs;    /* 3*n_faces, n - d*ndc */
    int32_t two_d;             /* Mesh::twoD() */
    int32_t empty_dir;         /* Mesh::emptyDir() */
    int32_t n_patches;
    const int32_t* patch_start; /* n_patches, face index of each patch's first face */
    const int32_t* patch_size;  /* n_patches */
    const double* C;            /* 3*n_cells cell centres (optional: linearUpwind / LUST momentum) */
    const double* Cf;           /* 3*n_faces face centres (optional, with C) */
    const double* skewVecs;     /* 3*n_faces, x_f - x'_f (Mesh::skewVecs); optional: NULL = not skewed.  The
                                   device flow step applies the reference's skew corrections when
                                   max |skewVecs|/|d| over internal faces exceeds 1e-8 (Mesh.cpp:596, 617-621) */
} vlm_mesh_desc;

/* Solver dictionary: SolverControls (src/fvm/linalg/LinearSolver.h:15-23) plus additive keys. */
typedef struct {
    char solver[32];          /* "PCG" | "PBiCGStab" | "Jacobi" | "GaussSeidel" | "symGaussSeidel" */
    char preconditioner[32];  /* "GAMG" | "DIC" | "DILU" | "diagonal" | "none" */
    double tolerance;
    double relTol;
    int32_t maxIter;
    int32_t minIter;
    int32_t nSweeps;
    /* ---- additive keys (zero-initialised struct = reference behaviour) ---- */
    char smoother[16];        /* GAMG smoother on the device: "" or "mcgs-jacobi" (level 0 multicolour
                                 Gauss-Seidel, forward colours pre / reversed post; Jacobi on the
                                 coarser levels) | "mcgs" (block-hybrid Gauss-Seidel on the coarser
                                 levels) | "jacobi" (every level) */
    char precision[16];       /* "" or "fp64" | "mixed" (FP32 GAMG V-cycle inside the FP64 PCG
                                 recurrence) | "mixed-dc" (FP32 inner PCG+GAMG inside FP64 defect
                                 correction; with a single reference row - the one row of A with a
                                 non-zero row sum, as setReference leaves it - the inner solve runs on
                                 the pure-Neumann operator with the constant mode projected out and
                                 the correction restores that mode) */
    int32_t reproducible;     /* 1: CFD_REPRODUCIBLE semantics: preconditioner -> diagonal,
                                 GS -> Jacobi, exact (order-independent) global sums */
    int32_t mergeLevels;      /* GAMG pairwise merges per level; 0 -> 2 (GAMG.cpp:96-99) */
    double innerRelTol;       /* mixed precision: inner FP32 solve relative tolerance; 0 -> 1e-4 */
} vlm_solver_ctrl;

/* SolverPerformance (src/fvm/linalg/LinearSolver.h:25-31). */
typedef struct {
    double initialResidual;
    double finalResidual;
    double residualSum;
    double normFactor;
    int32_t iterations;       /* Krylov iterations (mixed: total inner iterations) */
    int32_t converged;
    int32_t outerIterations;  /* mixed precision: FP64 defect-correction passes (else 0) */
    int32_t status;           /* vlm_status of the device solve (NONFINITE, SINGULAR, ...) */
    char solver[32];
} vlm_solver_perf;

/* ------------------------------------------------------------------ context / mesh */
vlm_status vlm_ctx_create(int device, vlm_ctx** out);
vlm_status vlm_ctx_destroy(vlm_ctx* ctx);
const char* vlm_last_error(const vlm_ctx* ctx); /* ctx may be NULL: last error of this thread */
/* Stream the context orders its work on (a cudaStream_t). */
void* vlm_ctx_stream(vlm_ctx* ctx);
/* The context's device name (cudaDeviceProp::name), for per-device tuning tables. */
vlm_status vlm_ctx_device_name(vlm_ctx* ctx, char* name, int32_t capacity);

vlm_status vlm_mesh_register(vlm_ctx* ctx, const vlm_mesh_desc* desc, int32_t merge_levels, vlm_mesh** out);
/* A batch of n_systems independent meshes registered as one device object (batched GAMG-PCG:
 * every kernel of an iteration covers all systems; reductions and convergence stay per system,
 * so each system's result is bit-identical to solving it alone).  Arrays of every entry point on a
 * batch concatenate the systems in order: cells, and internal faces (upper/lower) system after
 * system; face arrays of the assembly calls (gamma, flux) hold every system's internal faces
 * followed by every system's boundary faces; perf outputs have n_systems entries (per pass). */
vlm_status vlm_mesh_register_batch(vlm_ctx* ctx, int32_t n_systems, const vlm_mesh_desc* descs,
                                   int32_t merge_levels, vlm_mesh** out);
/* Registration flags (the _ex forms; 0 = the plain entry points).
 * VLM_MESH_DEVICE_AGGLOMERATION: the GAMG hierarchy is built on the device by a parallel handshake
 * matching of the heaviest couplings (magSf*ndc, GAMG.cpp:215) in place of the reference's
 * sequential pairwise pass (GAMG.cpp:40-94, buildHierarchy): the same level structure, other
 * aggregates (so iteration counts differ from the reference's by the aggregation's quality), for
 * meshes whose registration time matters (serving unseen sizes).  No reference counterpart. */
#define VLM_MESH_DEVICE_AGGLOMERATION 1
vlm_status vlm_mesh_register_ex(vlm_ctx* ctx, const vlm_mesh_desc* desc, int32_t merge_levels, int32_t flags,
                                vlm_mesh** out);
vlm_status vlm_mesh_register_batch_ex(vlm_ctx* ctx, int32_t n_systems, const vlm_mesh_desc* descs,
                                      int32_t merge_levels, int32_t flags, vlm_mesh** out);
vlm_status vlm_mesh_systems(vlm_mesh* mesh, int32_t* n_systems, int64_t* n_cells, int64_t* n_internal_faces,
                            int64_t* n_faces);
vlm_status vlm_mesh_release(vlm_mesh* mesh);

/* ------------------------------------------------------------------ device-side box mesh setup */
/* generateBox (src/fvm/mesh/RawMesh.cpp:391-502, BoxSpec) and the serial Mesh::build geometry
 * (src/fvm/mesh/Mesh.cpp:21-48, 135-153, 239-320, 600-626) computed by kernels on the context's
 * device; the arrays equal the reference's bit for bit.  They come back in host memory as a
 * vlm_mesh_desc (with C, Cf and skewVecs) to pass to vlm_mesh_register; the box owns them. */
typedef struct {
    int32_t n[3];          /* cells per direction */
    double lo[3];
    double hi[3];
    int32_t periodic[3];   /* cyclic pairs merged into internal faces */
    int32_t two_d;         /* n[2] == 1; the z sides become empty and are dropped */
    double beta[3];        /* tanhStretch grading per direction (RawMesh.cpp:387-389); 0 = uniform */
    const double* points;  /* optional: (n0+1)(n1+1)(n2+1)*3 vertex coordinates in generateBox order
                              (host); NULL = the graded box from lo, hi, beta */
} vlm_box_spec;
typedef struct vlm_box vlm_box;
vlm_status vlm_box_create(vlm_ctx* ctx, const vlm_box_spec* spec, vlm_box** out);
/* desc: pointers into the box's arrays (valid until vlm_box_destroy); patches in side order */
vlm_status vlm_box_desc(const vlm_box* box, vlm_mesh_desc* desc);
/* per patch of the desc, its box side: 0 xMin, 1 xMax, 2 yMin, 3 yMax, 4 zMin, 5 zMax */
vlm_status vlm_box_patch_sides(const vlm_box* box, int32_t* sides);
vlm_status vlm_box_destroy(vlm_box* box);

/* ------------------------------------------------------------------ linear algebra */
/* y = A x over the mesh's LDU matrix (host pointers; lower == NULL means symmetric). */
vlm_status vlm_amul(vlm_ctx* ctx, vlm_mesh* mesh, const double* diag, const double* upper,
                    const double* lower, const double* x, double* y);

/* solveLdu: x (in: initial guess, out: solution), host pointers. */
vlm_status vlm_ldu_solve(vlm_ctx* ctx, vlm_mesh* mesh, const double* diag, const double* upper,
                         const double* lower, const double* b, double* x, const vlm_solver_ctrl* ctrl,
                         vlm_solver_perf* perf);
/* Same, device pointers, ordered on vlm_ctx_stream(ctx); perf is written after completion. */
vlm_status vlm_ldu_solve_device(vlm_ctx* ctx, vlm_mesh* mesh, const double* diag, const double* upper,
                                const double* lower, const double* b, double* x, const vlm_solver_ctrl* ctrl,
                                vlm_solver_perf* perf);

/* One GAMG V-cycle w = M^-1 r with the device smoother named in ctrl (host pointers). */
vlm_status vlm_gamg_apply(vlm_ctx* ctx, vlm_mesh* mesh, const double* diag, const double* upper,
                          const double* lower, const double* r, double* w, const vlm_solver_ctrl* ctrl);

/* w = M^-1 r with the preconditioner named in ctrl->preconditioner: "none", "diagonal", "DIC",
 * "DILU" (natural-order factorisation and sweeps, level-scheduled on the device) or "GAMG"
 * (= vlm_gamg_apply).  Host pointers. */
vlm_status vlm_precond_apply(vlm_ctx* ctx, vlm_mesh* mesh, const double* diag, const double* upper,
                             const double* lower, const double* r, double* w, const vlm_solver_ctrl* ctrl);

/* Hierarchy introspection (for parity checks): number of levels, then per level sizes
 * {n, nFaces} and optional copies of l/u (nFaces), agg (n, empty on the coarsest level). */
vlm_status vlm_gamg_levels(vlm_mesh* mesh, int32_t* n_levels);
vlm_status vlm_gamg_level(vlm_mesh* mesh, int32_t level, int32_t* sizes, int32_t* l, int32_t* u, int32_t* agg);
/* Number of colours the device smoother uses on a level. */
vlm_status vlm_gamg_colours(vlm_mesh* mesh, int32_t level, int32_t* n_colours);

/* ------------------------------------------------------------------ assembly */
/* fvm::laplacian(gamma, psi, nonOrthCorr) for a scalar field with per-patch BCs
 * (bc_type[p]: 0 zeroGradient, 1 fixedValue with values bc_values[f - n_internal_faces], 2 symmetry
 * (zeroGradient for a scalar), 5 fixedGradient with the normal gradients in bc_values; other types
 * are rejected with VLM_ERR_BAD_ARG).
 * grad_scheme for the non-orthogonal correction: 0 Gauss linear, 1 leastSquares.
 * Outputs (host): diag[n_cells], upper[n_internal], source[n_cells],
 * internal_coeffs[n_boundary], boundary_source[n_boundary], ffc[n_faces], *has_ffc. */
vlm_status vlm_laplacian(vlm_ctx* ctx, vlm_mesh* mesh, const double* gamma, const double* psi,
                         const int32_t* bc_type, const double* bc_values, int32_t non_orth_corr,
                         int32_t grad_scheme, double* diag, double* upper, double* source,
                         double* internal_coeffs, double* boundary_source, double* ffc, int32_t* has_ffc);

/* fvc::grad of a scalar field, out[3*n_cells]. */
vlm_status vlm_grad(vlm_ctx* ctx, vlm_mesh* mesh, const double* psi, const int32_t* bc_type,
                    const double* bc_values, int32_t scheme, double* out);

/* fvc::div of a face flux (src/fvm/discretization/Fvc.h:294-304): out[n_cells] per unit volume. */
vlm_status vlm_div(vlm_ctx* ctx, vlm_mesh* mesh, const double* face_flux, double* out);

/* The pressure equation of the PISO/SIMPLE corrector (src/fvm/solvers/IncompressibleFlow.cpp:322-341,
 * projectDivergenceFree :62-71): for each of the n_non_orth+1 passes
 *     pEqn = fvm::laplacian(gamma, p) [non-orthogonal correction from grad(p)];  pEqn -= div_phi;
 *     pEqn.setReference(ref_cell, ref_value) (ref_cell < 0: none);  pEqn.solve(ctrl | final_ctrl);
 * with the GAMG-PCG solve on the device, p's boundary values corrected after each solve, and the
 * flux of the last pass (pEqn.flux(), n_faces) written to `flux` when not NULL.
 * gamma: n_faces face diffusivity (rAUf); div_phi: n_cells, per unit volume; p: n_cells in/out;
 * perf: n_non_orth+1 entries.  Host pointers. */
vlm_status vlm_pressure_solve(vlm_ctx* ctx, vlm_mesh* mesh, const double* gamma, const double* div_phi, double* p,
                              const int32_t* bc_type, const double* bc_values, int32_t ref_cell, double ref_value,
                              int32_t n_non_orth, int32_t grad_scheme, const vlm_solver_ctrl* ctrl,
                              const vlm_solver_ctrl* final_ctrl, vlm_solver_perf* perf, double* flux);
/* Batch form: ref_cells[n_systems] (local cell of each system, -1: none); perf[(n_non_orth+1)*n_systems]
 * (pass-major); device_pointers selects device (1) or host (0) arrays. */
vlm_status vlm_pressure_solve_batch(vlm_ctx* ctx, vlm_mesh* mesh, const double* gamma, const double* div_phi,
                                    double* p, const int32_t* bc_type, const double* bc_values,
                                    const int32_t* ref_cells, double ref_value, int32_t n_non_orth,
                                    int32_t grad_scheme, const vlm_solver_ctrl* ctrl, const vlm_solver_ctrl* final_ctrl,
                                    vlm_solver_perf* perf, double* flux, int32_t device_pointers);
/* Same with device pointers, ordered on vlm_ctx_stream(ctx). */
vlm_status vlm_pressure_solve_device(vlm_ctx* ctx, vlm_mesh* mesh, const double* gamma, const double* div_phi,
                                     double* p, const int32_t* bc_type, const double* bc_values, int32_t ref_cell,
                                     double ref_value, int32_t n_non_orth, int32_t grad_scheme,
                                     const vlm_solver_ctrl* ctrl, const vlm_solver_ctrl* final_ctrl,
                                     vlm_solver_perf* perf, double* flux);

/* Kernel launches executed on this mesh so far and its device memory footprint in bytes. */
vlm_status vlm_mesh_stats(vlm_mesh* mesh, int64_t* launches, int64_t* device_bytes);
/* Launch configuration of the coarse V-cycle tail (no reference counterpart: it only shapes
 * launches and leaves every result bit for bit as it is): the levels of at most max_rows rows of a
 * system (and the whole V-cycle of systems of at most full_rows level-0 rows) run in one launch on a
 * thread-block cluster of `cluster` CTAs (1, 2, 4 or 8).  0 keeps a value; row limits left at 0 scale
 * with the cluster.  Set it before the mesh's first solve or flow (recorded graphs are dropped; a
 * flow created before keeps launching the old configuration).  The tuner (voluma_b200/tune.py)
 * picks these per device and mesh size. */
vlm_status vlm_mesh_set_tail(vlm_mesh* mesh, int32_t cluster, int64_t max_rows, int64_t full_rows);
vlm_status vlm_mesh_get_tail(vlm_mesh* mesh, int32_t* cluster, int64_t* max_rows, int64_t* full_rows);
/* Fused launches on the V-cycle's Jacobi levels (no reference counterpart; results bit for bit as
 * unfused): on levels of at most pre_rows rows (all systems of the mesh) both pre-sweeps from zero
 * run as one pass, on levels of at most restrict_rows rows the residual and the restriction, and on
 * levels of at most post_rows rows the prolongation runs inside the first post-sweep.  A negative
 * value keeps a setting; 0 (the default) fuses nowhere.  Same timing rules as vlm_mesh_set_tail. */
vlm_status vlm_mesh_set_fusion(vlm_mesh* mesh, int64_t pre_rows, int64_t restrict_rows, int64_t post_rows);
/* Measurement hook (no reference counterpart): with `on`, the mesh's solves run their launches
 * directly (no graph) with a CUDA event pair around every level-0 smoothing sweep, in the solve's
 * own order; vlm_mesh_sweep_time returns the summed event times (ms) and the number of sweeps since
 * timing was switched on.  Results are unchanged. */
vlm_status vlm_mesh_time_sweeps(vlm_mesh* mesh, int32_t on);
vlm_status vlm_mesh_sweep_time(vlm_mesh* mesh, double* ms_total, int64_t* sweeps);
vlm_status vlm_mesh_get_fusion(vlm_mesh* mesh, int64_t* pre_rows, int64_t* restrict_rows, int64_t* post_rows);
/* Launch shape of the plane-streamed level-0 FP64 product of a box system, planned at registration:
 * pencil height in x-rows, shared-memory plane stages, CTAs; all 0 where it does not apply (more than
 * one system, an x extent not a multiple of 8, fewer than 3 planes, or VLM_BOX_STREAM=0 in the
 * environment at registration), and the four-slot kernel runs instead.  Results are the same bit
 * for bit either way. */
vlm_status vlm_mesh_get_stream(vlm_mesh* mesh, int32_t* pencil_rows, int32_t* stages, int32_t* ctas);
/* Measurement hook: times `reps` launches of one level-0 kernel on the matrix of the last solve
 * ("amul64", "spmv64", "smooth64", "smooth32", "residual64", "residual32"; a smooth launch is one
 * full multicolour sweep; "vcycle32" / "vcycle32_notail" one FP32 V-cycle with / without the
 * coarse tail, "tail32" the tail alone, bytes 0) with CUDA events on the context stream, from a
 * fixed state (right-hand side b, zero iterate).  Each launch is timed on its own after a read of a
 * 256 MB buffer has evicted its operands from the L2 cache; the suffix ":warm" times the launches
 * back to back instead (operands that fit stay in L2).  Outputs the mean ms per launch and the
 * algorithmic bytes of one launch (values + int32 addressing, each array once). */
vlm_status vlm_profile_kernel(vlm_ctx* ctx, vlm_mesh* mesh, const char* kernel, int32_t reps, double* ms,
                              double* bytes);

/* ------------------------------------------------------------------ host-only topology */
/* The GAMG agglomeration hierarchy and the smoother colouring the device uses, built on the
 * host without touching a GPU (buildHierarchy, src/fvm/linalg/GAMG.cpp:206-261).  */
typedef struct vlm_topology vlm_topology;
vlm_status vlm_topology_build(int32_t n_cells, int32_t n_internal_faces, const int32_t* owner,
                              const int32_t* neighbour, const double* magSf, const double* ndc,
                              int32_t merge_levels, vlm_topology** out);
vlm_status vlm_topology_levels(const vlm_topology* t, int32_t* n_levels);
/* sizes: {n, nFaces, len(agg), nColours}; any output may be NULL */
vlm_status vlm_topology_level(const vlm_topology* t, int32_t level, int32_t* sizes, int32_t* l, int32_t* u,
                              double* weight, int32_t* agg, int32_t* face_map, int8_t* face_flip,
                              int32_t* colour);
/* Whether the mesh is a generateBox mesh (src/fvm/mesh/RawMesh.cpp:391-502), read from its face
 * arrays: shape = {nx, ny, nz, periodic x, y, z, box layout}; nx = 0 when it is not a box.  The
 * last entry is 1 when level 0 of its solves runs the structured box kernels (every periodic extent
 * even and the natural-order colouring red-black).  No reference counterpart: the reference has no
 * structured path. */
vlm_status vlm_topology_box(const vlm_topology* t, int32_t* shape);
vlm_status vlm_topology_destroy(vlm_topology* t);

/* ------------------------------------------------------------------ failure detection */
/* Self-test of the bounded group barrier that the level-scheduled DIC/DILU and Gauss-Seidel kernels
 * use when one system spans several CTAs (no reference counterpart: the reference is serial).  Runs
 * `ctas` co-resident CTAs (1..64) through `rounds` barriers with each wait limited to `spin_limit`
 * polls; CTA `absent_cta` (when in range; -1 for none) returns before its first arrival, so the other
 * CTAs' wait runs out.  *barrier_status: 0, or VLM_ERR_TIMEOUT when a wait gave up (the kernel still
 * ends, and the context stays usable); passed[b]: barriers CTA b passed before that. */
vlm_status vlm_barrier_check(vlm_ctx* ctx, int32_t ctas, int64_t spin_limit, int32_t absent_cta, int32_t rounds,
                             int32_t* passed, int32_t* barrier_status);

/* ------------------------------------------------------------------ reductions */
/* Order-independent exact sum of n doubles on the device (host pointer in, host result). */
vlm_status vlm_exact_sum(vlm_ctx* ctx, const double* values, int64_t n, double* out);

/* ------------------------------------------------------------------ incompressible step */
/* IncompressibleFlow::step (src/fvm/solvers/IncompressibleFlow.cpp:138-370) on the device, for laminar
 * flow: momentum assembly (fvm::ddt + fvm::div(phi, U) - fvm::laplacian(nu, U), Fvm.h:18-182),
 * FvMatrix::relax (FvMatrix.h:111-131), the momentum predictor, A/H/HbyA and the Rhie-Chow flux
 * phiHbyA (IncompressibleFlow.cpp:244-292), the pressure equation with its non-orthogonal correctors,
 * the explicit pressure relaxation and U = HbyA - rAU grad p.  The mesh must be a single system
 * registered with geometry (and C / Cf for linearUpwind or LUST); it must outlive the flow.
 * Boundary conditions per patch: 0 zeroGradient, 1 fixedValue (noSlip = fixedValue 0), 2 symmetry
 * (slip plane, SymmetryBC of field/BoundaryCondition.h:194-205: U_b = U_P - (n.U_P) n with the
 * normal part implicit and zero flux; for p the same as zeroGradient), 3 inletOutlet for U
 * (InletOutletBC, BoundaryCondition.h:263-287: inlet value u_value where the face flux at the start
 * of the step is inflow, zeroGradient elsewhere; the flux is not fixed), 4 freestream (U: value
 * fraction 1/2 - (U_inf.n)/(2|U_inf|) towards u_value = U_inf, BoundaryCondition.h:289-302; p:
 * freestreamPressure towards p_value with fraction 1/2 + (U_inf.n)/(2|U_inf|), U_inf from the U
 * freestream condition of the same patch, :304-320), 5 fixedGradient (the value is the normal
 * gradient, :140-153), 6 pressureInletOutletVelocity for U (u_value = the tangential inflow
 * velocity, :343-364) and fixedFluxPressure for p (the gradient that makes the boundary flux the
 * boundary velocity's, set every corrector, :155-163 and IncompressibleFlow.cpp:17-29), 7
 * totalPressure for p (p_value = p0; p0 - |U_b|^2/2 on inflow faces, set at each step start,
 * :325-341), 8 Robin a phi + b dphi/dn = c (:166-192, coefficients in vlm_flow_ctrl u_robin /
 * p_robin; it fixes the value when a != 0), 9 advective for U (AdvectiveBC, :389-414 and
 * field/VolField.h:235-264: the outflow wave equation dU/dt + U_n dU/dn = 0 discretised with the
 * step's Euler / backward coefficients, a mixed condition with value fraction c / (c + U_n dc) towards
 * the boundary's own history; zero gradient when steady; optional far-field relaxation in
 * vlm_flow_ctrl u_advective).  Patch
 * values are uniform; vlm_flow_set_boundary_values sets the fixedValue
 * and inletOutlet values face by face (profiles such as a parabolic inlet).
 * In CFD_REPRODUCIBLE mode (reproducible = 1 in all three solver controls) a step reproduces the
 * reference's fields bit for bit. */
typedef struct vlm_flow vlm_flow;

typedef struct {
    double nu;                   /* kinematic viscosity */
    int32_t steady;              /* 1: SIMPLE (steadyState) */
    int32_t div_scheme;          /* 0 upwind, 1 linear, 2 linearUpwind, 3 LUST, 4 limitedLinear (k = div_coeff),
                                    5 vanLeer, 6 MUSCL, 7 minmod (Schemes.h:15-39, Fvm.h:47-72) */
    int32_t ddt_scheme;          /* 0 steadyState, 1 Euler, 2 backward */
    int32_t n_outer, n_corr, n_non_orth_corr, momentum_predictor; /* PimpleControls */
    double alpha_u, alpha_p;
    int32_t p_ref_cell;
    double p_ref_value;
    vlm_solver_ctrl U, p, p_final;
    double div_coeff;            /* limitedLinear's k ("limitedLinear k"); 0 -> 1 */
    int32_t grad_scheme;         /* IncompressibleFlow::gradScheme, also the mesh default (Mesh::setGradScheme)
                                    that fvm::div and the laplacians' non-orthogonal correction use:
                                    0 Gauss linear, 1 leastSquares */
    int32_t grad_p_scheme;       /* IncompressibleFlow::gradPScheme (momentum source, U correction):
                                    0 Gauss linear, 1 leastSquares, 2 GaussSkew (Fvc.h:233-262) */
    const double* u_robin;       /* boundary type 8, Robin a U + b dU/dn = c (RobinBC, field/BoundaryCondition.h:
                                    166-192): {a, b} per patch (host array, 2 x patches), c = the patch's
                                    u_value; NULL when no U patch is Robin */
    const double* p_robin;       /* the same for p: {a, b} per patch, c = p_value; NULL when none */
    const double* u_advective;   /* boundary type 9: {lInf, fieldInf x, y, z} per patch (host array, 4 x
                                    patches); lInf > 0 relaxes towards fieldInf over the length lInf
                                    (AdvectiveBC's fieldInf / lInf), lInf = 0 none; NULL: no far field */
} vlm_flow_ctrl;

typedef struct {
    double UInitialResidual, pInitialResidual, continuityError; /* StepInfo */
    int32_t iterations;          /* linear-solver iterations of the step */
    int32_t launches;            /* kernels the step ran (graph kernel nodes included) */
} vlm_step_info;

vlm_status vlm_flow_create(vlm_ctx* ctx, vlm_mesh* mesh, const vlm_flow_ctrl* ctrl, const int32_t* u_type,
                           const double* u_value, const int32_t* p_type, const double* p_value, vlm_flow** out);
/* IncompressibleFlow::initialize from host fields: U 3 per cell (NULL: keep), p per cell (NULL: keep). */
vlm_status vlm_flow_set_state(vlm_flow* flow, const double* U, const double* p);
/* Face-by-face boundary values (FixedValueBC::values, InletOutletBC refValue): u_face 3 per boundary
 * face (index f - n_internal_faces) for the fixedValue and inletOutlet U patches, p_face 1 per
 * boundary face for the fixedValue p patches; faces of other patches are ignored; NULL keeps. */
vlm_status vlm_flow_set_boundary_values(vlm_flow* flow, const double* u_face, const double* p_face);
/* One IncompressibleFlow::step(dt) (dt ignored when steady). */
vlm_status vlm_flow_step(vlm_flow* flow, double dt, vlm_step_info* info);
/* The steady loop of fvmFlow (apps/fvmFlow/fvmFlow.cpp:611-640): steps until U and p residuals are
 * below residual_tol (from the second iteration) or max_iter; *iterations = steps taken. */
vlm_status vlm_flow_run_steady(vlm_flow* flow, int32_t max_iter, double residual_tol, int32_t* iterations,
                               vlm_step_info* last);
/* Kernels run by the flow so far (all steps). */
int64_t vlm_flow_launches(vlm_flow* flow);
vlm_status vlm_flow_get_state(vlm_flow* flow, double* U, double* p, double* phi);
vlm_status vlm_flow_destroy(vlm_flow* flow);

/* Turbulence model and momentum forcing of a flow: the LES Smagorinsky model with optional Van
 * Driest damping (TurbulenceModel::correct, TurbulenceModel.cpp:226-250; LESModel::correctModel,
 * LESModels.cpp:64-153; Smagorinsky::nutCell, LESModels.cpp:274-287) and the momentum forcing of
 * IncompressibleFlow (MomentumForcing, IncompressibleFlow.h:40-47; the source terms at
 * IncompressibleFlow.cpp:186-202 and applyForcingCorrection, :115-142).  Set before the first step
 * (vlm_flow_set_model replaces IncompressibleFlow.updateTurbulence and .forcing). */
typedef struct vlm_flow_model {
    int32_t les;               /* 0 laminar, 1 Smagorinsky */
    double Cs;                 /* Smagorinsky constant (coeffs.Cs, 0.17) */
    int32_t van_driest;        /* damp the filter width near walls (vanDriest) */
    double Aplus, Cdelta;      /* Van Driest constants (coeffs.Aplus 26, coeffs.Cdelta 0.158) */
    double kappa;              /* von Karman constant (coeffs.kappa 0.41) */
    double delta_coeff;        /* filter width = delta_coeff * cbrt(V) (coeffs.deltaCoeff 1) */
    double nut_max_ratio;      /* nu_t is limited to nut_max_ratio * nu (nutMaxRatio 1e5) */
    double depth;              /* 2D meshes: extent in the empty direction (filter width sqrt(V / depth)) */
    const int32_t* wall_patch; /* per mesh patch: 1 = wall (PatchType::Wall), else 0; may be NULL (no walls) */
    int32_t forcing;           /* 0 none, 1 constant body force, 2 mean velocity */
    double force[3];           /* constant: force per unit mass */
    double Ubar[3];            /* mean velocity: target volume-averaged velocity */
    double relaxation;         /* mean velocity: gain of the pressure-gradient update (1) */
    double grad_p;             /* mean velocity: initial driving pressure gradient (0) */
} vlm_flow_model;

vlm_status vlm_flow_set_model(vlm_flow* flow, const vlm_flow_model* model);

/* Restart snapshot in the reference's format (restart::write / restart::read, io/Restart.cpp:105-190):
 * a directory with one binary file per array (U.bin, p.bin, phi.bin, the old time levels U_0 / U_00 /
 * phi_0 / phi_00 when the flow has them, nut.bin with a turbulence model; each an 8-byte magic
 * "CFDRST01", the count and the number of components, then the doubles in cell or face order) and
 * state.txt (time, dt, dt0, timeIndex, nOldTimes, gradP).  Files written by either side are read by
 * the other.  Set the model (vlm_flow_set_model) before reading; *found is 0 when dir has no
 * state.txt (nothing read).  A file that does not match the mesh is BAD_ARG. */
vlm_status vlm_flow_write_restart(vlm_flow* flow, const char* dir);
vlm_status vlm_flow_read_restart(vlm_flow* flow, const char* dir, int32_t* found);
/* nu_t per cell (nCells, of the last step's last outer pass) and the mean-velocity driving pressure
 * gradient; either pointer may be NULL. */
vlm_status vlm_flow_get_model_state(vlm_flow* flow, double* nut, double* grad_p);

/* ------------------------------------------------------------------ serving */
/* Continuous batching of incompressible solves on one device (no counterpart in the reference,
 * which runs one case per process): requests are admitted in arrival order when a slot is free and
 * their device-memory estimate fits in the unused HBM budget, run concurrently on their own
 * streams, keep all their state on the device until they finish, and give the same result alone
 * and in any mix. */
typedef struct vlm_server vlm_server;

typedef struct {
    const vlm_mesh_desc* mesh;  /* with geometry; copied at submission */
    const vlm_flow_ctrl* ctrl;  /* copied; ctrl->steady selects the steady loop or n_steps of dt */
    const int32_t* u_type;      /* per patch (copied) */
    const double* u_value;
    const int32_t* p_type;
    const double* p_value;
    const double* U0;           /* initial fields, 3 per cell / per cell (NULL: zero) */
    const double* p0;
    int32_t n_steps;            /* transient */
    double dt;
    int32_t max_iter;           /* steady: SIMPLE iteration cap */
    double residual_tol;        /* steady: convergence tolerance (fvmFlow residualTol) */
    double arrival;             /* server clock (s) at which the request arrives */
    int64_t device_bytes;       /* admission estimate (0: vlm_flow_request_bytes) */
    int32_t mesh_flags;         /* registration flags of the request's mesh (vlm_mesh_register_ex): 0, or
                                   VLM_MESH_DEVICE_AGGLOMERATION to build its GAMG hierarchy on the device */
} vlm_flow_request;

typedef struct {
    int64_t id;
    int32_t status;             /* VLM_OK, VLM_ERR_OOM (larger than the budget), or the failing call's status */
    int32_t iterations;         /* SIMPLE iterations / transient steps */
    double arrival, admitted, finished; /* server clock (s) */
    double UInitialResidual, pInitialResidual, continuityError; /* last step */
    int64_t device_bytes;       /* admission estimate used */
    int64_t launches;           /* kernels run for this request */
} vlm_flow_result;

int64_t vlm_flow_request_bytes(int32_t n_cells, int32_t n_faces);
vlm_status vlm_server_create(int32_t device, int64_t hbm_budget, int32_t max_active, vlm_server** out);
double vlm_server_clock(vlm_server* server);
vlm_status vlm_server_submit(vlm_server* server, const vlm_flow_request* request, int64_t* id);
/* Finished results in completion order (waits up to timeout seconds when none is ready). */
vlm_status vlm_server_collect(vlm_server* server, vlm_flow_result* out, int32_t capacity, int32_t* n, double timeout);
/* Final U (3 per cell), p and phi of a finished request (any pointer may be NULL). */
vlm_status vlm_server_result_fields(vlm_server* server, int64_t id, double* U, double* p, double* phi);
/* Stops admitting, finishes the requests already running, frees everything. */
vlm_status vlm_server_destroy(vlm_server* server);

/* Exact sum that allocates no device memory.  No counterpart in the reference.  For callers that
 * cannot call cudaMalloc where they need the sum (device memory owned by their own pool or fixed
 * budget; loops where an allocate/free pair would synchronise the device).  values and out are
 * device pointers; the work is ordered on `stream` (a cudaStream_t, NULL = default stream) and the
 * call returns before it completes.  Scratch: one fixed 299,016-byte __device__ array per device,
 * held until the process exits and shared by all calls; calls that overlap on the GPU race on it,
 * so order them on one stream.  The first call on a device looks the array up; every call clears
 * its counter on `stream` before the sum.  n <= 2^31-1, else VLM_ERR_BAD_ARG; the
 * message is available from vlm_last_error(NULL). */
vlm_status vlm_exact_sum_noalloc(const double* values, int64_t n, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VOLUMA_B200_H */
