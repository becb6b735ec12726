/*
 * chuanflow_b200 -- C ABI of the B200 (sm_100a) implementation of ChuanFlow's
 * 3D unstructured finite-volume SIMPLE path.
 *
 * Conventions
 *   - every entry point returns an int status: CFG_OK (0) or a CFG_E* code;
 *     cfg_last_error() gives the message of the last failure on the calling
 *     thread.  No C++ exception crosses this boundary.
 *   - meshes and contexts are opaque handles; a context owns all device
 *     memory of one case on one device and one CUDA stream, and is confined
 *     to the thread that uses it (no global mutable state is shared).
 *   - indices on this boundary are int64 (the reference's `label`), reals
 *     are double (its `scalar`); vectors are packed xyz triples.
 *   - host pointers unless the name says `_dev`.
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the ChuanFlow source tree).
 */
#ifndef CHUANFLOW_B200_H
#define CHUANFLOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFG_OK 0
#define CFG_EINVAL 1    /* bad argument or inconsistent input */
#define CFG_ECUDA 2     /* a CUDA call failed */
#define CFG_EMESH 3     /* invalid mesh (cfFatal in polyMesh / blockMesh) */
#define CFG_ESETUP 4    /* case set-up error (BC types, dictionary keys) */
#define CFG_ENOMEM 5
#define CFG_ENUMERIC 6  /* a check of the algorithm failed (e.g. unequal momentum diagonals) */

typedef struct cfg_mesh cfg_mesh;
typedef struct cfg_ctx cfg_ctx;

/* boundary-condition kinds, as volScalarField / volVectorField know them
 * (src/3d/include/cf/fvm/Fields.h:14-22, src/3d/src/fields/volFields.cpp:117-147,246-283) */
enum cfg_bc_type
{
    CFG_BC_FIXED_VALUE = 0,
    CFG_BC_ZERO_GRADIENT = 1,
    CFG_BC_FIXED_GRADIENT = 2,
    CFG_BC_SYMMETRY = 3,
    CFG_BC_OUTLET = 4,
    CFG_BC_WALL = 5,
    CFG_BC_EMPTY = 6
};

enum cfg_grad_scheme { CFG_GRAD_LINEAR = 0, CFG_GRAD_CORRECTED = 1, CFG_GRAD_LEAST_SQUARES = 2 };
/* upwind, linear and blend as fvm::div (src/3d/src/discrete/divScheme.cpp:11-62);
 * LINEAR_UPWIND is this library's extension (no reference counterpart): the
 * upwind matrix plus a deferred correction phi_f (grad U)_u.(Cf - C_u) of the
 * upwind cell's gradient (the case's grad scheme, U's conditions) on the
 * right-hand side, evaluated on the iterate each equation is assembled from */
enum cfg_div_scheme { CFG_DIV_UPWIND = 0, CFG_DIV_LINEAR = 1, CFG_DIV_BLEND = 2, CFG_DIV_LINEAR_UPWIND = 3 };
enum cfg_lin_method { CFG_SOLVE_CG = 0, CFG_SOLVE_BICGSTAB = 1 };
/* pressure preconditioner: the reference's Jacobi PCG, or this library's
 * multicolour DIC (no reference counterpart) */
enum cfg_precond
{
    CFG_PRECOND_JACOBI = 0,
    CFG_PRECOND_DIC = 1,
    CFG_PRECOND_MPNN = 2,
    CFG_PRECOND_AMG = 3,
    CFG_PRECOND_IR32 = 4,
    CFG_PRECOND_AMG_MPNN = 5
};
/* CFG_PRECOND_MPNN: flexible CG with the learned preconditioner (cfg_mpnn_*),
 * the reference's infinity-norm test, FP64 DIC-PCG when it stalls.
 * CFG_PRECOND_AMG: FP64 flexible CG, device-resident, preconditioned by an
 * FP32 aggregation-AMG V-cycle rebuilt from each outer iteration's matrix
 * (hierarchy structure once per context), the reference's infinity-norm test.
 * CFG_PRECOND_IR32: mixed precision -- the matrix rounded to FP32 each outer
 * iteration, FP32 multicolour DIC-PCG corrections (to 1e-4 relative) inside
 * an FP64 iterative refinement whose residual b - A x and infinity-norm test
 * (Matrix.cpp:166-180) are FP64; the inner iterations are what is counted.
 * CFG_PRECOND_MPNN and CFG_PRECOND_AMG_MPNN start each pressure solve from
 * the network's initial guess x0 + M(b - A x0), then iterate with flexible
 * CG preconditioned by the network (MPNN) or by the FP32 AMG V-cycle
 * (AMG_MPNN). */

/* Schemes (src/3d/include/cf/fvm/FvMatrix.h:30-38) */
typedef struct cfg_schemes
{
    int32_t div;        /* cfg_div_scheme, default upwind */
    int32_t laplacian_corrected; /* 1 = "corrected" (default), 0 = "none" */
    int32_t grad;       /* cfg_grad_scheme, default corrected */
    double blend_coeff; /* default 0.9 */
} cfg_schemes;

/* SimpleControls (src/3d/include/cf/fvm/SimpleSolver.h:13-64) plus the
 * GPU-only settings of the case dictionary's optional gpu{} block */
typedef struct cfg_simple_controls
{
    int32_t max_iterations;   /* 200 */
    double continuity_tol;    /* 1e-6 */
    double pcorr_tol;         /* 0 */
    double momentum_tol;      /* 0 */
    double linear_tol;        /* 1e-7 */
    int32_t linear_max_iter;  /* 2000 */
    int32_t non_orth_correctors; /* 2 */
    double relax_u;           /* 0.7 */
    double relax_p;           /* 0.3 */
    double p_relax_start;     /* 0 */
    double body_force[3];     /* 0 */
    double nu;                /* kinematic viscosity */
    /* gpu{} -- defaults reproduce the reference */
    int32_t p_precond;        /* cfg_precond, default JACOBI */
    int32_t verbose;          /* 1: print the reference's per-iteration log line */
    /* pressure reference cell, -1 = none (the reference has none: a case with
     * no fixed-value pressure patch leaves the singular Neumann system to CG).
     * A pinned cell follows OpenFOAM's fvMatrix::setReference: its source
     * gains diag * p_ref_value and its diagonal doubles. */
    int64_t p_ref_cell;
    double p_ref_value;
    /* SimpleControls::dt / uTimeOld (SimpleSolver.h:44-63, simpleSolver.cpp:
     * 75-97): dt > 0 puts fvm::ddt(U, Uold, dt) (Euler) into every sweep's
     * momentum equation, so the loop's fixed point is one implicit-Euler step
     * and rAU is bounded by dt.  u_time_old: 0 none, 1 the velocity at the
     * start of this call, 2 the field last given to cfg_fields_upload_old.
     * The reference refuses either without the other; so does this. */
    double dt;
    int32_t u_time_old;
    /* gpu{} uPreconditioner: the momentum BiCGStab's right preconditioner.
     * CFG_PRECOND_JACOBI (0, the reference's: z = p D^-1, Matrix.cpp:262-
     * 300) or CFG_PRECOND_AMG (3): the FP32 aggregation-AMG V-cycle of the
     * momentum matrix, one V-cycle for the three components at once, inside
     * the same FP64 BiCGStab and the same |r|inf / |b|inf test.  Other
     * values are refused. */
    int32_t u_precond;
} cfg_simple_controls;

/* SimpleResult (SimpleSolver.h:66-72) plus inner-solver statistics */
typedef struct cfg_simple_result
{
    int32_t iterations;
    int32_t converged;
    double final_continuity_error;
    double final_momentum_residual;
    double last_dp;            /* pDeltaMax of the last iteration */
    double last_continuity_corrected;
    int64_t u_inner_iterations; /* summed over components, passes and outer iterations */
    int64_t p_inner_iterations;
    int32_t diverged;
} cfg_simple_result;

/* SolverReport (src/common/include/cf/common/Matrix.h:58-64) */
typedef struct cfg_solver_report
{
    int32_t iterations;
    int32_t converged;
    double initial_residual;
    double final_residual;
} cfg_solver_report;

/* ---- errors ------------------------------------------------------------ */

/* Copies the last error message of this thread into buf; returns its length. */
size_t cfg_last_error(char* buf, size_t size);
const char* cfg_version(void);

/* ---- mesh ---------------------------------------------------------------- */

/* polyMesh(points, faces, owner, neighbour, patches)
 * (src/3d/include/cf/fvm/PolyMesh.h:30-34, src/3d/src/mesh/polyMesh.cpp:12-64).
 * Faces are given as a CSR of vertex lists.  Patch i covers faces
 * [patch_start[i], patch_start[i]+patch_size[i]).  Geometry is computed on the
 * host in the reference's operation order (polyMesh.cpp:83-288). */
int cfg_mesh_create(const double* points, int64_t n_points, const int64_t* face_offsets,
                    const int64_t* face_verts, int64_t n_faces, const int64_t* owner,
                    const int64_t* neighbour, int64_t n_internal, int32_t n_patches,
                    const char* const* patch_names, const char* const* patch_types,
                    const int64_t* patch_start, const int64_t* patch_size, cfg_mesh** out);

/* BlockMesh::create (src/3d/include/cf/fvm/BlockMesh.h:44-46,
 * src/3d/src/mesh/blockMesh.cpp:36-189).  side_names/side_types are in the
 * order xmin xmax ymin ymax zmin zmax; NULL gives the reference's defaults. */
int cfg_mesh_block(const double min[3], const double max[3], int64_t nx, int64_t ny, int64_t nz,
                   const char* const* side_names, const char* const* side_types, cfg_mesh** out);

/* The polyMesh GmshMesh::fromFile builds from volume elements
 * (src/3d/src/mesh/gmshMesh.cpp:578-760): tetrahedra (type 4), hexahedra (5)
 * and prisms (6) with gmsh's local node order; faces recovered cell by cell
 * and deduplicated, internal faces owned by the lower cell, boundary faces
 * grouped into patches named after the bounding-box plane they lie on (the
 * reader's rule for a file without surface groups), type "wall". */
int cfg_mesh_from_cells(const double* points, int64_t n_points, const int32_t* cell_types,
                        const int64_t* cell_offsets, const int64_t* cell_verts, int64_t n_cells, cfg_mesh** out);

/* GmshMesh::fromFile (src/3d/include/cf/fvm/GmshMesh.h:11-37,
 * src/3d/src/mesh/gmshMesh.cpp:534-776): an ASCII .msh 2.2 or 4.x file of
 * first-order tetrahedra, hexahedra and prisms; boundary faces named by the
 * physical groups of the surface elements (else by bounding-box plane);
 * patch types from names[i] -> types[i] (others "wall"). */
int cfg_mesh_read_gmsh(const char* path, int32_t n_types, const char* const* names, const char* const* types,
                       cfg_mesh** out);

/* polyMesh::movePoints (polyMesh.cpp:320-329): same topology, new points,
 * geometry recomputed. */
int cfg_mesh_move_points(cfg_mesh* mesh, const double* points, int64_t n_points);

/* Synthetic-mesh helper with no reference counterpart: displaces every
 * interior point of a blockMesh box by an independent uniform offset in
 * [-fraction*h, fraction*h) per axis (h the local cell size along that
 * axis), from a counter-based hash of (seed, point, axis). */
int cfg_mesh_jitter_interior(cfg_mesh* mesh, double fraction, uint64_t seed);

void cfg_mesh_destroy(cfg_mesh* mesh);

/* counts[5] = nPoints nCells nFaces nInternalFaces nPatches */
int cfg_mesh_counts(const cfg_mesh* mesh, int64_t counts[5]);
/* patch names/types (buffers of `size` bytes) and ranges */
int cfg_mesh_patch(const cfg_mesh* mesh, int32_t patch, char* name, size_t name_size, char* type,
                   size_t type_size, int64_t* start, int64_t* size);
int cfg_mesh_patch_id(const cfg_mesh* mesh, const char* name);
/* addressing copies: points nP*3, face_offsets nF+1, face_verts, owner nF, neighbour nInt */
int cfg_mesh_addressing(const cfg_mesh* mesh, double* points, int64_t* face_offsets,
                        int64_t* face_verts, int64_t* owner, int64_t* neighbour);
/* polyMesh geometry accessors (PolyMesh.h:51-65); any pointer may be NULL */
int cfg_mesh_geometry(const cfg_mesh* mesh, double* cell_volumes, double* cell_centres,
                      double* face_centres, double* face_sf, double* face_areas, double* delta_vec,
                      double* delta_coeff);
/* makeInternalOwnerWeights / makeFaceSkewVectors (src/3d/src/discrete/interpolate.cpp:28-48) */
int cfg_mesh_weights(const cfg_mesh* mesh, double* owner_weights, double* skew);
/* Device cell numbering (no reference counterpart; the reference keeps the
 * mesh order).  A context lays its cell arrays out in one of these orders;
 * every per-cell sum keeps the original face and column order, so results
 * are identical in all of them, and fields cross the ABI in the original
 * order.  COLOUR: cells grouped by their greedy first-fit colour (computed in
 * ascending original order), so each multicolour-DIC sweep reads contiguous
 * rows.  RCM: reverse Cuthill-McKee from a pseudo-peripheral cell, for
 * locality on meshes whose cells come in no spatial order.  DEFAULT: the
 * environment variable CHUANFLOW_CELL_ORDER (identity | colour | rcm |
 * rcm-colour), else IDENTITY (measured fastest on block and Delaunay meshes,
 * whose own order is already local). */
enum cfg_cell_order
{
    CFG_ORDER_DEFAULT = -1,
    CFG_ORDER_IDENTITY = 0,
    CFG_ORDER_COLOUR = 1,
    CFG_ORDER_RCM = 2,
    CFG_ORDER_RCM_COLOUR = 3
};
/* The numbering of `order` as new -> original cell index. */
int cfg_mesh_device_order(const cfg_mesh* mesh, int32_t order, int64_t* new_to_old);

/* ---- case context on one device ------------------------------------------ */

/* Uploads the mesh to `device` and allocates the case state there. `stream`
 * is a cudaStream_t (NULL = a stream created and owned by the context). */
int cfg_ctx_create(const cfg_mesh* mesh, int32_t device, void* stream, cfg_ctx** out);
/* cfg_ctx_create with an explicit device cell numbering (cfg_cell_order). */
int cfg_ctx_create_ordered(const cfg_mesh* mesh, int32_t device, void* stream, int32_t order, cfg_ctx** out);
void cfg_ctx_destroy(cfg_ctx* ctx);

/* volVectorField::setPatchValue / volScalarField::setPatchValue
 * (Fields.h:42, :90; volFields.cpp:57-62, :175-180).  field 'U' or 'p'. */
int cfg_set_patch_bc(cfg_ctx* ctx, char field, int32_t patch, int32_t bc_type, const double* value);
/* volVectorField::setFaceValue (Fields.h:97, volFields.cpp:187-201): a
 * per-face prescribed velocity for a boundary face; n faces at once. */
int cfg_set_face_values_U(cfg_ctx* ctx, int64_t n, const int64_t* faces, const double* values);
int cfg_clear_face_values_U(cfg_ctx* ctx);
int cfg_set_schemes(cfg_ctx* ctx, const cfg_schemes* schemes);

/* Field transfers.  U: nCells*3, p: nCells, phi: nFaces, all in the mesh's
 * original cell and face order; NULL skips a field. */
int cfg_fields_upload(cfg_ctx* ctx, const double* U, const double* p, const double* phi);
int cfg_fields_download(cfg_ctx* ctx, double* U, double* p, double* phi);
/* The velocity at the previous time level for cfg_simple_controls.u_time_old
 * = 2 (nCells x 3, original order): SimpleControls::uTimeOld. */
int cfg_fields_upload_old(cfg_ctx* ctx, const double* U_old);

/* The initial flux of src/3d/apps/simpleFoamApp.cpp:94-95 and
 * src/3d/apps/caseInit.h:18-31: boundary phi from U's conditions
 * (surfaceScalarField::correctBoundaryFlux), and when `u0` is non-NULL every
 * cell set to u0 and the internal flux interpolated from it. */
int cfg_fields_init_flux(cfg_ctx* ctx, const double* u0);

/* solveIncompressibleSimple (src/3d/include/cf/fvm/SimpleSolver.h:119-127,
 * src/3d/src/solvers/simpleSolver.cpp:33-394), laminar and steady.  Runs up
 * to controls->max_iterations outer iterations on the device fields. */
int cfg_simple_iterate(cfg_ctx* ctx, const cfg_simple_controls* controls, cfg_simple_result* result);

/* PisoControls (src/3d/include/cf/fvm/PisoSolver.h:13-40) plus the
 * viscosity and the GPU pressure preconditioner */
typedef struct cfg_piso_controls
{
    double dt;
    int32_t correctors;          /* 2 */
    double continuity_tol;       /* 1e-10 */
    double linear_tol;           /* 1e-8 */
    int32_t linear_max_iter;     /* 2000 */
    int32_t non_orth_correctors; /* 2 */
    double body_force[3];
    double nu;
    int32_t p_precond;           /* cfg_precond */
} cfg_piso_controls;

/* PisoStepResult (PisoSolver.h:42-50) */
typedef struct cfg_piso_result
{
    int32_t correctors_used;
    int32_t converged;
    int32_t diverged;
    double predicted_continuity_error;
    double continuity_error;
    double pressure_correction_max;
    int64_t u_inner_iterations;
    int64_t p_inner_iterations;
    double device_ms;
} cfg_piso_result;

/* solveTransientIncompressiblePiso (PisoSolver.h:92-100,
 * src/3d/src/solvers/pisoSolver.cpp:13-237): one implicit-Euler time step of
 * the device fields (momentum once, then the correctors, each solving the
 * full pressure from the previous iterate).  With a RANS model set up
 * (cfg_turbulence_setup) the model advances first with the step's dt and
 * supplies nu + nut on faces (pisoSolver.cpp:29-30); otherwise laminar. */
int cfg_piso_step(cfg_ctx* ctx, const cfg_piso_controls* controls, cfg_piso_result* result);

/* Wall time (ms) of the device work of the last cfg_simple_iterate call,
 * measured with CUDA events on the context's stream, and the launch count.
 * kernel_ms[0..7] split it by family: gradient, assembly, momentum solve,
 * pressure solve, flux/update, continuity, other, total. */
int cfg_last_timing(const cfg_ctx* ctx, double kernel_ms[8], int64_t* launches);

/* Opt-in CUDA-event timing of every linear-solver kernel launch on the
 * context's stream (no reference counterpart); while it is on, solver
 * iterations are launched one by one rather than as CUDA graphs.  Enabling
 * clears the counts; cfg_kernel_stats gives {launches, total ms} for the
 * first `slots` (at most CFG_KERNEL_SLOTS) of, in order: the PCG SpMV +
 * p.Ap, the x/r update + norms + r.z, the search-direction update; the four
 * BiCGStab kernels (p/z update, v = Az, t = As^, x/r update); the whole DIC
 * application z = M^-1 r; the AMG-preconditioned momentum BiCGStab's p
 * update, then its two V-cycles' finest pre-sweep and residual, everything
 * coarser (restriction to prolongation) and finest post-sweep (both
 * V-cycles of an iteration in these three slots), v = Az, s = r - alpha v,
 * t = As^ and x/r update.  out holds 2 * slots doubles. */
#define CFG_KERNEL_SLOTS 16
int cfg_kernel_timing(cfg_ctx* ctx, int32_t enable);
int cfg_kernel_stats(const cfg_ctx* ctx, double* out, int32_t slots);
/* The same slots' launches weighted by the vector components each launch
 * still iterated on (the fused three-component BiCGStab kernels skip a
 * converged component's rows; 1 per launch elsewhere), for per-launch byte
 * counts (no reference counterpart); out holds `slots` doubles. */
int cfg_kernel_components(const cfg_ctx* ctx, double* out, int32_t slots);

/* ---- the linear-solver call surface ------------------------------------ */

/* solveCG / solveBiCGStab on a CSR matrix (src/common/include/cf/common/Matrix.h:67-73,
 * src/common/src/Matrix.cpp:153-319): host CSR (rows sorted by column, the
 * diagonal present), b and x (x: initial guess in, solution out).  The
 * matrix and vectors are copied to the device and back inside the call. */
int cfg_sparse_solve(const cfg_ctx* ctx_or_null, int32_t device, int64_t n, const int64_t* row_start,
                     const int64_t* cols, const double* vals, const double* b, double* x, double tol,
                     int32_t max_iter, int32_t method, cfg_solver_report* report);

/* ---- the pressure-Poisson solve on its own (no reference counterpart) ---- */

enum cfg_poisson_method
{
    CFG_POISSON_JACOBI64 = 0,  /* FP64 Jacobi-PCG, the reference's solver */
    CFG_POISSON_DIC64 = 1,     /* FP64 multicolour-DIC PCG */
    CFG_POISSON_IR32 = 2,      /* FP32 DIC-PCG corrections inside FP64 iterative refinement */
    CFG_POISSON_FCG_MPNN = 3,  /* flexible CG with the learned preconditioner (cfg_mpnn_create),
                                * FP64 DIC-PCG from its iterate when it stalls */
    CFG_POISSON_FCG_AMG = 4,   /* FP64 flexible CG preconditioned by an FP32 aggregation-AMG
                                * V-cycle (same fallback) */
    CFG_POISSON_FCG_AMG_MPNN = 5 /* the same with the learned network correcting what each
                                  * V-cycle leaves: z = V(r) + N(r - A V(r)) */
};

typedef struct cfg_poisson_report
{
    int64_t inner_iterations;   /* PCG iterations, summed over refinement steps */
    int32_t outer_iterations;   /* refinement steps (1 for the FP64 methods) */
    int32_t converged;
    double true_rel_residual;   /* |b - A x|2 / |b|2 recomputed in FP64 */
    double device_ms;           /* CUDA-event time of the solve on the context's stream */
    double initial_rel_residual;
} cfg_poisson_report;

/* The context's pressure matrix set to the orthogonal part of laplacianFace
 * with unit face coefficient (laplacianScheme.cpp:176-215, sign -1) under
 * the patches' p conditions, plus a reference cell (-1: none) pinned as
 * OpenFOAM's fvMatrix::setReference does; its FP32 copy and both DIC
 * factors are prepared. */
int cfg_poisson_setup(cfg_ctx* ctx, int64_t ref_cell);

/* Solves that system for host b to |b - A x|2 / |b|2 <= rel_tol (FP64, true
 * residual); x holds the initial guess and receives the solution.  For
 * CFG_POISSON_IR32 each refinement step solves for the correction in FP32
 * to inner_rel_tol (at most inner_max_iter iterations); max_iter bounds all
 * PCG iterations. */
int cfg_poisson_solve(cfg_ctx* ctx, const double* b, double* x, int32_t method, double rel_tol, int32_t max_iter,
                      int32_t inner_max_iter, double inner_rel_tol, cfg_poisson_report* report);
/* The aggregation-AMG hierarchy of the cfg_poisson_setup system, built (or
 * refreshed for new values) here rather than inside the first AMG solve:
 * out[0] levels, out[1..8] rows per level, out[9] host structure set-up ms
 * (plain aggregation, Galerkin gather lists; once per mesh), out[10] value
 * set-up ms (device Galerkin sums and the coarsest dense inverse). */
int cfg_poisson_amg_setup(cfg_ctx* ctx, double out[11]);
/* One V-cycle of that hierarchy, z = V(r) (host vectors, original order):
 * the preconditioner as CFG_POISSON_FCG_AMG applies it, for tests. */
int cfg_poisson_amg_apply(cfg_ctx* ctx, const double* r, double* z);
/* The three-component V-cycle the AMG momentum BiCGStab applies, on the
 * same hierarchy: r and z hold three vectors one after another (3 n
 * values); component q is skipped, its z left as given, when done[q] != 0.
 * Each applied component equals cfg_poisson_amg_apply of it, for tests. */
int cfg_poisson_amg_apply3(cfg_ctx* ctx, const double* r, double* z, const int32_t done[3]);
/* Strength-of-connection aggregation for the pressure AMG hierarchy (the one
 * the SIMPLE and PISO pressure solves and the Poisson system use; no
 * counterpart in the reference, whose pressure solve is Jacobi-PCG,
 * src/common/src/Matrix.cpp:153-222).  With theta > 0 an entry (i, j) joins
 * the aggregation only when |a_ij| >= theta * max over k != i of |a_ik|, on
 * every level (coarse values: FP64 Galerkin sums of the operator the
 * hierarchy is first built for); a level that this coarsens by less than
 * half is aggregated plainly.  theta 0 (the default) is plain aggregation.
 * Set it before the first AMG pressure or Poisson solve: once the hierarchy
 * is built, a different theta is refused with CFG_EINVAL.  The momentum
 * hierarchy always aggregates plainly. */
int cfg_amg_strength(cfg_ctx* ctx, double theta);

/* ---- diagnostics used by the parity tests (no reference counterpart) ----- */

/* The equations of one outer iteration built from the context's current
 * fields: out receives gradPn (3N), the momentum diagonal (3N), the
 * momentum explicit operator h = rhs - (A x - diag x) at x = 0 (3N) and at
 * x = xprobe (3N), rAUf (F), div(phi) (N), the predictor continuity error
 * (1), the pressure diagonal (N), its h at 0 and at xprobe (2N), the
 * gradient of xprobe under p's conditions (3N), and phi corrected with
 * xprobe as the solved pressure (F).  Vector blocks are component-major. */
int cfg_probe_equations(cfg_ctx* ctx, const cfg_simple_controls* controls, const double* xprobe, double* out);

/* The multicolour DIC of the pressure matrix last assembled in the context
 * (by cfg_probe_equations or an outer iteration): its factor (1/rD per cell)
 * and one application z = M^-1 r, and the number of colours. */
int cfg_probe_dic(cfg_ctx* ctx, const double* r, double* z, double* rdinv, int32_t* n_colours);

/* fvc::grad of a cell field with fixed boundary face values bvals[f - nInternal]
 * (gradScheme.cpp:246-277); vol_quirk 1 selects the volScalarField overload's
 * internal face value for the linear scheme.  out: nCells*3. */
int cfg_gradient(cfg_ctx* ctx, const double* data, const double* bvals, int32_t scheme, int32_t vol_quirk,
                 double* out);

/* Jacobi-preconditioned CG on a CSR matrix that is already in device memory,
 * for callers that cannot let a library allocate: a solver inside a host
 * framework whose memory manager owns the whole GPU, or one that overlaps
 * other streams and cannot afford the device-wide synchronisation of
 * cudaMalloc / cudaFree.  No counterpart in the reference.  The same
 * algorithm as cfg_sparse_solve's CG; the caller passes device pointers
 * (row_start n+1 and cols int32, vals, b, x; x holds the initial guess and
 * receives the solution) and a cudaStream_t (NULL: the default stream), and
 * this call allocates nothing: its work vectors live in one static device
 * array of the library, sized for at most 262,144 rows (about 8.5 MB, held
 * on every GPU that loads the library until the process exits); larger n is
 * rejected with CFG_EINVAL.  The call waits on its stream once per chunk of
 * iterations to test convergence.  The first call on each device looks that
 * array's address up (cudaGetSymbolAddress, with the device current) and
 * keeps it for the life of the process, so make that first call before any
 * stream capture begins; after a cudaDeviceReset on that device the kept
 * address is stale, so do not call it again after a reset.
 * Calls share the array and keep no state between them, but two calls whose
 * work overlaps on the GPU (different streams or host threads at once) race
 * on it. */
int cfg_pcg_solve_static(int32_t device, int64_t n, const int32_t* row_start_dev, const int32_t* cols_dev,
                         const double* vals_dev, const double* b_dev, double* x_dev, double tol, int32_t max_iter,
                         void* stream, cfg_solver_report* report);

/* ---- case dictionary (the reference's case.dict grammar) ----------------- */

/* Runs a chflow-simple-foam case file end to end (src/3d/apps/simpleFoamApp.cpp:33-209
 * without turbulence/energy/output): mesh from block{}, patches{}, schemes{},
 * simple{} (with linearTol/linearMaxIter as in
 * src/coupling/apps/multiCoupledApp.cpp:41-57) and an optional gpu{} block.
 * Fields are returned through U/p/phi if non-NULL (sizes from counts). */
int cfg_run_case_file(const char* path, int32_t device, cfg_simple_result* result, int64_t counts[5],
                      double* U, double* p, double* phi);

/* Parses a case file on the host only (no device): writes a text summary
 * of the mesh counts, every patch's U/p conditions, schemes and controls. */
int cfg_case_inspect(const char* path, char* out, size_t size);

/* ---- output ----------------------------------------------------------------- */

/* VtkWriter (src/3d/include/cf/fvm/VtkWriter.h, src/3d/src/io/vtkWrite.cpp:33-131):
 * a .vtu of the mesh, every cell a polyhedron, with cell fields -- the
 * scalars in the order given, then the vectors.  binary = 0 writes the
 * reference's ASCII file byte for byte; 1 writes the same arrays raw in an
 * appended block (plus the polyhedron face offsets). */
int cfg_mesh_write_vtu(const cfg_mesh* mesh, const char* path, int32_t n_fields, const char* const* names,
                       const int32_t* n_comp, const double* const* data, int32_t binary);
/* the context's fields (original order): p, then k, epsilon, nut when a RANS
 * model is set up, then U */
int cfg_write_vtu(cfg_ctx* ctx, const char* path, int32_t binary);

/* writeFieldsHdf5 (src/3d/include/cf/fvm/Hdf5Writer.h:25, src/3d/src/io/hdf5Write.cpp:38-95):
 * an HDF5 file holding /points (n_points x 3 f64), /owner and /neighbour
 * (int64) and one 1-D f64 dataset of n_cells values per field under
 * /fields.  The reference writes it through the HDF5 C library and fails
 * without one; this library encodes the file format itself (superblock 0,
 * symbol-table groups, version-1 object headers, contiguous datasets), so
 * no HDF5 library is needed.  Field names must be non-empty, distinct and
 * free of '/'; at most 256 fields. */
int cfg_mesh_write_hdf5(const cfg_mesh* mesh, const char* path, int32_t n_fields, const char* const* names,
                        const double* const* data);
/* the context's cell fields (original order) as /fields/p, then k, epsilon
 * (omega for k-omega SST) and nut when a RANS model is set up, then Ux, Uy,
 * Uz */
int cfg_write_hdf5(cfg_ctx* ctx, const char* path);

/* ---- RANS turbulence -------------------------------------------------------- */

/* RansModel::create (src/3d/src/turbulence/turbulenceModel.cpp:54-104,
 * wallFunction.cpp) with model "kEpsilon" (kEpsilon.cpp), "kOmegaSST"
 * (kOmegaSST.cpp: Menter 2003 blend with the shortest-path cell wall
 * distance), "des" (desModel.cpp: the shielded length on k-epsilon) or
 * "gammaTransition" (transitionModel.cpp: k-epsilon with an intermittency
 * equation), or "laminar" (removes a model).  Spalding wall functions on
 * patches of type "wall"; k and the dissipation variable fixed on patches of
 * type "inlet".  Set up after the velocity conditions: the initial k = 1.5
 * (U_inlet intensity)^2 and epsilon = Cmu^0.25 k^1.5 / L, or for kOmegaSST
 * omega = k^0.5 / (Cmu^0.25 L) (L = length_scale, or 7% of the box diagonal
 * when length_scale <= 0).  The model is then advanced once per SIMPLE outer
 * iteration and supplies nu + nut on faces to the momentum equation
 * (simpleSolver.cpp:52, :97); `nu` is the molecular viscosity. */
int cfg_turbulence_setup(cfg_ctx* ctx, const char* model, double intensity, double length_scale, double relaxation,
                         double nu);
/* TurbulenceConfig's model options (TurbulenceModel.h:50-59), taken by the
 * next cfg_turbulence_setup (or detail-block model) of this context: C_DES
 * (des, default 0.61), reOnset, onsetWidth and gammaRate (gammaTransition;
 * defaults 0, -1 = 5% of the onset distance, 4). */
int cfg_turbulence_params(cfg_ctx* ctx, double c_des, double re_onset, double onset_width, double gamma_rate);
/* k, the dissipation variable (epsilon; omega for kOmegaSST), nut (nCells,
 * original order) and nu + nut on faces (nFaces); any pointer may be NULL. */
int cfg_turbulence_fields(cfg_ctx* ctx, double* k, double* eps, double* nut, double* nu_eff_face);

/* ---- learned pressure preconditioner (no reference counterpart) ------------ */

/* A message-passing network on the cell-face graph of the context's pressure
 * matrix (the cfg_poisson_setup system, else the last SIMPLE pressure
 * equation): z = r/diag + s (wout . h), h from `layers` residual layers of
 * width 32 with one-hop messages weighted by -a_ij/a_ii, s = rms(r).  FP32
 * master weights, BF16 in use, FP32 activations; trained on the device.
 * Parameters: 64 + layers * 2080 + 32 floats. */
int cfg_mpnn_create(cfg_ctx* ctx, int32_t layers, uint64_t seed);
int cfg_mpnn_params(const cfg_ctx* ctx, int64_t* n);
/* FP32 master weights: get and/or set (either may be NULL). */
int cfg_mpnn_weights(cfg_ctx* ctx, float* get, const float* set, int64_t n);
/* loss |A M(r) - r|^2 / |r|^2 of one residual sample and its gradient with
 * respect to the (BF16-rounded) weights; grad may be NULL. */
int cfg_mpnn_loss_grad(cfg_ctx* ctx, const double* r, double* loss, float* grad);
/* z = M(r) */
int cfg_mpnn_apply(cfg_ctx* ctx, const double* r, double* z);
/* Adam (lr) over n_samples residual samples (n_samples x nCells, original
 * order), `epochs` passes; losses[epoch] = mean loss (may be NULL). */
int cfg_mpnn_train(cfg_ctx* ctx, const double* samples, int32_t n_samples, int32_t epochs, float lr, double* losses);
/* The same on (residual, converged correction) pairs: r_k the residual a
 * pressure solve starts from, t_k the correction the plain solver converged
 * to from there (A t_k = r_k); the loss is the energy-norm error
 * e.Ae / t.At with e = M(r) - t, the error CG minimises.  targets has the
 * layout of samples.  cfg_mpnn_loss_grad_pair gives one pair's loss and
 * gradient. */
int cfg_mpnn_train_pairs(cfg_ctx* ctx, const double* samples, const double* targets, int32_t n_samples,
                         int32_t epochs, float lr, double* losses);
int cfg_mpnn_loss_grad_pair(cfg_ctx* ctx, const double* r, const double* t, double* loss, float* grad);
/* reps event-timed applications of the network on the context's current
 * pressure matrix: out[0] ms per application, out[1] ms per message-passing
 * layer launch (no reference counterpart). */
int cfg_mpnn_time(cfg_ctx* ctx, int32_t reps, double out[2]);
/* Keep (on = 1) up to max_samples training pairs of the SIMPLE / PISO
 * pressure solves: the residual each starts from (b - A x0 of its first
 * pass, original order) and the correction that pass converges to (x - x0);
 * on = 2 first drops those kept; on = 0 stops.  cfg_mpnn_train_collected
 * trains on the pairs in the energy norm (cfg_mpnn_train_pairs); n returns
 * how many are kept. */
int cfg_mpnn_collect(cfg_ctx* ctx, int32_t on, int32_t max_samples, int32_t* n);
int cfg_mpnn_train_collected(cfg_ctx* ctx, int32_t epochs, float lr, double* losses);
/* r = b - A x on the cfg_poisson_setup system (training samples from the
 * plain solver's iterates). */
int cfg_poisson_residual(cfg_ctx* ctx, const double* b, const double* x, double* r);

/* ---- detail blocks of a coupled 1D-3D network ------------------------- */

/* BlockMeasure (src/coupling/include/cf/coupling/CoupledNetwork.h:327-357),
 * the part a laminar block reports, plus inner-solver statistics */
typedef struct cfg_detail_measure
{
    int64_t cells;
    int32_t sweeps;       /* SIMPLE outer iterations of this lossAt */
    int32_t converged;
    int32_t diverged;
    double dp_pa;         /* rho * (volume-weighted p of the first cross-section - the last) */
    double imposed_q;     /* m3/s */
    double flux_in;       /* -sum phi over the inlet patch */
    double flux_out;      /* sum phi over the outlet patch */
    double inlet_area;
    double plug_speed;
    double device_ms;     /* device time of the SIMPLE iterations */
    int64_t u_inner_iterations;
    int64_t p_inner_iterations;
    int32_t status;       /* CFG_OK, or CFG_ENUMERIC for a non-finite or non-positive drop,
                           * the two results lossAt rejects (coupledNetwork.cpp:1146-1151) */
} cfg_detail_measure;

/* DetailBlock's constructor (coupledNetwork.cpp:462-620, 644-877): the first
 * patch of type "inlet" and of type "outlet" (opposed, equal areas), the flow
 * axis from the inlet area vector, the cross-sections (cells by axial centre,
 * grouped within 1e-9 of the extent) and the inlet profile "flat",
 * "parabolic" or "power1over7" (normalised to carry the rate exactly). */
int cfg_detail_setup(cfg_ctx* ctx, const char* inlet_shape, double rho);
/* DetailBlock::lossAt(q) (coupledNetwork.cpp:1080-1152, 878-926,
 * 1154-1195) for a laminar block: the boundary conditions of rate q, SIMPLE
 * with `controls` from the block's current fields (a coupling pass warm
 * starts), and the measured drop.  Returns CFG_ENUMERIC, with `out` filled,
 * when the drop is non-finite or non-positive, where lossAt raises. */
int cfg_detail_loss(cfg_ctx* ctx, double q, const cfg_simple_controls* controls, cfg_detail_measure* out);

/* DetailBlock's TurbulenceConfig (coupledNetwork.cpp:1112-1113): the block's
 * RANS model ("laminar" or "kEpsilon", see cfg_turbulence_setup), created at
 * its first lossAt after the inlet velocity is written. */
int cfg_detail_turbulence(cfg_ctx* ctx, const char* model, double intensity, double length_scale, double relaxation,
                          double nu);

/* A batch of detail-block contexts on one device (no reference counterpart:
 * solveCoupled1d3d evaluates its blocks one after another,
 * coupledNetwork.cpp:1454-1487).  The contexts stay owned by the caller and
 * must each have their own stream (the default of cfg_ctx_create). */
typedef struct cfg_batch cfg_batch;
int cfg_batch_create(int32_t n, cfg_ctx* const* blocks, cfg_batch** out);
void cfg_batch_destroy(cfg_batch* batch);
/* The schedule: `workers` blocks in flight at once (1 = one after another),
 * each block's solver kernels on a grid of at most `row_blocks_per_sm`
 * blocks per SM (0 = the context's own grid; -1 = by block size, one per
 * 32k cells between 1 and 4).  workers = 0 runs each pass as ONE CUDA-graph
 * launch: every block's outer iteration and measure are parallel branches
 * of a graph captured on the first pass (per schedule and controls), their
 * linear solvers iterate in device-side conditional while-nodes, and the
 * host only writes the blocks' boundary values before the launch and reads
 * their sums after it; it needs one outer iteration per pass, Jacobi or DIC
 * pressure and no gammaTransition model. */
int cfg_batch_set_schedule(cfg_batch* batch, int32_t workers, int32_t row_blocks_per_sm);
/* One coupling pass: lossAt(q[i]) of every block i with controls[i]; wall_ms
 * (may be NULL) is the pass's host wall time.  A block whose drop lossAt
 * would reject reports it in out[i].status; the pass still completes. */
int cfg_batch_loss(cfg_batch* batch, const double* q, const cfg_simple_controls* controls, cfg_detail_measure* out,
                   double* wall_ms);
/* A device-side copy of every block's U, p, phi, and its return: passes
 * repeated from the same fields (the same work under another schedule). */
int cfg_batch_save(cfg_batch* batch);
int cfg_batch_restore(cfg_batch* batch);
/* Chooses the schedule by measurement: every candidate runs the same pass
 * from the blocks' current fields (saved and restored around each), the
 * fastest is kept and then runs that pass for real; the chosen schedule and
 * each candidate's wall time are returned (times: 9 doubles, may be NULL;
 * -1 for a candidate the controls exclude).  Candidates (workers, row blocks
 * per SM): (1,0), (8,1), (16,1), (16,-1), (32,-1), (64,-1), and the
 * single-graph pass (0,1), (0,2), (0,-1); each is timed on a second run of
 * the pass (the first carries its graph captures). */
int cfg_batch_autotune(cfg_batch* batch, const double* q, const cfg_simple_controls* controls, int32_t* workers,
                       int32_t* row_blocks_per_sm, double* times);

#ifdef __cplusplus
}
#endif
#endif /* CHUANFLOW_B200_H */
