/*
 * rdst.h -- C ABI of the B200 fully-coupled density-based step.
 *
 * This is the drop-in boundary for rhoDST's implicit step
 * (libraries/finiteVolume/iteration/Single/Single.C:80-104 of rhoDST).  A
 * foam-extend host (an `iteration` subclass selected as
 * `timeIntegration GPU;`) marshals its fvMesh arrays and dictionary entries
 * into the structs below and calls rdst_step() where Single::iterate ran:
 *
 *   rhoDSTFlux_.computeFluxDST()        -> flux + residual kernels
 *   fvmDST::ddt(W) + fvmDST::fluxDST()  -> Jacobian/assembly kernels
 *   Eqn.solve(true)                     -> block GMRES/BiCGStab kernels
 *   #include "updateFields.H"           -> update kernel
 *   turbulence_.correct()               -> Spalart-Allmaras kernels
 *   runTime_.setCourantDST()            -> time-step kernels
 *
 * Plain C99: pointers and sizes only, no exceptions cross the ABI.  Host
 * arrays are borrowed for the duration of a call.  All device memory is
 * owned by the context and released by rdst_destroy().
 *
 * Array conventions follow foam's fvMesh:
 *   faces [0, n_internal_faces) are internal (owner < neighbour),
 *   faces [n_internal_faces, n_faces) are boundary faces grouped by patch;
 *   vectors are AoS xyz triplets ("N x 3").
 */
#ifndef RDST_H
#define RDST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Mirrors the reference's FatalError exits
 * (newbaseFluxDST.C:72-82, JacobianDST.C:80-89, newIteration.C:67-76) as
 * RDST_ERR_CONFIG; the message is available from rdst_last_error(). */
typedef enum rdst_status {
    RDST_OK = 0,
    RDST_ERR_CONFIG = 1,      /* unknown selector name / bad option value   */
    RDST_ERR_MESH = 2,        /* inconsistent mesh arrays                   */
    RDST_ERR_CUDA = 3,        /* CUDA runtime error                         */
    RDST_ERR_DIVERGED = 4,    /* NaN or non-positive rho/p after an update  */
    RDST_ERR_TIMEOUT = 5,     /* a bounded device wait gave up              */
    RDST_ERR_UNSUPPORTED = 6, /* a reference option this path rejects       */
    RDST_ERR_ARG = 7          /* null pointer / size out of range           */
} rdst_status;

/* Patch geometric type (foam polyPatch type). */
enum {
    RDST_PATCH_PATCH = 0,
    RDST_PATCH_WALL = 1,
    RDST_PATCH_SYMMETRY = 2,   /* symmetryPlane */
    RDST_PATCH_EMPTY = 3       /* 2D front/back: carries no flux */
};

/* Boundary condition of one primitive field on one patch (foam
 * fvPatchField type).  p and T use FIXED_VALUE/ZERO_GRADIENT/
 * INLET_OUTLET/SYMMETRY/FARFIELD; U uses all of them (SLIP = symmetry
 * treatment on a non-symmetry patch; FIXED_VALUE with 0 = no-slip wall). */
enum {
    RDST_BC_FIXED_VALUE = 0,
    RDST_BC_ZERO_GRADIENT = 1,
    RDST_BC_INLET_OUTLET = 2,
    RDST_BC_SYMMETRY = 3,
    RDST_BC_SLIP = 4,
    RDST_BC_FARFIELD = 5       /* farField{Pressure,Velocity,Temperature}DST */
};

typedef struct rdst_patch {
    int32_t start;             /* first face of the patch (foam face index) */
    int32_t size;
    int32_t type;              /* RDST_PATCH_*                               */
    int32_t bc_p, bc_U, bc_T;  /* RDST_BC_* per primitive field              */
    int32_t bc_nuTilda;        /* SA: FIXED_VALUE / ZERO_GRADIENT /
                                  INLET_OUTLET (farField: inletOutlet)      */
    double p_value;            /* fixedValue / inletValue / far-field p_inf  */
    double U_value[3];
    double T_value;
    double nuTilda_value;      /* SA: fixed/inlet value of nuTilda           */
} rdst_patch;

typedef struct rdst_mesh {
    int32_t n_cells;
    int32_t n_internal_faces;
    int32_t n_faces;            /* internal + boundary                        */
    int32_t n_patches;
    const int32_t* owner;       /* [n_faces]                                  */
    const int32_t* neighbour;   /* [n_internal_faces]                         */
    const double* Sf;           /* [n_faces*3] face area vectors              */
    const double* Cf;           /* [n_faces*3] face centres                   */
    const double* magSf;        /* [n_faces]                                  */
    const double* weights;      /* [n_faces] linear interpolation weights     */
    const double* deltaCoeffs;  /* [n_faces]                                  */
    const double* C;            /* [n_cells*3] cell centres                   */
    const double* V;            /* [n_cells]   cell volumes                   */
    const rdst_patch* patches;  /* [n_patches]                                */
    const double* wall_distance;/* [n_cells] or NULL (needed by SA models)    */
} rdst_mesh;

/* Per-step report (the reference's Info output + residual history). */
typedef struct rdst_step_report {
    double time;               /* physical time after the step               */
    double deltaT;             /* physical time step used by the step        */
    double courant;            /* global Courant (transient) / mean (steady) */
    double res_l2[5];          /* ||R_k * V||_2 over cells, k = rho..rhoE    */
    double res_mag;            /* sqrt(sum_cells |R|^2): the CFL-ramp norm
                                  of timeDST::setCourantDST (timeDST.C:330)  */
    double lin_initial[5];     /* linear solver initial residual (normalised)*/
    double lin_final[5];       /* linear solver final residual               */
    int32_t lin_iterations;    /* GMRES restarts / BiCGStab iterations       */
    int32_t flags;             /* bit0: field bounding was active;
                                  bit3: the (last) linear solve stopped at
                                  maxIter with neither tolerance nor relTol
                                  reached (foam's converged() false)        */
    double rdt_min, rdt_max;   /* min/max of the local 1/dtau                */
    double t_flux_ms, t_jacobian_ms, t_precond_ms, t_krylov_ms, t_update_ms;
} rdst_step_report;

typedef struct rdst_ctx rdst_ctx;

/* Create a context.  `keys`/`values` are the dictionary entries that select
 * the path, with foam's names (dotted for sub-dictionaries), e.g.
 *   "fluxScheme" "Kurganov"          (rhoDSTDict; newbaseFluxDST.C:64-84)
 *   "Jacobian" "Roe"                 (rhoDSTDict; JacobianDST.C:72-91)
 *   "timeIntegration.timeIntegration" "Single"
 *   "timeControls.neighbouring" "true" ...
 *   "ddtSchemes.default" "Euler" | "steadyStateDST" | "dual2ndDST"
 *   "interpolationSchemes.reconstruct(rho)" "OSPRE"
 *   "solvers.W.solver" "GMRES" | "BiCGStab" | "GaussSeidel" | "ILU" | "AMG"
 *   "solvers.W.preconditioner" "ILUC0" | "Cholesky" | "GaussSeidel" |
 *                              "ILUCp" | "AMG" | "diagonal" | "none"
 *   "solvers.W.nSweeps" "1"  "solvers.W.fillInLevel" "0"
 *   "fieldBounds.p" "0.001 10000"
 *   "thermo.R" / "thermo.Cp" / "transport.mu" / "transport.Pr" ...
 * (solver/preconditioner names as foam-extend registers them for the 5x5
 * block matrix, Vector5typedefs.C:1602-1708).  Unknown selector values
 * return RDST_ERR_CONFIG; reference options this path rejects
 * (directWaveSpeed false, SAMG, dual time with SARC1)
 * RDST_ERR_UNSUPPORTED.
 * Replaces createFields.H:115-152 (flux, Jacobian and iteration selection)
 * and timeDST::initialize (timeDST.C:67-208). */
rdst_status rdst_create(const rdst_mesh* mesh, int32_t n_options,
                        const char* const* keys, const char* const* values,
                        rdst_ctx** out);

/* Initial state from primitive fields (createFields.H:21-72):
 * rho = p psi, rhoU = rho U, rhoE = rho (h Cv/Cp + |U|^2/2).
 * nuTilda may be NULL for laminar runs. */
rdst_status rdst_set_primitive(rdst_ctx* ctx, const double* p, const double* U,
                               const double* T, const double* nuTilda);

/* Conservative state in and out (geometricFieldDST::set / retrieve).  The
 * first state set on a context also initialises the time control
 * (timeDST::initialize); later calls replace the fields only and keep the
 * Courant history, like foam fields written between time steps. */
rdst_status rdst_set_conservative(rdst_ctx* ctx, const double* rho,
                                  const double* rhoU, const double* rhoE);
rdst_status rdst_get_conservative(rdst_ctx* ctx, double* rho, double* rhoU,
                                  double* rhoE);
rdst_status rdst_get_primitive(rdst_ctx* ctx, double* p, double* U, double* T,
                               double* nuTilda);

/* Advance n_steps implicit steps (Single::iterate, Single.C:80-104).
 * `reports` may be NULL or hold n_steps entries. */
rdst_status rdst_step(rdst_ctx* ctx, int32_t n_steps, rdst_step_report* reports);

/* Evaluate the residual R(W) of the current state (computeFluxDST +
 * calcFields, baseFluxDST.C:223-255): out[n_cells*5], per unit volume,
 * components (rho, rhoU_x, rhoU_y, rhoU_z, rhoE). */
rdst_status rdst_residual(rdst_ctx* ctx, double* out);

/* Assemble the block system of the current state without solving and copy
 * it out in foam's LDU layout (fluxDST.C:73-127 + fvmDST.C:77-143):
 * diag[n_cells*25], upper[n_internal_faces*25] (row owner, column
 * neighbour), lower[n_internal_faces*25], source[n_cells*5]; each 5x5 block
 * row-major.  Any pointer may be NULL. */
rdst_status rdst_assemble(rdst_ctx* ctx, double* diag, double* upper,
                          double* lower, double* source);

/* Pressure (+ viscous) force on one patch, projected on the lift and drag
 * directions and normalised by (q_inf * A_ref): the forceCoeffs function
 * object used by the reference's RAE2822 / oneraM6Turb cases.
 * out[0] = C_l, out[1] = C_d, out[2] = C_m about `cofr` around `pitch_axis`. */
rdst_status rdst_forces(rdst_ctx* ctx, int32_t patch, const double lift_dir[3],
                        const double drag_dir[3], const double cofr[3],
                        const double pitch_axis[3], double p_ref,
                        double q_ref_times_area, double l_ref, double out[3]);

/* Message of the last failing call on this context ("" if none).  With
 * ctx == NULL: the message of the calling thread's last failing
 * context-free call (rdst_residual_norms_noalloc). */

/* ---- discrete adjoint of the steady residual ----
 * No counterpart in the reference: rhoDST has no adjoint.  R(W) is the
 * per-unit-volume residual that rdst_residual returns (no pseudo-time
 * term), convective and -- with transport options set -- viscous terms,
 * muEff = mu(T) + mu_t with mu_t frozen at the last turbulence update
 * (frozen-turbulence adjoint; the turbulence model is not linearized).  It
 * depends on the patch velocity values U_patch: the U_value of every patch
 * that is not a wall, so far field, inlet and outlet together (the free
 * stream); a wall's velocity is held.  In/outflow and sub/supersonic
 * branches of the boundary conditions are held at the current state's.
 *
 * Objective: the pressure force of one patch along a direction,
 *   J = scale * sum_{faces b of patch} (p_b - p_ref) S_b . direction
 * (scale = 1 / (q_ref A_ref) gives a drag or lift coefficient). */
typedef struct rdst_objective {
    int32_t patch;
    double direction[3];
    double p_ref;
    double scale;
} rdst_objective;

typedef struct rdst_adjoint_report {
    double J;
    double force[3];       /* scale * sum (p_b - p_ref) S_b = dJ/d(direction) */
    double dJ_dU[3];       /* total derivative wrt U_patch (all patches together) */
    double residual0;      /* ||dJ/dW||_2 */
    double residual;       /* ||dJ/dW - (dR/dW)^T psi||_2 at exit */
    int32_t iterations;    /* Krylov iterations */
    int32_t cycles;        /* GMRES restart cycles */
    double t_ms;           /* device time of the call */
} rdst_adjoint_report;

/* rdst_objective_gradient: J, the force vector, dJ/dW (N x 5, the state
 * order of rdst_get_conservative: rho, rhoU xyz, rhoE) and the explicit
 * dJ/dU_patch at the current state.  Any output may be NULL. */
rdst_status rdst_objective_gradient(rdst_ctx* ctx, const rdst_objective* obj, double* J, double force[3],
                                    double* dJdW, double dJdU[3]);
/* rdst_adjoint_product: u = (dR/dW)^T v (N x 5 each) and
 * dU = (dR/dU_patch)^T v, matrix-free at the current state. */
rdst_status rdst_adjoint_product(rdst_ctx* ctx, const double* v, double* u, double dU[3]);
/* rdst_tangent_product: Ju = (dR/dW) u (N x 5 each), the forward-mode
 * linearization of the same residual with the same held branches: the
 * exact counterpart of rdst_adjoint_product (v . Ju = ((dR/dW)^T v) . u). */
rdst_status rdst_tangent_product(rdst_ctx* ctx, const double* u, double* Ju);
/* rdst_boundary_branches: for every boundary face (face - n_internal_faces;
 * zero on empty patches) the previous mass flux and far-field Mach number
 * that chose the in/outflow and sub/supersonic branches of the current
 * boundary states, i.e. the branches the adjoint and tangent linearize.
 * No counterpart in the reference. */
rdst_status rdst_boundary_branches(rdst_ctx* ctx, double* phi_prev, double* mach);
/* rdst_set_geometry: replace the mesh metrics of the context (Sf, Cf,
 * magSf, weights, deltaCoeffs, C, V and the wall distance) with those of a
 * mesh of the same topology -- equal counts, owner/neighbour lists and patch
 * ranges, else RDST_ERR_MESH and the context is unchanged.  State, options
 * and boundary values stay; the next residual, step or adjoint call works on
 * the new geometry.  Shape derivatives use it: the explicit derivatives of
 * R and J with respect to a design variable that moves the mesh, at a fixed
 * state, without building a new context.  No counterpart in the reference
 * (rhoDST runs on static meshes). */
rdst_status rdst_set_geometry(rdst_ctx* ctx, const rdst_mesh* mesh);
/* rdst_adjoint: solves (dR/dW)^T psi = dJ/dW by GMRES(n_directions),
 * right-preconditioned with the transposed step Jacobian (block ILU(0) or
 * block Jacobi as the solvers.W preconditioner selects), restarted until
 * the residual falls by rel_tol or after max_cycles cycles; reports J and
 * dJ/dU_patch = dJ/dU_patch|explicit - psi^T dR/dU_patch.  psi (N x 5)
 * may be NULL.  Call it at a converged state (R ~ 0). */
rdst_status rdst_adjoint(rdst_ctx* ctx, const rdst_objective* obj, double rel_tol, int32_t max_cycles,
                         int32_t n_directions, double* psi, rdst_adjoint_report* report);

const char* rdst_last_error(const rdst_ctx* ctx);

/* Release the context and all its device memory. */
void rdst_destroy(rdst_ctx* ctx);

/* Held cells (no reference counterpart: the halo cells of an overlapping
 * domain decomposition, where the reference has processor patches): cells
 * with mask[i] != 0 (original numbering, n_cells entries) keep their state
 * in the steps -- their residual is zero (so they enter neither the
 * residual norms nor the CFL ramp) and their rows of the implicit system
 * are identity rows with no right-hand side.  Their states still enter the
 * neighbours' fluxes, as Dirichlet data set with rdst_set_conservative.
 * NULL clears the mask. */
rdst_status rdst_set_held_cells(rdst_ctx* ctx, const uint8_t* mask);

/* Replace nuTilda between steps (n_cells values, original numbering): its
 * boundary values and mu_t follow; the mean flow and the time-control
 * history are kept (the turbulence counterpart of rdst_set_conservative
 * after a first state, used for the halo cells of a decomposed run).
 * Held cells keep their nuTilda in the segregated nuTilda solve too. */
rdst_status rdst_set_nu_tilda(rdst_ctx* ctx, const double* nut);

/* The states of n listed cells (original numbering): six values per cell,
 * rho, rhoU (3), rhoE, nuTilda (0 without a turbulence model).  get reads
 * them; set writes them between steps with rdst_set_conservative's
 * semantics (boundary values and mu_t follow, time-control history kept),
 * so a decomposed run moves only its halo cells. */
rdst_status rdst_get_cells(rdst_ctx* ctx, int32_t n, const int32_t* cells, double* out);
rdst_status rdst_set_cells(rdst_ctx* ctx, int32_t n, const int32_t* cells, const double* in);
/* The same with the values in DEVICE memory of the context's GPU (cells
 * stays a host array): the halo of a decomposed run goes to and from NCCL
 * without a host copy.  get returns once the values are in out_dev; set
 * reads in_dev, which must be ready when it is called.  (No counterpart in
 * the reference, whose processor patches exchange inside foam-extend.) */
rdst_status rdst_get_cells_device(rdst_ctx* ctx, int32_t n, const int32_t* cells, double* out_dev);
rdst_status rdst_set_cells_device(rdst_ctx* ctx, int32_t n, const int32_t* cells, const double* in_dev);

/* Host-only helper (no GPU needed): recursive coordinate bisection of the
 * cell centres into n_parts parts, out_part[n_cells].  The GPU library uses
 * the same partition for its subdomain ILU(0) (block-Jacobi across parts,
 * as foam-extend's ILUC0 behaves across processor patches). */
rdst_status rdst_partition_cells(int32_t n_cells, const double* C,
                                 int32_t n_parts, int32_t* out_part);

/* Host-only helper (no GPU needed): recursive bisection of the cell graph
 * (internal faces owner/neighbour) by breadth-first distance from a
 * pseudo-peripheral cell, n_parts parts; the partition the library uses
 * with the option "ilu.partition" "graph" (foam-extend's decomposePar
 * methods, scotch or hierarchical, cut processors the same two ways). */
rdst_status rdst_partition_graph(int32_t n_cells, int32_t n_internal_faces,
                                 const int32_t* owner, const int32_t* neighbour,
                                 int32_t n_parts, int32_t* out_part);

/* Instrumentation (no reference counterpart).
 * rdst_stream: the CUDA stream (cudaStream_t) all of the context's kernels
 * run on, so a caller can record its own events around rdst_step.
 * rdst_launch_count: kernels launched by this context so far.
 * rdst_last_step_ms: device time of the last rdst_step call, from CUDA
 * events recorded on the context's stream at entry and after its last
 * kernel.
 * rdst_kernel_stats: with the option "profile" "true", the library records
 * CUDA events around every launch of the named kernel class inside
 * rdst_step ("spmv", "precond", "flux", "assemble", "factor", "orth",
 * "update") and returns its launch count and summed device time.
 * rdst_set_profile: switches that recording on or off for later steps
 * (the event records add device time of their own, so steps are timed
 * with it off).  No counterpart in the reference (instrumentation). */
void* rdst_stream(rdst_ctx* ctx);
int64_t rdst_launch_count(const rdst_ctx* ctx);
double rdst_last_step_ms(const rdst_ctx* ctx);
rdst_status rdst_kernel_stats(rdst_ctx* ctx, const char* kernel, int64_t* launches, double* total_ms);
rdst_status rdst_set_profile(rdst_ctx* ctx, int32_t on);

/* Allocation-free residual norms (no counterpart in the reference; an
 * addition for callers that may not allocate device memory: code running
 * during CUDA stream capture, where cudaMalloc is not capturable, hosts
 * whose device memory belongs to a pool allocator, and paths that cannot
 * pay cudaMalloc's implicit synchronisation).
 * R (n_cells x 5, per unit volume), V (n_cells) and out (6) are DEVICE
 * pointers owned by the caller; out[0] = sqrt(sum_i |R_i|^2) (res_mag of
 * rdst_step_report), out[1+k] = ||R_k V||_2 (res_l2).  Runs asynchronously
 * on `stream` (a cudaStream_t; NULL = legacy default stream) on the GPU
 * that holds R: V and out must live on the same GPU and `stream` must
 * belong to it; host pointers and buffers on different GPUs are rejected
 * with RDST_ERR_ARG before anything is launched.  The calling thread's
 * current device is left as it was.
 * Scratch is a fixed 192 KiB array in the library's device image, present
 * on every GPU that loads the library until the process exits; n_cells
 * above 1,048,576 is rejected with RDST_ERR_ARG.  Calls share that array:
 * calls whose kernels may overlap on the GPU race and must be serialised.
 * The first call on a device looks up the array's device address (a
 * one-time set-up); make that first call before any stream capture. */
rdst_status rdst_residual_norms_noalloc(int32_t n_cells, const double* R, const double* V,
                                        double* out, void* stream);

/* Library identification (e.g. "rdst-b200 sm_100a"). */
const char* rdst_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RDST_H */
