/*
 * cfsa_ns.h — C ABI of the B200 (sm_100a) Taylor-Hood P2/P1 Navier-Stokes PISO solver.
 *
 * This is the thin layer between the C++ NavierStokesSolver facade and the CUDA kernels.
 * Plain pointers and sizes only; host arrays in, host arrays out. Each entry point cites the
 * member of the reference's NavierStokesSolver (include/FEM/NavierStokes.hpp,
 * src/FEM/NavierStokes.cpp of sudo-shaka/Cell-Fluid-Structure-Analysis) that it replaces.
 *
 * Layouts (the reference's): velocity fields are [N2][3] doubles with the nv P1 vertices
 * first and the ne P2 edge nodes after them (N2 = nv + ne); pressure fields are [nv] doubles.
 *
 * Errors: every call returns a status code; the reference's bool returns map to
 * status == CFSA_OK. cfsa_ns_last_error(h) gives the message of the last failure.
 * Threading: one handle drives one CUDA stream on the device current at create time; a handle
 * is not thread-safe, distinct handles are independent.
 */
#ifndef CFSA_NS_H
#define CFSA_NS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CFSA_OK 0
#define CFSA_NOT_CONVERGED 1   /* a Krylov solve hit its iteration cap */
#define CFSA_BREAKDOWN 2       /* a Krylov solve broke down (zero denominator) */
#define CFSA_NAN 3             /* hasNans() after the step */
#define CFSA_CUDA_ERROR 4
#define CFSA_BAD_ARG 5
#define CFSA_NOT_INITIALIZED 6
#define CFSA_UNSUPPORTED 7

/* FluidBCType values (include/FEM/NavierStokes.hpp:13-19) */
#define CFSA_BC_WALL 0
#define CFSA_BC_INLET 1
#define CFSA_BC_OUTLET 2
#define CFSA_BC_INTERNAL 3
#define CFSA_BC_UNDEFINED 4

/* OutletType values (include/FEM/NavierStokes.hpp:21-25) */
#define CFSA_OUTLET_DIRICHLET 0
#define CFSA_OUTLET_NEUMANN 1

/* pressure Krylov method: the reference uses BiCGSTAB (src/FEM/NavierStokes.cpp:633), which is the
 * default here too; the Poisson matrix with penalty rows is SPD, so the CG variants are offered
 * (same system and stopping rule, fewer products; CFSA_KRYLOV_CG2L is the fastest). */
#define CFSA_KRYLOV_CG 0
#define CFSA_KRYLOV_BICGSTAB 1
/* CG with one reduction per iteration (Chronopoulos & Gear 1989): CG's iterates in exact
 * arithmetic, one fused product-and-reduction pass and one grid synchronisation per iteration */
#define CFSA_KRYLOV_CG1 2
/* CFSA_KRYLOV_CG1's recurrences with a two-level preconditioner: Jacobi plus an additive coarse
 * correction on geometric aggregates (boxes over the vertices, ~cfsa_ns_set_coarse_target of
 * them), M r = D^-1 r + P (P^T A P)^-1 P^T r. Same system and stopping rule, several times fewer
 * iterations on the Poisson operator; still one grid synchronisation per iteration. */
#define CFSA_KRYLOV_CG2L 3

/* arithmetic of the Krylov solves */
#define CFSA_PRECISION_FP64 0
/* momentum: FP32 operator and Krylov vectors; FP64 solution, true residual (reliable updates), dot
 * products and scalars; convergence decided on the FP64 true residual. Pressure in FP64. */
#define CFSA_PRECISION_MIXED 1
/* CFSA_PRECISION_MIXED plus, with CFSA_KRYLOV_CG2L, the pressure solve in float storage inside
 * FP64 defect correction. Each sweep restarts the CG, so the pressure solve takes more iterations
 * than in FP64 (1.8x on the 1M-tet cylinder), which costs more than float storage saves. */
#define CFSA_PRECISION_MIXED_FULL 2

/* Krylov convergence norm. REFERENCE: ||r|| <= tol ||b|| (NavierStokes.cpp:500,635). With the
 * 1e10 / 1e12 penalty rows in b this norm is dominated by the Dirichlet rows, so it constrains the
 * interior only loosely. JACOBI: ||D^-1/2 r|| <= tol ||D^-1/2 b||, D = diag of the operator, which
 * weighs the penalty rows down by their diagonal. */
#define CFSA_NORM_REFERENCE 0
#define CFSA_NORM_JACOBI 1

/* matrix ids for cfsa_ns_get_matrix */
#define CFSA_MAT_MASS 0       /* M  (buildMassMatrix, NavierStokes.cpp:227-310) */
#define CFSA_MAT_STIFFNESS 1  /* K  (buildStiffnessMatrix, NavierStokes.cpp:135-225) */
#define CFSA_MAT_GRAD_X 2     /* Gx (buildGradientMatrices, NavierStokes.cpp:70-133) */
#define CFSA_MAT_GRAD_Y 3
#define CFSA_MAT_GRAD_Z 4
#define CFSA_MAT_POISSON 5    /* L  (buildPoissonMatrix, NavierStokes.cpp:316-356) */
#define CFSA_MAT_MOMENTUM 6   /* M/dt + K + 1e10 on Inlet/Wall diagonals (NavierStokes.cpp:460-495) */
#define CFSA_MAT_POISSON_BC 7 /* L + 1e12 on outlet / reference diagonals (NavierStokes.cpp:604-626) */

typedef struct cfsa_ns cfsa_ns;

/* Mesh as the solver reads it (Mesh accessors used by NavierStokes.cpp). */
typedef struct {
  int64_t nv, nt, ne;
  const double *vertices;   /* [nv][3] */
  const int32_t *tets;      /* [nt][4] P1 vertex ids */
  const int32_t *tet_edges; /* [nt][6] edge-node ids 0..ne-1, local edges 01,02,03,12,13,23 */
  const int8_t *p1_bc;      /* [nv] FluidBCType */
  const int8_t *p2_bc;      /* [ne] FluidBCType */
  int64_t nbf;              /* boundary faces (for forces and shear); may be 0 */
  const int32_t *bface_verts; /* [nbf][3] */
  const int32_t *bface_tet;   /* [nbf] owning tet */
  const double *bface_normal; /* [nbf][3] */
  const double *bface_area;   /* [nbf] */
} cfsa_mesh_view;

typedef struct {
  double density;
  double viscosity;
} cfsa_fluid;

typedef struct {
  int32_t momentum_iters[3];  /* last step, per velocity component */
  int32_t pressure_iters;     /* last corrector solve */
  double momentum_residual[3];/* ||r||/||b|| at exit */
  double pressure_residual;
  int32_t momentum_outer[3];  /* FP64 reliable updates of x and r (mixed precision), else 0 */
  int32_t pressure_outer;     /* defect-correction sweeps of the mixed-precision pressure solve */
  int64_t steps;              /* PISO/SIMPLE steps taken since create */
  double time;                /* simulated time */
  double last_step_ms;        /* device time of the last stepping call, all its steps (CUDA events) */
  int64_t nnz_p2, nnz_p1;     /* matrix sizes */
  int64_t kernel_launches;    /* device kernels launched by the last stepping call */
  int64_t krylov_iters[2];    /* Krylov iterations in the last stepping call: momentum, pressure */
  double phase_ms[3];         /* last PISO step on the device: momentum predictor, pressure solve,
                                 everything else (CUDA events inside the step) */
} cfsa_ns_stats;

/* kernel ids for cfsa_ns_profile_kernel */
#define CFSA_KERNEL_MOMENTUM_SPMV 0 /* 3-right-hand-side SELL product of the momentum BiCGSTAB */
#define CFSA_KERNEL_PRESSURE_SPMV 1 /* SELL product of the pressure CG */
/* the whole resident pressure solve (CFSA_KRYLOV_CG2L or _CG1) on the last step's system, fused
 * product and vector updates inside one kernel: avg_ms per solve, alg_bytes = iterations x bytes
 * per iteration (operator, row metadata, each vector read or written once, coarse inverse) */
#define CFSA_KERNEL_PRESSURE_SOLVE 2
/* the FP32 3-right-hand-side product of the mixed-precision momentum solve */
#define CFSA_KERNEL_MOMENTUM_SPMV_F32 3

/* NavierStokesSolver::initialize (include/FEM/NavierStokes.hpp:91-92; NavierStokes.cpp:10-68):
 * uploads the mesh, builds the CSR patterns, assembles M, K, G, L on the device and zeroes the
 * fields. The inlet value in effect at create time is zero (as in the reference's CLI path);
 * call cfsa_ns_initialize_fields after setting the inlet to reproduce initialize() with a
 * preset inlet. */
int cfsa_ns_create(const cfsa_mesh_view *mesh, const cfsa_fluid *fluid, cfsa_ns **out);
void cfsa_ns_destroy(cfsa_ns *h);
const char *cfsa_ns_last_error(const cfsa_ns *h);

/* Sizes: out[0..3] = nv, ne, N2, nt. */
int cfsa_ns_sizes(const cfsa_ns *h, int64_t out[4]);

/* ---- setters (include/FEM/NavierStokes.hpp:166-186) ---- */
int cfsa_ns_set_dt(cfsa_ns *h, double dt);                                /* setDt */
int cfsa_ns_set_tolerances(cfsa_ns *h, double momentum, double pressure); /* setTolerance (routed) */
int cfsa_ns_set_max_iterations(cfsa_ns *h, int momentum, int pressure);   /* NavierStokes.cpp:499,634 */
int cfsa_ns_set_num_corrections(cfsa_ns *h, int n);                        /* setNumberOfCorrections */
int cfsa_ns_set_relaxation(cfsa_ns *h, double relax_u, double relax_p);    /* setRelaxU / setRelaxP */
int cfsa_ns_set_outlet(cfsa_ns *h, int outlet_type, double outlet_pressure); /* setOutletType/Pressure */
int cfsa_ns_set_reference_node(cfsa_ns *h, int node);                      /* setReferencePressureNode */
int cfsa_ns_set_inlet_uniform(cfsa_ns *h, const double u[3]);             /* setMeanInletVelocity */
int cfsa_ns_set_inlet_profile(cfsa_ns *h, const double *u /*[N2][3]*/);   /* new: per-node inlet */
int cfsa_ns_set_pressure_solver(cfsa_ns *h, int krylov);                   /* new: CG or BiCGSTAB */
/* new: momentum Krylov method, CFSA_KRYLOV_BICGSTAB (default; the reference's Jacobi BiCGSTAB,
 * src/FEM/NavierStokes.cpp:498-515) or CFSA_KRYLOV_CG (Jacobi-preconditioned CG on the same
 * system: M/dt + K + the 1e10 Dirichlet penalty is symmetric positive definite because the
 * convection term is explicit; one sparse product per iteration instead of two; same stopping
 * rule). With a mixed precision the CG runs in FP32 with FP64 reliable updates, like BiCGSTAB. */
int cfsa_ns_set_momentum_solver(cfsa_ns *h, int krylov);
/* new: aggregate count the CFSA_KRYLOV_CG2L coarse space aims for (default 256, 1..1024, others
 * are rejected with CFSA_BAD_ARG). The aggregates are boxes of a uniform grid, so the number
 * actually occupied can exceed the target (256 requested gives 432 on the 1M-tet cylinder); the
 * host Cholesky of the coarse matrix grows with the cube of the occupied count (~0.1 s at 432 on
 * that mesh). The coarse space is rebuilt with the Poisson operator. Its per-aggregate arrays (6 doubles each) share
 * the solve kernel's shared memory with the row staging: a coarse space that does not fit (very
 * large targets on very large meshes) fails the next step with CFSA_CUDA_ERROR and says so in
 * cfsa_ns_last_error. */
int cfsa_ns_set_coarse_target(cfsa_ns *h, int target);
/* new: aggregates of the current CFSA_KRYLOV_CG2L coarse space (built on demand; 0 for the other
 * methods or when the coarse operator was not SPD) */
int cfsa_ns_get_coarse_size(cfsa_ns *h, int *nc);
int cfsa_ns_set_precision(cfsa_ns *h, int precision);                      /* new: FP64 or mixed */
int cfsa_ns_set_convergence_norm(cfsa_ns *h, int norm);                     /* new: see CFSA_NORM_* */
/* Fluid viscosity; stiffness (scaled by 1/viscosity, NavierStokes.cpp:153) is re-assembled. */
int cfsa_ns_set_viscosity(cfsa_ns *h, double viscosity);

/* initialize() field set-up (NavierStokes.cpp:22-46): zero fields, inlet nodes take the current
 * inlet value, time reset to 0. */
int cfsa_ns_initialize_fields(cfsa_ns *h);

/* build_sparse_matrices (include/FEM/NavierStokes.hpp:97-102): re-assemble M, K, G, L on the
 * device from the current vertex coordinates (patterns are reused). */
int cfsa_ns_assemble(cfsa_ns *h);
/* Mesh motion (Mesh::updateGeometry, include/Mesh/Mesh.hpp:98-101): new vertex coordinates
 * [nv][3]; re-assembles. */
int cfsa_ns_update_vertices(cfsa_ns *h, const double *xyz);
/* New boundary tags (coupled BC remapping, src/Numerics/CoupledSolver.cpp:113-129). */
int cfsa_ns_update_boundary_tags(cfsa_ns *h, const int8_t *p1_bc, const int8_t *p2_bc);

/* ---- stepping ---- */
int cfsa_ns_piso_step(cfsa_ns *h);                          /* pisoStep, NavierStokes.cpp:374-414 */
int cfsa_ns_piso_steps(cfsa_ns *h, int n, int *n_done);     /* n x pisoStep, one sync at the end */
int cfsa_ns_simple_step(cfsa_ns *h);                        /* simpleStep, NavierStokes.cpp:968-1009 */
int cfsa_ns_momentum_predictor(cfsa_ns *h);                 /* solveMomentumPredictor, :416-524 */
int cfsa_ns_pressure_poisson(cfsa_ns *h);                   /* solvePressurePoisson, :586-668 */
/* solvePressureBiCGSTAB (src/FEM/NavierStokes.cpp:773-802): solves L x = rhs with Jacobi BiCGSTAB
 * on the raw Poisson matrix (no outlet or reference penalty) from a zero initial guess, stopping at
 * ||r|| <= tol ||rhs|| or after maxit iterations (the reference uses tol 1e-8, maxit 1000).
 * rhs, x: [nv] host arrays; x receives the last iterate. Returns CFSA_NOT_CONVERGED or
 * CFSA_BREAKDOWN when the solve fails (the reference's false). The solver's fields are unchanged. */
int cfsa_ns_solve_pressure_bicgstab(cfsa_ns *h, const double *rhs, double *x, double tol, int maxit);
int cfsa_ns_correct_velocity(cfsa_ns *h);                   /* correctVelocity, :702-771 */

/* ---- fields ---- */
int cfsa_ns_get_velocity(cfsa_ns *h, double *u /*[N2][3]*/);          /* getVelocity */
int cfsa_ns_get_velocity_star(cfsa_ns *h, double *u /*[N2][3]*/);
int cfsa_ns_get_pressure(cfsa_ns *h, double *p /*[nv]*/);             /* getPressure */
int cfsa_ns_get_pressure_correction(cfsa_ns *h, double *p /*[nv]*/);
/* new (the reference's getters are synchronous, getVelocity/getPressure): stream-ordered
 * read-back of the current u ([N2][3]) or p ([nv]) into a host array. The call snapshots the field
 * on the device after the work enqueued so far and returns at once; the copy to `u` / `p` runs
 * while later steps compute. The host array must stay valid, and is complete, only after
 * cfsa_ns_wait_outputs (or a later read-back of the same field, which waits for the previous one
 * to release the snapshot first). Pinned host memory makes the copy truly asynchronous. */
int cfsa_ns_get_velocity_async(cfsa_ns *h, double *u /*[N2][3]*/);
int cfsa_ns_get_pressure_async(cfsa_ns *h, double *p /*[nv]*/);
int cfsa_ns_wait_outputs(cfsa_ns *h);
int cfsa_ns_set_fields(cfsa_ns *h, const double *u /*[N2][3] or NULL*/, const double *p /*[nv] or NULL*/);
int cfsa_ns_get_time(const cfsa_ns *h, double *t);                    /* getTime */
/* new: binary state file for restarts (the reference has none: its VTK output cannot be read
 * back). cfsa_ns_save_state writes u ([N2][3]), p ([nv]), the time and the step count after a
 * header holding a format tag, N2 and nv; cfsa_ns_load_state reads such a file into a handle
 * whose mesh has the same N2 and nv (CFSA_BAD_ARG otherwise, or on an I/O error, with the reason
 * in cfsa_ns_last_error). Operators, parameters and the inlet are not part of the file. */
int cfsa_ns_save_state(cfsa_ns *h, const char *path);
int cfsa_ns_load_state(cfsa_ns *h, const char *path);
int cfsa_ns_get_stats(const cfsa_ns *h, cfsa_ns_stats *s);

/* ---- operators ---- */
/* computeDivergence (NavierStokes.cpp:670-700) of a host velocity field. */
int cfsa_ns_compute_divergence(cfsa_ns *h, const double *u /*[N2][3]*/, double *div /*[nv]*/);
/* computeAdvectionRHS (NavierStokes.cpp:526-584) of the current velocity. */
int cfsa_ns_compute_advection(cfsa_ns *h, double *conv /*[N2][3]*/);
/* computeShearStress / computePressureForces / computeTotalFluidForces (NavierStokes.cpp:841-965)
 * of the current fields; outputs [nv][3]. Requires boundary faces in the mesh view. */
int cfsa_ns_compute_shear_stress(cfsa_ns *h, double *out);
int cfsa_ns_compute_pressure_forces(cfsa_ns *h, double *out);
int cfsa_ns_compute_total_fluid_forces(cfsa_ns *h, double *out);

/* ---- matrices (CSR, ascending columns) ---- */
int cfsa_ns_get_matrix_size(cfsa_ns *h, int which, int64_t *nrows, int64_t *nnz);
int cfsa_ns_get_matrix(cfsa_ns *h, int which, int64_t *rowptr, int32_t *cols, double *vals);
/* 1/rowsum(M) (NavierStokes.cpp:290-306) */
int cfsa_ns_get_inv_lumped_mass(cfsa_ns *h, double *out /*[N2]*/);

/* ---- diagnostics (no counterpart in the reference) ---- */
/* Times `iters` back-to-back launches of one step kernel on the handle's stream with CUDA events,
 * on the current device data, without touching the solver state. avg_ms: mean duration of one
 * launch; alg_bytes: algorithmic bytes one launch must move (matrix values and column indices,
 * row metadata, each vector element read or written once). */
int cfsa_ns_profile_kernel(cfsa_ns *h, int which, int iters, double *avg_ms, double *alg_bytes);
/* Bound on the polls a CTA of the resident pressure solvers (CG, CFSA_KRYLOV_CG1, CG2L) makes at
 * a grid barrier before it gives up: the solve then stops, the step fails with CFSA_CUDA_ERROR
 * ("gave up waiting at a grid barrier"), time does not advance, and the handle stays usable.
 * polls < 0 restores the default (2^25 polls, over a second); 0 gives up at the first wait, which
 * tests use to exercise the failure path. */
int cfsa_ns_set_barrier_spin_limit(cfsa_ns *h, int64_t polls);

/* ---- allocation-free operator (no counterpart in the reference) ---- */
/* Divergence (the computeDivergence operator above) for callers that cannot allocate device
 * memory when they call it: a host framework whose caching pool allocator has already reserved
 * the whole device (cudaMalloc then fails with out-of-memory although the pool has room), and
 * coupling loops that call the operator many times per step, where cudaMalloc/cudaFree would
 * synchronise the device and stall the caller's other streams. Inputs and outputs are the
 * caller's device arrays: u_dev [3][N2] component-major doubles (all x, then all y, then all z),
 * div_dev [nv] doubles. The per-tet intermediate lives in a file-scope static device array of
 * 1,048,576 doubles (8 MiB), held by every GPU that loads this library until the process exits;
 * meshes with more tets are rejected with CFSA_BAD_ARG. The first call on a device looks that
 * array's address up, so make the first call before any stream capture. Every call shares the one
 * array and every entry a call reads is written by the same call first, so nothing needs
 * clearing; calls that overlap on the GPU (other threads or other handles) race on it.
 * The kernels run on the handle's stream, not on the caller's: finish writing u_dev first (for
 * example, synchronise the stream that produced it). The call returns once div_dev is written and
 * leaves the caller's current device as it found it. */
int cfsa_ns_compute_divergence_noalloc(cfsa_ns *h, const double *u_dev, double *div_dev);

/* ---- output ---- */
/* io::exportToVtk(filename, const NavierStokesSolver&, scale) (src/IO/VtkExport.cpp:49-84,
 * 238-268): legacy ASCII VTK unstructured grid of the P1 mesh (points scaled by `scale`), point
 * data FluidBoundaryType, pressure and velocity (scaled) on the P1 vertices, formatted as the
 * reference writes them. The fields are copied from the device asynchronously while the points
 * and cells are formatted. `fields` adds (new) boundary-force vectors per vertex: */
#define CFSA_VTK_SHEAR_STRESS 1    /* computeShearStress (NavierStokes.cpp:874-944) */
#define CFSA_VTK_PRESSURE_FORCES 2 /* computePressureForces (NavierStokes.cpp:841-873) */
int cfsa_ns_write_vtk(cfsa_ns *h, const char *path, double scale, int fields);

/* ---- discrete adjoint (no counterpart in the reference) ----
 * Reverse mode through the PISO steps exactly as the forward kernels compute them (every Krylov
 * solve taken as the exact linear solve it converges to). The differentiated map is
 *   (inlet values g [N2][3], viscosity) -> J(u^N, p^N),
 * N PISO steps from the state (u^0, p^0) held when cfsa_ns_adjoint_forward starts, which is held
 * fixed (its adjoint is returned as dJ/du0, dJ/dp0 so that callers can chain). The pair
 * forward/backward is used like a torch.autograd.Function: forward runs and records, backward
 * takes the objective (or a caller seed dJ/du^N, dJ/dp^N) and returns the gradients.
 * Objectives read the fields computeShearStress / getPressure expose (NavierStokes.cpp:874-944). */
#define CFSA_OBJECTIVE_WALL_SHEAR 0    /* mean over wall vertices with lo <= x[axis] <= hi of |s_v|^2,
                                          s = computeShearStress (traction per vertex) */
#define CFSA_OBJECTIVE_PRESSURE_DROP 1 /* mean p over inlet vertices - mean p over outlet vertices */

typedef struct {
  int32_t kind; /* CFSA_OBJECTIVE_* */
  int32_t axis; /* wall-shear patch: coordinate axis 0..2 */
  double lo, hi;
} cfsa_objective;

typedef struct {
  int64_t steps;             /* recorded forward steps N */
  int32_t checkpoint_every;  /* steps per checkpoint segment */
  int32_t checkpoints;       /* stored (u, p) checkpoints */
  int64_t recomputed_steps;  /* forward steps re-run by the last backward pass */
  int64_t momentum_iters;    /* adjoint Krylov iterations of the last backward pass */
  int64_t pressure_iters;
  double forward_ms;         /* device time of the forward pass (CUDA events) */
  double backward_ms;        /* device time of the last backward pass, recomputation included */
  int64_t record_bytes;      /* device memory held by checkpoints and step records */
  int64_t kernel_launches;   /* device kernels launched by the last backward pass */
} cfsa_adjoint_stats;

/* Objective value on the current fields. */
int cfsa_ns_objective(cfsa_ns *h, const cfsa_objective *obj, double *J);
/* Forward half: runs nsteps PISO steps (same kernels and results as cfsa_ns_piso_steps) and keeps
 * a checkpoint of (u, p) every checkpoint_every steps plus the per-step data of the last segment
 * (u^n on P1 vertices and u* of each step). checkpoint_every <= 0 chooses the largest segment
 * whose step records fit in half of the free device memory (no recomputation when all steps
 * fit). The backward pass re-runs each earlier segment from its checkpoint. Any later change of
 * parameters, inlet values, tags or geometry invalidates the recording. */
int cfsa_ns_adjoint_forward(cfsa_ns *h, int nsteps, int checkpoint_every, int *n_done);
/* Backward half for a built-in objective, evaluated on the recorded final state. Outputs may be
 * NULL: J; grad_inlet [N2][3] = dJ/dg (zero off inlet nodes); grad_viscosity = dJ/dnu;
 * grad_u0 [N2][3], grad_p0 [nv]. The solver's fields are left at the recorded final state. */
int cfsa_ns_adjoint_backward(cfsa_ns *h, const cfsa_objective *obj, double *J, double *grad_inlet,
                             double *grad_viscosity, double *grad_u0, double *grad_p0);
/* Backward half from a caller seed dJ/du^N [N2][3], dJ/dp^N [nv] and the explicit dJ/dnu. */
int cfsa_ns_adjoint_backward_seed(cfsa_ns *h, const double *dJ_du, const double *dJ_dp,
                                  double dJ_dviscosity, double *grad_inlet, double *grad_viscosity,
                                  double *grad_u0, double *grad_p0);
int cfsa_ns_get_adjoint_stats(cfsa_ns *h, cfsa_adjoint_stats *out);

#ifdef __cplusplus
}
#endif

#endif /* CFSA_NS_H */
