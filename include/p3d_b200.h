/*
 * p3d_b200 -- B200-native matrix-free Q2-P1disc Stokes operators for pTatin3d.
 *
 * Plain C ABI: every entry point takes plain pointers and sizes, returns an
 * int status (P3D_OK == 0, never exits), and does not expose CUDA or torch
 * types beyond an opaque stream handle (a cudaStream_t passed as void*; NULL
 * means the default stream).
 *
 * Reference interfaces replaced (paths relative to the pTatin3d tree):
 *   - the A11 SpMVOp callback triple {SpMVOp_MatMult, SpMVOp_SetUp,
 *     SpMVOp_Destroy} of struct _p_MatA11MF       include/stokes_operators.h:47-62
 *   - MFStokesWrapper_A11_CUDA / _Tensor / _AVX     src/stokes_operators_cuda.cu:457-532,
 *                                                   src/stokes_operators_tensor.c:181-288,
 *                                                   src/stokes_operators_avx.c:206-315
 *   - MatGetDiagonal_MFStokes_A11 / MFStokesWrapper_diagA11
 *                                                   src/stokes_operators.c:1060-1099,
 *                                                   src/stokes_operators_mf.c:67-131
 *   - MatMult_MFStokes_A12 / A21 (MFStokesWrapper_A12/_A21)
 *                                                   src/stokes_operators.c:1284-1486,
 *                                                   src/stokes_operators_mf.c:788-933
 *   - MatMult_MFStokes_A (fused A11+A12+A21)        src/stokes_operators.c:884-967,
 *                                                   src/stokes_operators_mf.c:707-786
 *   - BCListInsertLocalZero / BCListInsertDirichlet_MatMult /
 *     BCListInsertValueIntoDirichletSlot            src/dmda_bcs.c:409-611
 *   - PCMG interpolation/restriction Mats (DMCreateInterpolation on the Q2
 *     node lattice)                                 src/ptatin_driver_linear_ts.c:850,986-990
 *
 * Data layout (identical to the reference's ghosted local arrays):
 *   velocity / coordinates : node-lexicographic (x fastest) on the ghosted
 *                            node lattice gx*gy*gz, 3 interleaved components
 *   viscosity              : eta[e*27 + q], e lexicographic over the local
 *                            elements (x fastest), q = qi + 3qj + 9qk
 *   pressure (P1disc)      : p[e*4 + i], basis [1, xh, yh, zh]
 */
#ifndef P3D_B200_H
#define P3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------- status ---- */
#define P3D_OK 0
#define P3D_ERR_ARG 1     /* bad argument / size mismatch                  */
#define P3D_ERR_CUDA 2    /* a CUDA runtime call failed (message retained) */
#define P3D_ERR_STATE 3   /* call out of order (e.g. apply before setup)   */
#define P3D_ERR_NOMEM 4   /* device allocation failed                      */
#define P3D_ERR_NOCONV 5  /* a solve hit its iteration limit               */
#define P3D_ERR_BREAKDOWN 6 /* a solve produced a non-finite residual      */
#define P3D_ERR_TIMEOUT 7 /* a bounded wait ran out                        */
#define P3D_ERR_CANCELLED 8 /* a served request was cancelled              */

/* ---------------------------------------------------------- meshes ---- */
/* Dirichlet bits: bit (3*face + component), faces in this order.  A bit is
 * honoured only on faces flagged in `global_faces` (faces of the local block
 * that lie on the global domain boundary). */
enum { P3D_FACE_IMIN = 0, P3D_FACE_IMAX, P3D_FACE_JMIN, P3D_FACE_JMAX, P3D_FACE_KMIN, P3D_FACE_KMAX };
#define P3D_BC_BIT(face, comp) (1u << (3u * (unsigned)(face) + (unsigned)(comp)))

typedef struct p3d_mesh_desc {
  int32_t mx, my, mz;        /* local (owned) elements per direction              */
  int32_t gx, gy, gz;        /* ghosted node-lattice extent of the local arrays   */
  int32_t ox, oy, oz;        /* lattice index of the first node of element (0,0,0) */
  uint32_t dirichlet;        /* P3D_BC_BIT mask                                   */
  uint32_t global_faces;     /* bit f set: local face f lies on the global boundary */
} p3d_mesh_desc;

/* Fill a desc for one process owning a whole mx*my*mz mesh (no ghosts). */
int p3d_mesh_desc_whole(int32_t mx, int32_t my, int32_t mz, uint32_t dirichlet, p3d_mesh_desc *out);

/* --------------------------------------------------- device operator --- */
typedef struct p3d_op p3d_op; /* opaque: one mesh + coefficients resident in HBM */

#define P3D_PREC_F64 64
#define P3D_PREC_F32 32

#define P3D_GEOM_AUTO 0    /* affine fast path when every element is a parallelepiped */
#define P3D_GEOM_GENERAL 1 /* per-quadrature-point Jacobian from the coordinates      */
#define P3D_GEOM_AFFINE 2  /* the Jacobian of the element centre at every Gauss point:
                              exact for parallelepipeds; on any other mesh it is the
                              reference's low-order operator MatMult_MFStokes_A11LowOrder
                              (ONEPOINTQ, src/stokes_operators.c:1207-1278,
                              src/stokes_operators_mf.c:353-488)                     */
#define P3D_GEOM_LOWORDER P3D_GEOM_AFFINE

#define P3D_BC_NONE 0      /* raw element apply: y += sum_e A_e x  (SpMVOp contract)   */
#define P3D_BC_MATMULT 1   /* MatMult contract: Dirichlet columns zeroed, rows y_k = x_k */

/* Create an operator on device `device` for the mesh; precision P3D_PREC_*. */
int p3d_op_create(const p3d_mesh_desc *mesh, int precision, int device, p3d_op **op);
int p3d_op_destroy(p3d_op *op);
/* Upload geometry and coefficients (host arrays, FP64).  coords: 3*gx*gy*gz,
 * eta: 27*mx*my*mz.  Re-callable whenever the reference's Mat state changes
 * (src/stokes_operators_cuda.cu:413-421). geom_mode: P3D_GEOM_*. */
int p3d_op_set_coefficients(p3d_op *op, const double *coords, const double *eta, int geom_mode);
/* Same, from device arrays already in HBM (FP64). */
int p3d_op_set_coefficients_device(p3d_op *op, const double *coords_dev, const double *eta_dev, int geom_mode);
int p3d_op_set_bc_mode(p3d_op *op, int bc_mode);
/* Which geometry path setup selected (P3D_GEOM_GENERAL or P3D_GEOM_AFFINE). */
int p3d_op_geometry_mode(const p3d_op *op, int *mode);
/* Sizes: velocity dofs 3*gx*gy*gz, pressure dofs 4*mx*my*mz. */
int p3d_op_sizes(const p3d_op *op, int64_t *n_velocity, int64_t *n_pressure);

/* Device-pointer applies, asynchronous on `stream`.  Element type is the
 * operator's precision (double* for F64, float* for F32).  All ADD into y
 * (the caller zeroes y, as MatMult_MFStokes_A11 does at
 * src/stokes_operators.c:1181); with P3D_BC_MATMULT the Dirichlet rows are
 * overwritten with x instead. */
int p3d_a11_apply(p3d_op *op, const void *x, void *y, void *stream);
/* MatMult contract, y = A11 x (MatMult_MFStokes_A11, src/stokes_operators.c:1142-1205,
 * which zeroes Yu and then adds): y is overwritten and never read, which
 * saves the read of y that the "+=" form needs. */
int p3d_a11_mult(p3d_op *op, const void *x, void *y, void *stream);
/* The MatMult of k operators at once (no counterpart in the reference,
 * which applies one operator per process): y[i] = A11_i x[i] for k <= 32
 * operators of the same mesh shape, precision, geometry path and boundary
 * mode (the solves of a served batch), in one zeroing launch and one
 * element-kernel launch whose grid covers the bricks of every member. */
#define P3D_GROUP_MAX 32
int p3d_a11_mult_grouped(p3d_op *const ops[], const void *const x[], void *const y[], int32_t k, void *stream);
int p3d_a11_diagonal(p3d_op *op, void *d, void *stream);           /* d += diag(A11); Dirichlet slots = 1 with MATMULT */
int p3d_a12_apply(p3d_op *op, const void *p, void *yu, void *stream);  /* yu += A12 p; Dirichlet rows 0 with MATMULT */
int p3d_a21_apply(p3d_op *op, const void *u, void *yp, void *stream);  /* yp += A21 u; Dirichlet columns zeroed with MATMULT */
int p3d_stokes_apply(p3d_op *op, const void *u, const void *p, void *yu, void *yp, void *stream); /* [A11 A12; A21 0] */

/* Residual of the Stokes equations (FormFunction_Stokes with FormFunctionLocal_U
 * and FormFunctionLocal_P, src/stokes_form_function.c:99-243, 357-564), FP64
 * device arrays: the Dirichlet values phi (3*nn, read at Dirichlet dofs only;
 * NULL = 0) are inserted into u, then
 *   ru = A11 u + A12 p - f_u,   rp = A21 u - f_p,
 * with f_u = sum_q w detJ N fu_q (fu: 3 per Gauss point, 81*nel, the Fu of the
 * reference's QPntVolCoefStokes; NULL = 0) and f_p = sum_q w detJ Np fp_q (fp:
 * 27*nel, the Fp; NULL = 0); finally the Dirichlet rows are ru_k = u_k - phi_k.
 * Calls on one operator must not overlap (the operator's boundary mode is
 * switched for the element pass). */
int p3d_stokes_residual(p3d_op *op, const double *u, const double *p, const double *phi, const double *fu,
                        const double *fp, double *ru, double *rp, void *stream);

/* Host-buffer apply with the reference CUDA backend's synchronous contract
 * (src/stokes_operators_cuda.cu:457-532): copies x in, applies into a zeroed
 * device y, copies y out (y = A11 x, overwriting y as the reference backend's
 * CopyFrom_A11_CUDA does; its caller has zeroed Yu, so this equals the
 * SpMVOp "+=" contract), and returns when y is complete. */
int p3d_a11_apply_host(p3d_op *op, const double *x_host, double *y_host);
/* Split p3d_a11_apply_host into `chunks` z-ranges of brick layers (0 =
 * automatic: 16 for meshes of 4M dofs and more, else 1) whose host->device
 * copies, applies and device->host copies overlap on three streams. */
int p3d_op_set_host_chunks(p3d_op *op, int chunks);
/* enable != 0: p3d_a11_apply_host page-locks (cudaHostRegister) each host
 * array it is given that is not page-locked yet, once, and keeps it so, which
 * lets the copies of every later apply run at full PCIe speed.  The reference
 * backend copies PETSc's pageable local arrays on every MatMult
 * (src/stokes_operators_cuda.cu:403,453); a MatShell binding that reuses the
 * DM's local vectors turns this on once.  Registered arrays must stay
 * allocated until the operator is destroyed or this is called with enable = 0,
 * which unregisters them (at most 16 ranges per operator; beyond that, and
 * where registration fails, the copies go the pageable way). */
int p3d_op_set_host_register(p3d_op *op, int enable);

/* Same result as p3d_a11_apply_host, without allocating any device memory
 * (no counterpart in the reference).  For callers that may not call
 * cudaMalloc/cudaFree, e.g. a MatShell callback running while the application
 * owns the device memory pool.  The x/y staging lives in a fixed file-scope
 * device array of P3D_NOALLOC_MAX_DOFS doubles each, resident on every device
 * that loads the library until the process exits; larger meshes return
 * P3D_ERR_ARG.  The first call on a device looks up that array's address
 * (cudaGetSymbolAddress), so make it before any stream capture; that address
 * is kept, so do not use this entry point again after resetting the device
 * (cudaDeviceReset) in the same process.  Calls share the array: calls whose
 * work overlaps on the GPU race. */
#define P3D_NOALLOC_MAX_DOFS 107811 /* 3 * 33^3: a 16^3-element Q2 mesh */
int p3d_a11_apply_host_noalloc(p3d_op *op, const double *x_host, double *y_host);

/* --------------------------------------- multigrid transfer (DMDA) ---- */
/* Trilinear prolongation on the node lattice, coarse (cnx,cny,cnz) nodes ->
 * fine (2c-1) nodes, `ndof` interleaved components; xf = P xc (overwrite).
 * Restriction is the transpose: xc = P^T xf (overwrite).  `prec` selects
 * double or float element type. */
int p3d_mg_prolong(int prec, int cnx, int cny, int cnz, int ndof, const void *xc, void *xf, void *stream);
int p3d_mg_restrict(int prec, int cnx, int cny, int cnz, int ndof, const void *xf, void *xc, void *stream);

/* ------------------------------------------------ z-slab exchange ---- */
/* One node plane of a z-slab partitioned velocity vector (3 components per
 * node of the (2mx+1) x (2my+1) plane): y_plane += recv, then the plane's
 * Dirichlet rows (x/y face bits of `dirichlet`) reset to x_plane.  The
 * receiving half of DMLocalToGlobal(ADD) on a shared slab plane followed by
 * the MatMult row convention (src/stokes_operators.c:1192-1201).  Device
 * arrays of `prec`; asynchronous on `stream`. */
int p3d_slab_add_plane(int prec, int32_t mx, int32_t my, uint32_t dirichlet, const void *recv, const void *x_plane,
                       void *y_plane, void *stream);

/* ------------------------------- material points -> Gauss points ---- */
/* Viscosity and density of material points (markers) onto the 27 Gauss
 * points of every element of one whole mx*my*mz mesh, by the projection types
 * of the reference's rheology update (coefficient_projection_type in
 * pTatin_EvaluateRheologyNonlinearities, src/rheology.c:150-185):
 *   P3D_PROJ_NULL            keep the Gauss-point values (case -1)
 *   P3D_PROJ_P0_ARITHMETIC   element average of the markers' eta (arithmetic,
 *   P3D_PROJ_P0_HARMONIC     harmonic or geometric) and of rho (arithmetic) on
 *   P3D_PROJ_P0_GEOMETRIC    all 27 points; an element without markers gets
 *                            0/0 (MPntPStokesProj_P0,
 *                            src/material_point_utils.c:2567-2808)
 *   P3D_PROJ_Q1              nodal average on the Q2 lattice (Q1 weights at
 *                            the element corners, 1 at the other Q2 nodes;
 *                            nodes without weight get 0), then Q1
 *                            interpolation of the corners clamped to the
 *                            element's nodal range
 *                            (SwarmUpdateGaussPropertiesLocalL2Projection_Q1_MPntPStokes,
 *                            src/material_point_utils.c:604-891)
 *   P3D_PROJ_ONE2ONE         marker p is Gauss point p, n == 27*nel
 *                            (SwarmUpdateGaussPropertiesOne2OneMap_MPntPStokes, :803-840)
 * Markers (device arrays, the fields of MPntStd / MPntPStokes): wil[n]
 * element index (x fastest; markers outside [0, nel) are skipped), xi[3n]
 * local coordinates in [-1,1]^3 (Q1 only), eta_p[n], rho_p[n].  Output:
 * eta_q, rho_q [27*nel] device arrays (element-major, q = qi + 3qj + 9qk).
 * `workspace`: device memory of p3d_marker_project_workspace bytes, 8-byte
 * aligned (may be NULL when that is 0).  After P3D_PROJ_Q1 it holds the nodal
 * viscosity [nn] followed by the nodal density [nn], nn = (2mx+1)(2my+1)(2mz+1)
 * (the input of p3d_solver_setup_nodal).  Asynchronous on `stream`. */
#define P3D_PROJ_NULL (-1)
#define P3D_PROJ_P0_ARITHMETIC 0
#define P3D_PROJ_Q1 1
#define P3D_PROJ_ONE2ONE 4
#define P3D_PROJ_P0_HARMONIC 10
#define P3D_PROJ_P0_GEOMETRIC 20
int p3d_marker_project_workspace(int32_t mx, int32_t my, int32_t mz, int type, int64_t *bytes);
int p3d_marker_project(int32_t mx, int32_t my, int32_t mz, int type, int64_t n, const int32_t *wil, const double *xi,
                       const double *eta_p, const double *rho_p, double *eta_q, double *rho_q, void *workspace,
                       void *stream);

/* ------------------------------------------------------ Stokes solve --- */
/* Device-resident solve of the Q2-P1disc Stokes system on one whole mesh:
 * outer FGMRES (FP64 residual and orthogonalisation) right-preconditioned by
 * the block upper-triangular factorisation [A11 A12; 0 S]^{-1}, S the
 * viscosity-scaled pressure mass matrix (exact 4x4 block inverse per element),
 * A11^{-1} by one geometric-multigrid V-cycle: Jacobi-preconditioned
 * Chebyshev smoothing with the matrix-free A11 on every level above the
 * coarsest, trilinear node-lattice transfers, and a Galerkin coarse operator
 * P^T A P inverted densely.  With mg_precision = P3D_PREC_F32 the smoother
 * applies, transfers and stored coefficients run in FP32 while the outer
 * Krylov iteration, the Schur update, the Jacobi diagonal and the coarse solve
 * stay FP64.  Replaces the PETSc solver stack the reference configures in
 * pTatin3dStokesKSPConfigureFSGMG / pTatin3dCreateStokesOperators
 * (src/ptatin_driver_linear_ts.c:558-882). */
typedef struct p3d_solver p3d_solver;

typedef struct p3d_solver_opts {
  int32_t nlevels;      /* multigrid levels, >= 1 (mesh coarsened by 2 per level)   */
  int32_t cheb_its;     /* Chebyshev iterations per pre/post smoothing              */
  double cheb_lo;       /* smoothing interval [cheb_lo*lmax, cheb_hi*lmax]          */
  double cheb_hi;       /*   (the reference's -esteig 0,0.2,0,1.1)                  */
  int32_t esteig_its;   /* CG-Lanczos iterations estimating lmax(D^{-1}A)           */
  int32_t mg_precision; /* P3D_PREC_F64 or P3D_PREC_F32 (mixed precision)           */
  int32_t restart;      /* FGMRES restart length (<= P3D_MAX_RESTART)               */
  int32_t max_it;       /* outer iteration limit                                    */
  double rtol;          /* ||r_k|| <= max(rtol*||r_0||, atol)                       */
  double atol;
  int32_t use_graph;    /* capture the preconditioner in a CUDA graph               */
  int32_t verbose;
  int32_t inner_its;    /* velocity-block solve inside the preconditioner: 0 = one
                           V-cycle; k > 0 = k conjugate-gradient iterations on A11
                           preconditioned by the V-cycle (the reference's inner
                           -fieldsplit_u_ksp); with inner_rtol > 0, at most k    */
  int32_t coarse_op;    /* operators of the coarse levels: P3D_COARSE_GALERKIN
                           (P^T A P, 27-point block stencils probed from the
                           finer level) or P3D_COARSE_REDISC (matrix-free
                           rediscretisation with restricted viscosity)            */
  int32_t schur_eta;    /* viscosity weighting of the pressure mass matrix in the
                           Schur approximation: P3D_SCHUR_ETA_QP (1/eta at every
                           quadrature point, the reference's ScaledMassMatrix) or
                           P3D_SCHUR_ETA_GEOMEAN (1/eta_e, eta_e the element's
                           geometric-mean viscosity)                              */
  int32_t coarse_eta;   /* Gauss-point viscosity of rediscretised coarse levels:
                           P3D_COARSE_ETA_GEOMEAN (geometric mean of the nearest
                           finer Gauss points) or P3D_COARSE_ETA_Q1 (the
                           reference's Q1 projection hierarchy: nodal projection,
                           scaled restriction, clamped interpolation)            */
  double inner_rtol;    /* > 0: the inner conjugate gradients stop once
                           |b - A11 x| <= inner_rtol |b| (-fieldsplit_u_ksp_rtol,
                           1e-2 in the reference's sinker tests) or after
                           inner_its iterations.  The loop runs on the device: a
                           conditional WHILE node of the captured preconditioner
                           graph, its condition set from the device-held residual.
                           0: a fixed inner_its iterations                        */
} p3d_solver_opts;

#define P3D_COARSE_ETA_GEOMEAN 0
#define P3D_COARSE_ETA_Q1 1
#define P3D_SCHUR_ETA_QP 0
#define P3D_SCHUR_ETA_GEOMEAN 1
#define P3D_COARSE_GALERKIN 0
#define P3D_COARSE_REDISC 1

#define P3D_MAX_RESTART 120   /* FGMRES basis vectors kept                        */
#define P3D_COARSE_MAX_DOFS 16384 /* largest coarse level inverted densely        */

typedef struct p3d_solve_stats {
  int32_t iterations;   /* outer FGMRES iterations                                  */
  int32_t converged;
  double r0, rfinal;    /* unpreconditioned residual 2-norms                        */
  double setup_ms, solve_ms;
  double lmax_fine;     /* estimated lmax(D^{-1}A) on the finest level              */
  int32_t coarse_dofs;
  int32_t inner_iterations; /* inner conjugate-gradient iterations of the solve
                               (tolerance-driven inner solves; 0 otherwise)      */
  int32_t group_members;    /* most solves this one shared its launches with,
                               itself included (1: solved alone)                 */
} p3d_solve_stats;

int p3d_solver_default_opts(p3d_solver_opts *opts);
/* Upper estimate of the device memory a solver of this mesh and options
 * holds after setup (used to admit solves by HBM footprint). */
int p3d_solver_estimate_bytes(const p3d_mesh_desc *mesh, const p3d_solver_opts *opts, int64_t *bytes);
/* mesh: a whole mesh (p3d_mesh_desc_whole); mx,my,mz divisible by 2^(nlevels-1). */
int p3d_solver_create(const p3d_mesh_desc *mesh, const p3d_solver_opts *opts, int device, p3d_solver **solver);
/* Device FP64 arrays: coords 3*nn, eta 27*nel.  Builds the hierarchy, the
 * operators, smoother bounds, the coarse inverse and the Schur blocks. */
int p3d_solver_setup(p3d_solver *s, const double *coords_dev, const double *eta_dev);
/* The same with the finest level's nodal viscosity [nn] given: the Q1
 * coefficient hierarchy (coarse_op P3D_COARSE_REDISC, coarse_eta
 * P3D_COARSE_ETA_Q1) restricts it instead of a projection of eta_dev.  This is
 * the reference's hierarchy for projection type 1, whose nodal field comes from
 * the markers (SwarmUpdateGaussPropertiesLocalL2Projection_Q1_MPntPStokes_Hierarchy,
 * src/material_point_utils.c:1267-1360); p3d_marker_project leaves that field
 * in its workspace.  Other options return P3D_ERR_ARG. */
int p3d_solver_setup_nodal(p3d_solver *s, const double *coords_dev, const double *eta_dev, const double *eta_nodes_dev);
/* Right-hand side from a Gauss-point density field and gravity vector
 * (Dirichlet rows zero); or set b directly (device arrays). */
int p3d_solver_set_rhs_body_force(p3d_solver *s, const double *rho_dev, double gx, double gy, double gz);
int p3d_solver_set_rhs(p3d_solver *s, const double *bu_dev, const double *bp_dev);
/* Solve; u (3*nn) and p (4*nel) are device FP64 arrays holding the initial
 * guess on entry and the solution on return. */
int p3d_solver_solve(p3d_solver *s, double *u_dev, double *p_dev, p3d_solve_stats *stats);
/* Solve k <= 32 solvers of one mesh shape and option set (each set up, with
 * its right-hand side) together: the FGMRES iterations of all members run in
 * lock-step, and every kernel of an iteration -- operators, smoothers,
 * transfers, stencils, coarse solves, Gram-Schmidt -- is one launch over all
 * members, the block preconditioner of all members one captured graph (no
 * counterpart in the reference, which solves one system per process).  Each
 * member keeps its own Krylov basis, step lengths and stopping test; a member
 * that converges, breaks down or reaches max_it leaves the group (its u, p
 * written) and the others go on.  Members need one V-cycle per outer
 * iteration (inner_its = 0, inner_rtol = 0) and at least 2 levels.  u[i],
 * p[i]: device initial guesses in, solutions out; stats[i] per member
 * (solve_ms from the start to the member's own exit; group_members the
 * largest group it shared launches with); status[i] (may be NULL): P3D_OK,
 * P3D_ERR_NOCONV, P3D_ERR_BREAKDOWN or P3D_ERR_CANCELLED per member.
 * Returns P3D_OK when every member converged, else a member's failure
 * status. */
int p3d_solver_solve_grouped(p3d_solver *const solvers[], int32_t k, double *const u[], double *const p[],
                             p3d_solve_stats stats[], int32_t status[]);
/* One application of the block preconditioner (testing / external Krylov). */
int p3d_solver_apply_pc(p3d_solver *s, const double *ru, const double *rp, double *zu, double *zp);
/* y = A_l x with the FP64 velocity operator of multigrid level `level`
 * (0 = coarsest), Dirichlet rows identity (testing the hierarchy). */
int p3d_solver_level_apply(p3d_solver *s, int level, const double *x_dev, double *y_dev);
int p3d_solver_destroy(p3d_solver *s);

/* ------------------------------------------------------- solve server --- */
/* A persistent request loop for independent Stokes solves of uneven mesh
 * sizes (no counterpart in the reference, which runs one solve per process).
 * Requests are admitted first-in first-out as soon as one of `max_active`
 * workers and the device memory they need (p3d_solver_estimate_bytes) are
 * free; a worker also takes the queued requests of the head's shape that fit
 * and solves them as one group (shared launches, p3d_server_set_group_max).
 * Groups of different shapes run concurrently, each on its own stream, with
 * their state resident in HBM.  Solvers are pooled by mesh and options and
 * reused by later requests of the same shape. */
typedef struct p3d_server p3d_server;

typedef struct p3d_request {
  int32_t mx, my, mz;     /* whole mesh, elements per direction                   */
  uint32_t dirichlet;     /* P3D_BC_BIT mask                                      */
  const double *coords;   /* host, 3*(2mx+1)(2my+1)(2mz+1)                        */
  const double *eta;      /* host, 27*mx*my*mz Gauss-point viscosity              */
  const double *rho;      /* host, 27*mx*my*mz Gauss-point density                */
  double gx, gy, gz;      /* gravity                                              */
  double *u, *p;          /* host outputs, 3*nn and 4*nel (valid after the result) */
  p3d_solver_opts opts;
  int64_t tag;            /* returned in the result                               */
} p3d_request;

typedef struct p3d_result {
  int64_t tag;
  int32_t status;         /* P3D_OK, P3D_ERR_NOCONV (u, p hold the last iterate), ... */
  int32_t iterations;
  double rel_residual;    /* ||r|| / ||r0||                                       */
  double wait_ms;         /* submit -> admitted                                   */
  double run_ms;          /* admitted -> solution copied to the host              */
  double latency_ms;      /* submit -> solution copied to the host                */
} p3d_result;

typedef struct p3d_server_stats {
  int64_t submitted, admitted, completed;
  int32_t active, queued;
  int64_t device_bytes, peak_device_bytes; /* estimated bytes held by pooled solvers */
  int32_t solvers_created, solvers_reused;
  int64_t grouped;        /* requests that shared launches with another one     */
  int64_t groups;         /* rolling groups that had two or more members        */
} p3d_server_stats;

int p3d_server_create(int device, int64_t hbm_budget_bytes, int32_t max_active, p3d_server **server);
/* Up to group_max (1..32, default 8) requests of one mesh shape and option
 * set are solved as one rolling group (the lock-step solve of
 * p3d_solver_solve_grouped: one launch per kernel for all of them).  Queued
 * requests of the group's shape join it at the start of a restart cycle; a
 * member leaves, and its result is posted, as soon as it converges, fails,
 * is cancelled or reaches max_it, while the others go on.  A request joins
 * a group ahead of queued requests of other shapes only if none of them
 * arrived more than the overtake bound before it (default 2000 ms,
 * p3d_server_set_group_overtake_ms), so groups cannot keep a worker from
 * the other shapes indefinitely.  1 solves every request on its own.
 * Requests with an inner velocity solve or one level are always solved
 * alone. */
int p3d_server_set_group_max(p3d_server *server, int32_t group_max);
/* Requests whose mesh has more than max_elements elements (default 16384,
 * i.e. 25^3) are solved alone: grouping pays where the launches of one
 * solve cannot fill the device (small meshes) and costs the memory of every
 * member at once.  0 groups nothing. */
int p3d_server_set_group_elements(p3d_server *server, int64_t max_elements);
/* The overtake bound of the rolling groups in milliseconds (>= 0). */
int p3d_server_set_group_overtake_ms(p3d_server *server, int32_t ms);
/* Non-blocking.  The request's host arrays must stay valid until its result
 * has been returned by p3d_server_poll. */
int p3d_server_submit(p3d_server *server, const p3d_request *request);
/* Up to max_results finished solves.  timeout_ms > 0: waits up to that long
 * for the first and returns P3D_ERR_TIMEOUT (with *n = 0) when none finished
 * in time; timeout_ms <= 0 returns at once (P3D_OK, possibly *n = 0). */
int p3d_server_poll(p3d_server *server, p3d_result *results, int32_t max_results, int32_t timeout_ms, int32_t *n);
/* Cancel the request with this tag.  A queued request completes at once, a
 * running one after its current outer iteration; its result has status
 * P3D_ERR_CANCELLED (u, p hold the last iterate of a running one) and its
 * execution slot and memory go back to the pool.  P3D_ERR_ARG when no queued
 * or running request has the tag (for example one that already finished). */
int p3d_server_cancel(p3d_server *server, int64_t tag);
int p3d_server_get_stats(p3d_server *server, p3d_server_stats *stats);
/* Finishes every submitted solve, then frees the pool. */
int p3d_server_destroy(p3d_server *server);

/* -------------------------------------------------------- diagnostics --- */
/* Last error message of the calling thread (static storage, never NULL). */
const char *p3d_last_error(void);
/* Number of kernels this library launched since load (all devices). */
int64_t p3d_kernel_launch_count(void);
/* Failure injection for tests of the error paths (host side; no GPU fault):
 * after `after` more successful device allocations by this library, every
 * further one fails with P3D_ERR_NOMEM, as an exhausted device would.  A
 * negative value switches the injection off (the default). */
int p3d_debug_fail_allocations_after(int64_t after);
/* Test aid for reads of memory nothing wrote: with fill in [0, 255] every
 * device allocation of this library is filled with that byte before it is
 * handed out (0xFF: every double and float reads as a NaN; 0x3F: as a
 * finite value near 5e-4 / 0.75), so a result that depends on the former
 * contents of reused memory shows up.  fill < 0 switches it off (the
 * default). */
int p3d_debug_poison_allocations(int32_t fill);
/* Library version string. */
const char *p3d_version(void);

#ifdef __cplusplus
}
#endif
#endif /* P3D_B200_H */
