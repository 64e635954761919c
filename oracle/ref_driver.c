/*
 * Driver for the reference's own element kernels, compiled unmodified from
 * the pTatin3d source tree against the PETSc stand-in headers in
 * oracle/shim (see oracle/Makefile).  It supplies the few accessor functions
 * those kernels call (DM coordinates, element connectivity, quadrature-point
 * records, Gauss rule) over plain arrays for ONE process owning the whole
 * mesh, and exports plain-C entry points:
 *
 *   ref_setup(mx,my,mz, coords[3*nn], eta[27*nel])
 *   ref_a11(variant, x[3*nn], y[3*nn])   variant 0=tensor 1=avx 2=ref 3=low-order (MFStokesWrapper_A11PC)
 *   ref_diag(y[3*nn]), ref_a12(p[4*nel], yu[3*nn]), ref_a21(u[3*nn], yp[4*nel]),
 *   ref_a12_avx(p, yu), ref_a_avx(u, p, yu, yp)
 *   ref_marker_project(type, n, wil, xi, eta_p, rho_p, eta_q, rho_q)
 *       the material-point -> Gauss-point projections of the rheology update
 *       (src/rheology.c:150-185; material_point_utils.c, quadrature.c)
 *   ref_solcx_norms(eta0, eta1, xc, n, u, p, norms[4])
 *       error norms of a discrete solution against the SolCx analytic
 *       solution, as the verification model prints them
 *       (src/models/analytics_vv/analytics_vv.c:313-357, src/inorms.c:188-363)
 *
 * Each adds element contributions exactly as the reference's SpMVOp_MatMult
 * callback does (the caller zeroes y and applies Dirichlet rows/columns).
 *
 * TEST INFRASTRUCTURE ONLY: built into oracle/_ref/libp3dref.so, used by
 * tests/ and bench.py's CPU-baseline leg.  The product never links it.
 */
#include <omp.h>
#include <stdarg.h>
#include <sys/time.h>

#include "petsc.h"
#include "ptatin3d.h"
#include "private/ptatin_impl.h"
#include "ptatin3d_stokes.h"
#include "stokes_operators.h"
#include "MPntStd_def.h"
#include "MPntPStokes_def.h"
#include "material_point_utils.h"
#include "inorms.h"
#include "models/analytics_vv/SolCxSolution.h"

/* kernels provided by the reference objects */
PetscErrorCode MFStokesWrapper_A11_Tensor(MatA11MF, Quadrature, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFStokesWrapper_A11_AVX(MatA11MF, Quadrature, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFStokesWrapper_A11(MatA11MF, Quadrature, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFStokesWrapper_A11PC(Quadrature, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFStokesWrapper_diagA11(Quadrature, DM, PetscScalar[]);
PetscErrorCode MFStokesWrapper_A12(Quadrature, DM, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFStokesWrapper_A21(Quadrature, DM, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFStokesWrapper_A12_AVX(Quadrature, DM, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFStokesWrapper_A_AVX(Quadrature, DM, PetscScalar[], DM, PetscScalar[], PetscScalar[], PetscScalar[]);
/* projections provided by the reference objects (material_point_utils.c, quadrature.c) */
PetscErrorCode MPntPStokesProj_P0(CoefficientAveragingType, const int, MPntStd[], MPntPStokes[], DM, Quadrature);
void QuadratureCreateGauss_3pnt_3D(PetscInt *ngp, PetscReal **q_coor, PetscReal **q_weight);

struct _p_shim_Vec {
  PetscScalar *a;
  long n;
};
struct _p_shim_DM {
  int kind; /* 0 velocity (Q2 lattice, stencil 2), 1 pressure (P1disc, stencil 0) */
  PetscInt M, N, P, dof, sw;
  PetscInt nel, npe;
  PetscInt *e;
  struct _p_shim_Vec coords;
  int clone; /* made by DMDADuplicateLayout: shares e and coords, freed by DMDestroy */
};

static struct _p_shim_DM g_dau, g_dap;
static struct _p_Quadrature g_Q;
static QPntVolCoefStokes *g_cells = NULL;
static PetscReal *g_qxi = NULL, *g_qw = NULL;

/* ---------------------------------------------------------- accessors --- */
PetscErrorCode PetscPrintf(MPI_Comm c, const char fmt[], ...) { (void)c; (void)fmt; return 0; }
PetscErrorCode PetscTime(PetscLogDouble *t)
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  *t = tv.tv_sec + 1e-6 * tv.tv_usec;
  return 0;
}
PetscErrorCode MPI_Comm_rank(MPI_Comm c, PetscMPIInt *r) { (void)c; *r = 0; return 0; }
PetscErrorCode MPI_Comm_size(MPI_Comm c, PetscMPIInt *r) { (void)c; *r = 1; return 0; }
PetscErrorCode MPI_Allreduce(const void *a, void *b, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c)
{
  (void)o; (void)c;
  memcpy(b, a, (size_t)n * (t == MPI_DOUBLE ? sizeof(double) : sizeof(int)));
  return 0;
}

/* closed-form 3-point Gauss-Legendre rule on [a,b], ascending nodes */
PetscErrorCode PetscDTGaussQuadrature(PetscInt npoints, PetscReal a, PetscReal b, PetscReal *x, PetscReal *w)
{
  if (npoints != 3) return PETSC_ERR_SUP;
  const double s = sqrt(3.0 / 5.0);
  const double xs[3] = {-s, 0.0, s}, ws[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  for (int i = 0; i < 3; i++) {
    x[i] = 0.5 * (b - a) * xs[i] + 0.5 * (b + a);
    w[i] = 0.5 * (b - a) * ws[i];
  }
  return 0;
}

PetscErrorCode DMGetCoordinateDM(DM dm, DM *cdm) { *cdm = dm; return 0; }
PetscErrorCode DMGetCoordinatesLocal(DM dm, Vec *c) { *c = &dm->coords; return 0; }
PetscErrorCode VecGetArray(Vec v, PetscScalar **a) { *a = v->a; return 0; }
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a) { (void)v; *a = NULL; return 0; }
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a) { *a = v->a; return 0; }
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar **a) { (void)v; *a = NULL; return 0; }
PetscErrorCode PetscOptionsGetBool(void *o, const char p[], const char n[], PetscBool *v, PetscBool *s) { (void)o; (void)p; (void)n; (void)v; if (s) *s = PETSC_FALSE; return 0; }
PetscErrorCode PetscOptionsGetInt(void *o, const char p[], const char n[], PetscInt *v, PetscBool *s) { (void)o; (void)p; (void)n; (void)v; if (s) *s = PETSC_FALSE; return 0; }
PetscErrorCode PetscOptionsGetReal(void *o, const char p[], const char n[], PetscReal *v, PetscBool *s) { (void)o; (void)p; (void)n; (void)v; if (s) *s = PETSC_FALSE; return 0; }
PetscErrorCode DMDAGetInfo(DM dm, PetscInt *dim, PetscInt *M, PetscInt *N, PetscInt *P, PetscInt *m, PetscInt *n,
                           PetscInt *p, PetscInt *dof, PetscInt *sw, DMBoundaryType *bx, DMBoundaryType *by,
                           DMBoundaryType *bz, DMDAStencilType *st)
{
  (void)bx; (void)by; (void)bz; (void)st;
  if (dim) *dim = 3;
  if (M) *M = dm->M;
  if (N) *N = dm->N;
  if (P) *P = dm->P;
  if (m) *m = 1;
  if (n) *n = 1;
  if (p) *p = 1;
  if (dof) *dof = dm->dof;
  if (sw) *sw = dm->sw;
  return 0;
}
PetscErrorCode DMDAGetGhostCorners(DM dm, PetscInt *x, PetscInt *y, PetscInt *z, PetscInt *m, PetscInt *n, PetscInt *p)
{
  if (x) *x = 0;
  if (y) *y = 0;
  if (z) *z = 0;
  if (m) *m = dm->M;
  if (n) *n = dm->N;
  if (p) *p = dm->P;
  return 0;
}
PetscErrorCode DMDAGetCorners(DM dm, PetscInt *x, PetscInt *y, PetscInt *z, PetscInt *m, PetscInt *n, PetscInt *p)
{
  return DMDAGetGhostCorners(dm, x, y, z, m, n, p);
}
/* first owned element's first node and the owned element counts (one process) */
PetscErrorCode DMDAGetCornersElementQ2(DM dm, PetscInt *sei, PetscInt *sej, PetscInt *sek, PetscInt *mx, PetscInt *my,
                                       PetscInt *mz)
{
  if (sei) *sei = 0;
  if (sej) *sej = 0;
  if (sek) *sek = 0;
  if (mx) *mx = (dm->M - 1) / 2;
  if (my) *my = (dm->N - 1) / 2;
  if (mz) *mz = (dm->P - 1) / 2;
  return 0;
}

PetscErrorCode DMDAGetElements_pTatinQ2P1(DM dm, PetscInt *nel, PetscInt *npe, const PetscInt **e)
{
  if (nel) *nel = dm->nel;
  if (npe) *npe = dm->npe;
  if (e) *e = dm->e;
  return 0;
}

PetscErrorCode VolumeQuadratureGetAllCellData_Stokes(Quadrature Q, QPntVolCoefStokes *coeffs[])
{
  *coeffs = (QPntVolCoefStokes *)Q->shim_cells;
  return 0;
}
PetscErrorCode VolumeQuadratureGetCellData_Stokes(Quadrature Q, QPntVolCoefStokes coeffs[], PetscInt cidx, QPntVolCoefStokes *cell[])
{
  *cell = &coeffs[cidx * Q->npoints];
  return 0;
}

/* local dof indices of an element: 3 interleaved components per node */
PetscErrorCode StokesVelocity_GetElementLocalIndices(PetscInt idx[], PetscInt elnid[])
{
  for (int n = 0; n < 27; n++)
    for (int d = 0; d < 3; d++) idx[3 * n + d] = 3 * elnid[n] + d;
  return 0;
}
PetscErrorCode StokesPressure_GetElementLocalIndices(PetscInt idx[], PetscInt elnid[])
{
  for (int n = 0; n < 4; n++) idx[n] = elnid[n];
  return 0;
}
PetscErrorCode DMDASetValuesLocalStencil_AddValues_Stokes_Velocity(PetscScalar *F, PetscInt eqn[], PetscScalar Fe[])
{
  for (int k = 0; k < 81; k++) F[eqn[k]] += Fe[k];
  return 0;
}
PetscErrorCode DMDASetValuesLocalStencil_AddValues_Stokes_Pressure(PetscScalar *F, PetscInt eqn[], PetscScalar Fe[])
{
  for (int k = 0; k < 4; k++) F[eqn[k]] += Fe[k];
  return 0;
}
PetscErrorCode DMDAGetElementCoordinatesQ2_3D(PetscScalar elcoords[], PetscInt elnid[], PetscScalar LA_gcoords[])
{
  for (int n = 0; n < 27; n++)
    for (int d = 0; d < 3; d++) elcoords[3 * n + d] = LA_gcoords[3 * elnid[n] + d];
  return 0;
}
PetscErrorCode DMDAGetVectorElementFieldQ2_3D(PetscScalar elfield[], PetscInt elnid[], PetscScalar LA_gfield[])
{
  return DMDAGetElementCoordinatesQ2_3D(elfield, elnid, LA_gfield);
}
PetscErrorCode DMDAGetScalarElementField(PetscScalar elfield[], PetscInt npe, PetscInt elnid[], PetscScalar LA_gfield[])
{
  for (int n = 0; n < npe; n++) elfield[n] = LA_gfield[elnid[n]];
  return 0;
}

/* DM / Vec calls of the material-point projections, for one process owning
 * the whole lattice (local vectors = global vectors, no ghosts) */
PetscErrorCode DMDADuplicateLayout(DM da1, PetscInt dof2, PetscInt sw2, DMDAStencilType st2, DM *da2)
{
  (void)st2;
  DM d = (DM)malloc(sizeof(*d));
  if (!d) return PETSC_ERR_MEM;
  *d = *da1;
  d->dof = dof2;
  d->sw = sw2;
  d->clone = 1;
  *da2 = d;
  return 0;
}
PetscErrorCode DMDestroy(DM *dm)
{
  if (dm && *dm && (*dm)->clone) free(*dm);
  if (dm) *dm = NULL;
  return 0;
}
PetscErrorCode DMDASetElementType_Q2(DM dm) { (void)dm; return 0; }
PetscErrorCode DMDAGetRefinementFactor(DM dm, PetscInt *rx, PetscInt *ry, PetscInt *rz)
{
  (void)dm;
  if (rx) *rx = 2;
  if (ry) *ry = 2;
  if (rz) *rz = 2;
  return 0;
}
PetscErrorCode DMDAGetLocalSizeElementQ2(DM dm, PetscInt *mx, PetscInt *my, PetscInt *mz)
{
  if (mx) *mx = (dm->M - 1) / 2;
  if (my) *my = (dm->N - 1) / 2;
  if (mz) *mz = (dm->P - 1) / 2;
  return 0;
}
static PetscErrorCode shim_vec_new(DM dm, Vec *v)
{
  Vec x = (Vec)malloc(sizeof(*x));
  if (!x) return PETSC_ERR_MEM;
  x->n = (long)dm->dof * dm->M * dm->N * dm->P;
  x->a = (PetscScalar *)calloc((size_t)x->n, sizeof(PetscScalar));
  *v = x;
  return x->a ? 0 : PETSC_ERR_MEM;
}
static PetscErrorCode shim_vec_free(Vec *v)
{
  if (v && *v) {
    free((*v)->a);
    free(*v);
    *v = NULL;
  }
  return 0;
}
PetscErrorCode DMGetGlobalVector(DM dm, Vec *v) { return shim_vec_new(dm, v); }
PetscErrorCode DMGetLocalVector(DM dm, Vec *v) { return shim_vec_new(dm, v); }
PetscErrorCode DMRestoreGlobalVector(DM dm, Vec *v) { (void)dm; return shim_vec_free(v); }
PetscErrorCode DMRestoreLocalVector(DM dm, Vec *v) { (void)dm; return shim_vec_free(v); }
PetscErrorCode PetscObjectSetName(PetscObject o, const char name[]) { (void)o; (void)name; return 0; }
PetscErrorCode VecZeroEntries(Vec v)
{
  memset(v->a, 0, sizeof(PetscScalar) * (size_t)v->n);
  return 0;
}
PetscErrorCode DMLocalToGlobalBegin(DM dm, Vec l, InsertMode mode, Vec g)
{
  (void)dm;
  for (long i = 0; i < g->n; i++) g->a[i] = (mode == ADD_VALUES) ? g->a[i] + l->a[i] : l->a[i];
  return 0;
}
PetscErrorCode DMLocalToGlobalEnd(DM dm, Vec l, InsertMode mode, Vec g) { (void)dm; (void)l; (void)mode; (void)g; return 0; }
PetscErrorCode DMGlobalToLocalBegin(DM dm, Vec g, InsertMode mode, Vec l)
{
  (void)dm; (void)mode;
  memcpy(l->a, g->a, sizeof(PetscScalar) * (size_t)l->n);
  return 0;
}
PetscErrorCode DMGlobalToLocalEnd(DM dm, Vec g, InsertMode mode, Vec l) { (void)dm; (void)g; (void)mode; (void)l; return 0; }
/* PETSc's VecPointwiseDivide sets w_i = 0 where y_i = 0 */
PetscErrorCode VecPointwiseDivide(Vec w, Vec x, Vec y)
{
  for (long i = 0; i < w->n; i++) w->a[i] = (y->a[i] != 0.0) ? x->a[i] / y->a[i] : 0.0;
  return 0;
}
PetscErrorCode Q2GetElementLocalIndicesDOF(PetscInt idx[], PetscInt ndof, PetscInt elnid[])
{
  for (int d = 0; d < ndof; d++)
    for (int n = 0; n < 27; n++) idx[ndof * n + d] = ndof * elnid[n] + d;
  return 0;
}
PetscErrorCode DMDASetValuesLocalStencil_AddValues_DOF(PetscScalar *F, PetscInt ndof, PetscInt eqn[], PetscScalar Fe[])
{
  for (int k = 0; k < 27 * ndof; k++) F[eqn[k]] += Fe[k];
  return 0;
}

/* ------------------------------------------------------------- entry --- */
void ref_teardown(void)
{
  free(g_dau.e); g_dau.e = NULL;
  free(g_dap.e); g_dap.e = NULL;
  free(g_dau.coords.a); g_dau.coords.a = NULL;
  free(g_cells); g_cells = NULL;
  free(g_qxi); g_qxi = NULL;
  free(g_qw); g_qw = NULL;
}

/* Build the one-process mesh: node lattice (2mx+1)x(2my+1)x(2mz+1), the
 * lexicographic Q2 connectivity, the P1disc element-major pressure layout
 * and the quadrature-point records (eta per QP; other fields zero). */
int ref_setup(int mx, int my, int mz, const double *coords, const double *eta)
{
  ref_teardown();
  int X = 2 * mx + 1, Y = 2 * my + 1, Z = 2 * mz + 1;
  long nn = (long)X * Y * Z, nel = (long)mx * my * mz;
  g_dau.kind = 0; g_dau.M = X; g_dau.N = Y; g_dau.P = Z; g_dau.dof = 3; g_dau.sw = 2;
  g_dau.nel = (PetscInt)nel; g_dau.npe = 27;
  g_dau.e = (PetscInt *)malloc(sizeof(PetscInt) * 27 * (nel + 1));
  long cnt = 0;
  for (int ek = 0; ek < mz; ek++)
    for (int ej = 0; ej < my; ej++)
      for (int ei = 0; ei < mx; ei++, cnt++)
        for (int c = 0; c < 3; c++)
          for (int b = 0; b < 3; b++)
            for (int a = 0; a < 3; a++)
              g_dau.e[27 * cnt + a + 3 * b + 9 * c] = (2 * ei + a) + X * ((2 * ej + b) + Y * (2 * ek + c));
  g_dau.coords.n = 3 * nn;
  g_dau.coords.a = (double *)malloc(sizeof(double) * 3 * nn);
  memcpy(g_dau.coords.a, coords, sizeof(double) * 3 * nn);

  g_dap.kind = 1; g_dap.M = mx; g_dap.N = my; g_dap.P = mz; g_dap.dof = 4; g_dap.sw = 0;
  g_dap.nel = (PetscInt)nel; g_dap.npe = 4;
  g_dap.e = (PetscInt *)malloc(sizeof(PetscInt) * 4 * (nel + 1));
  for (long e = 0; e < nel; e++)
    for (int d = 0; d < 4; d++) g_dap.e[4 * e + d] = (PetscInt)(4 * e + d);
  g_dap.coords = g_dau.coords;

  g_cells = (QPntVolCoefStokes *)calloc((size_t)nel * 27, sizeof(QPntVolCoefStokes));
  for (long k = 0; k < nel * 27; k++) g_cells[k].eta = eta[k];
  memset(&g_Q, 0, sizeof g_Q);
  g_Q.dim = 3; g_Q.type = VOLUME_QUAD; g_Q.npoints = 27; g_Q.n_elements = (PetscInt)nel;
  g_Q.shim_cells = g_cells;
  PetscInt ngp = 0;
  QuadratureCreateGauss_3pnt_3D(&ngp, &g_qxi, &g_qw); /* the Gauss rule of the volume quadrature */
  g_Q.q_xi_coor = g_qxi;
  g_Q.q_weight = g_qw;
  return 0;
}

int ref_a11(int variant, double *x, double *y)
{
  switch (variant) {
  case 0: return MFStokesWrapper_A11_Tensor(NULL, &g_Q, &g_dau, x, y);
  case 1: return MFStokesWrapper_A11_AVX(NULL, &g_Q, &g_dau, x, y);
  case 2: return MFStokesWrapper_A11(NULL, &g_Q, &g_dau, x, y);
  case 3: return MFStokesWrapper_A11PC(&g_Q, &g_dau, x, y);
  default: return PETSC_ERR_SUP;
  }
}
int ref_diag(double *y) { return MFStokesWrapper_diagA11(&g_Q, &g_dau, y); }
int ref_a12(double *p, double *yu) { return MFStokesWrapper_A12(&g_Q, &g_dau, &g_dap, p, yu); }
int ref_a21(double *u, double *yp) { return MFStokesWrapper_A21(&g_Q, &g_dau, &g_dap, u, yp); }
/* the AVX back end's A12 and fused [A11 A12; A21 0] (what MatMult_MFStokes_A12 and
 * MatMult_MFStokes_A call when __AVX__ is defined, src/stokes_operators.c:927,1323) */
int ref_a12_avx(double *p, double *yu) { return MFStokesWrapper_A12_AVX(&g_Q, &g_dau, &g_dap, p, yu); }
int ref_a_avx(double *u, double *p, double *yu, double *yp) { return MFStokesWrapper_A_AVX(&g_Q, &g_dau, u, &g_dap, p, yu, yp); }
/* Gauss-point eta / rho [27*nel] from n markers by the reference's projection
 * `type` (-1 none, 0/10/20 P0 arithmetic/harmonic/geometric, 1 Q1, 4 one-to-one;
 * src/rheology.c:150-185).  eta_q / rho_q hold the current values on entry. */
int ref_marker_project(int type, int n, const int *wil, const double *xi, const double *eta_p, const double *rho_p,
                       double *eta_q, double *rho_q)
{
  const long nq = (long)g_Q.n_elements * 27;
  for (long k = 0; k < nq; k++) {
    g_cells[k].eta = eta_q[k];
    g_cells[k].rho = rho_q[k];
  }
  MPntStd *std = (MPntStd *)calloc((size_t)(n > 0 ? n : 1), sizeof(MPntStd));
  MPntPStokes *stk = (MPntPStokes *)calloc((size_t)(n > 0 ? n : 1), sizeof(MPntPStokes));
  if (!std || !stk) { free(std); free(stk); return PETSC_ERR_MEM; }
  for (int p = 0; p < n; p++) {
    std[p].wil = wil[p];
    if (xi) for (int d = 0; d < 3; d++) std[p].xi[d] = xi[3 * p + d];
    stk[p].eta = eta_p[p];
    stk[p].rho = rho_p[p];
  }
  int rc;
  switch (type) {
  case -1: rc = 0; break;
  case 0: rc = MPntPStokesProj_P0(CoefAvgARITHMETIC, n, std, stk, &g_dau, &g_Q); break;
  case 10: rc = MPntPStokesProj_P0(CoefAvgHARMONIC, n, std, stk, &g_dau, &g_Q); break;
  case 20: rc = MPntPStokesProj_P0(CoefAvgGEOMETRIC, n, std, stk, &g_dau, &g_Q); break;
  case 1: rc = SwarmUpdateGaussPropertiesLocalL2Projection_Q1_MPntPStokes(n, std, stk, &g_dau, &g_Q); break;
  case 4: rc = SwarmUpdateGaussPropertiesOne2OneMap_MPntPStokes(n, std, stk, &g_Q); break;
  default: rc = PETSC_ERR_SUP;
  }
  for (long k = 0; k < nq; k++) {
    eta_q[k] = g_cells[k].eta;
    rho_q[k] = g_cells[k].rho;
  }
  free(std);
  free(stk);
  return rc;
}
/* [v_L2, symmetric-gradient H1 seminorm, H1, p_L2] errors of (u [3*nn], p [4*nel])
 * against SolCx(eta0, eta1, xc, n) on the mesh given to ref_setup */
int ref_solcx_norms(double eta0, double eta1, double xc, int n, double *u, double *p, double *norms)
{
  ParamsSolCx prm;
  int rc = SolCxParamsSetValues(&prm, eta0, eta1, xc, n);
  if (rc) return rc;
  struct _p_shim_Vec sv, sp;
  sv.a = u;
  sv.n = (long)g_dau.dof * g_dau.M * g_dau.N * g_dau.P;
  sp.a = p;
  sp.n = (long)g_dap.dof * g_dap.M * g_dap.N * g_dap.P;
  return Evaluate_uL2_symuH1_pL2(&g_dau, &g_dap, &sv, &sp, &g_Q, EvaluateV_SolCx, EvaluateE_SolCx, EvaluateP_SolCx,
                                 (void *)&prm, &norms[0], &norms[1], &norms[2], &norms[3]);
}
/* the analytic velocity [3] and pressure at a point */
int ref_solcx_exact(double eta0, double eta1, double xc, int n, double *pos, double *vel, double *pressure)
{
  ParamsSolCx prm;
  int rc = SolCxParamsSetValues(&prm, eta0, eta1, xc, n);
  if (rc) return rc;
  if ((rc = EvaluateV_SolCx(pos, vel, (void *)&prm))) return rc;
  return EvaluateP_SolCx(pos, pressure, (void *)&prm);
}
/* the velocity DM and the volume quadrature of the mesh given to ref_setup
 * (what pTatin3d hands an A11 back end through struct _p_MatA11MF) */
DM ref_velocity_dm(void) { return &g_dau; }
Quadrature ref_quadrature(void) { return &g_Q; }
int ref_set_threads(int n) { omp_set_num_threads(n); return 0; }
int ref_max_threads(void) { return omp_get_max_threads(); }
