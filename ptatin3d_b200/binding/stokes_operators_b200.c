/*
 * The "b200" back end of pTatin3d's matrix-free A11 operator: the SpMVOp
 * triple {SpMVOp_MatMult, SpMVOp_SetUp, SpMVOp_Destroy} of struct _p_MatA11MF
 * (include/stokes_operators.h:47-62) over libp3d_b200.  A pTatin3d
 * maintainer drops this file into src/ and registers the three functions
 * under "b200" in MatA11MFCreate (src/stokes_operators.c:120-139):
 *
 *   ierr = PetscFunctionListAdd(&MatMult_flist,"b200",MFStokesWrapper_A11_B200);CHKERRQ(ierr);
 *   ierr = PetscFunctionListAdd(&SetUp_flist,"b200",MFA11SetUp_B200);CHKERRQ(ierr);
 *   ierr = PetscFunctionListAdd(&Destroy_flist,"b200",MFA11Destroy_B200);CHKERRQ(ierr);
 *
 * It replaces the "cuda" back end (src/stokes_operators_cuda.cu:240-532):
 * the same SpMVOp contract (Yu += sum_e A_e ufield on the ghosted local arrays,
 * the caller zeroes Yu and handles the Dirichlet rows and columns,
 * src/stokes_operators.c:1171-1201), the same re-upload of coordinates and
 * viscosity when the Mat's state changes (:413-421 there), no exit() on
 * errors (CUDA failures come back as PETSc errors).  The local vectors PETSc
 * hands over are pageable; the operator page-locks them on first use so that
 * later MatMults copy at full PCIe speed (they stay registered until the
 * back end is destroyed).
 *
 * The repository compiles and tests this file against its PETSc stand-in
 * headers and the reference's own kernels (oracle/Makefile, target `bind`;
 * tests/test_gpu_binding.py).
 */
#include <petscdm.h>
#include <ptatin3d.h>
#include <ptatin3d_stokes.h>
#include <dmda_element_q2p1.h>
#include <stokes_operators.h>

#include "p3d_b200.h"

typedef struct {
  p3d_op *op;
  PetscObjectState state; /* Mat state the device coefficients belong to */
  double *eta;            /* viscosity extracted from the quadrature records, [27*nel] */
  PetscInt nel;
} B200Ctx;

static PetscErrorCode B200Check(int rc)
{
  if (rc) SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "p3d_b200: %s", p3d_last_error());
  return 0;
}

PetscErrorCode MFA11SetUp_B200(MatA11MF mf)
{
  PetscErrorCode ierr;
  B200Ctx *c;
  p3d_mesh_desc d;
  PetscInt esi, esj, esk, mx, my, mz, gsi, gsj, gsk, gx, gy, gz;

  PetscFunctionBegin;
  ierr = PetscMalloc1(1, &c); CHKERRQ(ierr);
  memset(c, 0, sizeof(*c));
  ierr = DMDAGetCornersElementQ2(mf->daUVW, &esi, &esj, &esk, &mx, &my, &mz); CHKERRQ(ierr);
  ierr = DMDAGetGhostCorners(mf->daUVW, &gsi, &gsj, &gsk, &gx, &gy, &gz); CHKERRQ(ierr);
  d.mx = mx; d.my = my; d.mz = mz;                /* owned elements */
  d.gx = gx; d.gy = gy; d.gz = gz;                /* ghosted local node lattice */
  d.ox = esi - gsi; d.oy = esj - gsj; d.oz = esk - gsk;
  d.dirichlet = 0; d.global_faces = 0;            /* boundary conditions stay with MatMult_MFStokes_A11 */
  ierr = B200Check(p3d_op_create(&d, P3D_PREC_F64, 0, &c->op)); CHKERRQ(ierr);
  ierr = B200Check(p3d_op_set_bc_mode(c->op, P3D_BC_NONE)); CHKERRQ(ierr);
  ierr = B200Check(p3d_op_set_host_register(c->op, 1)); CHKERRQ(ierr);
  c->state = -1;
  c->nel = mx * my * mz;
  mf->ctx = c;
  PetscFunctionReturn(0);
}

PetscErrorCode MFStokesWrapper_A11_B200(MatA11MF mf, Quadrature volQ, DM dau, PetscScalar ufield[], PetscScalar Yu[])
{
  PetscErrorCode ierr;
  B200Ctx *c = (B200Ctx *)mf->ctx;
  QPntVolCoefStokes *qp;
  Vec gcoords;
  const PetscScalar *LA_gcoords;
  const PetscInt *elnidx;
  PetscInt e, q, nel, nen;

  PetscFunctionBegin;
  if (!c) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_WRONG, "b200 back end used before its SetUp");
  if (c->state != mf->state) { /* coefficients changed since the last upload */
    ierr = DMDAGetElements_pTatinQ2P1(dau, &nel, &nen, &elnidx); CHKERRQ(ierr);
    if (nel != c->nel) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_SIZ, "the DM's elements differ from the back end's");
    ierr = VolumeQuadratureGetAllCellData_Stokes(volQ, &qp); CHKERRQ(ierr);
    if (!c->eta) { ierr = PetscMalloc1(27 * c->nel, &c->eta); CHKERRQ(ierr); }
    for (e = 0; e < c->nel; e++)
      for (q = 0; q < 27; q++) c->eta[27 * e + q] = qp[27 * e + q].eta;
    ierr = DMGetCoordinatesLocal(dau, &gcoords); CHKERRQ(ierr);
    ierr = VecGetArrayRead(gcoords, &LA_gcoords); CHKERRQ(ierr);
    ierr = B200Check(p3d_op_set_coefficients(c->op, LA_gcoords, c->eta, P3D_GEOM_AUTO)); CHKERRQ(ierr);
    ierr = VecRestoreArrayRead(gcoords, &LA_gcoords); CHKERRQ(ierr);
    c->state = mf->state;
  }
  /* Yu = A ufield; the caller zeroed Yu (src/stokes_operators.c:1181), so this is the += of the contract */
  ierr = B200Check(p3d_a11_apply_host(c->op, ufield, Yu)); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

PetscErrorCode MFA11Destroy_B200(MatA11MF mf)
{
  B200Ctx *c = (B200Ctx *)mf->ctx;
  PetscFunctionBegin;
  if (c) {
    p3d_op_destroy(c->op); /* also unregisters the page-locked local arrays */
    if (c->eta) PetscFree(c->eta);
    PetscFree(c);
    mf->ctx = NULL;
  }
  PetscFunctionReturn(0);
}
