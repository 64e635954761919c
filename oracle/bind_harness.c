/*
 * Test harness of the reference-side binding ptatin3d_b200/binding/
 * stokes_operators_b200.c: it fills a struct _p_MatA11MF (the reference's
 * include/stokes_operators.h:47-62) with the binding's SpMVOp triple, as
 * MatA11MFCreate/MatA11MFSetup do for a registered back end
 * (src/stokes_operators.c:101-157, 226-273), over the one-process DM and
 * quadrature of oracle/ref_driver.c, and calls it through those function
 * pointers the way MatMult_MFStokes_A11 does (src/stokes_operators.c:1185).
 *
 * TEST INFRASTRUCTURE ONLY: built into oracle/_ref/libp3dbind.so (oracle/Makefile,
 * target `bind`) and used by tests/.
 */
#include "petsc.h"
#include "ptatin3d.h"
#include "private/ptatin_impl.h"
#include "ptatin3d_stokes.h"
#include "stokes_operators.h"

PetscErrorCode MFA11SetUp_B200(MatA11MF);
PetscErrorCode MFStokesWrapper_A11_B200(MatA11MF, Quadrature, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFA11Destroy_B200(MatA11MF);
DM ref_velocity_dm(void);
Quadrature ref_quadrature(void);

static struct _p_MatA11MF g_mf;

/* SetUp of the back end on the mesh of the last ref_setup */
int bind_setup(void)
{
  memset(&g_mf, 0, sizeof g_mf);
  g_mf.daUVW = ref_velocity_dm();
  g_mf.volQ = ref_quadrature();
  g_mf.state = 0;
  g_mf.SpMVOp_MatMult = MFStokesWrapper_A11_B200;
  g_mf.SpMVOp_SetUp = MFA11SetUp_B200;
  g_mf.SpMVOp_Destroy = MFA11Destroy_B200;
  int rc = g_mf.SpMVOp_SetUp(&g_mf);
  if (!rc) g_mf.is_setup = PETSC_TRUE;
  return rc;
}
/* the Mat's state advances (PetscObjectStateIncrease after new coefficients) */
int bind_touch(void)
{
  g_mf.state++;
  return 0;
}
/* Yu += A11 ufield on the local arrays, through the SpMVOp pointer */
int bind_matmult(double *ufield, double *Yu)
{
  return g_mf.SpMVOp_MatMult(&g_mf, g_mf.volQ, g_mf.daUVW, ufield, Yu);
}
int bind_destroy(void)
{
  int rc = g_mf.SpMVOp_Destroy(&g_mf);
  g_mf.is_setup = PETSC_FALSE;
  return rc;
}
