/*
 * Stand-in for the reference's ptatin3d_stokes.h: declares only the
 * quadrature-point accessors and local-index helpers the element kernels
 * call.  The coefficient record itself comes from the reference header
 * QPntVolCoefStokes_def.h.  Test infrastructure only.
 */
#ifndef P3D_SHIM_PTATIN3D_STOKES_H
#define P3D_SHIM_PTATIN3D_STOKES_H
#include "ptatin3d.h"
#include "QPntVolCoefStokes_def.h"
#include "dmda_bcs.h"
PetscErrorCode StokesVelocity_GetElementLocalIndices(PetscInt el_localIndices[], PetscInt elnid[]);
PetscErrorCode StokesPressure_GetElementLocalIndices(PetscInt el_localIndices[], PetscInt elnid[]);
PetscErrorCode VolumeQuadratureGetAllCellData_Stokes(Quadrature Q, QPntVolCoefStokes *coeffs[]);
PetscErrorCode VolumeQuadratureGetCellData_Stokes(Quadrature Q, QPntVolCoefStokes coeffs[], PetscInt cidx, QPntVolCoefStokes *cell[]);
PetscErrorCode DMDASetValuesLocalStencil_AddValues_Stokes_Velocity(PetscScalar *fields_F, PetscInt u_eqn[], PetscScalar Fe_u[]);
PetscErrorCode DMDASetValuesLocalStencil_AddValues_Stokes_Pressure(PetscScalar *fields_F, PetscInt p_eqn[], PetscScalar Fe_p[]);
#endif
