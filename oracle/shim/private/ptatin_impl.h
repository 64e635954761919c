/*
 * Stand-in for the reference's private/ptatin_impl.h: the element kernels
 * only read volQ->npoints, so the quadrature object here carries the fields
 * the oracle driver fills in.  Test infrastructure only.
 */
#ifndef P3D_SHIM_PTATIN_IMPL_H
#define P3D_SHIM_PTATIN_IMPL_H
#include "ptatin3d.h"
#include "ptatin3d_stokes.h"
struct _p_Quadrature {
  PetscInt dim;
  QuadratureType type;
  PetscInt npoints;
  PetscReal *q_xi_coor;
  PetscReal *q_weight;
  PetscInt n_elements;
  DataBucket properties_db;
  void *shim_cells; /* QPntVolCoefStokes array [n_elements * npoints] */
};
#endif
