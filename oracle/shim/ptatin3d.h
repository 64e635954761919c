/*
 * Stand-in for the reference's top-level ptatin3d.h when compiling only the
 * element kernels into the CPU oracle: it declares the handful of opaque
 * pTatin types those kernels mention and nothing else (no swarms, no MPI
 * data exchangers).  Test infrastructure only.
 */
#ifndef P3D_SHIM_PTATIN3D_H
#define P3D_SHIM_PTATIN3D_H
#include "petsc.h"
#include "ptatin3d_defs.h"
typedef struct _p_pTatinCtx *pTatinCtx;
typedef struct _p_pTatinModel *pTatinModel;
typedef struct _p_PhysCompStokes *PhysCompStokes;
typedef struct _p_PhysCompEnergy *PhysCompEnergy;
typedef struct _p_Quadrature *Quadrature;
typedef struct _p_SurfaceQuadrature *SurfaceQuadrature;
typedef enum { LINE_QUAD = 0, SURFACE_QUAD, VOLUME_QUAD } QuadratureType;
typedef struct _p_DataBucket *DataBucket;
typedef struct _p_DataEx *DataEx;
#endif
