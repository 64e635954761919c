/*
 * Minimal PETSc stand-in used ONLY to compile the reference's element-kernel
 * sources (stokes_operators_{tensor,avx,mf}.c, element_utils_q2.c) and its
 * material-point projections (material_point_utils.c, quadrature.c) into the
 * CPU oracle under oracle/_ref.  Nothing here is PETSc; it declares just the
 * types, macros and accessor functions those files name.  The accessors are
 * implemented by oracle/ref_driver.c over plain arrays.
 *
 * Test infrastructure only: nothing in the product links this.
 */
#ifndef P3D_SHIM_PETSC_H
#define P3D_SHIM_PETSC_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

typedef int PetscErrorCode;
typedef int PetscInt;
typedef int PetscMPIInt;
typedef double PetscReal;
typedef double PetscScalar;
typedef double PetscLogDouble;
typedef long long PetscObjectState;
typedef int PetscClassId;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_DOUBLE 1
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_INT 2
#define PETSC_COMM_WORLD 0
#define PETSC_COMM_SELF 0
#define MPIU_INT MPI_INT
#define MPIU_REAL MPI_DOUBLE
#define MPIU_SUM MPI_SUM
#define PetscObjectComm(o) 0

typedef struct _p_shim_DM  *DM;
typedef struct _p_shim_Vec *Vec;
typedef struct _p_shim_Mat *Mat;
typedef struct _p_shim_IS  *IS;
typedef struct _p_shim_KSP *KSP;
typedef struct _p_shim_SNES *SNES;
typedef struct _p_shim_PC  *PC;
typedef struct _p_shim_Obj *PetscObject;
typedef struct _p_shim_Viewer *PetscViewer;
typedef struct _p_shim_FList *PetscFunctionList;
typedef struct _p_shim_Random *PetscRandom;
typedef struct _p_shim_Section *PetscSection;
typedef struct _p_shim_LG *ISLocalToGlobalMapping;
typedef struct { PetscScalar x, y, z; } DMDACoor3d;
typedef struct { PetscScalar x, y; } DMDACoor2d;
typedef enum { DMDA_STENCIL_STAR, DMDA_STENCIL_BOX } DMDAStencilType;
typedef enum { DM_BOUNDARY_NONE } DMBoundaryType;
typedef enum { INSERT_VALUES, ADD_VALUES } InsertMode;
typedef enum { PETSC_ERR_SUP = 56, PETSC_ERR_ARG_SIZ = 60, PETSC_ERR_ARG_WRONG = 62,
               PETSC_ERR_ARG_CORRUPT = 64, PETSC_ERR_USER = 83, PETSC_ERR_ARG_NULL = 85,
               PETSC_ERR_MEM = 55, PETSC_ERR_ARG_OUTOFRANGE = 63, PETSC_ERR_LIB = 76 } PetscErrorCodeEnum;
typedef enum { PETSC_VIEWER_DEFAULT = 0, PETSC_VIEWER_ASCII_VTK } PetscViewerFormat;

#define PETSC_EXTERN extern
#define PETSC_STATIC_INLINE static inline
#define PETSC_DECIDE (-1)
#define PETSC_DEFAULT (-2)
#define PETSC_NULL NULL
#define PETSC_FUNCTION_NAME __func__
#define PetscFunctionBegin do {} while (0)
#define PetscFunctionReturn(x) return (x)
#define CHKERRQ(e) do { if (e) return (e); } while (0)
#define CHKERRABORT(c, e) do { if (e) abort(); } while (0)
#define CHKMEMQ
#define SETERRQ(c, n, s) return (n)
#define SETERRQ1(c, n, s, a) return (n)
#define SETERRQ2(c, n, s, a, b) return (n)
#define SETERRQ3(c, n, s, a, b, d) return (n)
#define SETERRQ4(c, n, s, a, b, d, e) return (n)
#define PetscMin(a, b) (((a) < (b)) ? (a) : (b))
#define PetscMax(a, b) (((a) > (b)) ? (a) : (b))
#define PetscAbsReal(a) fabs(a)
#define PetscAbsScalar(a) fabs(a)
#define PetscSqrtReal(a) sqrt(a)
#define PetscSqr(a) ((a) * (a))
#define PetscRealPart(a) (a)
#define PetscPowReal(a, b) pow(a, b)
#define PetscExpReal(a) exp(a)
#define PetscSinReal(a) sin(a)
#define PetscCosReal(a) cos(a)
#define PETSC_PI 3.14159265358979323846
#define PETSC_MAX_REAL 1.7976931348623157e+308
#define PETSC_MACHINE_EPSILON 2.2204460492503131e-16
#define PetscUnlikely(x) (x)
#define PetscLikely(x) (x)
#define PETSC_MAX_PATH_LEN 4096

/* memory */
#define PetscMalloc(n, p) ((*(void **)(p) = malloc((size_t)(n))) ? 0 : PETSC_ERR_MEM)
#define PetscMalloc1(n, p) PetscMalloc((size_t)(n) * sizeof(**(p)), (p))
#define PetscCalloc1(n, p) ((*(void **)(p) = calloc((size_t)(n), sizeof(**(p)))) ? 0 : PETSC_ERR_MEM)
#define PetscFree(p) (free(p), (p) = NULL, 0)
#define PetscMemzero(p, n) (memset((p), 0, (size_t)(n)), 0)
#define PetscMemcpy(d, s, n) (memcpy((d), (s), (size_t)(n)), 0)

/* logging and printing: no-ops */
#define PetscLogFlops(n) 0
#define PetscLogEventBegin(e, a, b, c, d) 0
#define PetscLogEventEnd(e, a, b, c, d) 0
#define PetscInfo(o, s) 0
#define PetscInfo1(o, s, a) 0
PetscErrorCode PetscPrintf(MPI_Comm c, const char fmt[], ...);
PetscErrorCode PetscTime(PetscLogDouble *t);
PetscErrorCode MPI_Comm_rank(MPI_Comm c, PetscMPIInt *r);
PetscErrorCode MPI_Comm_size(MPI_Comm c, PetscMPIInt *r);
PetscErrorCode MPI_Allreduce(const void *a, void *b, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c);

/* the accessors the element kernels call; implemented in oracle/ref_driver.c */
PetscErrorCode PetscDTGaussQuadrature(PetscInt npoints, PetscReal a, PetscReal b, PetscReal *x, PetscReal *w);
PetscErrorCode DMGetCoordinateDM(DM dm, DM *cdm);
PetscErrorCode DMGetCoordinatesLocal(DM dm, Vec *c);
PetscErrorCode VecGetArray(Vec v, PetscScalar **a);
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a);
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a);
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar **a);
PetscErrorCode PetscOptionsGetBool(void *o, const char pre[], const char name[], PetscBool *v, PetscBool *set);
PetscErrorCode PetscOptionsGetInt(void *o, const char pre[], const char name[], PetscInt *v, PetscBool *set);
PetscErrorCode PetscOptionsGetReal(void *o, const char pre[], const char name[], PetscReal *v, PetscBool *set);
PetscErrorCode DMDAGetInfo(DM, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *,
                           PetscInt *, PetscInt *, PetscInt *, DMBoundaryType *, DMBoundaryType *,
                           DMBoundaryType *, DMDAStencilType *);
PetscErrorCode DMDAGetGhostCorners(DM, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *);
PetscErrorCode DMDAGetCorners(DM, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *);
#endif
