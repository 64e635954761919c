/*
 * Link-time stand-ins for the symbols that the reference's
 * material_point_utils.c and quadrature.c name in code the oracle never runs
 * (marker I/O and VTK output, data-bucket access, the multi-level Q1
 * hierarchy's PETSc Mat calls, element-type objects).  They exist so that
 * oracle/_ref/libp3dref.so links with every symbol defined; each function
 * returns a nonzero error code (PETSC_ERR_SUP) if it is ever reached.
 *
 * TEST INFRASTRUCTURE ONLY.
 */
#define P3D_STUB_UNSUPPORTED 56

int DMCreateInjection(void) { return P3D_STUB_UNSUPPORTED; }
int DMCreateInterpolationScale(void) { return P3D_STUB_UNSUPPORTED; }
int DMDAEQ1_GetElementLocalIndicesDOF(void) { return P3D_STUB_UNSUPPORTED; }
int DMDAEQ1_GetScalarElementField_3D(void) { return P3D_STUB_UNSUPPORTED; }
int DMDAEQ1_SetValuesLocalStencil_AddValues_DOF(void) { return P3D_STUB_UNSUPPORTED; }
int DMDAGetElementsQ1(void) { return P3D_STUB_UNSUPPORTED; }
int DMView(void) { return P3D_STUB_UNSUPPORTED; }
int ElementTypeCreate_Q2(void) { return P3D_STUB_UNSUPPORTED; }
int ElementTypeDestroy_Q2(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPEnergyGetField_diffusivity(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPEnergyGetField_heat_source(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPEnergyPVTUWriteAllPPointDataFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPEnergySetField_diffusivity(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPEnergySetField_heat_source(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPEnergyVTKWriteBinaryAppendedDataAllFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPEnergyVTKWriteBinaryAppendedHeaderAllFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesGetField_density(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesGetField_eta_effective(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesPVTUWriteAllPPointDataFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesPlGetField_plastic_strain(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesPlGetField_yield_indicator(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesPlPVTUWriteAllPPointDataFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesPlSetField_plastic_strain(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesPlSetField_yield_indicator(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesPlVTKWriteBinaryAppendedDataAllFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesPlVTKWriteBinaryAppendedHeaderAllFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesSetField_density(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesSetField_eta_effective(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesVTKWriteBinaryAppendedDataAllFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntPStokesVTKWriteBinaryAppendedHeaderAllFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdGetField_global_coord(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdGetField_local_coord(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdGetField_local_element_index(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdGetField_phase_index(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdGetField_point_index(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdPVTUWriteAllPPointDataFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdSetField_global_coord(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdSetField_local_coord(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdSetField_local_element_index(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdSetField_phase_index(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdSetField_point_index(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdVTKWriteBinaryAppendedDataAllFields(void) { return P3D_STUB_UNSUPPORTED; }
int MPntStdVTKWriteBinaryAppendedHeaderAllFields(void) { return P3D_STUB_UNSUPPORTED; }
int MatDestroy(void) { return P3D_STUB_UNSUPPORTED; }
int MatMult(void) { return P3D_STUB_UNSUPPORTED; }
int MatRestrict(void) { return P3D_STUB_UNSUPPORTED; }
int PetscMPIIntCast(void) { return P3D_STUB_UNSUPPORTED; }
int PetscSNPrintf(void) { return P3D_STUB_UNSUPPORTED; }
int PetscViewerASCIIOpen(void) { return P3D_STUB_UNSUPPORTED; }
int PetscViewerDestroy(void) { return P3D_STUB_UNSUPPORTED; }
int PetscViewerPopFormat(void) { return P3D_STUB_UNSUPPORTED; }
int PetscViewerPushFormat(void) { return P3D_STUB_UNSUPPORTED; }
int VecDestroy(void) { return P3D_STUB_UNSUPPORTED; }
int VecPointwiseMult(void) { return P3D_STUB_UNSUPPORTED; }
int VecReciprocal(void) { return P3D_STUB_UNSUPPORTED; }
int VecView(void) { return P3D_STUB_UNSUPPORTED; }
int pTatinGenerateParallelVTKName(void) { return P3D_STUB_UNSUPPORTED; }
int pTatinGenerateVTKName(void) { return P3D_STUB_UNSUPPORTED; }
int ptatinDataBucketDestroy(void) { return P3D_STUB_UNSUPPORTED; }
int ptatinDataBucketGetDataFieldByName(void) { return P3D_STUB_UNSUPPORTED; }
int ptatinDataBucketGetDataFields(void) { return P3D_STUB_UNSUPPORTED; }
int ptatinDataBucketGetSizes(void) { return P3D_STUB_UNSUPPORTED; }
int ptatinDataBucketQueryDataFieldByName(void) { return P3D_STUB_UNSUPPORTED; }
int ptatinDataBucketView(void) { return P3D_STUB_UNSUPPORTED; }
int ptatinDataFieldAccessPoint(void) { return P3D_STUB_UNSUPPORTED; }
int ptatinDataFieldGetAccess(void) { return P3D_STUB_UNSUPPORTED; }
int ptatinDataFieldRestoreAccess(void) { return P3D_STUB_UNSUPPORTED; }
int ptatinDataFieldVerifyAccess(void) { return P3D_STUB_UNSUPPORTED; }

const char MPntPEnergy_classname[] = "MPntPEnergy";
const char MPntPStokesPl_classname[] = "MPntPStokesPl";
const char MPntPStokes_classname[] = "MPntPStokes";
const char MPntStd_classname[] = "MPntStd";
const int MPntPEnergy_nmembers = 0;
const int MPntPStokesPl_nmembers = 0;
const int MPntPStokes_nmembers = 0;
const int QPntVolCoefEnergy_nmembers = 0;
const int QPntVolCoefStokes_nmembers = 0;
