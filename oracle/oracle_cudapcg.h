/*
 * oracle_cudapcg.h -- TEST INFRASTRUCTURE ONLY (the parity checker, never the product).
 *
 * Types and constants of chfem's cudapcg C ABI, restated so that the CPU oracle
 * (oracle_cudapcg.c) can be built without the reference tree.  The struct layout and
 * the flag values must equal the reference's, because the reference's own host code
 * (femhmg.c) fills cudapcgModel_t through the constructor callback it registers:
 *   - flag values ............ chfem/src/femhmg/cudapcg/includes.h:9-44
 *   - default precision/keys . chfem/src/femhmg/cudapcg/includes.h:46-80 (FP64, 16-bit keys)
 *   - cudapcgModel_t ......... chfem/src/femhmg/cudapcg/includes.h:93-129
 * When the oracle is linked with the reference host code (oracle/Makefile, target `ref`)
 * it is compiled with -DORACLE_USE_REF_HEADERS and takes these types from the
 * reference header itself, so both sides see one definition.
 */
#ifndef ORACLE_CUDAPCG_H
#define ORACLE_CUDAPCG_H

#ifdef ORACLE_USE_REF_HEADERS
#include "cudapcg.h"
#else
#include <stdint.h>

#define CUDAPCG_TRUE 1
#define CUDAPCG_FALSE 0
#define CUDAPCG_NBN 0
#define CUDAPCG_EBE 1
#define CUDAPCG_POREMAP_IMG 0
#define CUDAPCG_POREMAP_NUM 1
#define CUDAPCG_TOLERANCE 0.00001
#define CUDAPCG_MAX_ITERATIONS 100000
#define CUDAPCG_L2_NORM 0
#define CUDAPCG_INF_NORM 1
#define CUDAPCG_ERROR_NORM 2
#define CUDAPCG_THERMAL_2D 0
#define CUDAPCG_THERMAL_3D 1
#define CUDAPCG_ELASTIC_2D 2
#define CUDAPCG_ELASTIC_3D 3
#define CUDAPCG_FLUID_2D 4
#define CUDAPCG_FLUID_3D 5
#define CUDAPCG_CG_SOLVER 0
#define CUDAPCG_MINRES_SOLVER 1
#define CUDAPCG_CG3_SOLVER 2
#define CUDAPCG_MINRES3_SOLVER 3
#define CUDAPCG_CG2_SOLVER 4
#define CUDAPCG_MINRES2_SOLVER 5
#define CUDAPCG_XREDUCE_NONE 0
#define CUDAPCG_XREDUCE_ONLYDIR 1
#define CUDAPCG_XREDUCE_FULL 2

typedef double cudapcgVar_t;
typedef double cudapcgTol_t;
typedef unsigned short int cudapcgMap_t;
typedef uint8_t cudapcgFlag_t;
typedef unsigned int cudapcgIdMap_t;
typedef uint16_t parametricScalarField_t;

typedef struct _pcgmodel {
  char *name;
  cudapcgFlag_t freeAllowed_flag;
  cudapcgFlag_t parStrategy_flag;
  cudapcgFlag_t poremap_flag;
  cudapcgFlag_t parametric_density_field_flag;
  cudapcgFlag_t SBS_flag;
  unsigned int nrows;
  unsigned int ncols;
  unsigned int nlayers;
  unsigned int nelem;
  unsigned int nvars;
  unsigned int nvarspernode;
  unsigned int nkeys;
  unsigned int localmtxdim;
  unsigned int nporenodes;
  unsigned int nbordernodes;
  unsigned int nhmgvars;
  double limits_density_field[2];
  cudapcgMap_t *image;
  parametricScalarField_t *parametric_density_field;
  cudapcgFlag_t *pore_map;
  cudapcgFlag_t *border_pore_map;
  cudapcgIdMap_t *periodic2DOF_map;
  cudapcgIdMap_t *DOF2periodic_map;
} cudapcgModel_t;
#endif /* ORACLE_USE_REF_HEADERS */

#ifdef __cplusplus
extern "C" {
#endif

/* cudapcg C ABI (chfem/src/femhmg/cudapcg/cudapcg.h:19-62), CPU FP64 implementation. */
cudapcgFlag_t cudapcgInit(cudapcgFlag_t analysis_flag, cudapcgFlag_t parStrategy_flag);
cudapcgFlag_t cudapcgEnd(void);
cudapcgFlag_t cudapcgSetModelConstructorFcn(cudapcgFlag_t (*fcn)(cudapcgModel_t **, const void *));
cudapcgFlag_t cudapcgBuildModel(const void *data);
cudapcgModel_t *cudapcgNewModel(void);
cudapcgFlag_t cudapcgSetModel(cudapcgModel_t *model);
cudapcgFlag_t cudapcgSetNumTol(cudapcgTol_t t);
cudapcgFlag_t cudapcgSetMaxIterations(unsigned int n);
cudapcgFlag_t cudapcgSetXReduceMode(cudapcgFlag_t flag);
cudapcgFlag_t cudapcgSetXReduceShift(unsigned int shift);
cudapcgFlag_t cudapcgSetXReduceScale(double scl);
cudapcgFlag_t cudapcgSetReduceStabFactor(double scl);
cudapcgFlag_t cudapcgSetSolver(cudapcgFlag_t flag);
cudapcgFlag_t cudapcgSetPreconditioner(cudapcgFlag_t flag);
cudapcgFlag_t cudapcgSetResNorm(cudapcgFlag_t flag);
cudapcgFlag_t cudapcgAllocateArrays(void);
cudapcgFlag_t cudapcgFreeArrays(void);
cudapcgFlag_t cudapcgSetRHS(cudapcgVar_t *RHS);
cudapcgFlag_t cudapcgSetX0(cudapcgVar_t *x0, cudapcgFlag_t mustInterpolate);
cudapcgFlag_t cudapcgSetImage(cudapcgMap_t *img);
cudapcgFlag_t cudapcgSetParametricDensityField(parametricScalarField_t *field, double fmin, double fmax);
cudapcgFlag_t cudapcgSetPoreMap(cudapcgFlag_t *pores);
cudapcgFlag_t cudapcgSetPeriodic2DOFMap(cudapcgIdMap_t *vars);
cudapcgFlag_t cudapcgSetDOF2PeriodicMap(cudapcgIdMap_t *nodes);
cudapcgFlag_t cudapcgSetLclMtxs(cudapcgVar_t *LclMtxs);
cudapcgFlag_t cudapcgSolve(cudapcgVar_t *x);
cudapcgFlag_t cudapcgSetHeaderString(char *header);
cudapcgFlag_t cudapcgPrintSolverReport(void);
cudapcgFlag_t cudapcgPrintSolverReport2(char *dest);
cudapcgFlag_t cudapcgPrintSolverMetrics(void);
cudapcgFlag_t cudapcgPrintSolverMetrics2(char *dest);
unsigned int cudapcgGetNumIterations(void);
unsigned int cudapcgGetMaxNumIterations(void);
cudapcgVar_t cudapcgGetResidual(void);

/* ---- oracle-only entry points (checker access for tests) ---------------------------- */

/* One operator apply y = A x on the current model (reference data formats). */
int oracle_apply(const double *x, double *y);
/* One Jacobi apply y = M^-1 x on the current model. */
int oracle_precond(const double *x, double *y);
/* Number of unknowns of the current model (0 if none). */
unsigned int oracle_nvars(void);
/* Copies of what the reference host code handed over the ABI, for map/RHS parity. */
unsigned int oracle_captured_count(int which);          /* 0 keys,1 p2dof,2 dof2p,3 porekeys,4 lclmtx,5 rhs,6 x */
int oracle_copy_captured(int which, void *dst, unsigned int bytes);
/* Residual history of the last solve: oracle_history(NULL,0) returns its length. */
unsigned int oracle_history(double *dst, unsigned int n);
/* Per-solve log: iterations and residual of every solve since the last reset. */
unsigned int oracle_solve_log(unsigned int *iters, double *residuals, unsigned int n);
void oracle_reset_log(void);
/* Quiet mode: suppress per-solve prints. */
void oracle_set_quiet(int quiet);

#ifdef __cplusplus
}
#endif
#endif /* ORACLE_CUDAPCG_H */
