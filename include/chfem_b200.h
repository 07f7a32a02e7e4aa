/*
 * chfem_b200.h -- C ABI of libchfem_b200.so, the host model layer of chfem_b200.
 *
 * Part 1 mirrors chfem's femhmg API (chfem/src/femhmg/femhmg.h:6-35): same names, argument
 * meaning and call order, so the reference's CLI driver (chfem/src/main.c) or its CPython
 * wrapper (chfem/src/chfem_wrapper.c) can run on this library.  3D analyses only (thermal,
 * elastic, Stokes permeability); 2D inputs and the scalar-density-field input are rejected
 * with an error message.
 *
 * Part 2 (chfemB200*) has no counterpart in the reference: precision and multi-RHS
 * switches, one-call runs for bindings, per-solve statistics, and map/RHS/tensor access for
 * parity tests.
 */
#ifndef CHFEM_B200_H
#define CHFEM_B200_H

#include <stdint.h>
#include "cudapcg_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef uint8_t logical;
typedef uint16_t hmgFlag_t;
typedef double var;
typedef uint8_t cudapcgFlag_b200;

/* ---------------- Part 1: femhmg API (femhmg.h:6-35) ----------------------------------- */
/* femhmg.c:135-394 */   logical hmgInit(char *data_filename, char *elem_filename, char *sdf_filename, uint8_t *data);
/* femhmg.c:396-450 */   logical hmgEnd(void);
/* femhmg.c:452-455 */   void hmgSetXReduceFlag(uint8_t flag);
/* femhmg.c:457-460 */   void hmgSetParallelStrategyFlag(uint8_t flag);
/* femhmg.c:462-465 */   void hmgSetSolverFlag(uint8_t flag);
/* femhmg.c:467-470 */   void hmgSetPreConditionerFlag(uint8_t flag);
/* femhmg.c:472-475 */   void hmgSetStoppingCriteria(uint8_t flag);
/* femhmg.c:477-515 */   logical hmgSetPoreMappingStrategy(uint8_t flag);
/* femhmg.c:561-846 */   void hmgFindInitialGuesses(unsigned int nlevels);
/* femhmg.c:548-552 */   void hmgExportX(logical flag);
/* femhmg.c:554-559 */   void hmgImportX(char *file);
/* femhmg.c:516-546 */   void hmgSetHomogenizationFlag(hmgFlag_t flag);
/* femhmg.c:848-1198 */  void hmgSolveHomogenization(void);
/* femhmg.c:1200-1321 */ void hmgPrintModelData(void);
/* femhmg.c:1347-1354 */ void hmgPrintConstitutiveMtx(void);
/* femhmg.c:1326-1329 */ var *hmgGetConstitutiveMtx(void);
/* femhmg.c:1331-1334 */ unsigned int hmgGetConstitutiveMtxDim(void);
/* femhmg.c:1336-1339 */ var *hmgGetThermalExpansion(void);
/* femhmg.c:1341-1344 */ unsigned int hmgGetThermalExpansionDim(void);
/* femhmg.c:1356-1367 */ logical hmgSaveConstitutiveMtx(const char *filename);
/* femhmg.c:1395-1400 */ void hmgSaveFields(logical mustExport_flag, logical byElems_flag);
/* femhmg.c:1369-1383 */ void hmgKeepTrackOfAnalysisReport(uint8_t flag);
/* femhmg.c:1385-1393 */ uint8_t hmgPrintReport(const char *filename);

/* ---------------- Part 2: extensions (no counterpart in the reference) ----------------- */
#define CHFEM_B200_PREC_FP64 0
#define CHFEM_B200_PREC_MIXED 1

/* Precision of the next solves: FP64 (default) or mixed (FP32 fields, FP64 reductions). */
void chfemB200SetPrecision(int mode);
/* Solve all load cases of an analysis in one block multi-RHS solve (1) or one by one (0). */
void chfemB200SetMultiRHS(int on);
/* Quiet mode: 1 suppresses the progress prints of the model layer. */
void chfemB200SetQuiet(int quiet);
/* Last error message ("" when none). */
const char *chfemB200LastError(void);

/* Per-load-case statistics of the last hmgSolveHomogenization. */
typedef struct {
  int n_cases;
  int direction[6];
  unsigned int iterations[6];
  double residual[6];
  double solve_seconds[6];   /* device time of each solve (CUDA events) */
  double rhs_seconds;        /* host wall time spent assembling right-hand sides */
  double update_seconds;     /* host wall time spent in effective-tensor updates */
  double total_seconds;      /* wall time of hmgSolveHomogenization */
  unsigned long long kernel_launches;
  unsigned int ndof;
  double setup_seconds;      /* host wall time of the solver set-up (context, uploads, allocations) */
  double solve_call_seconds; /* host wall time of the solve calls (work-vector allocation, device
                                solve, result readout) */
  double teardown_seconds;   /* host wall time of releasing the solver's device memory */
} chfemB200SolveStats;
int chfemB200GetSolveStats(chfemB200SolveStats *out);

/* One-call run for bindings (the reference's chfem.wrapper.run contract, chfem_wrapper.c:7-89):
   voxels: uint8 image in C order of a (z,y,x) array; nf: settings file; direction 0..6;
   solver 0..3; precondition 0/1; x0_file may be NULL.  Fills C (C_dim entries, row-major)
   and returns the tensor dimension (3 or 6), or 0 on error. */
int chfemB200Run(const uint8_t *voxels, const char *nf, int direction, int solver, int precondition,
                 int precision, int multirhs, double *C_out);

/* Batched thermal homogenization of many independent images (no counterpart in the reference,
   which homogenizes one image per run): sample s is an nx*ny*nz uint8 image in C order of a
   (z,y,x) array (the .raw layout), whose colours colors[0..nmat-1] have conductivities
   conductivity[0..nmat-1] (nmat <= 4; unit voxel, NBN, PCG with Jacobi, L2 stopping test).  All
   samples and their 3 load cases are solved together on the GPU (cudapcgB200SolveThermalBatch).
   Fills C_out[9s..9s+8] (row-major 3x3 tensor of sample s) and, when not NULL,
   iterations[3s + k].  precision: 0 FP64, 1 mixed.  Returns 1 when every load case converged,
   2 when some stopped at maxit, 0 on error (chfemB200LastError). */
typedef struct {
  unsigned int nx, ny, nz;
  const uint8_t *voxels;
  unsigned int nmat;
  uint8_t colors[4];
  double conductivity[4];
} chfemB200ThermalSample;
int chfemB200RunThermalBatch(unsigned int nsamples, const chfemB200ThermalSample *samples, double tol,
                             unsigned int maxit, int precision, double *C_out, unsigned int *iterations,
                             double *solve_seconds);
/* Statistics of the last chfemB200RunThermalBatch (the solver's cudapcgB200BatchStats). */
int chfemB200LastBatchStats(cudapcgB200BatchStats *out);

/* Parity access to the current model's maps and matrices (0 if unavailable).
   which: 0 node keys (uint16, N), 1 node->DOF map (uint32, N), 2 DOF->node map (uint32, nV+nB),
          3 interface fluid keys (uint8, nB), 4 local matrices (double), 5 last RHS (double, ndof),
          6 element material map (uint16, N), 7 CB matrices (double) */
unsigned long long chfemB200ModelArraySize(int which);
int chfemB200CopyModelArray(int which, void *dst, unsigned long long bytes);
/* Assemble the RHS of load case `direction` into dst (ndof doubles). */
int chfemB200AssembleRHS(int direction, double *dst);
/* Effective-tensor column of load case `direction` from a solution x (ndof doubles). */
int chfemB200UpdateC(int direction, const double *x, double *C_out);
/* Right-hand side of the thermal-expansion load (a unit temperature rise; elastic models with
   %thermal_expansion) into dst (ndof doubles): femhmg_elastic_3D.c:464-505,
   femhmg_elastic_2D.c:277-300. */
int chfemB200AssembleThermalExpansionRHS(double *dst);
/* The effective thermal expansion (6 values, 3 in 2D, into alpha_out) from that load's solution
   x (ndof doubles) and the effective tensor C (C_dim doubles), the stress sums taken on the host:
   femhmg_elastic_3D.c:863-1074, femhmg_elastic_2D.c:388-528. */
int chfemB200UpdateThermalExpansion(const double *x, const double *C, double *alpha_out);
/* Export the solution and its field for every load case of the next solve (as hmgSaveFields
   does; for the one-call chfemB200Run, which re-initializes the model). */
void chfemB200SetExportFields(int on);
/* Initial guesses for the next hmgSolveHomogenization / chfemB200Run (used once, then cleared):
   x0[k] for load case k (k < ncases; NULL entries start from zero), nvars doubles each, in host
   memory or (on_device) device memory that stays valid until the solve returns.  They take
   the place of the recursive coarse-grid guesses (-r); an -xi file still takes precedence. */
int chfemB200SetInitialGuesses(int ncases, const double *const *x0, int on_device);
/* Effective-tensor column of load case `direction` from its volume term (the moments of
   cudapcgB200SolveLoadCases) plus the host face term; copies the whole tensor to C_out. */
int chfemB200UpdateCFromVolume(int direction, const double *volume, double *C_out);
/* Model sizes: [nx, ny, nz, nelem, ndof, nV, nB, nmat, analysis] */
int chfemB200ModelInfo(unsigned int *info9);

#ifdef __cplusplus
}
#endif
#endif /* CHFEM_B200_H */
