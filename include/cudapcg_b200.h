/*
 * cudapcg_b200.h -- C ABI of libcudapcg_b200.so, the B200 (sm_100a) solver library of
 * chfem_b200.
 *
 * Part 1 is a drop-in for chfem's cudapcg library: same names, argument meaning, data
 * formats and 1/0 return convention as chfem/src/femhmg/cudapcg/cudapcg.h:19-62, with
 * cudapcgVar_t = double and 16-bit material keys (the reference defaults,
 * chfem/src/femhmg/cudapcg/includes.h:46-80).  A caller built against the reference header
 * links against this library unchanged.  Differences by design:
 *   - errors return 0 and leave a message for cudapcgB200LastError(); the library never
 *     calls exit() or cudaDeviceReset() (reference: error_handling.h:6-14, cudapcg.cu:201);
 *   - 2D analyses (CUDAPCG_THERMAL_2D, CUDAPCG_ELASTIC_2D, CUDAPCG_FLUID_2D) run with the
 *     reference's 2D formats (4-bit key fields, dense 4x4 / 8x8 / 12x12 element matrices, up
 *     to 16 materials); the scalar density field (cudapcgSetParametricDensityField)
 *     applies to thermal and elastic models, 3D and 2D;
 *   - the 2-vector solvers (CG2/MINRES2, solvers/cg2.cu, pcg2.cu, minres2.cu, pminres2.cu)
 *     run for Stokes, 3D and 2D: cudapcgSolve then writes the 3 (2D: 2) reduced velocity sums
 *     of the solution (x[0..2], scaled by cudapcgSetXReduceScale) and
 *     <model name>_xreduce_metrics_<n>.bin;
 *     for thermal / elastic models they return an error (the reference's host never runs them
 *     there, femhmg.c:852-856).
 *
 * Part 2 (cudapcgB200* / chfemB200*) has no counterpart in the reference: precision mode,
 * operator access for tests, solve statistics.
 */
#ifndef CUDAPCG_B200_H
#define CUDAPCG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef CUDAPCG_TRUE
#define CUDAPCG_TRUE 1
#define CUDAPCG_FALSE 0
#define CUDAPCG_NBN 0
#define CUDAPCG_EBE 1
#define CUDAPCG_POREMAP_IMG 0
#define CUDAPCG_POREMAP_NUM 1
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
/* includes.h:42-44: how the 2-vector solvers reduce the solution */
#define CUDAPCG_XREDUCE_NONE 0
#define CUDAPCG_XREDUCE_ONLYDIR 1
#define CUDAPCG_XREDUCE_FULL 2
typedef double cudapcgVar_t;
typedef double cudapcgTol_t;
typedef unsigned short int cudapcgMap_t;
typedef uint8_t cudapcgFlag_t;
typedef unsigned int cudapcgIdMap_t;
typedef uint16_t parametricScalarField_t;

/* Same field order as chfem/src/femhmg/cudapcg/includes.h:93-129. */
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
#endif

/* ---------------- Part 1: drop-in cudapcg ABI (cudapcg.h:19-62) ---------------------- */
/* cudapcg.cu:108-183 */ cudapcgFlag_t cudapcgInit(cudapcgFlag_t analysis_flag, cudapcgFlag_t parStrategy_flag);
/* cudapcg.cu:185-203 */ cudapcgFlag_t cudapcgEnd(void);
/* cudapcg.cu:250-254 */ cudapcgFlag_t cudapcgSetModelConstructorFcn(cudapcgFlag_t (*fcn)(cudapcgModel_t **, const void *));
/* cudapcg.cu:256-293 */ cudapcgFlag_t cudapcgBuildModel(const void *data);
/* cudapcg.cu:205-236 */ cudapcgModel_t *cudapcgNewModel(void);
/* cudapcg.cu:238-247 */ cudapcgFlag_t cudapcgSetModel(cudapcgModel_t *model);
/* cudapcg.cu:94 */      cudapcgFlag_t cudapcgSetNumTol(cudapcgTol_t t);
/* cudapcg.cu:95 */      cudapcgFlag_t cudapcgSetMaxIterations(unsigned int n);
/* cudapcg.cu:96 */      cudapcgFlag_t cudapcgSetXReduceMode(cudapcgFlag_t flag);
/* cudapcg.cu:97 */      cudapcgFlag_t cudapcgSetXReduceShift(unsigned int shift);
/* cudapcg.cu:98 */      cudapcgFlag_t cudapcgSetXReduceScale(double scl);
/* cudapcg.cu:99 */      cudapcgFlag_t cudapcgSetReduceStabFactor(double scl);
/* cudapcg.cu:100 */     cudapcgFlag_t cudapcgSetSolver(cudapcgFlag_t flag);
/* cudapcg.cu:101 */     cudapcgFlag_t cudapcgSetPreconditioner(cudapcgFlag_t flag);
/* cudapcg.cu:102 */     cudapcgFlag_t cudapcgSetResNorm(cudapcgFlag_t flag);
/* cudapcg.cu:377-381 */ cudapcgFlag_t cudapcgAllocateArrays(void);
/* cudapcg.cu:383-387 */ cudapcgFlag_t cudapcgFreeArrays(void);
/* cudapcg.cu:312-317 */ cudapcgFlag_t cudapcgSetRHS(cudapcgVar_t *RHS);
/* cudapcg.cu:295-310 */ cudapcgFlag_t cudapcgSetX0(cudapcgVar_t *x0, cudapcgFlag_t mustInterpolate);
/* cudapcg.cu:319-325 */ cudapcgFlag_t cudapcgSetImage(cudapcgMap_t *img);
/* cudapcg.cu:327-334 */ cudapcgFlag_t cudapcgSetParametricDensityField(parametricScalarField_t *field, double fmin, double fmax);
/* cudapcg.cu:336-346 */ cudapcgFlag_t cudapcgSetPoreMap(cudapcgFlag_t *pores);
/* cudapcg.cu:348-355 */ cudapcgFlag_t cudapcgSetPeriodic2DOFMap(cudapcgIdMap_t *vars);
/* cudapcg.cu:357-363 */ cudapcgFlag_t cudapcgSetDOF2PeriodicMap(cudapcgIdMap_t *nodes);
/* cudapcg.cu:365-375 */ cudapcgFlag_t cudapcgSetLclMtxs(cudapcgVar_t *LclMtxs);
/* cudapcg.cu:389-409 */ cudapcgFlag_t cudapcgSolve(cudapcgVar_t *x);  /* CG2/MINRES2: x[0..2] = reduced sums;
                                                                        x = NULL (CG/MINRES): the solution stays
                                                                        on the device only */
/* cudapcg.cu:411-434 */ cudapcgFlag_t cudapcgSetHeaderString(char *header);
/* cudapcg.cu:434-448 */ cudapcgFlag_t cudapcgPrintSolverReport(void);
/* cudapcg.cu:450-469 */ cudapcgFlag_t cudapcgPrintSolverReport2(char *dest);
/* cudapcg.cu:471-482 */ cudapcgFlag_t cudapcgPrintSolverMetrics(void);
/* cudapcg.cu:484-499 */ cudapcgFlag_t cudapcgPrintSolverMetrics2(char *dest);
/* cudapcg.cu:103 */     unsigned int cudapcgGetNumIterations(void);
/* cudapcg.cu:104 */     unsigned int cudapcgGetMaxNumIterations(void);
/* cudapcg.cu:105 */     cudapcgVar_t cudapcgGetResidual(void);

/* ---------------- Part 2: extensions (no counterpart in the reference) ---------------- */
#define CHFEM_B200_FP64 0   /* FP64 storage and arithmetic (parity mode, default)            */
#define CHFEM_B200_MIXED 1  /* FP32 fields/operator, FP64 dots, stopping test, replacement  */

/* Last error message of this library ("" when none). */
const char *cudapcgB200LastError(void);
/* Precision mode for the next solves (CHFEM_B200_FP64 or CHFEM_B200_MIXED).  Mixed applies to
   THERMAL_3D and ELASTIC_3D; FLUID_3D models always solve in FP64 (its (P)MINRES recurrence
   nears breakdown on the indefinite Stokes system, where FP32 rounding stalls it). */
cudapcgFlag_t cudapcgB200SetPrecision(int mode);
/* Mixed mode: replace the recursive residual by b - A x every k iterations (0 = never). */
cudapcgFlag_t cudapcgB200SetResidualReplacement(unsigned int k);
/* Iterations per CUDA-graph launch of the device-resident loop (even, >= 2). */
cudapcgFlag_t cudapcgB200SetIterationsPerLaunch(unsigned int k);
/* y = A x on the current model (host buffers of nvars doubles); for parity tests. */
cudapcgFlag_t cudapcgB200ApplyOperator(const double *x, double *y);
/* y = M^-1 x (Jacobi) on the current model. */
cudapcgFlag_t cudapcgB200ApplyPreconditioner(const double *x, double *y);
/* Block solve of nrhs load cases of the current model at once (3 for thermal, 3 or 6 for
   elastic; CG/PCG): rhs[k], x_out[k] are host buffers of nvars doubles, x0 may be NULL or hold
   NULL entries; x0_interpolate: 0 each x0[k] is a host vector of nvars doubles, 1 a host
   solution on the model coarsened by 2 per axis, prolonged as cudapcgSetX0(x0, 1) does, 2 a
   device vector of nvars doubles.  Each right-hand side runs the
   recurrence and stopping test of cudapcgSolve; the operator reads the model once per block
   apply.  iterations/residuals (nrhs entries) may be NULL.  Returns 1 when every right-hand
   side met the tolerance. */
cudapcgFlag_t cudapcgB200SolveBlock(unsigned int nrhs, const double *const *rhs, const double *const *x0,
                                    int x0_interpolate, double *const *x_out, unsigned int *iterations,
                                    double *residuals);
/* y[k] = A v[k] for nrhs host vectors of nvars doubles (3 thermal, 3 or 6 elastic) through the
   block operator pass that cudapcgB200SolveBlock runs; for parity tests. */
cudapcgFlag_t cudapcgB200ApplyBlockOperator(unsigned int nrhs, const double *const *v, double *const *y);
/* Block solve of the homogenization load cases of the current model with the right-hand sides
   assembled and the effective-tensor volume term reduced on the device, so that no full-length
   vector crosses to or from the host.  Load case k: thermal/elastic, the macroscopic jump
   jump[k] along axis[k] (0 x, 1 y, 2 z) in DOF component comp[k], entering through the voxels
   on the +axis cell boundary (femhmg_thermal_3D.c:122-236, femhmg_elastic_3D.c:130-511);
   Stokes (MINRES/PMINRES), a unit body force along axis[k] (femhmg_fluid_3D.c:112-182; comp
   and jump unused).  CB: the effective-tensor matrices of the host layer -- nmat x ns x 8dof
   (thermal ns = 3, elastic ns = 6) or Stokes 3 x 24 followed by the 8 body-force weights.
   moments[k*ns + s] = sum over voxels of (CB x)_s for case k (Stokes: the mean-velocity sums),
   to which the caller adds the boundary face term.  x0 / x0_interpolate as for
   cudapcgB200SolveBlock; x_out may be NULL or hold NULL entries (no copy back).  Returns 1 when
   every case met the tolerance. */
cudapcgFlag_t cudapcgB200SolveLoadCases(unsigned int nrhs, const int *axis, const int *comp, const double *jump,
                                        const double *CB, unsigned int ns, const double *const *x0, int x0_interpolate,
                                        double *moments, double *const *x_out, unsigned int *iterations,
                                        double *residuals);
/* Batched thermal homogenization (no counterpart in the reference, which homogenizes one image
   per run): nsamples independent periodic models of any sizes, each with its own 1..4
   conductivities, solved together with all 3 load cases (X, Y, Z) of every sample; each load
   case of each sample keeps its own PCG scalars and L2 stopping test (pcg.cu:100-224) and stops
   on its own.  Sample s: dims[3s..3s+2] = nrows (y), ncols (x), nlayers (z); keys[s] its 16-bit
   node keys (as cudapcgSetImage takes them, nrows*ncols*nlayers entries); Kdense[s] its nmat[s]
   dense 8x8 conductivity matrices; CB[s] its nmat[s] 3x8 flux-averaging matrices (the host
   layer's effective-tensor matrices).  The load-case right-hand sides are built on the device.
   Out: moments[9s + 3k + row] = sum over voxels of (CB x_k)_row for load case k (add the face
   term and divide by the voxel count for the tensor); iterations/residuals [3s + k] may be NULL.
   precision CHFEM_B200_FP64 or CHFEM_B200_MIXED (FP32 fields; FP64 x, dots, replacement).
   The operator's tile shape (32 x 4, 8 or 16 nodes) is timed once per batch signature and
   remembered.  Returns 1 when every load case converged, 2 when some stopped at maxit, 0 on
   error (cudapcgB200BatchLastError).  Independent of the cudapcgInit model. */
typedef struct {
  double setup_seconds;   /* device time of the initial pass */
  double solve_seconds;   /* device time of the iterations and the tensor reduction */
  double wall_seconds;    /* whole call, uploads included */
  unsigned int max_iterations;
  unsigned int converged; /* load cases that met the tolerance */
  unsigned long long kernel_launches;
  int tile_cols;          /* chosen tile: 32 x tile_cols nodes */
  int ctas_operator, ctas_pointwise;
  double tile_ms[3];      /* timed operator pass for tiles 32x4, 32x8, 32x16 (0 when cached) */
} cudapcgB200BatchStats;
int cudapcgB200SolveThermalBatch(unsigned int nsamples, const unsigned int *dims, const uint16_t *const *keys,
                                 const unsigned int *nmat, const double *const *Kdense, const double *const *CB, double tol,
                                 unsigned int maxit, int precision, int precondition, double *moments,
                                 unsigned int *iterations, double *residuals, cudapcgB200BatchStats *stats);
const char *cudapcgB200BatchLastError(void);
/* Exported field of a solution still on the device (chfem's -e output,
   femhmg_thermal_3D.c:674-1111, femhmg_elastic_3D.c:1800-2650): the nodal heat flux (3 per node)
   or stress (6 per node, Voigt xx yy zz yz xz xy), each node's value the mean over its 8 voxels
   of the voxel's field at that node's corner; boundary voxels see the load case's jump (the
   displaced component comp on their +axis face nodes).  block_index -1: the solution of the last
   cudapcgSolve; k >= 0: right-hand side k of the last block solve.  props: conductivity per
   material (thermal) or (E, nu) per material (elastic).  field_out: host, nf * nodes doubles. */
cudapcgFlag_t cudapcgB200ComputeFields(int block_index, int axis, int comp, double jump, const double *props,
                                       double *field_out);
/* The one-by-one load-case loop on the device (femhmg.c:1030-1110 without the host's RHS
   assembly, x copy and updateC loop): cudapcgB200SetLoadCaseRHS builds the right-hand side of
   load case (axis, comp, jump) from the node keys and element matrices (thermal / elastic) or
   the pore map (Stokes: CB = the model's 3x24 + 8 velocity-averaging entries, axis = flow
   direction), as the host's assembly (femhmg_thermal_3D.c / femhmg_elastic_3D.c / _fluid_3D.c
   assembleRHS); after cudapcgSolve, cudapcgB200VolumeTerm returns the volume term sum_e CB_e x_e
   of the tensor column (ns = 3 thermal / Stokes, 6 elastic; CB per material in the layout of
   cudapcgB200SolveLoadCases).  The face term is the caller's (a few boundary voxels). */
cudapcgFlag_t cudapcgB200SetLoadCaseRHS(int axis, int comp, double jump, const double *CB);
cudapcgFlag_t cudapcgB200VolumeTerm(const double *CB, unsigned int ns, double *moments);
/* Node material keys built on the device from the voxel image's colours (thermal / elastic,
   NBN): colors = rows x cols x slices bytes with x fastest (the .raw order, femhmg.c:1644-1700),
   each voxel split into refinement^3 model voxels; material_of_color[256] = the material index
   of each colour (-1: not listed, which is an error).  Replaces building the keys on the host
   and cudapcgSetImage(keys) (femhmg.c:1000-1004, femhmg_3D.c:19-75): one byte per voxel
   crosses PCIe instead of two. */
cudapcgFlag_t cudapcgB200SetImageColors(const uint8_t *colors, unsigned int rows, unsigned int cols, unsigned int slices,
                                        unsigned int refinement, const int *material_of_color);
/* Stokes (FLUID_3D) DOF-number maps built on the device from the image's colours, in place of
   building them on the host and cudapcgSetPeriodic2DOFMap / SetPoreMap / SetDOF2PeriodicMap
   (femhmg_fluid_3D.c:370-491 numbers them on the host): material_of_color as for
   cudapcgB200SetImageColors, pore = material 0; pore nodes are numbered first, then interface
   nodes, each in node order.  The model's nporenodes, nbordernodes, nvars and nhmgvars are set
   from the numbering (also in the caller's model struct), and *npore, *nborder return them. */
cudapcgFlag_t cudapcgB200SetPoreImageColors(const uint8_t *colors, unsigned int rows, unsigned int cols, unsigned int slices,
                                            unsigned int refinement, const int *material_of_color, unsigned int *npore,
                                            unsigned int *nborder);
/* The current Stokes model's node->DOF (N), DOF->node (nporenodes + nbordernodes) and interface
   key (nbordernodes) maps copied to host buffers (any may be NULL); for tests. */
cudapcgFlag_t cudapcgB200GetPoreMaps(uint32_t *dof_of_node, uint32_t *node_of_dof, uint8_t *border_keys);
/* Initial guess of the next cudapcgSolve from a device vector of nvars doubles (the device
   counterpart of cudapcgSetX0(x0, 0); cleared by cudapcgSetX0(NULL, 0)). */
cudapcgFlag_t cudapcgB200SetX0Device(const double *x0);
/* Statistics of the last solve. */
typedef struct {
  unsigned int iterations;
  double residual;
  double solve_seconds;        /* device time of the iteration loop (CUDA events) */
  double setup_seconds;        /* device time of init + initial-guess handling */
  unsigned long long kernel_launches;  /* kernels of this library launched by the last solve */
  int precision;
  int found;
} cudapcgB200Stats;
cudapcgFlag_t cudapcgB200GetStats(cudapcgB200Stats *out);
/* Device-side operator timing: runs `reps` applies of the current model's operator on its
   work vectors and returns the mean duration in seconds (CUDA events); for roofline reports. */
double cudapcgB200TimeOperator(unsigned int reps);
/* Mean device duration (s, CUDA events on the library's stream) of `reps` launches of one
   kernel of the iteration on the current model and its work vectors:
   which 0 plain operator apply, 1 PCG operator pass (direction formed on the fly + dot),
   2 PCG pointwise update pass, 3 (P)MINRES operator pass, 4 (P)MINRES direction pass,
   5 block PCG operator pass and 6 block PCG pointwise pass (thermal: 3 right-hand sides,
   elastic: 6; see cudapcgB200SolveBlock).
   The solver scalars are reset first; results of the work vectors are meaningless after. */
double cudapcgB200TimeKernel(int which, unsigned int reps);
/* Operator apply that allocates nothing (no counterpart in the reference).  For callers that
   cannot allocate device memory -- an embedder whose device memory belongs to its own
   allocator or pool, or a loop that must not pay cudaMalloc's implicit synchronisation:
   y = A v and *vAv = v.Av for a THERMAL_3D (1) or ELASTIC_3D (3) model, all FP64, every
   pointer a caller-owned device buffer: keys (nrows*ncols*nlayers 16-bit node keys), Kdense
   (nmat dense element matrices of (8*dof)^2 doubles, i.e. the SparseQ1 thermal rows expanded
   to 8x8), v and y (nvars doubles), vAv (1 double); y and vAv must not overlap v, keys or
   Kdense (rejected).  Scratch lives in a fixed 66 KB file-scope device array held by every
   GPU that loads the library until exit; its address is looked up on every call made outside
   stream capture, and a call under capture uses the one of the last uncaptured call on that
   device (so the first call on a device, and the first after a device reset, must be made
   outside capture).  Calls that overlap on the GPU share that array and race.  Any model size
   is accepted (the operator runs on at most 8192 CTAs, one reduction slot each); each
   dimension must stay below 2^31 - 16.  stream: a cudaStream_t (NULL for the default stream).
   Returns 1, or 0 with cudapcgB200LastError() set. */
int cudapcgB200ApplyOperatorNoAlloc(int analysis_flag, unsigned int nrows, unsigned int ncols, unsigned int nlayers,
                                    unsigned int nmat, const uint16_t *keys, const double *Kdense, const double *v,
                                    double *y, double *vAv, void *stream);
/* Number of bytes the library holds on the device for the current model and arrays. */
unsigned long long cudapcgB200DeviceBytes(void);
/* The solver's device blocks come from the current device's default stream-ordered memory pool,
   which keeps freed blocks (up to a quarter of the device's memory) mapped for the next model
   (cudapcgEnd returns them to the pool, not to the driver).  This hands every kept block of the pool back to the driver.  Returns 1, or 0
   with cudapcgB200LastError() set. */
int cudapcgB200TrimMemory(void);

#ifdef __cplusplus
}
#endif
#endif /* CUDAPCG_B200_H */
