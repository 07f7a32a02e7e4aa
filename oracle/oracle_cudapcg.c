/*
 * oracle_cudapcg.c -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the parity oracle of the chfem_b200 build: a CPU, FP64, OpenMP restatement
 * of chfem's cudapcg solver library (the matrix-free voxel-FEM operator, its Jacobi
 * preconditioner and the CG / PCG / MINRES / PMINRES loops) operating on exactly the data
 * formats the reference's host code hands over the cudapcg C ABI.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it, and only as the
 * checker.  The product (chfem_b200/) never links or calls it.
 *
 * Each function cites the reference file:line it follows (paths inside cortezpedro/chfem).
 * Scope: 3D thermal (1 DOF/node), 3D elastic (3 DOF/node), 3D Stokes with the DOF-number
 * pore map (CUDAPCG_POREMAP_NUM; the image pore map is turned into it), including the 2-vector
 * solvers with on-the-fly reduction of the solution (CG2/PCG2/MINRES2/PMINRES2, Stokes); the
 * scalar density field; 2D thermal (1 DOF/node), 2D elastic (2 DOF/node) and 2D Stokes (2
 * velocities + pressure, the 2-vector solvers included) on pixel images.
 *
 * Operator restatement.  The reference applies A node-by-node: for node i and each of the
 * 8 voxels (elements) around it, i is local node e of element e, and the row block of the
 * element matrix K_m(e) that belongs to local node e is multiplied with the 8 nodal values
 * of that element (chfem/src/femhmg/cudapcg/kernels/matrix_free.cu:125-164 thermal,
 * :416-459 elastic, :689-732 Stokes pore rows, :936-977 Stokes interface rows).  This
 * oracle does the same with dense element matrices; the thermal "SparseQ1" 40-entry
 * storage (matrix_free.cu:191-323, femhmg_thermal_3D.c:42-120) is expanded to the dense
 * 8x8 form once, when the local matrices are set.
 */
#define _GNU_SOURCE
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <omp.h>
#include "oracle_cudapcg.h"

/* ------------------------------------------------------------------------------------ */
/* Element geometry.  Local node k of an element sits at (row,col,layer) offset          */
/* (DROW,DCOL,DLAY)[k] from local node 0 (matrix_free.cu:147-160: WALK_RIGHT = col+1,    */
/* WALK_UP = row-1, WALK_FAR = layer+1).                                                  */
static const int DROW[8] = {0, 0, -1, -1, 0, 0, -1, -1};
static const int DCOL[8] = {0, 1, 1, 0, 0, 1, 1, 0};
static const int DLAY[8] = {0, 0, 0, 0, 1, 1, 1, 1};

static inline unsigned int wrapi(int v, unsigned int n) { return (unsigned int)((v % (int)n + (int)n) % (int)n); }
/* PERIODICNUM_3D (chfem/src/femhmg/cudapcg/kernels/utils.h:82): row fastest. */
static inline unsigned int pnum(int r, int c, int l, unsigned int R, unsigned int C, unsigned int L) {
  return wrapi(r, R) + wrapi(c, C) * R + wrapi(l, L) * R * C;
}

/* The 27 periodic neighbours of node (r,c,l), indexed (dr+1) + 3(dc+1) + 9(dl+1). */
static inline void neighbours27(int r, int c, int l, unsigned int R, unsigned int C, unsigned int L, unsigned int *nb) {
  unsigned int rr[3] = {wrapi(r - 1, R), (unsigned int)r, wrapi(r + 1, R)};
  unsigned int cc[3] = {wrapi(c - 1, C) * R, (unsigned int)c * R, wrapi(c + 1, C) * R};
  unsigned int ll[3] = {wrapi(l - 1, L) * R * C, (unsigned int)l * R * C, wrapi(l + 1, L) * R * C};
  for (int k = 0; k < 3; k++)
    for (int j = 0; j < 3; j++)
      for (int t = 0; t < 3; t++) nb[t + 3 * j + 9 * k] = rr[t] + cc[j] + ll[k];
}
/* Neighbour slot of local node b of the element in which the centre node is local node e. */
#define NBIDX(e, b) ((DROW[b] - DROW[e] + 1) + 3 * (DCOL[b] - DCOL[e] + 1) + 9 * (DLAY[b] - DLAY[e] + 1))

/* ------------------------------------------------------------------------------------ */
typedef struct {
  cudapcgModel_t *model;
  unsigned int analysis;   /* CUDAPCG_THERMAL_2D / 3D, ELASTIC_2D / 3D, FLUID_2D / 3D */
  int dim2;                /* 2D analysis: pixel images, 4-node elements, 4-bit key fields */
  unsigned int par;        /* NBN / EBE */
  cudapcgTol_t tol;
  unsigned int maxit;
  unsigned int solver_flag;
  int precond;
  int resnorm;
  int x0_set;
  char *header;
  unsigned int iteration;
  double residual;
  double total_time, mean_time;
  int found;
  double *x, *r, *d, *q, *s;
  /* 2-vector solvers: reduction mode, shift (loaded velocity component), scale, solve count */
  unsigned int xr_mode, xr_shift;
  double xr_scale;
  unsigned long count;
  double *Kd;        /* dense element matrices, nkeys x (ed x ed) */
  unsigned int ed;   /* element matrix dimension: 8, 24 or 32 */
  unsigned int nkeys;
  unsigned short *keys; /* per-node material key (NBN form), derived for EBE */
  /* scalar density field (cudapcgSetParametricDensityField): per voxel a 16-bit code q, the
     voxel's element matrix scaled by fmin + (fmax - fmin) q / 65535 */
  parametricScalarField_t *sdf;
  double sdf_min, sdf_max;
} oracle_solver_t;

static oracle_solver_t *S = NULL;
static int is_fluid(void) { return S->analysis == CUDAPCG_FLUID_3D || S->analysis == CUDAPCG_FLUID_2D; }
static cudapcgFlag_t (*model_ctor)(cudapcgModel_t **, const void *) = NULL;
static int g_quiet = 0;

/* captured inputs (checker access): 0 image/keys, 1 node->DOF, 2 DOF->node, 3 pore map,
   4 local matrices, 5 right-hand side, 6 solution, 7 density codes, 8 density range */
#define CAP_SLOTS 9
static void *cap_ptr[CAP_SLOTS] = {0};
static unsigned int cap_n[CAP_SLOTS] = {0};
static size_t cap_elsz[CAP_SLOTS] = {sizeof(cudapcgMap_t), sizeof(cudapcgIdMap_t), sizeof(cudapcgIdMap_t),
                                     sizeof(cudapcgFlag_t), sizeof(double), sizeof(double), sizeof(double),
                                     sizeof(parametricScalarField_t), sizeof(double)};
static double *hist = NULL;
static unsigned int hist_n = 0, hist_cap = 0;
#define LOG_CAP 4096
static unsigned int log_it[LOG_CAP];
static double log_res[LOG_CAP];
static unsigned int log_n = 0;

static void capture(int which, const void *src, unsigned int n) {
  free(cap_ptr[which]);
  cap_ptr[which] = malloc((size_t)n * cap_elsz[which] + 1);
  if (cap_ptr[which] && src) memcpy(cap_ptr[which], src, (size_t)n * cap_elsz[which]);
  cap_n[which] = n;
}
static void hist_push(double v) {
  if (hist_n == hist_cap) {
    hist_cap = hist_cap ? 2 * hist_cap : 1024;
    hist = (double *)realloc(hist, sizeof(double) * hist_cap);
  }
  hist[hist_n++] = v;
}

/* ------------------------------------------------------------------------------------ */
/* Stopping-test helpers: chfem/src/femhmg/cudapcg/solvers/stopping_criteria.cu:7-14.    */
/* The reference's bit-trick square root (solvers_utils.cu:39-53) is a sqrt             */
/* approximation refined by Newton steps; the oracle uses libm sqrt, which differs only */
/* in the printed residual, never in the stop decision (that compares squares).          */
static int above_tol(double delta, double delta0, double tol) { return fabs(delta) > tol * tol * fabs(delta0); }
static double eval_res(double delta, double delta0) { return sqrt(fabs(delta) / fabs(delta0)); }

/* ------------------------------------------------------------------------------------ */
/* BLAS-1 (chfem/src/femhmg/cudapcg/kernels/vector.cu:21-110, :463-492, :540-573).        */
static double dot(const double *a, const double *b, unsigned int n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < (long)n; i++) s += a[i] * b[i];
  return s;
}
static double absmax(const double *a, unsigned int n) {
  double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static)
  for (long i = 0; i < (long)n; i++) { double v = fabs(a[i]); if (v > m) m = v; }
  return m;
}
static void zeros(double *a, unsigned int n) { memset(a, 0, sizeof(double) * n); }
static void axpy_iny(double *y, const double *x, double a, unsigned int n) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; i++) y[i] += a * x[i];
}
static void axpy_to(const double *y, const double *x, double a, unsigned int n, double *res) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; i++) res[i] = y[i] + a * x[i];
}
static void arrcpy(const double *v, unsigned int n, double *res) { memmove(res, v, sizeof(double) * n); }

/* ------------------------------------------------------------------------------------ */
/* Thermal SparseQ1 expansion.  Row a of the Q1 conductivity matrix is non-zero on the    */
/* diagonal and on the 4 nodes that share no edge with a; the 40 stored values list the   */
/* non-zeros of rows 0..7 in ascending column order (femhmg_thermal_3D.c:42-120,          */
/* matrix_free.cu:191-323 whose K[mat+j] walk follows the same order).                    */
static int shares_edge(int a, int b) {
  int dif = (DROW[a] != DROW[b]) + (DCOL[a] != DCOL[b]) + (DLAY[a] != DLAY[b]);
  return dif == 1;
}
static void expand_sparseq1(const double *sp, double *dense8) {
  int p = 0;
  for (int a = 0; a < 8; a++)
    for (int b = 0; b < 8; b++) dense8[a * 8 + b] = shares_edge(a, b) ? 0.0 : sp[p++];
}

/* Node key from a per-voxel material map (EBE input, cudapcgSetImage with               */
/* elem_material_map, femhmg.c:1001-1004).  Voxel v is the element whose local node 3 is  */
/* node v (femhmg_3D.c:45-49), so the element in which node (r,c,l) is local node e is   */
/* voxel (r-DROW[e]-1, c-DCOL[e], l-DLAY[e]).  Key layout: femhmg_3D.c:19-75.            */
static void keys_from_elements(const cudapcgMap_t *em, unsigned int R, unsigned int C, unsigned int L, unsigned short *keys) {
  unsigned int N = R * C * L;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)N; i++) {
    int r = (int)(i % R), c = (int)((i / R) % C), l = (int)(i / ((long)R * C));
    unsigned int k = 0;
    for (int e = 0; e < 8; e++) k |= ((unsigned int)em[pnum(r - DROW[e] - 1, c - DCOL[e], l - DLAY[e], R, C, L)] & 3u) << (2 * e);
    keys[i] = (unsigned short)k;
  }
}

/* ------------------------------------------------------------------------------------ */
/* Operator y = A x (reference formulation, FP64).                                        */
/* Scale of the voxel in which node (r, c, l) is local node e: 1 without a density field;
   with one, fmin + (fmax - fmin) q / 65535 of that voxel, the voxel at (r - DROW[e] - 1,
   c - DCOL[e], l - DLAY[e]) (matrix_free.cu:2283-2295 lists the 8 voxels around a node in this
   order, kernel_applyPreConditioner_thermal_3D_ElemByElem_ScalarDensityField). */
static double sdf_scale(int r, int c, int l, int e, unsigned int R, unsigned int C, unsigned int L) {
  if (!S->sdf) return 1.0;
  const unsigned int v = pnum(r - DROW[e] - 1, c - DCOL[e], l - DLAY[e], R, C, L);
  return S->sdf_min + (S->sdf_max - S->sdf_min) * (double)S->sdf[v] * (1.0 / 65535.0);
}

static void apply_thermal_elastic(const double *v, double *y) {
  cudapcgModel_t *m = S->model;
  const unsigned int R = m->nrows, C = m->ncols, L = m->nlayers, N = R * C * L;
  const unsigned int nd = (S->analysis == CUDAPCG_ELASTIC_3D) ? 3 : 1;
  const unsigned int ed = 8 * nd;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)N; i++) {
    int r = (int)(i % R), c = (int)((i / R) % C), l = (int)(i / ((long)R * C));
    unsigned int nb[27];
    neighbours27(r, c, l, R, C, L, nb);
    unsigned int key = S->keys[i];
    double acc[3] = {0, 0, 0};
    for (int e = 0; e < 8; e++) {
      const double *K = S->Kd + (size_t)((key >> (2 * e)) & 3u) * ed * ed;
      const double f = sdf_scale(r, c, l, e, R, C, L);
      for (int b = 0; b < 8; b++) {
        unsigned int j = nb[NBIDX(e, b)];
        for (unsigned int ci = 0; ci < nd; ci++) {
          const double *row = K + (size_t)(e * nd + ci) * ed + b * nd;
          double s = 0.0;
          for (unsigned int cj = 0; cj < nd; cj++) s += row[cj] * v[(size_t)j * nd + cj];
          acc[ci] += f * s;
        }
      }
    }
    for (unsigned int ci = 0; ci < nd; ci++) y[(size_t)i * nd + ci] = acc[ci];
  }
}

/* Stokes, DOF-number pore map (matrix_free.cu:674-732 pore rows, :926-977 interface rows; */
/* layout [3*nVel interleaved velocities | nVel+nBorder pressures], matrix_free.cu:5012-5047). */
static void apply_fluid(const double *v, double *y) {
  cudapcgModel_t *m = S->model;
  const unsigned int R = m->nrows, C = m->ncols, L = m->nlayers;
  const unsigned int nV = m->nporenodes, nB = m->nbordernodes;
  const double *K = S->Kd;
  const cudapcgIdMap_t *dmap = m->periodic2DOF_map, *nmap = m->DOF2periodic_map;
#pragma omp parallel for schedule(static)
  for (long id = 0; id < (long)(nV + nB); id++) {
    unsigned int node = nmap[id];
    int r = (int)(node % R), c = (int)((node / R) % C), l = (int)(node / (R * C));
    int pore = id < (long)nV;
    unsigned int fkey = pore ? 255u : m->border_pore_map[id - nV];
    double rv[3] = {0, 0, 0}, rp = 0.0;
    unsigned int nb[27];
    neighbours27(r, c, l, R, C, L, nb);
    for (int e = 0; e < 8; e++) {
      if (!((fkey >> e) & 1u)) continue;
      for (int b = 0; b < 8; b++) {
        unsigned int dof = dmap[nb[NBIDX(e, b)]];
        if (dof < nV) {
          const double *vv = v + 3 * (size_t)dof;
          if (pore)
            for (int ci = 0; ci < 3; ci++)
              rv[ci] += K[(3 * e + ci) * 32 + 3 * b] * vv[0] + K[(3 * e + ci) * 32 + 3 * b + 1] * vv[1] + K[(3 * e + ci) * 32 + 3 * b + 2] * vv[2];
          rp += K[(24 + e) * 32 + 3 * b] * vv[0] + K[(24 + e) * 32 + 3 * b + 1] * vv[1] + K[(24 + e) * 32 + 3 * b + 2] * vv[2];
        }
        double vp = v[3 * (size_t)nV + dof];
        if (pore)
          for (int ci = 0; ci < 3; ci++) rv[ci] += K[(3 * e + ci) * 32 + 24 + b] * vp;
        rp -= K[(24 + e) * 32 + 24 + b] * vp;
      }
    }
    if (pore) { y[3 * id] = rv[0]; y[3 * id + 1] = rv[1]; y[3 * id + 2] = rv[2]; }
    y[3 * (size_t)nV + id] = rp;
  }
}

/* 2D thermal / elastic (matrix_free.cu:70-95, :353-385): node i = (row, col) is local node e of
   the pixel (row - DROW[e] - 1, col - DCOL[e]) and that pixel's local node b sits at
   (row - DROW[e] + DROW[b], col - DCOL[e] + DCOL[b]); the key holds the pixel's material in bits
   [4e, 4e + 4) (femhmg_2D.c:14-46); element matrices are dense (4 nd) x (4 nd), row-major. */
/* Density scale of the pixel in which node (r, c) is local node e, the pixel at
   (r - DROW[e] - 1, c - DCOL[e]); 1 without a density field (matrix_free.cu:1800-1880 and
   :2748-2850: each pixel's element matrix, of its own material, scaled by its density) */
static double sdf_scale_2d(int r, int c, int e, unsigned int R, unsigned int C) {
  if (!S->sdf) return 1.0;
  const unsigned int v = wrapi(r - DROW[e] - 1, R) + wrapi(c - DCOL[e], C) * R;
  return S->sdf_min + (S->sdf_max - S->sdf_min) * (double)S->sdf[v] * (1.0 / 65535.0);
}

static void apply_2d(const double *v, double *y) {
  cudapcgModel_t *m = S->model;
  const unsigned int R = m->nrows, C = m->ncols, N = R * C;
  const unsigned int nd = (S->analysis == CUDAPCG_ELASTIC_2D) ? 2 : 1, ed = 4 * nd;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)N; i++) {
    const int r = (int)(i % R), c = (int)(i / R);
    const unsigned int key = S->keys[i];
    double acc[2] = {0, 0};
    for (int e = 0; e < 4; e++) {
      const double *K = S->Kd + (size_t)((key >> (4 * e)) & 15u) * ed * ed;
      const double f = sdf_scale_2d(r, c, e, R, C);
      for (int b = 0; b < 4; b++) {
        const unsigned int j = wrapi(r - DROW[e] + DROW[b], R) + wrapi(c - DCOL[e] + DCOL[b], C) * R;
        for (unsigned int ci = 0; ci < nd; ci++) {
          double s = 0.0;
          for (unsigned int cj = 0; cj < nd; cj++) s += K[(e * nd + ci) * ed + b * nd + cj] * v[(size_t)j * nd + cj];
          acc[ci] += f * s;
        }
      }
    }
    for (unsigned int ci = 0; ci < nd; ci++) y[(size_t)i * nd + ci] = acc[ci];
  }
}
/* 2D Jacobi (matrix_free.cu:51-68, :325-346): the node's diagonal entries over its 4 pixels,
   each scaled by the pixel's density under a density field (matrix_free.cu:1350-1365,
   :1398-1416) */
static void inv_diag_2d(double *dinv) {
  cudapcgModel_t *m = S->model;
  const unsigned int R = m->nrows, C = m->ncols, N = R * C;
  const unsigned int nd = (S->analysis == CUDAPCG_ELASTIC_2D) ? 2 : 1, ed = 4 * nd;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)N; i++) {
    const int r = (int)(i % R), c = (int)(i / R);
    const unsigned int key = S->keys[i];
    for (unsigned int ci = 0; ci < nd; ci++) {
      double s = 0.0;
      for (int e = 0; e < 4; e++)
        s += sdf_scale_2d(r, c, e, R, C) * S->Kd[(size_t)((key >> (4 * e)) & 15u) * ed * ed + (e * nd + ci) * ed + e * nd + ci];
      dinv[(size_t)i * nd + ci] = 1.0 / s;
    }
  }
}
/* 2D node key from a per-pixel material map (EBE input) */
static void keys_from_elements_2d(const cudapcgMap_t *em, unsigned int R, unsigned int C, unsigned short *keys) {
  for (long i = 0; i < (long)R * C; i++) {
    const int r = (int)(i % R), c = (int)(i / R);
    unsigned int k = 0;
    for (int e = 0; e < 4; e++) k |= ((unsigned int)em[wrapi(r - DROW[e] - 1, R) + wrapi(c - DCOL[e], C) * R] & 15u) << (4 * e);
    keys[i] = (unsigned short)k;
  }
}

/* 2D Stokes, DOF-number pore map (matrix_free.cu:484-518 pore rows, :628-660 interface rows):
   the 12 x 12 element matrix [K G; G^T Stab] enters as [K G; G^T -Stab] over the node's fluid
   pixels; velocity columns of non-pore neighbours are dropped (no slip); vector layout
   [2 nVel interleaved velocities | nVel + nBorder pressures]. */
static void apply_fluid_2d(const double *v, double *y) {
  cudapcgModel_t *m = S->model;
  const unsigned int R = m->nrows, C = m->ncols;
  const unsigned int nV = m->nporenodes, nB = m->nbordernodes;
  const double *K = S->Kd;
  const cudapcgIdMap_t *dmap = m->periodic2DOF_map, *nmap = m->DOF2periodic_map;
#pragma omp parallel for schedule(static)
  for (long id = 0; id < (long)(nV + nB); id++) {
    const unsigned int node = nmap[id];
    const int r = (int)(node % R), c = (int)(node / R);
    const int pore = id < (long)nV;
    const unsigned int fkey = pore ? 15u : m->border_pore_map[id - nV];
    double rv[2] = {0, 0}, rp = 0.0;
    for (int e = 0; e < 4; e++) {
      if (!((fkey >> e) & 1u)) continue;
      for (int b = 0; b < 4; b++) {
        const unsigned int dof = dmap[wrapi(r - DROW[e] + DROW[b], R) + wrapi(c - DCOL[e] + DCOL[b], C) * R];
        if (dof < nV) {
          const double *vv = v + 2 * (size_t)dof;
          if (pore)
            for (int ci = 0; ci < 2; ci++) rv[ci] += K[(2 * e + ci) * 12 + 2 * b] * vv[0] + K[(2 * e + ci) * 12 + 2 * b + 1] * vv[1];
          rp += K[(8 + e) * 12 + 2 * b] * vv[0] + K[(8 + e) * 12 + 2 * b + 1] * vv[1];
        }
        const double vp = v[2 * (size_t)nV + dof];
        if (pore)
          for (int ci = 0; ci < 2; ci++) rv[ci] += K[(2 * e + ci) * 12 + 8 + b] * vp;
        rp -= K[(8 + e) * 12 + 8 + b] * vp;
      }
    }
    if (pore) { y[2 * id] = rv[0]; y[2 * id + 1] = rv[1]; }
    y[2 * (size_t)nV + id] = rp;
  }
}
/* 2D Stokes Jacobi (matrix_free.cu:461-469, :608-616) */
static void inv_diag_fluid_2d(double *dinv) {
  cudapcgModel_t *m = S->model;
  const unsigned int nV = m->nporenodes, nB = m->nbordernodes;
  const double *K = S->Kd;
  double dv[2] = {0, 0}, dp = 0.0;
  for (int e = 0; e < 4; e++) {
    for (int ci = 0; ci < 2; ci++) dv[ci] += K[(2 * e + ci) * 13];
    dp -= K[(8 + e) * 13];
  }
#pragma omp parallel for schedule(static)
  for (long id = 0; id < (long)nV; id++) {
    for (int ci = 0; ci < 2; ci++) dinv[2 * id + ci] = 1.0 / dv[ci];
    dinv[2 * (size_t)nV + id] = 1.0 / dp;
  }
#pragma omp parallel for schedule(static)
  for (long b = 0; b < (long)nB; b++) {
    const unsigned int fk = m->border_pore_map[b];
    double s = 0.0;
    for (int e = 0; e < 4; e++) s -= K[(8 + e) * 13] * (double)((fk >> e) & 1u);
    dinv[3 * (size_t)nV + b] = 1.0 / s;
  }
}

static void Aprod(const double *v, double *y) {
  if (S->analysis == CUDAPCG_FLUID_2D) apply_fluid_2d(v, y);
  else if (S->dim2) apply_2d(v, y);
  else if (S->analysis == CUDAPCG_FLUID_3D) apply_fluid(v, y);
  else apply_thermal_elastic(v, y);
}
/* Aprod with the reference's (scl, scl_prev) form: y = scl*A v + scl_prev*y (wrappers.cu:711-906). */
static void Aprod_scl(const double *v, double scl, double scl_prev, double *y, double *tmp) {
  Aprod(v, tmp);
  unsigned int n = S->model->nvars;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; i++) y[i] = scl * tmp[i] + scl_prev * y[i];
}

/* Jacobi diagonal inverse, recomputed from keys like the reference                       */
/* (matrix_free.cu:167-188 thermal, :388-408 elastic, :663-672 and :912-925 Stokes).       */
static void inv_diag(double *dinv) {
  cudapcgModel_t *m = S->model;
  if (S->analysis == CUDAPCG_FLUID_2D) { inv_diag_fluid_2d(dinv); return; }
  if (S->dim2) { inv_diag_2d(dinv); return; }
  if (S->analysis == CUDAPCG_FLUID_3D) {
    const unsigned int nV = m->nporenodes, nB = m->nbordernodes;
    const double *K = S->Kd;
    double dv[3] = {0, 0, 0}, dp = 0.0;
    for (int e = 0; e < 8; e++) {
      for (int ci = 0; ci < 3; ci++) dv[ci] += K[(3 * e + ci) * 33];
      dp -= K[(24 + e) * 33];
    }
#pragma omp parallel for schedule(static)
    for (long id = 0; id < (long)nV; id++) {
      for (int ci = 0; ci < 3; ci++) dinv[3 * id + ci] = 1.0 / dv[ci];
      dinv[3 * (size_t)nV + id] = 1.0 / dp;
    }
#pragma omp parallel for schedule(static)
    for (long b = 0; b < (long)nB; b++) {
      unsigned int fk = m->border_pore_map[b];
      double s = 0.0;
      for (int e = 0; e < 8; e++) s -= K[(24 + e) * 33] * (double)((fk >> e) & 1u);
      dinv[4 * (size_t)nV + b] = 1.0 / s;
    }
    return;
  }
  const unsigned int N = m->nrows * m->ncols * m->nlayers;
  const unsigned int nd = (S->analysis == CUDAPCG_ELASTIC_3D) ? 3 : 1, ed = 8 * nd;
  const unsigned int R = m->nrows, C = m->ncols, L = m->nlayers;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)N; i++) {
    unsigned int key = S->keys[i];
    const int r = (int)(i % R), c = (int)((i / R) % C), l = (int)(i / ((long)R * C));
    for (unsigned int ci = 0; ci < nd; ci++) {
      double s = 0.0;
      for (int e = 0; e < 8; e++) {
        const double *K = S->Kd + (size_t)((key >> (2 * e)) & 3u) * ed * ed;
        s += sdf_scale(r, c, l, e, R, C, L) * K[(e * nd + ci) * ed + e * nd + ci];
      }
      dinv[(size_t)i * nd + ci] = 1.0 / s;
    }
  }
}
static double *g_dinv = NULL;
/* res = scl1 * M^-1 v1 + scl2 * v2 (wrappers.cu:438-628). */
static void apply_precond(const double *v1, const double *v2, double scl1, double scl2, double *res) {
  unsigned int n = S->model->nvars;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; i++) res[i] = scl1 * v1[i] * g_dinv[i] + (v2 ? scl2 * v2[i] : 0.0);
}
/* res = M v1: implemented for Stokes only, with the stencil constants of                */
/* matrix_free.cu:5672-5693 (used for both NBN and SBS, wrappers.cu:663-673); the        */
/* thermal/elastic versions are warnings that leave res untouched (wrappers.cu:635-648).  */
static void apply_invprecond(const double *v1, double scl1, double *res) {
  cudapcgModel_t *m = S->model;
  if (S->analysis == CUDAPCG_FLUID_2D) {  /* the 2D stencil constants are the diagonal's (4, -4/9, -n/9) */
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)m->nvars; i++) res[i] = scl1 * v1[i] / g_dinv[i];
    return;
  }
  if (S->analysis != CUDAPCG_FLUID_3D) return;
  const unsigned int nV = m->nporenodes, nB = m->nbordernodes;
#pragma omp parallel for schedule(static)
  for (long id = 0; id < (long)nV; id++) {
    for (int ci = 0; ci < 3; ci++) res[3 * id + ci] = scl1 * v1[3 * id + ci] * (1.0 / 0.28125);
    res[3 * (size_t)nV + id] = scl1 * v1[3 * (size_t)nV + id] * (1.0 / -2.25);
  }
#pragma omp parallel for schedule(static)
  for (long b = 0; b < (long)nB; b++) {
    unsigned int fk = m->border_pore_map[b];
    double cnt = 0.0;
    for (int e = 0; e < 8; e++) cnt += (double)((fk >> e) & 1u);
    res[4 * (size_t)nV + b] = scl1 * v1[4 * (size_t)nV + b] * (cnt / -18.0);
  }
}
/* scl * v^T M^-1 v (wrappers.cu:997-1141). */
static double dot_precond(const double *v, double scl) {
  unsigned int n = S->model->nvars;
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < (long)n; i++) s += v[i] * v[i] * g_dinv[i];
  return scl * s;
}

/* ------------------------------------------------------------------------------------ */
/* Coarse-to-fine prolongation for recursive initial guesses: wrappers.cu:290-303 and     */
/* image.cu:20-123 (x2 injection at even nodes, then periodic midpoint fill along rows,   */
/* cols and layers).                                                                      */
static void interpl2(const double *v, unsigned int rows, unsigned int cols, unsigned int layers, unsigned int stride, double *res) {
  unsigned int lay = layers < 1 ? 1 : layers;
  size_t nvox = (size_t)rows * cols * lay;
  memset(res, 0, sizeof(double) * nvox * stride);
  unsigned int rc = rows / 2, cc = cols / 2, lc = lay / 2;
  size_t ncoarse = (size_t)cc * rc * (lc + (lc < 1));
  for (size_t i = 0; i < ncoarse; i++) {
    size_t ii = i % rc, jj = (i % ((size_t)cc * rc)) / rc, kk = i / ((size_t)cc * rc);
    size_t idx = 2 * ii + 2 * jj * rows + 2 * kk * (size_t)rows * cols;
    for (unsigned int j = 0; j < stride; j++) res[stride * idx + j] = 2.0 * v[stride * i + j];
  }
  size_t RC = (size_t)rows * cols;
  for (size_t i = 0; i < nvox; i++) {          /* rows */
    size_t ii = i % rows, jj = (i % RC) / rows, kk = i / RC;
    if ((ii & 1) && !(jj & 1) && !(kk & 1)) {
      size_t up = i - 1 + rows * (!(i % rows)), dn = i + 1 - rows * (!((i + 1) % rows));
      for (unsigned int j = 0; j < stride; j++) res[stride * i + j] = 0.5 * res[stride * up + j] + 0.5 * res[stride * dn + j];
    }
  }
  for (size_t i = 0; i < nvox; i++) {          /* cols */
    size_t jj = (i % RC) / rows, kk = i / RC, il = i % RC;
    if ((jj & 1) && !(kk & 1)) {
      size_t lf = (il + (RC - rows)) % RC + kk * RC, rt = (il + rows) % RC + kk * RC;
      for (unsigned int j = 0; j < stride; j++) res[stride * i + j] = 0.5 * res[stride * lf + j] + 0.5 * res[stride * rt + j];
    }
  }
  if (layers >= 1)
    for (size_t i = 0; i < nvox; i++) {        /* layers */
      size_t kk = i / RC;
      if (kk & 1) {
        size_t nr = (i + (nvox - RC)) % nvox, fr = (i + RC) % nvox;
        for (unsigned int j = 0; j < stride; j++) res[stride * i + j] = 0.5 * res[stride * nr + j] + 0.5 * res[stride * fr + j];
      }
    }
}

/* ------------------------------------------------------------------------------------ */
/* Model management: cudapcg.cu:108-293.                                                  */
static cudapcgFlag_t ctor_simple(cudapcgModel_t **ptr, const void *data) {
  if (!data) return CUDAPCG_FALSE;
  *ptr = (cudapcgModel_t *)data;
  return CUDAPCG_TRUE;
}
static void free_model(cudapcgModel_t *m) {
  if (!m) return;
  free(m->name); free(m->image); free(m->parametric_density_field); free(m->pore_map);
  free(m->border_pore_map); free(m->periodic2DOF_map); free(m->DOF2periodic_map);
  free(m);
}
static void free_arrays(void) {
  if (!S) return;
  if (!S->x0_set) { free(S->x); S->x = NULL; }
  free(S->d); free(S->q); free(S->s); free(g_dinv);
  S->d = S->q = S->s = NULL; g_dinv = NULL;
}

static void alloc_model_arrays(void);
cudapcgModel_t *cudapcgNewModel(void) {
  cudapcgModel_t *m = (cudapcgModel_t *)calloc(1, sizeof(cudapcgModel_t));
  if (!m) return NULL;
  m->freeAllowed_flag = CUDAPCG_TRUE;
  m->parStrategy_flag = CUDAPCG_NBN;
  m->poremap_flag = CUDAPCG_POREMAP_NUM;
  return m;
}

cudapcgFlag_t cudapcgEnd(void) {
  if (!S) return CUDAPCG_FALSE;
  if (S->model && S->model->freeAllowed_flag) free_model(S->model);
  free(S->x); free(S->r); free(S->d); free(S->q); free(S->s); free(S->Kd); free(S->keys); free(S->sdf); free(S->header);
  free(g_dinv); g_dinv = NULL;
  free(S); S = NULL;
  return CUDAPCG_TRUE;  /* the oracle never resets a device */
}

cudapcgFlag_t cudapcgInit(cudapcgFlag_t analysis_flag, cudapcgFlag_t par) {
  cudapcgEnd();
  if (analysis_flag != CUDAPCG_THERMAL_3D && analysis_flag != CUDAPCG_ELASTIC_3D && analysis_flag != CUDAPCG_FLUID_3D &&
      analysis_flag != CUDAPCG_THERMAL_2D && analysis_flag != CUDAPCG_ELASTIC_2D && analysis_flag != CUDAPCG_FLUID_2D) {
    fprintf(stderr, "oracle: analysis %d is not restated\n", analysis_flag);
    return CUDAPCG_FALSE;
  }
  if ((analysis_flag == CUDAPCG_FLUID_3D || analysis_flag == CUDAPCG_FLUID_2D) && par != CUDAPCG_NBN) {
    printf("ERROR: EBE solver is unavailable for FLUID analysis.\n");
    return CUDAPCG_FALSE;
  }
  S = (oracle_solver_t *)calloc(1, sizeof(oracle_solver_t));
  if (!S) return CUDAPCG_FALSE;
  S->analysis = analysis_flag; S->par = par;
  S->dim2 = (analysis_flag == CUDAPCG_THERMAL_2D || analysis_flag == CUDAPCG_ELASTIC_2D || analysis_flag == CUDAPCG_FLUID_2D);
  S->tol = CUDAPCG_TOLERANCE; S->maxit = CUDAPCG_MAX_ITERATIONS;
  S->solver_flag = CUDAPCG_CG_SOLVER; S->precond = 1; S->resnorm = CUDAPCG_L2_NORM;
  S->xr_mode = CUDAPCG_XREDUCE_FULL; S->xr_shift = 0; S->xr_scale = 1.0;  /* cudapcg.cu:154-156 */
  S->residual = 1.0;
  S->header = strdup("");
  if (!model_ctor) model_ctor = ctor_simple;
  return CUDAPCG_TRUE;
}

cudapcgFlag_t cudapcgSetModelConstructorFcn(cudapcgFlag_t (*fcn)(cudapcgModel_t **, const void *)) {
  if (!fcn) return CUDAPCG_FALSE;
  model_ctor = fcn;
  return CUDAPCG_TRUE;
}

static void alloc_model_arrays(void) {
  cudapcgModel_t *m = S->model;
  free(S->r); S->r = (double *)calloc(m->nvars, sizeof(double));
  if (!is_fluid()) {
    if (!m->image) m->image = (cudapcgMap_t *)calloc(m->nelem, sizeof(cudapcgMap_t));
  } else {
    if (!m->periodic2DOF_map) m->periodic2DOF_map = (cudapcgIdMap_t *)calloc(m->nelem, sizeof(cudapcgIdMap_t));
    if (!m->border_pore_map) m->border_pore_map = (cudapcgFlag_t *)calloc(m->nbordernodes + 1, 1);
    if (!m->DOF2periodic_map) m->DOF2periodic_map = (cudapcgIdMap_t *)calloc(m->nporenodes + m->nbordernodes + 1, sizeof(cudapcgIdMap_t));
    if (m->poremap_flag == CUDAPCG_POREMAP_IMG && !m->pore_map) m->pore_map = (cudapcgFlag_t *)calloc(m->nelem, 1);
  }
}

/* Image pore map (CUDAPCG_POREMAP_IMG, femhmg.c:962-965): the host hands over every node's
   fluid key (bit e set when the node's local voxel e is pore) with the node->DOF map, and the
   reference's image kernels walk the nodes with them (matrix_free.cu:4707-4958).  The operator
   is the same; here the DOF->node map and the interface keys are scattered from the two maps
   (node i with a non-zero key and DOF id d is the node of DOF d; an interface DOF d >= nV
   takes the node's key) and the DOF-number restatement runs. */
static void maps_from_pore_image(void) {
  cudapcgModel_t *m = S->model;
  const unsigned int nV = m->nporenodes, nVB = m->nporenodes + m->nbordernodes;
  for (unsigned int i = 0; i < m->nelem; i++) {
    const unsigned int k = m->pore_map[i];
    if (!k) continue;
    const unsigned int d = m->periodic2DOF_map[i];
    if (d >= nVB) continue;
    m->DOF2periodic_map[d] = i;
    if (d >= nV) m->border_pore_map[d - nV] = (cudapcgFlag_t)k;
  }
}

cudapcgFlag_t cudapcgBuildModel(const void *data) {
  if (!S) return CUDAPCG_FALSE;
  if (!S->model) S->model = cudapcgNewModel();
  else if (S->model->freeAllowed_flag) { free_model(S->model); S->model = cudapcgNewModel(); }
  if (!model_ctor(&S->model, data)) return CUDAPCG_FALSE;
  if (is_fluid() && S->model->poremap_flag != CUDAPCG_POREMAP_NUM && S->model->poremap_flag != CUDAPCG_POREMAP_IMG) {
    fprintf(stderr, "oracle: unknown pore map flag\n");
    return CUDAPCG_FALSE;
  }
  free_arrays();
  alloc_model_arrays();
  return CUDAPCG_TRUE;
}

cudapcgFlag_t cudapcgSetModel(cudapcgModel_t *model) {
  if (!S) return CUDAPCG_FALSE;
  if (S->model && S->model->freeAllowed_flag) free_model(S->model);
  S->model = model;
  free_arrays();
  alloc_model_arrays();
  return CUDAPCG_TRUE;
}

cudapcgFlag_t cudapcgSetNumTol(cudapcgTol_t t) { if (!S) return 0; S->tol = t; return 1; }
cudapcgFlag_t cudapcgSetMaxIterations(unsigned int n) { if (!S) return 0; S->maxit = n; return 1; }
/* cudapcg.cu:96-99.  The stabilisation factor only rescales the terms of a sum in the      */
/* reference (xreduce.cu:8-13); the oracle sums in FP64 directly.                          */
cudapcgFlag_t cudapcgSetXReduceMode(cudapcgFlag_t f) { if (!S) return 0; S->xr_mode = f <= CUDAPCG_XREDUCE_FULL ? f : CUDAPCG_XREDUCE_FULL; return 1; }
cudapcgFlag_t cudapcgSetXReduceShift(unsigned int s) { if (!S) return 0; S->xr_shift = s; return 1; }
cudapcgFlag_t cudapcgSetXReduceScale(double s) { if (!S) return 0; S->xr_scale = s; return 1; }
cudapcgFlag_t cudapcgSetReduceStabFactor(double s) { (void)s; return S ? 1 : 0; }
/* cudapcg.cu:597-671: 3-vector variants run the same iterates; the 2-vector variants run the restatements below. */
cudapcgFlag_t cudapcgSetSolver(cudapcgFlag_t flag) {
  if (!S) return 0;
  if (flag > CUDAPCG_MINRES2_SOLVER) { printf("ERROR: Invalid \"solverFlag\" (%d).\n", flag); return 0; }
  S->solver_flag = flag;
  return 1;
}
cudapcgFlag_t cudapcgSetPreconditioner(cudapcgFlag_t flag) { if (!S) return 0; S->precond = flag > 0; return 1; }
cudapcgFlag_t cudapcgSetResNorm(cudapcgFlag_t flag) { if (!S) return 0; S->resnorm = flag > CUDAPCG_ERROR_NORM ? CUDAPCG_L2_NORM : flag; return 1; }
unsigned int cudapcgGetNumIterations(void) { return S ? S->iteration : 0; }
unsigned int cudapcgGetMaxNumIterations(void) { return S ? S->maxit : 0; }
cudapcgVar_t cudapcgGetResidual(void) { return S ? S->residual : 0; }

cudapcgFlag_t cudapcgAllocateArrays(void) {
  if (!S || !S->model) return 0;
  unsigned int n = S->model->nvars;
  if (!S->x) S->x = (double *)calloc(n, sizeof(double));
  if (!S->d) S->d = (double *)calloc(n, sizeof(double));
  if (!S->q) S->q = (double *)calloc(n, sizeof(double));
  if (!S->s) S->s = (double *)calloc(n, sizeof(double));
  if (!g_dinv) g_dinv = (double *)calloc(n, sizeof(double));
  return 1;
}
cudapcgFlag_t cudapcgFreeArrays(void) { if (!S) return 0; free_arrays(); return 1; }

cudapcgFlag_t cudapcgSetRHS(cudapcgVar_t *RHS) {
  if (!S || !S->model) return 0;
  memcpy(S->r, RHS, sizeof(double) * S->model->nvars);
  capture(5, RHS, S->model->nvars);
  return 1;
}

/* setX0_cg (solvers/cg.cu:15-31) */
cudapcgFlag_t cudapcgSetX0(cudapcgVar_t *x0, cudapcgFlag_t mustInterpolate) {
  if (!S || !S->model) return 0;
  cudapcgModel_t *m = S->model;
  if (!x0) {
    if (!S->x0_set) return 1;
    S->x0_set = 0;
    if (S->x) zeros(S->x, m->nvars);
    return 1;
  }
  if (!S->x) S->x = (double *)calloc(m->nvars, sizeof(double));
  if (mustInterpolate) {
    unsigned int nd = m->nvars / m->nelem;
    interpl2(x0, m->nrows, m->ncols, m->nlayers, nd, S->x);
  } else {
    memcpy(S->x, x0, sizeof(double) * m->nvars);
  }
  S->x0_set = 1;
  return 1;
}

cudapcgFlag_t cudapcgSetImage(cudapcgMap_t *img) {
  if (!S || !S->model) return 0;
  cudapcgModel_t *m = S->model;
  memcpy(m->image, img, sizeof(cudapcgMap_t) * m->nelem);
  capture(0, img, m->nelem);
  free(S->keys);
  S->keys = (unsigned short *)malloc(sizeof(unsigned short) * m->nelem);
  if (S->par == CUDAPCG_EBE && S->dim2) keys_from_elements_2d(img, m->nrows, m->ncols, S->keys);
  else if (S->par == CUDAPCG_EBE) keys_from_elements(img, m->nrows, m->ncols, m->nlayers, S->keys);
  else for (unsigned int i = 0; i < m->nelem; i++) S->keys[i] = img[i];
  return 1;
}
/* cudapcg.cu:327-334: the density codes of every voxel and their range; a thermal model has one
   material (femhmg.c:256-262 normalises it), whose key is zero everywhere. */
cudapcgFlag_t cudapcgSetParametricDensityField(parametricScalarField_t *f, double fmin, double fmax) {
  if (!S || !S->model || !f) return 0;
  cudapcgModel_t *m = S->model;
  free(S->sdf);
  S->sdf = (parametricScalarField_t *)malloc(sizeof(parametricScalarField_t) * m->nelem);
  memcpy(S->sdf, f, sizeof(parametricScalarField_t) * m->nelem);
  S->sdf_min = fmin;
  S->sdf_max = fmax;
  if (!S->keys) S->keys = (unsigned short *)calloc(m->nelem, sizeof(unsigned short));
  capture(7, f, m->nelem);
  const double range[2] = {fmin, fmax};
  capture(8, range, 2);
  return 1;
}
cudapcgFlag_t cudapcgSetPoreMap(cudapcgFlag_t *pores) {
  if (!S || !S->model) return 0;
  if (S->model->poremap_flag == CUDAPCG_POREMAP_IMG) {  /* cudapcg.cu:339-341: one key per node */
    memcpy(S->model->pore_map, pores, S->model->nelem);
    capture(3, pores, S->model->nelem);
    return 1;
  }
  memcpy(S->model->border_pore_map, pores, S->model->nbordernodes);
  capture(3, pores, S->model->nbordernodes);
  return 1;
}
cudapcgFlag_t cudapcgSetPeriodic2DOFMap(cudapcgIdMap_t *vars) {
  if (!S || !S->model) return 0;
  memcpy(S->model->periodic2DOF_map, vars, sizeof(cudapcgIdMap_t) * S->model->nelem);
  capture(1, vars, S->model->nelem);
  return 1;
}
cudapcgFlag_t cudapcgSetDOF2PeriodicMap(cudapcgIdMap_t *nodes) {
  if (!S || !S->model) return 0;
  if (S->model->poremap_flag != CUDAPCG_POREMAP_NUM) return 0;  /* cudapcg.cu:360 */
  unsigned int n = S->model->nporenodes + S->model->nbordernodes;
  memcpy(S->model->DOF2periodic_map, nodes, sizeof(cudapcgIdMap_t) * n);
  capture(2, nodes, n);
  return 1;
}
cudapcgFlag_t cudapcgSetLclMtxs(cudapcgVar_t *L) {
  if (!S || !S->model) return 0;
  cudapcgModel_t *m = S->model;
  S->nkeys = m->nkeys;
  capture(4, L, m->nkeys * m->localmtxdim);
  free(S->Kd);
  if (S->analysis == CUDAPCG_FLUID_2D) {  /* one 12 x 12 matrix (femhmg_fluid_2D.c:41-80) */
    S->ed = 12;
    S->Kd = (double *)malloc(sizeof(double) * 144);
    memcpy(S->Kd, L, sizeof(double) * 144);
  } else if (S->analysis == CUDAPCG_THERMAL_2D || S->analysis == CUDAPCG_ELASTIC_2D) {  /* dense 4x4 / 8x8 */
    S->ed = S->analysis == CUDAPCG_THERMAL_2D ? 4 : 8;
    S->Kd = (double *)malloc(sizeof(double) * S->ed * S->ed * m->nkeys);
    memcpy(S->Kd, L, sizeof(double) * S->ed * S->ed * m->nkeys);
  } else if (S->analysis == CUDAPCG_THERMAL_3D) {
    S->ed = 8;
    S->Kd = (double *)malloc(sizeof(double) * 64 * m->nkeys);
    for (unsigned int k = 0; k < m->nkeys; k++) expand_sparseq1(L + 40 * k, S->Kd + 64 * k);
  } else if (S->analysis == CUDAPCG_ELASTIC_3D) {
    S->ed = 24;
    S->Kd = (double *)malloc(sizeof(double) * 576 * m->nkeys);
    memcpy(S->Kd, L, sizeof(double) * 576 * m->nkeys);
  } else {
    S->ed = 32;
    S->Kd = (double *)malloc(sizeof(double) * 1024);
    memcpy(S->Kd, L, sizeof(double) * 1024);
  }
  return 1;
}

/* ------------------------------------------------------------------------------------ */
/* Solvers.                                                                               */
static void report_line(double stop_metric, double delta, double delta0) {
  if (g_quiet) return;
  if (S->resnorm != CUDAPCG_ERROR_NORM) printf("%siteration: %d, residual: %.3e\n", S->header, S->iteration, stop_metric);
  else printf("%siteration: %d, residual: %.3e, error: %.3e\n", S->header, S->iteration, eval_res(delta, delta0), stop_metric);
}
static void finish(double stop_metric, double delta, double delta0, int l2_uses_delta) {
  if (S->resnorm == CUDAPCG_L2_NORM && l2_uses_delta) {
    S->residual = eval_res(delta, delta0);
    S->found = !above_tol(delta, delta0, S->tol);
  } else {
    S->residual = stop_metric;
    S->found = S->residual <= S->tol;
  }
}
static void log_solve(void) { if (log_n < LOG_CAP) { log_it[log_n] = S->iteration; log_res[log_n] = S->residual; log_n++; } }

/* solve_pcg (solvers/pcg.cu:28-243) and solve_cg (solvers/cg.cu:62-260). */
static void solve_cg_family(int pre) {
  cudapcgModel_t *m = S->model;
  const unsigned int n = m->nvars, nstop = m->nhmgvars;
  double *x = S->x, *r = S->r, *d = S->d, *q = S->q, *tmp = S->s;
  if (!S->x0_set) zeros(x, n);
  zeros(q, n);
  double a, delta, delta0, delta_old, stop_metric = 1.0, res0;
  int cont = 1;
  S->iteration = 0;
  hist_n = 0;
  if (pre) { apply_precond(r, NULL, 1.0, 0.0, d); delta0 = dot(r, d, n); }
  else delta0 = dot(r, r, n);
  res0 = (S->resnorm == CUDAPCG_INF_NORM) ? absmax(r, n) : delta0;
  if (fabs(res0) < 1e-12) {
    S->residual = 0.0; S->found = 1;
    if (!g_quiet) printf("%sNull solution satisfied %s.\n", S->header, pre ? "PCG" : "CG");
    return;
  }
  if (S->x0_set) {
    Aprod(x, q);
    axpy_iny(r, q, -1.0, n);
    if (pre) { apply_precond(r, NULL, 1.0, 0.0, d); delta = dot(r, d, n); }
    else delta = dot(r, r, n);
    if (!above_tol(delta, delta0, S->tol)) {
      S->residual = eval_res(delta, delta0); S->found = 1;
      if (!g_quiet) printf("%sInitial guess satisfied %s.\n", S->header, pre ? "PCG" : "CG");
      return;
    }
  } else delta = delta0;
  delta_old = delta;
  hist_push(S->resnorm == CUDAPCG_INF_NORM ? absmax(r, n) / res0 : (S->resnorm == CUDAPCG_L2_NORM ? eval_res(delta, delta0) : 1.0));
  /* first iteration */
  S->iteration++;
  if (!pre) arrcpy(r, n, d);
  Aprod(d, q);
  a = delta / dot(d, q, n);
  axpy_iny(x, d, a, n);
  axpy_iny(r, q, -a, n);
  if (pre) { apply_precond(r, NULL, 1.0, 0.0, q); delta = dot(r, q, n); }
  else delta = dot(r, r, n);
  for (;;) {
    switch (S->resnorm) {
      case CUDAPCG_L2_NORM: stop_metric = eval_res(delta, delta0); cont = above_tol(delta, delta0, S->tol); break;
      case CUDAPCG_INF_NORM: stop_metric = absmax(r, n) / res0; cont = stop_metric > S->tol; break;
      default:
        stop_metric = fabs(a) * absmax(d, nstop) / absmax(x, nstop);
        cont = !((stop_metric <= S->tol) || !above_tol(delta, delta0, S->tol));
    }
    hist_push(stop_metric);
    if (!(cont && S->iteration < S->maxit)) break;
    S->iteration++;
    axpy_to(pre ? q : r, d, delta / delta_old, n, d);
    Aprod(d, q);
    a = delta / dot(d, q, n);
    axpy_iny(x, d, a, n);
    axpy_iny(r, q, -a, n);
    delta_old = delta;
    if (pre) { apply_precond(r, NULL, 1.0, 0.0, q); delta = dot(r, q, n); }
    else delta = dot(r, r, n);
  }
  (void)tmp;
  report_line(stop_metric, delta, delta0);
  finish(stop_metric, delta, delta0, 1);
}

/* solve_pminres (solvers/pminres.cu:28-247): preconditioned conjugate residual. */
static void solve_pminres(void) {
  cudapcgModel_t *m = S->model;
  const unsigned int n = m->nvars, nstop = m->nhmgvars;
  double *x = S->x, *r = S->r, *d = S->d, *q = S->q, *s = S->s;
  double *tmp = (double *)malloc(sizeof(double) * n);
  if (!S->x0_set) zeros(x, n);
  zeros(q, n);
  double a, b, delta, delta0, delta_old, stop_metric = 1.0, res0;
  int cont = 1;
  S->iteration = 0;
  hist_n = 0;
  res0 = (S->resnorm == CUDAPCG_INF_NORM) ? absmax(r, n) : dot_precond(r, 1.0);
  apply_precond(r, NULL, 1.0, 0.0, q);
  Aprod_scl(q, 1.0, 0.0, s, tmp);
  delta0 = dot(q, s, n);
  if (fabs(res0) < 1e-12) {
    S->residual = 0.0; S->found = 1; zeros(x, n);
    if (!g_quiet) printf("%sNull solution satisfied MINRES.\n", S->header);
    free(tmp); return;
  }
  if (S->x0_set) {
    Aprod_scl(x, -1.0, 1.0, r, tmp);
    apply_precond(r, NULL, 1.0, 0.0, q);
    Aprod_scl(q, 1.0, 0.0, s, tmp);
    delta = dot(q, s, n);
    if (!above_tol(delta, delta0, S->tol)) {
      S->residual = eval_res(delta, delta0); S->found = 1;
      if (!g_quiet) printf("%sInitial guess satisfied MINRES.\n", S->header);
      free(tmp); return;
    }
  } else delta = delta0;
  delta_old = delta;
  hist_push(1.0);
  S->iteration++;
  arrcpy(q, n, d);
  arrcpy(s, n, q);
  a = delta / dot_precond(q, 1.0);
  axpy_iny(x, d, a, n);
  axpy_iny(r, q, -a, n);
  apply_precond(r, NULL, 1.0, 0.0, r);
  Aprod_scl(r, 1.0, 0.0, s, tmp);
  delta_old = delta;
  delta = dot(r, s, n);
  apply_invprecond(r, 1.0, r);
  for (;;) {
    switch (S->resnorm) {
      case CUDAPCG_L2_NORM:
        stop_metric = dot_precond(r, 1.0);
        cont = above_tol(stop_metric, res0, S->tol);
        stop_metric = eval_res(stop_metric, res0);
        break;
      case CUDAPCG_INF_NORM: stop_metric = absmax(r, n) / res0; cont = stop_metric > S->tol; break;
      default: stop_metric = fabs(a) * absmax(d, nstop) / absmax(x, nstop); cont = stop_metric > S->tol;
    }
    hist_push(stop_metric);
    if (!(cont && S->iteration < S->maxit)) break;
    S->iteration++;
    b = delta / delta_old;
    apply_precond(r, d, 1.0, b, d);
    axpy_to(s, q, b, n, q);
    a = delta / dot_precond(q, 1.0);
    axpy_iny(x, d, a, n);
    axpy_iny(r, q, -a, n);
    apply_precond(r, NULL, 1.0, 0.0, r);
    Aprod_scl(r, 1.0, 0.0, s, tmp);
    delta_old = delta;
    delta = dot(r, s, n);
    apply_invprecond(r, 1.0, r);
  }
  report_line(stop_metric, delta, delta0);
  S->residual = stop_metric;
  S->found = S->residual <= S->tol;
  free(tmp);
}

/* solve_minres (solvers/minres.cu:58-260): unpreconditioned conjugate residual. */
static void solve_minres(void) {
  cudapcgModel_t *m = S->model;
  const unsigned int n = m->nvars, nstop = m->nhmgvars;
  double *x = S->x, *r = S->r, *d = S->d, *q = S->q, *s = S->s;
  double *tmp = (double *)malloc(sizeof(double) * n);
  if (!S->x0_set) zeros(x, n);
  zeros(q, n);
  double a, b, delta, delta0, delta_old, stop_metric = 1.0, res0;
  int cont = 1;
  S->iteration = 0;
  hist_n = 0;
  Aprod_scl(r, 1.0, 0.0, s, tmp);
  delta0 = dot(r, s, n);
  res0 = (S->resnorm == CUDAPCG_INF_NORM) ? absmax(r, n) : dot(r, r, n);
  if (fabs(res0) < 1e-12) {
    S->residual = 0.0; S->found = 1; zeros(x, n);
    if (!g_quiet) printf("%sNull solution satisfied MINRES.\n", S->header);
    free(tmp); return;
  }
  if (S->x0_set) {
    Aprod_scl(x, -1.0, 1.0, r, tmp);
    Aprod_scl(r, 1.0, 0.0, s, tmp);
    delta = dot(r, s, n);
    if (!above_tol(delta, delta0, S->tol)) {
      S->residual = eval_res(delta, delta0); S->found = 1;
      if (!g_quiet) printf("%sInitial guess satisfied MINRES.\n", S->header);
      free(tmp); return;
    }
  } else delta = delta0;
  delta_old = delta;
  hist_push(1.0);
  S->iteration++;
  arrcpy(r, n, d);
  arrcpy(s, n, q);
  a = delta / dot(q, q, n);
  axpy_iny(x, d, a, n);
  axpy_iny(r, q, -a, n);
  Aprod_scl(r, 1.0, 0.0, s, tmp);
  delta = dot(r, s, n);
  for (;;) {
    switch (S->resnorm) {
      case CUDAPCG_L2_NORM:
        stop_metric = dot(r, r, n);
        cont = above_tol(stop_metric, res0, S->tol);
        stop_metric = eval_res(stop_metric, res0);
        break;
      case CUDAPCG_INF_NORM: stop_metric = absmax(r, n) / res0; cont = stop_metric > S->tol; break;
      default: stop_metric = fabs(a) * absmax(d, nstop) / absmax(x, nstop); cont = stop_metric > S->tol;
    }
    hist_push(stop_metric);
    if (!(cont && S->iteration < S->maxit)) break;
    S->iteration++;
    b = delta / delta_old;
    axpy_to(s, q, b, n, q);
    axpy_to(r, d, b, n, d);
    a = delta / dot(q, q, n);
    axpy_iny(x, d, a, n);
    axpy_iny(r, q, -a, n);
    Aprod_scl(r, 1.0, 0.0, s, tmp);
    delta_old = delta;
    delta = dot(r, s, n);
  }
  report_line(stop_metric, delta, delta0);
  S->residual = stop_metric;
  S->found = S->residual <= S->tol;
  free(tmp);
}

/* ------------------------------------------------------------------------------------ */
/* 2-vector solvers (solvers/cg2.cu, pcg2.cu, minres2.cu, pminres2.cu): only r and d are   */
/* kept; the solution is never stored, only reduced on the fly into the per-component sums */
/* of its velocity part (xreduce.cu:4-27), which are the effective-permeability column.    */
/*   NONE    res[c][it] = a * sum_j d[Dj+c]   (the sums are accumulated at the end)        */
/*   ONLYDIR x[j] += a d[Dj+shift];  res[shift][it] = sum_j x[j]                           */
/*   FULL    x[i] += a d[i] (velocity DOFs);  res[c][it] = sum_j x[Dj+c]                    */
/* with D = nvarspernode = 3 velocities per node, 2 on a 2D image (femhmg.c:75, :82).       */
typedef struct {
  double *res[3];
  double *xa;          /* reduction accumulator (ONLYDIR: nV values, FULL: D nV, NONE: none) */
  unsigned int nv;     /* velocity nodes */
  unsigned int D;      /* velocity components per node */
} xred_t;

static double sum_stride(const double *v, unsigned int nv, unsigned int stride, unsigned int c) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long j = 0; j < (long)nv; j++) s += v[(size_t)j * stride + c];
  return s;
}
static void xred_update(xred_t *X, unsigned int it, double a, const double *d) {
  const unsigned int nv = X->nv;
  switch (S->xr_mode) {
    case CUDAPCG_XREDUCE_NONE:
      for (unsigned int c = 0; c < X->D; c++) X->res[c][it] = a * sum_stride(d, nv, X->D, c);
      break;
    case CUDAPCG_XREDUCE_ONLYDIR:
#pragma omp parallel for schedule(static)
      for (long j = 0; j < (long)nv; j++) X->xa[j] += a * d[X->D * (size_t)j + S->xr_shift];
      X->res[S->xr_shift][it] = sum_stride(X->xa, nv, 1, 0);
      break;
    default:
      axpy_iny(X->xa, d, a, X->D * nv);
      for (unsigned int c = 0; c < X->D; c++) X->res[c][it] = sum_stride(X->xa, nv, X->D, c);
  }
}
/* the x0 stored in d enters the accumulator and the first sums (cg2.cu:131-146) */
static void xred_x0(xred_t *X, const double *d) {
  const unsigned int nv = X->nv;
  if (S->xr_mode == CUDAPCG_XREDUCE_ONLYDIR) {
#pragma omp parallel for schedule(static)
    for (long j = 0; j < (long)nv; j++) X->xa[j] += d[X->D * (size_t)j + S->xr_shift];
  } else if (S->xr_mode == CUDAPCG_XREDUCE_FULL) {
    memcpy(X->xa, d, sizeof(double) * X->D * nv);
  }
  for (unsigned int c = 0; c < X->D; c++) X->res[c][0] = sum_stride(d, nv, X->D, c);
}
/* the largest |x| the solver holds, for the error norm of CG2/PCG2 (cg2.cu:181); without */
/* an accumulator (NONE) the denominator is 1, as in (P)MINRES2                            */
static double xred_absmax(const xred_t *X) {
  if (S->xr_mode == CUDAPCG_XREDUCE_NONE) return 1.0;
  return absmax(X->xa, S->xr_mode == CUDAPCG_XREDUCE_ONLYDIR ? X->nv : X->D * X->nv);
}
/* save_xreduce (xreduce.cu:29-48) and the result (pcg2.cu:262-280) */
static void xred_finish(xred_t *X, unsigned int it, double *res_x) {
  const double scl = S->xr_scale;
  for (unsigned int c = 0; c < X->D; c++)
    for (unsigned int j = 0; j <= it; j++) X->res[c][j] *= scl;
  char fn[2048];
  snprintf(fn, sizeof fn, "%s_xreduce_metrics_%lu.bin", S->model->name ? S->model->name : "", S->count);
  FILE *f = fopen(fn, "wb");
  if (f) {
    if (S->xr_mode != CUDAPCG_XREDUCE_ONLYDIR) for (unsigned int c = 0; c < X->D; c++) fwrite(X->res[c], sizeof(double), it + 1, f);
    else fwrite(X->res[S->xr_shift], sizeof(double), it + 1, f);
    fclose(f);
  }
  for (unsigned int c = 0; c < X->D; c++) {
    double *p = X->res[c];
    switch (S->xr_mode) {
      case CUDAPCG_XREDUCE_NONE:
        for (unsigned int j = it; j > 0; j--) p[j - 1] += p[j];
        res_x[c] = p[0];
        break;
      case CUDAPCG_XREDUCE_ONLYDIR: res_x[c] = S->xr_shift == c ? p[it] : 0.0; break;
      default: res_x[c] = p[it];
    }
  }
}

/* solve_pcg2 (pcg2.cu:24-290) / solve_cg2 (cg2.cu:62-320) */
static void solve_cg2_family(int pre, xred_t *X, double *res_x) {
  cudapcgModel_t *m = S->model;
  const unsigned int n = m->nvars, nstop = m->nhmgvars;
  double *r = S->r, *d = S->d, *q = S->q;
  double a = 0.0, delta, delta0, delta_old, stop_metric = 1.0, res0;
  int cont = 1;
  S->iteration = 0;
  hist_n = 0;
  if (pre) { apply_precond(r, NULL, 1.0, 0.0, q); delta0 = dot(r, q, n); }
  else delta0 = dot(r, r, n);
  res0 = (S->resnorm == CUDAPCG_INF_NORM) ? absmax(r, n) : delta0;
  if (fabs(res0) < 1e-12) {
    S->residual = 0.0; S->found = 1;
    if (!g_quiet) printf("%sNull solution satisfied %s.\n", S->header, pre ? "PCG" : "CG");
    return;
  }
  if (S->x0_set) {
    Aprod_scl(d, -1.0, 1.0, r, q);
    if (pre) { apply_precond(r, NULL, 1.0, 0.0, q); delta = dot(r, q, n); }
    else delta = dot(r, r, n);
    xred_x0(X, d);
    if (!above_tol(delta, delta0, S->tol)) {
      S->residual = eval_res(delta, delta0); S->found = 1;
      if (!g_quiet) printf("%sInitial guess satisfied %s.\n", S->header, pre ? "PCG" : "CG");
      return;
    }
  } else delta = delta0;
  delta_old = delta;
  for (;;) {
    S->iteration++;
    if (S->iteration == 1) { if (pre) apply_precond(r, NULL, 1.0, 0.0, d); else arrcpy(r, n, d); }
    else if (pre) apply_precond(r, d, 1.0, delta / delta_old, d);
    else axpy_to(r, d, delta / delta_old, n, d);
    Aprod(d, q);
    a = delta / dot(d, q, n);
    xred_update(X, S->iteration, a, d);
    axpy_iny(r, q, -a, n);
    delta_old = delta;
    if (pre) { apply_precond(r, NULL, 1.0, 0.0, q); delta = dot(r, q, n); }
    else delta = dot(r, r, n);
    switch (S->resnorm) {
      case CUDAPCG_L2_NORM: stop_metric = eval_res(delta, delta0); cont = above_tol(delta, delta0, S->tol); break;
      case CUDAPCG_INF_NORM: stop_metric = absmax(r, n) / res0; cont = stop_metric > S->tol; break;
      default:
        stop_metric = fabs(a) * absmax(d, nstop) / xred_absmax(X);
        cont = !((stop_metric <= S->tol) || !above_tol(delta, delta0, S->tol));
    }
    hist_push(stop_metric);
    if (!(cont && S->iteration < S->maxit)) break;
  }
  report_line(stop_metric, delta, delta0);
  finish(stop_metric, delta, delta0, 1);
  xred_finish(X, S->iteration, res_x);
}

/* solve_pminres2 (pminres2.cu:20-278) / solve_minres2 (minres2.cu:62-320): preconditioned   */
/* conjugate residual with r and d only (A d is applied twice per iteration, A M^-1 r once). */
static void solve_minres2_family(int pre, xred_t *X, double *res_x) {
  cudapcgModel_t *m = S->model;
  const unsigned int n = m->nvars, nstop = m->nhmgvars;
  double *r = S->r, *d = S->d, *q = S->q, *t = S->s;
  double a = 0.0, b, delta, delta0, delta_old, stop_metric = 1.0, res0;
  int cont = 1;
  S->iteration = 0;
  hist_n = 0;
  if (S->resnorm == CUDAPCG_INF_NORM) res0 = absmax(r, n);
  else res0 = pre ? dot_precond(r, 1.0) : dot(r, r, n);
  if (pre) apply_precond(r, NULL, 1.0, 0.0, r);
  Aprod(r, q);
  delta0 = dot(r, q, n);
  if (pre) apply_invprecond(r, 1.0, r);
  if (fabs(res0) < 1e-12) {
    S->residual = 0.0; S->found = 1;
    if (!g_quiet) printf("%sNull solution satisfied MINRES.\n", S->header);
    return;
  }
  if (S->x0_set) {
    Aprod_scl(d, -1.0, 1.0, r, q);
    if (pre) apply_precond(r, NULL, 1.0, 0.0, r);
    Aprod(r, q);
    delta = dot(r, q, n);
    if (pre) apply_invprecond(r, 1.0, r);
    xred_x0(X, d);
    if (!above_tol(delta, delta0, S->tol)) {
      S->residual = eval_res(delta, delta0); S->found = 1;
      if (!g_quiet) printf("%sInitial guess satisfied MINRES.\n", S->header);
      return;
    }
  } else delta = delta0;
  delta_old = delta;
  for (;;) {
    S->iteration++;
    b = S->iteration == 1 ? 0.0 : delta / delta_old;
    if (pre) apply_precond(r, S->iteration == 1 ? NULL : d, 1.0, b, d);
    else if (S->iteration == 1) arrcpy(r, n, d);
    else axpy_to(r, d, b, n, d);
    Aprod(d, q);
    if (pre) { apply_precond(q, NULL, 1.0, 0.0, t); a = delta / dot(q, t, n); }
    else a = delta / dot(q, q, n);
    xred_update(X, S->iteration, a, d);
    axpy_iny(r, q, -a, n);
    if (pre) apply_precond(r, NULL, 1.0, 0.0, r);
    Aprod(r, q);
    delta_old = delta;
    delta = dot(r, q, n);
    if (pre) apply_invprecond(r, 1.0, r);
    switch (S->resnorm) {
      case CUDAPCG_L2_NORM:
        stop_metric = pre ? dot_precond(r, 1.0) : dot(r, r, n);
        cont = above_tol(stop_metric, res0, S->tol);
        stop_metric = eval_res(stop_metric, res0);
        break;
      case CUDAPCG_INF_NORM: stop_metric = absmax(r, n) / res0; cont = stop_metric > S->tol; break;
      default: stop_metric = fabs(a) * absmax(d, nstop); cont = stop_metric > S->tol;
    }
    hist_push(stop_metric);
    if (!(cont && S->iteration < S->maxit)) break;
  }
  report_line(stop_metric, delta, delta0);
  S->residual = stop_metric;
  S->found = S->residual <= S->tol;
  xred_finish(X, S->iteration, res_x);
}

static void solve_two_vector(double *res_x) {
  cudapcgModel_t *m = S->model;
  xred_t X;
  X.nv = m->nporenodes;
  X.D = S->analysis == CUDAPCG_FLUID_2D ? 2 : 3;
  double *buf = (double *)calloc((size_t)3 * (S->maxit + 1), sizeof(double));
  for (int c = 0; c < 3; c++) X.res[c] = buf + (size_t)c * (S->maxit + 1);
  X.xa = (S->xr_mode == CUDAPCG_XREDUCE_NONE) ? NULL
       : (double *)calloc(S->xr_mode == CUDAPCG_XREDUCE_ONLYDIR ? X.nv : X.D * (size_t)X.nv, sizeof(double));
  /* the x0 lives in d (cudapcg.cu:302) */
  if (S->x0_set) memcpy(S->d, S->x, sizeof(double) * m->nvars);
  for (unsigned int c = 0; c < X.D; c++) res_x[c] = 0.0;
  const int minres = S->solver_flag == CUDAPCG_MINRES2_SOLVER;
  if (minres) solve_minres2_family(S->precond, &X, res_x);
  else solve_cg2_family(S->precond, &X, res_x);
  free(X.xa);
  free(buf);
}

/* cudapcgSolve (cudapcg.cu:389-409). */
cudapcgFlag_t cudapcgSolve(cudapcgVar_t *res_x) {
  if (!S || !S->model || !res_x) return 0;
  double t0 = omp_get_wtime();
  int must_free = (S->d == NULL);
  cudapcgAllocateArrays();
  if (is_fluid() && S->model->poremap_flag == CUDAPCG_POREMAP_IMG) maps_from_pore_image();
  inv_diag(g_dinv);
  S->found = 0;
  S->count++;
  if (S->solver_flag >= CUDAPCG_CG2_SOLVER) {
    if (!is_fluid()) {
      printf("ERROR: the 2-vector solvers are restated for Stokes; use CG3/MINRES3.\n");
      if (must_free) free_arrays();
      return 0;
    }
    solve_two_vector(res_x);
    capture(6, res_x, S->analysis == CUDAPCG_FLUID_2D ? 2 : 3);
  } else {
    int minres = (S->solver_flag == CUDAPCG_MINRES_SOLVER || S->solver_flag == CUDAPCG_MINRES3_SOLVER);
    if (minres) { if (S->precond) solve_pminres(); else solve_minres(); }
    else solve_cg_family(S->precond);
    memcpy(res_x, S->x, sizeof(double) * S->model->nvars);
    capture(6, S->x, S->model->nvars);
  }
  S->total_time = omp_get_wtime() - t0;
  S->mean_time = S->iteration ? S->total_time / S->iteration : 0.0;
  log_solve();
  if (must_free) free_arrays();
  return (cudapcgFlag_t)S->found;
}

cudapcgFlag_t cudapcgSetHeaderString(char *header) {
  if (!S) return 0;
  free(S->header);
  S->header = strdup(header ? header : "");
  return 1;
}
cudapcgFlag_t cudapcgPrintSolverMetrics(void) {
  if (!S) return 0;
  if (!g_quiet) {
    printf("%sMean time per iteration: %.2e s\n", S->header, S->mean_time);
    printf("%sElapsed time: %.2e s\n", S->header, S->total_time);
  }
  return 1;
}
cudapcgFlag_t cudapcgPrintSolverMetrics2(char *dest) {
  if (!dest || !S) return 0;
  sprintf(dest, "%sMean time per iteration: %.2e s\n%sElapsed time: %.2e s\n", S->header, S->mean_time, S->header, S->total_time);
  return 1;
}
cudapcgFlag_t cudapcgPrintSolverReport(void) {
  if (!S) return 0;
  if (!g_quiet) {
    if (S->found) printf("%sPCG solver found a solution in %d iterations.\n", S->header, S->iteration);
    else printf("%sPCG solver did not converge within provided max number of iterations (%d).\n", S->header, S->maxit);
    printf("%sResidual: %e\n", S->header, S->residual);
  }
  return cudapcgPrintSolverMetrics();
}
cudapcgFlag_t cudapcgPrintSolverReport2(char *dest) {
  if (!dest || !S) return 0;
  sprintf(dest, "%sPCG solver ran through %d iterations.\n%sResidual: %e\n%sMean time per iteration: %.2e s\n%sElapsed time: %.2e s\n",
          S->header, S->iteration, S->header, S->residual, S->header, S->mean_time, S->header, S->total_time);
  return 1;
}

/* ------------------------------------------------------------------------------------ */
/* Oracle-only entry points.                                                              */
int oracle_apply(const double *x, double *y) {
  if (!S || !S->model || !S->Kd) return 0;
  if (!is_fluid() && !S->keys) return 0;
  Aprod(x, y);
  return 1;
}
int oracle_precond(const double *x, double *y) {
  if (!S || !S->model || !S->Kd) return 0;
  double *dinv = (double *)malloc(sizeof(double) * S->model->nvars);
  double *save = g_dinv;
  g_dinv = dinv;
  inv_diag(dinv);
  apply_precond(x, NULL, 1.0, 0.0, y);
  g_dinv = save;
  free(dinv);
  return 1;
}
unsigned int oracle_nvars(void) { return (S && S->model) ? S->model->nvars : 0; }
unsigned int oracle_captured_count(int which) { return (which >= 0 && which < CAP_SLOTS) ? cap_n[which] : 0; }
int oracle_copy_captured(int which, void *dst, unsigned int bytes) {
  if (which < 0 || which >= CAP_SLOTS || !cap_ptr[which]) return 0;
  size_t have = (size_t)cap_n[which] * cap_elsz[which];
  memcpy(dst, cap_ptr[which], bytes < have ? bytes : have);
  return 1;
}
unsigned int oracle_history(double *dst, unsigned int n) {
  if (dst) memcpy(dst, hist, sizeof(double) * (n < hist_n ? n : hist_n));
  return hist_n;
}
unsigned int oracle_solve_log(unsigned int *iters, double *residuals, unsigned int n) {
  unsigned int k = n < log_n ? n : log_n;
  if (iters) memcpy(iters, log_it, sizeof(unsigned int) * k);
  if (residuals) memcpy(residuals, log_res, sizeof(double) * k);
  return log_n;
}
void oracle_reset_log(void) { log_n = 0; }
void oracle_set_quiet(int quiet) { g_quiet = quiet; }
