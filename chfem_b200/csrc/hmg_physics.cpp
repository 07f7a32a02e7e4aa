// hmg_physics.cpp -- physics of the chfem_b200 host layer: node keys and pore maps, element
// matrices, right-hand sides and effective-tensor updates (3D; 2D thermal and elastic at the end).
//
// Reference behaviour followed (chfem/src/femhmg/physical_phenomena/):
//   node keys ................. femhmg_3D.c:19-75
//   Stokes fluid keys, DOF ids  femhmg_fluid_3D.c:370-491 (pore nodes first, then interface
//                               nodes, each in ascending node order)
//   element matrices .......... femhmg_thermal_3D.c:42-120, femhmg_elastic_3D.c:51-128,
//                               femhmg_fluid_3D.c:41-110
//   right-hand sides .......... femhmg_thermal_3D.c:122-236, femhmg_elastic_3D.c:130-511,
//                               femhmg_fluid_3D.c:112-182
//   effective tensor .......... femhmg_thermal_3D.c:355-500, femhmg_elastic_3D.c:1075-1343,
//                               femhmg_fluid_3D.c:184-285
// The reference hard-codes the element matrices as closed-form tables and writes each load
// case as its own loop.  Here the matrices are integrated from the trilinear shape functions
// with 2x2x2 Gauss quadrature (exact for these integrands), and every load case is the same
// generic statement: a unit macroscopic gradient/strain enters as a jump of one field
// component across the periodic +face of the cell, RHS = -K_e * jump on the voxels whose
// +face lies on that boundary, and the tensor column is the volume average of
// (flux or stress matrix) * (x + jump).
#include "hmg.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <omp.h>

namespace chfem_host {

static inline int drow(int k) { return -((k & 3) >> 1); }
static inline int dcol(int k) { return ((k & 3) == 1 || (k & 3) == 2) ? 1 : 0; }
static inline int dlay(int k) { return k >> 2; }
// Local node coordinates in the unit cube: x = +col, y = -row, z = -layer.  The reference's
// Stokes element matrix (femhmg_fluid_3D.c:57-91) is written with z = +layer instead (its
// u_x-u_z couplings have the opposite sign to a z = -layer derivation); `zflip` selects that.
static inline int nxi(int k) { return dcol(k); }
static inline int neta(int k) { return -drow(k); }
static inline int nzeta(int k, bool zflip) { return zflip ? dlay(k) : 1 - dlay(k); }
static inline bool shares_edge(int a, int b) {
  return ((drow(a) != drow(b)) + (dcol(a) != dcol(b)) + (dlay(a) != dlay(b))) == 1;
}
static inline long wrapl(long v, long n) { v %= n; return v < 0 ? v + n : v; }

// Node of local node k of voxel (r,c,l).
static inline long elem_node(long r, long c, long l, int k, long R, long C, long L) {
  return wrapl(r + 1 + drow(k), R) + wrapl(c + dcol(k), C) * R + wrapl(l + dlay(k), L) * R * C;
}
// Voxel in which node (r,c,l) is local node e.
static inline long node_elem(long r, long c, long l, int e, long R, long C, long L) {
  return wrapl(r - drow(e) - 1, R) + wrapl(c - dcol(e), C) * R + wrapl(l - dlay(e), L) * R * C;
}

// ---- shape functions and 2-point Gauss quadrature on [0,1]^3 --------------------------
struct QP { double p[3]; double w; };
static void gauss(QP* q) {
  const double g[2] = {0.5 - 0.5 / std::sqrt(3.0), 0.5 + 0.5 / std::sqrt(3.0)};
  int n = 0;
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) { q[n].p[0] = g[i]; q[n].p[1] = g[j]; q[n].p[2] = g[k]; q[n].w = 0.125; n++; }
}
static inline double f1(int node_at_one, double t) { return node_at_one ? t : 1.0 - t; }
static inline double df1(int node_at_one) { return node_at_one ? 1.0 : -1.0; }
static void shape(int a, const double* p, double& phi, double* grad, bool zflip) {
  const int cx = nxi(a), cy = neta(a), cz = nzeta(a, zflip);
  const double fx = f1(cx, p[0]), fy = f1(cy, p[1]), fz = f1(cz, p[2]);
  phi = fx * fy * fz;
  grad[0] = df1(cx) * fy * fz;
  grad[1] = fx * df1(cy) * fz;
  grad[2] = fx * fy * df1(cz);
}

// ---- maps -----------------------------------------------------------------------------
// Stokes: the fluid key of every node (bit e: the voxel in which the node is local node e is
// pore, material index 0), the pore voxels, and the counts of pore nodes (key 255) and
// interface nodes (0 < key < 255) -- the sizes of the DOF numbering (femhmg_fluid_3D.c:370-424),
// which itself runs in build_maps or on the device (cudapcgB200SetPoreImageColors).
static bool count_pore_nodes_2d(Model& m, std::string& err);
bool count_pore_nodes(Model& m, std::string& err) {
  if (m.dim2) return count_pore_nodes_2d(m, err);
  const long R = m.ny, C = m.nx, L = m.nz, N = m.N;
  m.fluid_keys.assign(N, 0);
  long pores = 0, nv = 0, nb = 0;
#pragma omp parallel for reduction(+ : pores, nv, nb) schedule(static)
  for (long i = 0; i < N; i++) {
    const long r = i % R, c = (i / R) % C, l = i / (R * C);
    unsigned k = 0;
    for (int e = 0; e < 8; e++) k |= (unsigned)(m.elem_mat[node_elem(r, c, l, e, R, C, L)] == 0) << e;
    m.fluid_keys[i] = (uint8_t)k;
    pores += (m.elem_mat[i] == 0);
    nv += (k == 255);
    nb += (k != 0 && k != 255);
  }
  m.nporeelem = pores;
  if (nv + nb >= (long)0xffffffffL || 4 * nv + nb >= (long)0xffffffffL) { err = "too many Stokes unknowns for 32-bit DOF ids"; return false; }
  m.nV = nv;
  m.nB = nb;
  m.ndof = 4 * nv + nb;
  return true;
}

static bool build_maps_2d(Model& m, std::string& err);
static void build_local_matrices_2d(Model& m);
static void assemble_rhs_2d(const Model& m, int dir, double* rhs);
static void update_C_2d(Model& m, int dir, const double* x);
static void assemble_rhs_thermal_expansion_2d(const Model& m, double* rhs);

bool build_maps(Model& m, std::string& err) {
  if (m.dim2) return build_maps_2d(m, err);
  const long R = m.ny, C = m.nx, L = m.nz, N = m.N;
  if (m.analysis != FLUID) {
    if (m.nmat > 4) { err = "more than 4 materials cannot be encoded in 16-bit node keys"; return false; }
    m.keys.assign(N, 0);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; i++) {
      const long r = i % R, c = (i / R) % C, l = i / (R * C);
      unsigned k = 0;
      for (int e = 0; e < 8; e++) k |= ((unsigned)m.elem_mat[node_elem(r, c, l, e, R, C, L)] & 3u) << (2 * e);
      m.keys[i] = (uint16_t)k;
    }
    m.ndof = N * m.nd;
    return true;
  }
  if (!count_pore_nodes(m, err)) return false;
  m.dof_of_node.assign(N, 0);
  long id = 0;
  for (long i = 0; i < N; i++)
    if (m.fluid_keys[i] == 255) m.dof_of_node[i] = (uint32_t)id++;
  m.nV = id;
  for (long i = 0; i < N; i++)
    if (m.fluid_keys[i] != 255 && m.fluid_keys[i] != 0) m.dof_of_node[i] = (uint32_t)id++;
  m.nB = id - m.nV;
  if (id >= (long)0xffffffffL) { err = "too many Stokes unknowns for 32-bit DOF ids"; return false; }
  m.node_of_dof.assign(m.nV + m.nB, 0);
  m.border_keys.assign(m.nB, 0);
  for (long i = 0; i < N; i++) {
    const uint8_t k = m.fluid_keys[i];
    if (!k) continue;
    const uint32_t d = m.dof_of_node[i];
    m.node_of_dof[d] = (uint32_t)i;
    if (k != 255) m.border_keys[d - m.nV] = k;
  }
  m.ndof = 4 * m.nV + m.nB;
  return true;
}

// ---- element matrices -------------------------------------------------------------------
void build_local_matrices(Model& m) {
  if (m.dim2) { build_local_matrices_2d(m); return; }
  QP q[8];
  gauss(q);
  double phi[8][8], grad[8][8][3];  // [qp][node]
  for (int g = 0; g < 8; g++)
    for (int a = 0; a < 8; a++) shape(a, q[g].p, phi[g][a], grad[g][a], m.analysis == FLUID);
  // integrals of products
  double KL[8][8] = {{0}}, GI[8][3] = {{0}}, PI[8] = {0}, DD[8][8][3][3] = {{{{0}}}}, GP[8][3][8] = {{{0}}};
  for (int g = 0; g < 8; g++)
    for (int a = 0; a < 8; a++) {
      PI[a] += q[g].w * phi[g][a];
      for (int i = 0; i < 3; i++) GI[a][i] += q[g].w * grad[g][a][i];
      for (int b = 0; b < 8; b++) {
        for (int i = 0; i < 3; i++) {
          KL[a][b] += q[g].w * grad[g][a][i] * grad[g][b][i];
          GP[a][i][b] += q[g].w * grad[g][a][i] * phi[g][b];
          for (int j = 0; j < 3; j++) DD[a][b][i][j] += q[g].w * grad[g][a][i] * grad[g][b][j];
        }
      }
    }
  if (m.analysis == THERMAL) {
    m.lcl.assign(40 * m.nmat, 0.0);
    m.Kdense.assign(64 * m.nmat, 0.0);
    m.CB.assign(24 * m.nmat, 0.0);  // [mat][stress s][node a]
    for (unsigned k = 0; k < m.nmat; k++) {
      const double kp = m.props[k];
      int p = 0;
      for (int a = 0; a < 8; a++)
        for (int b = 0; b < 8; b++) {
          const double v = kp * KL[a][b];
          m.Kdense[64 * k + 8 * a + b] = shares_edge(a, b) ? 0.0 : v;
          if (!shares_edge(a, b)) m.lcl[40 * k + p++] = v;
        }
      for (int s = 0; s < 3; s++)
        for (int a = 0; a < 8; a++) m.CB[24 * k + 8 * s + a] = kp * GI[a][s];
    }
  } else if (m.analysis == ELASTIC) {
    m.lcl.assign(576 * m.nmat, 0.0);
    m.CB.assign(144 * m.nmat, 0.0);
    for (unsigned k = 0; k < m.nmat; k++) {
      const double E = m.props[2 * k], nu = m.props[2 * k + 1];
      const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = E / (2.0 * (1.0 + nu));
      double D[6][6] = {{0}};
      for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) D[i][j] = lam;
        D[i][i] = lam + 2.0 * mu;
        D[3 + i][3 + i] = mu;
      }
      // B rows (Voigt: xx, yy, zz, yz, xz, xy) at each quadrature point
      double Kel[24][24] = {{0}}, Bav[6][24] = {{0}};
      for (int g = 0; g < 8; g++) {
        double B[6][24] = {{0}};
        for (int a = 0; a < 8; a++) {
          const double* dg = grad[g][a];
          B[0][3 * a + 0] = dg[0];
          B[1][3 * a + 1] = dg[1];
          B[2][3 * a + 2] = dg[2];
          B[3][3 * a + 1] = dg[2]; B[3][3 * a + 2] = dg[1];
          B[4][3 * a + 0] = dg[2]; B[4][3 * a + 2] = dg[0];
          B[5][3 * a + 0] = dg[1]; B[5][3 * a + 1] = dg[0];
        }
        double DB[6][24] = {{0}};
        for (int s = 0; s < 6; s++)
          for (int c = 0; c < 24; c++) {
            double t = 0.0;
            for (int u = 0; u < 6; u++) t += D[s][u] * B[u][c];
            DB[s][c] = t;
          }
        for (int r = 0; r < 24; r++)
          for (int c = 0; c < 24; c++) {
            double t = 0.0;
            for (int s = 0; s < 6; s++) t += B[s][r] * DB[s][c];
            Kel[r][c] += q[g].w * t;
          }
        for (int s = 0; s < 6; s++)
          for (int c = 0; c < 24; c++) Bav[s][c] += q[g].w * DB[s][c];
      }
      for (int r = 0; r < 24; r++)
        for (int c = 0; c < 24; c++) m.lcl[576 * k + 24 * r + c] = Kel[r][c];
      for (int s = 0; s < 6; s++)
        for (int c = 0; c < 24; c++) m.CB[144 * k + 24 * s + c] = Bav[s][c];
    }
    m.Kdense = m.lcl;
  } else {
    // Stokes, unit voxel, mu = 1: [K G; G^T Stab], K = int(grad u : grad v + grad u^T : grad v),
    // G = int(d_i phi_a psi_b), Stab = (1/6) * Q1 Laplacian (the pressure stabilisation
    // of femhmg_fluid_3D.c:44-45).
    m.lcl.assign(1024, 0.0);
    for (int a = 0; a < 8; a++)
      for (int i = 0; i < 3; i++) {
        for (int b = 0; b < 8; b++)
          for (int j = 0; j < 3; j++) m.lcl[(3 * a + i) * 32 + 3 * b + j] = (i == j ? KL[a][b] : 0.0) + DD[a][b][j][i];
        for (int b = 0; b < 8; b++) {
          m.lcl[(3 * a + i) * 32 + 24 + b] = GP[a][i][b];
          m.lcl[(24 + b) * 32 + 3 * a + i] = GP[a][i][b];
        }
      }
    for (int a = 0; a < 8; a++)
      for (int b = 0; b < 8; b++) m.lcl[(24 + a) * 32 + 24 + b] = KL[a][b] / 6.0;
    m.CB.assign(80, 0.0);
    for (int i = 0; i < 3; i++)
      for (int a = 0; a < 8; a++) m.CB[24 * i + 3 * a + i] = PI[a];
    for (int a = 0; a < 8; a++) m.CB[72 + a] = PI[a];
    m.Kdense = m.lcl;
  }
}

// ---- load cases -----------------------------------------------------------------------
// 2D: thermal X, Y; elastic X, Y, XY (direction flags 0, 1, 5; femhmg.c:868-896)
int load_case_count(const Model& m) { return m.dim2 ? (m.analysis == ELASTIC ? 3 : 2) : (m.analysis == ELASTIC ? 6 : 3); }
void load_case_list(const Model& m, int* dirs) {
  for (int i = 0; i < load_case_count(m); i++) dirs[i] = i;
  if (m.dim2 && m.analysis == ELASTIC) dirs[2] = 5;
}
int tensor_dim(const Model& m) { return m.dim2 ? (m.analysis == ELASTIC ? 3 : 2) : (m.analysis == ELASTIC ? 6 : 3); }
int tensor_column(const Model& m, int dir) { return (m.dim2 && dir == 5) ? 2 : dir; }
// (axis of the jump, displaced component) of a load case; X Y Z YZ XZ XY
void case_axis(const Model& m, int dir, int& axis, int& comp) {
  if (m.analysis != ELASTIC) { axis = dir; comp = 0; return; }
  if (m.dim2) { axis = dir == 0 ? 0 : 1; comp = dir == 1 ? 1 : 0; return; }
  static const int AX[6] = {0, 1, 2, 1, 2, 1}, CO[6] = {0, 1, 2, 2, 0, 0};
  axis = AX[dir]; comp = CO[dir];
}
static const int FACE[3][4] = {{1, 2, 5, 6}, {2, 3, 6, 7}, {0, 1, 2, 3}};
long axis_len(const Model& m, int axis) { return axis == 0 ? m.nx : (axis == 1 ? m.ny : m.nz); }

// Voxels whose +axis face is the cell's +axis boundary: last column (x), first row (y),
// first layer (z) -- femhmg_thermal_3D.c:144, :178, :212.
template <typename F>
static void for_boundary_voxels(const Model& m, int axis, F f) {
  const long R = m.ny, C = m.nx, L = m.nz;
  if (axis == 0) { for (long l = 0; l < L; l++) for (long r = 0; r < R; r++) f(r, C - 1, l); }
  else if (axis == 1) { for (long l = 0; l < L; l++) for (long c = 0; c < C; c++) f(0, c, l); }
  else { for (long c = 0; c < C; c++) for (long r = 0; r < R; r++) f(r, c, 0); }
}

void assemble_rhs(const Model& m, int dir, double* rhs) {
  if (m.dim2) { assemble_rhs_2d(m, dir, rhs); return; }
  std::memset(rhs, 0, sizeof(double) * m.ndof);
  const long R = m.ny, C = m.nx, L = m.nz;
  if (m.analysis == FLUID) {  // unit body force along dir: int(phi_a) at every pore-node velocity
    const long N = m.N;
    for (long e = 0; e < N; e++) {
      if (m.elem_mat[e] != 0) continue;
      const long r = e % R, c = (e / R) % C, l = e / (R * C);
      for (int a = 0; a < 8; a++) {
        const uint32_t d = m.dof_of_node[elem_node(r, c, l, a, R, C, L)];
        if (d < (uint32_t)m.nV) rhs[3 * (size_t)d + dir] += m.CB[72 + a];
      }
    }
    return;
  }
  int axis, comp;
  case_axis(m, dir, axis, comp);
  const double jump = (double)axis_len(m, axis);
  const int nd = m.nd, ed = 8 * nd;
  for_boundary_voxels(m, axis, [&](long r, long c, long l) {
    const long e = r + c * R + l * R * C;
    const double* K = m.Kdense.data() + (size_t)m.elem_mat[e] * ed * ed;
    const double f_e = sdf_scale(m, e);
    for (int a = 0; a < 8; a++) {
      const long n = elem_node(r, c, l, a, R, C, L);
      for (int ci = 0; ci < nd; ci++) {
        double s = 0.0;
        for (int f = 0; f < 4; f++) s += K[(a * nd + ci) * ed + FACE[axis][f] * nd + comp];
        rhs[n * nd + ci] -= f_e * s * jump;
      }
    }
  });
}

// sum_e f_e CB_e x_e over all voxels (flux or stress components; f_e the voxel's density
// scale, 1 without a density field)
static void volume_term_3d(const Model& m, const double* x, double* acc) {
  const long R = m.ny, C = m.nx, L = m.nz, N = m.N;
  const int nd = m.nd, ns = (m.analysis == ELASTIC) ? 6 : 3, ec = 8 * nd;
  for (int s = 0; s < 6; s++) acc[s] = 0.0;
#pragma omp parallel
  {
    double loc[6] = {0, 0, 0, 0, 0, 0};
#pragma omp for schedule(static)
    for (long e = 0; e < N; e++) {
      const long r = e % R, c = (e / R) % C, l = e / (R * C);
      const double* CB = m.CB.data() + (size_t)m.elem_mat[e] * ns * ec;
      const double f_e = sdf_scale(m, e);
      for (int a = 0; a < 8; a++) {
        const long n = elem_node(r, c, l, a, R, C, L);
        for (int ci = 0; ci < nd; ci++) {
          const double v = f_e * x[n * nd + ci];
          for (int s = 0; s < ns; s++) loc[s] += CB[s * ec + a * nd + ci] * v;
        }
      }
    }
#pragma omp critical
    for (int s = 0; s < ns; s++) acc[s] += loc[s];
  }
}

void update_C(Model& m, int dir, const double* x) {
  if (m.dim2) { update_C_2d(m, dir, x); return; }
  const long R = m.ny, C = m.nx, L = m.nz, N = m.N;
  if (m.analysis == FLUID) {
    double c0 = 0, c1 = 0, c2 = 0;
#pragma omp parallel for reduction(+ : c0, c1, c2) schedule(static)
    for (long e = 0; e < N; e++) {
      if (m.elem_mat[e] != 0) continue;
      const long r = e % R, c = (e / R) % C, l = e / (R * C);
      for (int a = 0; a < 8; a++) {
        const uint32_t d = m.dof_of_node[elem_node(r, c, l, a, R, C, L)];
        if (d < (uint32_t)m.nV) {
          c0 += m.CB[3 * a] * x[3 * (size_t)d];
          c1 += m.CB[24 + 3 * a + 1] * x[3 * (size_t)d + 1];
          c2 += m.CB[48 + 3 * a + 2] * x[3 * (size_t)d + 2];
        }
      }
    }
    const double scl = m.voxel * m.voxel / (double)N;
    m.C[0 + dir] = c0 * scl; m.C[3 + dir] = c1 * scl; m.C[6 + dir] = c2 * scl;
    return;
  }
  int axis, comp;
  case_axis(m, dir, axis, comp);
  const double jump = (double)axis_len(m, axis);
  const int nd = m.nd, ns = (m.analysis == ELASTIC) ? 6 : 3, ec = 8 * nd;
  double acc[6];
  volume_term_3d(m, x, acc);
  for_boundary_voxels(m, axis, [&](long r, long c, long l) {
    const long e = r + c * R + l * R * C;
    const double* CB = m.CB.data() + (size_t)m.elem_mat[e] * ns * ec;
    const double f_e = sdf_scale(m, e);
    for (int f = 0; f < 4; f++)
      for (int s = 0; s < ns; s++) acc[s] += f_e * CB[s * ec + FACE[axis][f] * nd + comp] * jump;
  });
  for (int s = 0; s < ns; s++) m.C[s * ns + dir] = acc[s] / (double)N;
}

// ---- thermal expansion (femhmg_elastic_3D.c:464-505 RHS, :863-1074 effective expansion) ----
// A unit temperature rise gives material m the eigenstrain alpha_m (1,1,1,0,0,0) and the stress
// sigma_m = D_m alpha_m (1,1,1,0,0,0) = alpha_m E_m / (1 - 2 nu_m) on the normal components.
// The reference evaluates the element load B^T sigma at the voxel centre, where every shape
// gradient is 1/4 (+-1, +-1, +-1), with the sign + where the node sits at coordinate 1.
// effective expansion: C alpha = beta, n = 6 (3D) or 3 (2D), elimination with partial pivoting
static void solve_expansion(Model& m, const double* beta, int n) {
  double M[6][7];
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < n; j++) M[i][j] = m.C[n * i + j];
    M[i][n] = beta[i];
  }
  for (int i = 0; i < n; i++) {
    int p = i;
    for (int j = i + 1; j < n; j++) if (std::fabs(M[j][i]) > std::fabs(M[p][i])) p = j;
    if (p != i) for (int k = 0; k <= n; k++) std::swap(M[i][k], M[p][k]);
    for (int j = i + 1; j < n; j++) {
      const double s = M[j][i] / M[i][i];
      for (int k = i; k <= n; k++) M[j][k] -= s * M[i][k];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double v = M[i][n];
    for (int j = i + 1; j < n; j++) v -= M[i][j] * m.thermal_expansion[j];
    m.thermal_expansion[i] = v / M[i][i];
  }
  for (int i = n; i < 6; i++) m.thermal_expansion[i] = 0.0;
}

static double thermal_stress(const Model& m, int mat) {
  const double E = m.props[2 * mat], nu = m.props[2 * mat + 1];
  return m.alpha[mat] * E / (1.0 - 2.0 * nu);
}

void assemble_rhs_thermal_expansion(const Model& m, double* rhs) {
  if (m.dim2) { assemble_rhs_thermal_expansion_2d(m, rhs); return; }
  std::memset(rhs, 0, sizeof(double) * m.ndof);
  const long R = m.ny, C = m.nx, L = m.nz, N = m.N;
  double f[4][24];
  for (unsigned mat = 0; mat < m.nmat && mat < 4; mat++) {
    const double sn = thermal_stress(m, (int)mat);
    for (int a = 0; a < 8; a++) {
      const int x = dcol(a), y = -drow(a), z = 1 - dlay(a);
      f[mat][3 * a + 0] = 0.25 * sn * (x ? 1.0 : -1.0);
      f[mat][3 * a + 1] = 0.25 * sn * (y ? 1.0 : -1.0);
      f[mat][3 * a + 2] = 0.25 * sn * (z ? 1.0 : -1.0);
    }
  }
  for (long e = 0; e < N; e++) {
    const long r = e % R, c = (e / R) % C, l = e / (R * C);
    const double* fe = f[m.elem_mat[e]];
    for (int a = 0; a < 8; a++) {
      const long n = elem_node(r, c, l, a, R, C, L);
      for (int ci = 0; ci < 3; ci++) rhs[3 * n + ci] += fe[3 * a + ci];
    }
  }
}

// volume: sum_e CB_e x_e of the thermal-expansion solution (6 values).  The mean strain of the
// periodic fluctuation, which the reference also adds (C times it), is zero: every node enters
// the sum once per local index and the centre gradients of the 8 shape functions sum to zero.
void update_thermal_expansion(Model& m, const double* volume) {
  double count[4] = {0, 0, 0, 0};
  const long ref3 = (long)m.refinement * m.refinement * m.refinement;
  for (uint8_t c : m.colors) count[m.props_keys[c]] += (double)ref3;
  double stress[6], beta[6];
  for (int k = 0; k < 6; k++) stress[k] = volume[k];
  for (unsigned mat = 0; mat < m.nmat && mat < 4; mat++)
    for (int k = 0; k < 3; k++) stress[k] -= count[mat] * thermal_stress(m, (int)mat);
  for (int k = 0; k < 6; k++) beta[k] = -stress[k] / (double)m.N;
  solve_expansion(m, beta, 6);
}

int voxel_material(const Model& m, long r, long c, long l) {
  if (!m.elem_mat.empty()) return m.elem_mat[r + c * (long)m.ny + l * (long)m.ny * m.nx];
  const long ref = m.refinement;
  return m.props_keys[m.colors[(size_t)(l / ref) * m.frows * m.fcols + (size_t)(r / ref) * m.fcols + (size_t)(c / ref)]];
}

// The effective-tensor column of load case dir from the volume term sum_e CB_e x_e (reduced on
// the device, cudapcgB200SolveLoadCases) plus the boundary face term -- the same sums as
// update_C, split where the device takes over.
void update_C_from_volume(Model& m, int dir, const double* volume) {
  if (m.analysis == FLUID) {
    const double scl = m.voxel * m.voxel / (double)m.N;
    for (int s = 0; s < 3; s++) m.C[3 * s + dir] = volume[s] * scl;
    return;
  }
  int axis, comp;
  case_axis(m, dir, axis, comp);
  const double jump = (double)axis_len(m, axis);
  const int nd = m.nd, ns = (m.analysis == ELASTIC) ? 6 : 3, ec = 8 * nd;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int s = 0; s < ns; s++) acc[s] = volume[s];
  for_boundary_voxels(m, axis, [&](long r, long c, long l) {
    const double* CB = m.CB.data() + (size_t)voxel_material(m, r, c, l) * ns * ec;
    for (int f = 0; f < 4; f++)
      for (int s = 0; s < ns; s++) acc[s] += CB[s * ec + FACE[axis][f] * nd + comp] * jump;
  });
  for (int s = 0; s < ns; s++) m.C[s * ns + dir] = acc[s] / (double)m.N;
}

// ---- 2D: pixel images (femhmg_2D.c, femhmg_thermal_2D.c, femhmg_elastic_2D.c) ----------
// A pixel (r, c) has its local node k at node (r + 1 + drow(k), c + dcol(k)), k = 0..3 (left
// bottom, right bottom, right top, left top; x = +col, y = -row); node (r, c) is local node e of
// pixel (r - drow(e) - 1, c - dcol(e)).  Node keys hold a pixel's material in 4 bits per local
// index (16 materials).  Element matrices are integrated with 2 x 2 Gauss points on the unit
// square; elasticity is plane strain (the reference's default build) unless
// CHFEM_B200_PLANE_STRESS=1 (its ELASTIC_2D_PLANESTRESS build).
static inline long elem_node_2d(long r, long c, int k, long R, long C) { return wrapl(r + 1 + drow(k), R) + wrapl(c + dcol(k), C) * R; }
static inline long node_elem_2d(long r, long c, int e, long R, long C) { return wrapl(r - drow(e) - 1, R) + wrapl(c - dcol(e), C) * R; }
static const int FACE2D[2][2] = {{1, 2}, {2, 3}};  // local nodes on the +x and +y sides

static bool build_maps_2d(Model& m, std::string& err) {
  const long R = m.ny, C = m.nx, N = m.N;
  if (m.analysis == FLUID) {  // femhmg_fluid_2D.c:370-460: pore nodes (key 15) first, then interface nodes
    if (!count_pore_nodes_2d(m, err)) return false;
    m.dof_of_node.assign(N, 0);
    long id = 0;
    for (long i = 0; i < N; i++)
      if (m.fluid_keys[i] == 15) m.dof_of_node[i] = (uint32_t)id++;
    for (long i = 0; i < N; i++)
      if (m.fluid_keys[i] != 15 && m.fluid_keys[i] != 0) m.dof_of_node[i] = (uint32_t)id++;
    m.node_of_dof.assign(m.nV + m.nB, 0);
    m.border_keys.assign(m.nB, 0);
    for (long i = 0; i < N; i++) {
      const uint8_t k = m.fluid_keys[i];
      if (!k) continue;
      const uint32_t d = m.dof_of_node[i];
      m.node_of_dof[d] = (uint32_t)i;
      if (k != 15) m.border_keys[d - m.nV] = k;
    }
    return true;
  }
  if (m.nmat > 16) { err = "more than 16 materials cannot be encoded in 16-bit 2D node keys"; return false; }
  m.keys.assign(N, 0);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; i++) {
    const long r = i % R, c = i / R;
    unsigned k = 0;
    for (int e = 0; e < 4; e++) k |= ((unsigned)m.elem_mat[node_elem_2d(r, c, e, R, C)] & 15u) << (4 * e);
    m.keys[i] = (uint16_t)k;
  }
  m.ndof = N * m.nd;
  return true;
}

// Stokes: fluid key of every node (bit e: the pixel in which the node is local node e is pore,
// material 0), pore nodes (key 15) and interface nodes (0 < key < 15); DOFs 3 per pore node
// (2 velocities, pressure) and 1 per interface node
static bool count_pore_nodes_2d(Model& m, std::string& err) {
  const long R = m.ny, C = m.nx, N = m.N;
  m.fluid_keys.assign(N, 0);
  long pores = 0, nv = 0, nb = 0;
  for (long i = 0; i < N; i++) {
    const long r = i % R, c = i / R;
    unsigned k = 0;
    for (int e = 0; e < 4; e++) k |= (unsigned)(m.elem_mat[node_elem_2d(r, c, e, R, C)] == 0) << e;
    m.fluid_keys[i] = (uint8_t)k;
    pores += (m.elem_mat[i] == 0);
    nv += (k == 15);
    nb += (k != 0 && k != 15);
  }
  if (3 * nv + nb >= (long)0xffffffffL) { err = "too many Stokes unknowns for 32-bit DOF ids"; return false; }
  m.nporeelem = pores;
  m.nV = nv;
  m.nB = nb;
  m.ndof = 3 * nv + nb;
  return true;
}

// Plane constitutive matrix of material k (xx, yy, xy): plane strain, or plane stress under
// CHFEM_B200_PLANE_STRESS=1 (femhmg_elastic_2D.c:56-200)
void plane_D(const Model& m, int k, double D[3][3]) {
  const char* ps = getenv("CHFEM_B200_PLANE_STRESS");
  const double E = m.props[2 * k], nu = m.props[2 * k + 1];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) D[i][j] = 0.0;
  if (ps && ps[0] == '1') {
    const double f = E / (1.0 - nu * nu);
    D[0][0] = D[1][1] = f; D[0][1] = D[1][0] = f * nu; D[2][2] = f * 0.5 * (1.0 - nu);
  } else {
    const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = E / (2.0 * (1.0 + nu));
    D[0][0] = D[1][1] = lam + 2.0 * mu; D[0][1] = D[1][0] = lam; D[2][2] = mu;
  }
}

static void build_local_matrices_2d(Model& m) {
  const double g[2] = {0.5 - 0.5 / std::sqrt(3.0), 0.5 + 0.5 / std::sqrt(3.0)};
  double grad[4][4][2];  // [qp][node][x, y]
  for (int q = 0; q < 4; q++) {
    const double px = g[q & 1], py = g[q >> 1];
    for (int a = 0; a < 4; a++) {
      const int cx = nxi(a), cy = neta(a);
      grad[q][a][0] = df1(cx) * f1(cy, py);
      grad[q][a][1] = f1(cx, px) * df1(cy);
    }
  }
  if (m.analysis == FLUID) {
    // unit pixel, mu = 1 (femhmg_fluid_2D.c:41-80): [K G; G^T Stab], K = int(grad u : grad v +
    // grad u^T : grad v), G = int(d_i phi_a psi_b), Stab = (1/6) * Q1 Laplacian; CB: the velocity
    // average (2 x 8) and the body-force load (4)
    double phi[4][4];
    for (int q = 0; q < 4; q++)
      for (int a = 0; a < 4; a++) phi[q][a] = f1(nxi(a), g[q & 1]) * f1(neta(a), g[q >> 1]);
    m.lcl.assign(144, 0.0);
    m.CB.assign(20, 0.0);
    for (int q = 0; q < 4; q++)
      for (int a = 0; a < 4; a++) {
        for (int b = 0; b < 4; b++) {
          const double kl = grad[q][a][0] * grad[q][b][0] + grad[q][a][1] * grad[q][b][1];
          for (int i = 0; i < 2; i++) {
            for (int j = 0; j < 2; j++) m.lcl[(2 * a + i) * 12 + 2 * b + j] += 0.25 * ((i == j ? kl : 0.0) + grad[q][a][j] * grad[q][b][i]);
            const double gp = 0.25 * grad[q][a][i] * phi[q][b];
            m.lcl[(2 * a + i) * 12 + 8 + b] += gp;
            m.lcl[(8 + b) * 12 + 2 * a + i] += gp;
          }
          m.lcl[(8 + a) * 12 + 8 + b] += 0.25 * kl / 6.0;
        }
        for (int i = 0; i < 2; i++) m.CB[8 * i + 2 * a + i] += 0.25 * phi[q][a];
        m.CB[16 + a] += 0.25 * phi[q][a];
      }
    m.Kdense = m.lcl;
    return;
  }
  const int nd = m.nd, ed = 4 * nd;
  m.lcl.assign((size_t)ed * ed * m.nmat, 0.0);
  if (m.analysis == THERMAL) {
    m.CB.assign((size_t)8 * m.nmat, 0.0);  // [mat][flux s][node a]
    for (unsigned k = 0; k < m.nmat; k++) {
      const double kp = m.props[k];
      for (int q = 0; q < 4; q++)
        for (int a = 0; a < 4; a++) {
          for (int b = 0; b < 4; b++)
            m.lcl[16 * k + 4 * a + b] += 0.25 * kp * (grad[q][a][0] * grad[q][b][0] + grad[q][a][1] * grad[q][b][1]);
          for (int s = 0; s < 2; s++) m.CB[8 * k + 4 * s + a] += 0.25 * kp * grad[q][a][s];
        }
    }
  } else {
    m.CB.assign((size_t)24 * m.nmat, 0.0);  // [mat][stress s (xx, yy, xy)][dof]
    for (unsigned k = 0; k < m.nmat; k++) {
      double D[3][3];
      plane_D(m, (int)k, D);
      for (int q = 0; q < 4; q++) {
        double B[3][8] = {{0}};
        for (int a = 0; a < 4; a++) {
          B[0][2 * a] = grad[q][a][0];
          B[1][2 * a + 1] = grad[q][a][1];
          B[2][2 * a] = grad[q][a][1]; B[2][2 * a + 1] = grad[q][a][0];
        }
        double DB[3][8];
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 8; c++) DB[r][c] = D[r][0] * B[0][c] + D[r][1] * B[1][c] + D[r][2] * B[2][c];
        for (int i = 0; i < 8; i++)
          for (int j = 0; j < 8; j++) m.lcl[64 * k + 8 * i + j] += 0.25 * (B[0][i] * DB[0][j] + B[1][i] * DB[1][j] + B[2][i] * DB[2][j]);
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 8; c++) m.CB[24 * k + 8 * r + c] += 0.25 * DB[r][c];
      }
    }
  }
  m.Kdense = m.lcl;
}

// Pixels whose +axis side is the cell's +axis boundary: last column (x), first row (y)
// (femhmg_thermal_2D.c:101-140)
template <typename F>
static void for_boundary_pixels(const Model& m, int axis, F f) {
  const long R = m.ny, C = m.nx;
  if (axis == 0) { for (long r = 0; r < R; r++) f(r, C - 1); }
  else { for (long c = 0; c < C; c++) f(0, c); }
}

static void assemble_rhs_2d(const Model& m, int dir, double* rhs) {
  std::memset(rhs, 0, sizeof(double) * m.ndof);
  const long R = m.ny, C = m.nx;
  if (m.analysis == FLUID) {  // unit body force along dir at every pore-node velocity (femhmg_fluid_2D.c:84-124)
    for (long e = 0; e < m.N; e++) {
      if (m.elem_mat[e] != 0) continue;
      const long r = e % R, c = e / R;
      for (int a = 0; a < 4; a++) {
        const uint32_t d = m.dof_of_node[elem_node_2d(r, c, a, R, C)];
        if (d < (uint32_t)m.nV) rhs[2 * (size_t)d + dir] += m.CB[16 + a];
      }
    }
    return;
  }
  int axis, comp;
  case_axis(m, dir, axis, comp);
  const double jump = (double)(axis == 0 ? m.nx : m.ny);
  const int nd = m.nd, ed = 4 * nd;
  for_boundary_pixels(m, axis, [&](long r, long c) {
    const double* K = m.Kdense.data() + (size_t)m.elem_mat[r + c * R] * ed * ed;
    const double f_e = sdf_scale(m, r + c * R);
    for (int a = 0; a < 4; a++) {
      const long n = elem_node_2d(r, c, a, R, C);
      for (int ci = 0; ci < nd; ci++) {
        double s = 0.0;
        for (int f = 0; f < 2; f++) s += K[(a * nd + ci) * ed + FACE2D[axis][f] * nd + comp];
        rhs[n * nd + ci] -= f_e * s * jump;
      }
    }
  });
}

// sum_e f_e CB_e x_e over all pixels (flux or stress components; f_e the pixel's density scale,
// 1 without a density field; femhmg_thermal_2D.c:293-372, femhmg_elastic_2D.c:638-742)
static void volume_term_2d(const Model& m, const double* x, double* acc) {
  const long R = m.ny, C = m.nx, N = m.N;
  const int nd = m.nd, ns = tensor_dim(m), ec = 4 * nd;
  for (int s = 0; s < 3; s++) acc[s] = 0.0;
#pragma omp parallel
  {
    double loc[3] = {0, 0, 0};
#pragma omp for schedule(static)
    for (long e = 0; e < N; e++) {
      const long r = e % R, c = e / R;
      const double* CB = m.CB.data() + (size_t)m.elem_mat[e] * ns * ec;
      double le[3] = {0, 0, 0};
      for (int a = 0; a < 4; a++) {
        const long n = elem_node_2d(r, c, a, R, C);
        for (int ci = 0; ci < nd; ci++)
          for (int s = 0; s < ns; s++) le[s] += CB[s * ec + a * nd + ci] * x[n * nd + ci];
      }
      const double f_e = sdf_scale(m, e);
      for (int s = 0; s < ns; s++) loc[s] += f_e * le[s];
    }
#pragma omp critical
    for (int s = 0; s < ns; s++) acc[s] += loc[s];
  }
}

static void update_C_2d(Model& m, int dir, const double* x) {
  const long R = m.ny, C = m.nx, N = m.N;
  if (m.analysis == FLUID) {  // femhmg_fluid_2D.c:245-300: mean velocity times h^2
    double c0 = 0, c1 = 0;
    for (long e = 0; e < N; e++) {
      if (m.elem_mat[e] != 0) continue;
      const long r = e % R, c = e / R;
      for (int a = 0; a < 4; a++) {
        const uint32_t d = m.dof_of_node[elem_node_2d(r, c, a, R, C)];
        if (d < (uint32_t)m.nV) {
          c0 += m.CB[2 * a] * x[2 * (size_t)d];
          c1 += m.CB[8 + 2 * a + 1] * x[2 * (size_t)d + 1];
        }
      }
    }
    const double scl = m.voxel * m.voxel / (double)N;
    m.C[0 + dir] = c0 * scl;
    m.C[2 + dir] = c1 * scl;
    return;
  }
  int axis, comp;
  case_axis(m, dir, axis, comp);
  const double jump = (double)(axis == 0 ? m.nx : m.ny);
  const int nd = m.nd, ns = tensor_dim(m), ec = 4 * nd, col = tensor_column(m, dir);
  double acc[3];
  volume_term_2d(m, x, acc);
  for_boundary_pixels(m, axis, [&](long r, long c) {
    const double* CB = m.CB.data() + (size_t)m.elem_mat[r + c * R] * ns * ec;
    const double f_e = sdf_scale(m, r + c * R);
    for (int f = 0; f < 2; f++)
      for (int s = 0; s < ns; s++) acc[s] += f_e * CB[s * ec + FACE2D[axis][f] * nd + comp] * jump;
  });
  for (int s = 0; s < ns; s++) m.C[s * ns + col] = acc[s] / (double)N;
}

// ---- 2D thermal expansion (femhmg_elastic_2D.c:277-300 RHS, :388-528 effective expansion) ----
// A unit temperature rise gives material m the in-plane eigenstrain alpha_m (1, 1, 0) and the
// stress D_m alpha_m (1, 1, 0), D_m the plane matrix of the element matrices (plane strain:
// alpha E / ((1 + nu)(1 - 2 nu)) on both normal components).  The element load is B^T sigma at
// the pixel centre, where every shape gradient is +-1/2 (+ where the node sits at coordinate 1).
// Under plane stress the reference's helpers (femhmg_elastic_2D.c:849-866, :868-906) take
// E / (1 - nu) for the factor of D, which is not the plane-stress matrix of its own element
// matrices (E / (1 - nu^2), :148-200): a homogeneous image would not return its own alpha.  Here
// both use the element matrices' D.
static void thermal_stress_2d(const Model& m, int mat, double s[2]) {
  double D[3][3];
  plane_D(m, mat, D);
  s[0] = m.alpha[mat] * (D[0][0] + D[0][1]);
  s[1] = m.alpha[mat] * (D[1][0] + D[1][1]);
}

static void assemble_rhs_thermal_expansion_2d(const Model& m, double* rhs) {
  std::memset(rhs, 0, sizeof(double) * m.ndof);
  const long R = m.ny, C = m.nx, N = m.N;
  std::vector<double> f((size_t)8 * m.nmat);
  for (unsigned mat = 0; mat < m.nmat; mat++) {
    double sn[2];
    thermal_stress_2d(m, (int)mat, sn);
    for (int a = 0; a < 4; a++) {
      f[8 * mat + 2 * a] = 0.5 * sn[0] * (nxi(a) ? 1.0 : -1.0);
      f[8 * mat + 2 * a + 1] = 0.5 * sn[1] * (neta(a) ? 1.0 : -1.0);
    }
  }
  for (long e = 0; e < N; e++) {
    const long r = e % R, c = e / R;
    const double* fe = f.data() + 8 * (size_t)m.elem_mat[e];
    for (int a = 0; a < 4; a++) {
      const long n = elem_node_2d(r, c, a, R, C);
      rhs[2 * n] += fe[2 * a];
      rhs[2 * n + 1] += fe[2 * a + 1];
    }
  }
}

// The effective expansion from the solution x of the unit-temperature load: mean stress
// sum_e (CB_e x_e - sigma_e) / N, and alpha_eff = C^-1 (-mean stress).  The mean strain of the
// periodic fluctuation, which the reference also multiplies by C and adds, is zero: the centre
// gradients of the 4 shape functions sum to zero and every node enters once per local index.
void update_thermal_expansion_2d(Model& m, const double* x) {
  double stress[3];
  volume_term_2d(m, x, stress);
  std::vector<double> count(m.nmat, 0.0);
  for (long e = 0; e < m.N; e++) count[m.elem_mat[e]] += 1.0;
  for (unsigned mat = 0; mat < m.nmat; mat++) {
    double sn[2];
    thermal_stress_2d(m, (int)mat, sn);
    stress[0] -= count[mat] * sn[0];
    stress[1] -= count[mat] * sn[1];
  }
  double beta[3];
  for (int k = 0; k < 3; k++) beta[k] = -stress[k] / (double)m.N;
  solve_expansion(m, beta, 3);
}

// The effective thermal expansion from the solution x of the unit-temperature load, with the
// stress sums taken on the host (the device path reduces the 3D volume term on the GPU)
void thermal_expansion_from_solution(Model& m, const double* x) {
  if (m.dim2) { update_thermal_expansion_2d(m, x); return; }
  double volume[6];
  volume_term_3d(m, x, volume);
  update_thermal_expansion(m, volume);
}

}  // namespace chfem_host
