// hmg.h -- internal model of the chfem_b200 host layer (3D thermal / elastic / Stokes, 2D
// thermal / elastic).
//
// Index conventions are chfem's (chfem/src/femhmg/femhmg.c:1644-1709,
// physical_phenomena/femhmg_3D.c:4-75): voxel and node index i = row + col*ny + layer*ny*nx,
// row fastest; a voxel e = (r,c,l) has its local node 3 ("left, top, near") at node e and
// its local node k at node (r + 1 + drow(k), c + dcol(k), l + dlay(k)) (periodic).
// Physical axes: x = +col, y = -row, z = -layer (right-handed), so the +x, +y, +z faces of
// a voxel hold local nodes {1,2,5,6}, {2,3,6,7} and {0,1,2,3}.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace chfem_host {

enum Analysis { THERMAL = 0, ELASTIC = 1, FLUID = 2 };

struct Model {
  // settings (.nf, femhmg.c:1456-1586)
  int analysis = -1;
  bool dim2 = false;                 // 2D image (%image_dimensions with 0 layers): pixels, nz = 1
  int solver_flag = 0;
  double voxel = 1.0;
  double tol = 1e-6;
  unsigned maxit = 10000;
  unsigned nx = 0, ny = 0, nz = 0;   // voxels per axis after refinement
  unsigned refinement = 1;
  unsigned nmat = 0;
  double props[512] = {0};
  int props_keys[256];               // colour -> material index (-1 when not listed)
  double alpha[256] = {0};
  bool has_thermal_expansion = false;
  double thermal_expansion[6] = {0, 0, 0, 0, 0, 0};  // effective, Voigt xx yy zz yz xz xy
  double xreduce_stab = -1.0;        // %xreduce_scale_factor (negative: not given)
  std::string nf, nf_noext, raw;
  // sizes
  long N = 0;                        // voxels = periodic nodes
  long ndof = 0;
  unsigned nd = 1;                   // DOF per node (thermal 1, elastic 3 (2D: 2); Stokes layout is special)
  unsigned C_dim = 9;
  // the image as read: one colour byte per voxel of the file, x fastest (refinement not applied)
  std::vector<uint8_t> colors;
  unsigned frows = 0, fcols = 0, fslices = 0;
  // maps (thermal / elastic: built on the host only when a host path needs them, else the
  // device builds the node keys from the colours)
  bool host_maps = false;
  std::vector<uint16_t> elem_mat;    // material index per voxel
  std::vector<uint16_t> keys;        // 16-bit node keys (thermal/elastic)
  std::vector<uint8_t> fluid_keys;   // 8-bit node fluid keys (Stokes)
  std::vector<uint32_t> dof_of_node; // Stokes: node -> DOF id
  std::vector<uint32_t> node_of_dof; // Stokes: DOF id -> node
  std::vector<uint8_t> border_keys;  // Stokes: fluid keys of interface nodes
  long nV = 0, nB = 0, nporeelem = 0;
  // local matrices in the cudapcg formats, and the stress (flux, velocity) averaging matrices
  std::vector<double> lcl;           // thermal 40/mat, elastic 576/mat, Stokes 1024; 2D: dense 16 / 64 per mat
  std::vector<double> CB;            // thermal 8x3 (avg gradient)*k per mat, elastic 6x24 per mat, Stokes 3x24
  std::vector<double> Kdense;        // dense element matrices (8nd x 8nd per material; Stokes 32x32)
  // scalar density field (-f): per model voxel a 16-bit code q; the voxel's element matrix is
  // scaled by sdf_min + (sdf_max - sdf_min) q / 65535 (femhmg.c:1760-1835); empty without one
  int data_type = 0;                 // %data_type of the field file: 0 float32, 1 float64
  std::vector<uint16_t> sdf;
  double sdf_range[2] = {0.0, 0.0};  // [min, max] of the quantised products
  // results
  double C[36] = {0};
  std::vector<double> rhs;
};

// scale of voxel e's element matrix (1 without a density field)
inline double sdf_scale(const Model& m, long e) {
  return m.sdf.empty() ? 1.0 : (double)m.sdf[e] * (1.0 / 65535.0) * (m.sdf_range[1] - m.sdf_range[0]) + m.sdf_range[0];
}

// physics (hmg_physics.cpp)
bool build_maps(Model& m, std::string& err);
bool count_pore_nodes(Model& m, std::string& err);
void build_local_matrices(Model& m);
void assemble_rhs(const Model& m, int direction, double* rhs);
void update_C(Model& m, int direction, const double* x);
// thermal expansion load case (elastic): right-hand side of a unit temperature rise, and the
// effective expansion from the tensor C and the volume term of its solution
void assemble_rhs_thermal_expansion(const Model& m, double* rhs);
void update_thermal_expansion(Model& m, const double* volume);
// 2D: from the solution itself (xx, yy, xy into thermal_expansion[0..2])
void update_thermal_expansion_2d(Model& m, const double* x);
// 3D or 2D, from the solution itself (the stress sums on the host)
void thermal_expansion_from_solution(Model& m, const double* x);
// 2D elastic: plane constitutive matrix of material k (xx, yy, xy) used by the element matrices
void plane_D(const Model& m, int k, double D[3][3]);
// material index of model voxel (r, c, l) (refined grid), from elem_mat or from the colours
int voxel_material(const Model& m, long r, long c, long l);
void update_C_from_volume(Model& m, int direction, const double* volume);
void case_axis(const Model& m, int direction, int& axis, int& comp);
long axis_len(const Model& m, int axis);
int load_case_count(const Model& m);
// number of flux / stress components of the tensor (thermal 3, elastic 6; 2D: 2, 3)
int tensor_dim(const Model& m);
// column of the effective tensor that load case `direction` fills (2D elastic XY: 2)
int tensor_column(const Model& m, int direction);
void load_case_list(const Model& m, int* dirs);

}  // namespace chfem_host
