// hmg.cpp -- femhmg-compatible host API of chfem_b200 (3D; 2D thermal / elastic): settings and image input,
// model set-up, the load-case loop over the cudapcg C ABI, output.
//
// Follows chfem/src/femhmg/femhmg.c: hmgInit :135-394, readData :1456-1586 (tag grammar and
// the 12-entry scan limit), readMaterialMapRAW/Numpy :1644-1758 (x-fastest file order
// transposed to the row-fastest internal order, with %refinement replication),
// hmgSolveHomogenization :848-1198 (solver set-up, direction loop, -xi/-xo files, updateC).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/chfem_b200.h"
#include "../../include/cudapcg_b200.h"
#include "hmg.h"

using namespace chfem_host;

namespace {

Model* g_m = nullptr;
std::string g_err;
// solver-side flags (femhmg.c:26-29 defaults)
int g_par = CUDAPCG_NBN, g_solver = CUDAPCG_CG_SOLVER, g_precond = 1, g_stopcrit = CUDAPCG_L2_NORM;
int g_poremap = CUDAPCG_POREMAP_NUM;
int g_precision = CHFEM_B200_PREC_FP64, g_multirhs = 0, g_quiet = 0;
int g_dir_set = 0, g_dir = 6;
int g_xreduce = CUDAPCG_XREDUCE_FULL;  // femhmg.c:23
bool g_export_x = false;
bool g_export_fields = false;

std::string g_x0_file;
bool g_use_x0 = false;
int g_recursions = 0;
// recursive initial guesses: per load case, the solution on the model coarsened by 2 per axis
// (prolonged by the library, cudapcgSetX0(x0, 1)); empty where none was found
std::vector<double> g_x0_coarse[6];
bool g_have_coarse = false;
// caller-provided initial guesses for the next homogenization (chfemB200SetInitialGuesses)
const double* g_x0_user[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
int g_x0_user_device = 0;
bool g_report = false;
std::string g_report_text;
chfemB200SolveStats g_stats;

#define SAY(...) do { if (!g_quiet) printf(__VA_ARGS__); } while (0)

void fail(const std::string& e) {
  g_err = e;
  fprintf(stderr, "chfem_b200: %s\n", e.c_str());
}

// -e (femhmg.c:1112-1118): the solution and its field per load case, as the reference writes
// them -- thermal <nf>_temperature_<dir>.bin and _flux_ (3 per node); elastic _displacement_ and
// _stress_ (6 per node); Stokes _velocity_ (3 per node, pore nodes) and _pressure_ (fluid nodes).
// block_index: the block solve's right-hand side holding this case (-1: the last single solve).
void write_bin(const std::string& fn, const double* v, size_t n) {
  FILE* f = fopen(fn.c_str(), "wb");
  if (!f) { SAY("WARNING: cannot write %s\n", fn.c_str()); return; }
  fwrite(v, sizeof(double), n, f);
  fclose(f);
}
// 2D exported field (flux k grad T, 2 per node; stress D eps, 3 per node: xx, yy, xy, with D the
// plane-strain or plane-stress matrix of the element matrices): at each node the mean over its 4
// pixels of the pixel's field at the node's corner, each pixel on the cell's +axis side seeing
// the load case's jump on its +axis side nodes (a node gathers its 4 corner values: no
// accumulation race).  Under plane stress the reference's stress helper takes E / (1 - nu) for
// the factor of D (femhmg_elastic_2D.c:815-847), not its element matrices' E / (1 - nu^2).
std::vector<double> fields_2d(const Model& m, int dir, const double* x) {
  const long R = m.ny, C = m.nx, N = m.N;
  const int nd = m.nd, nf = m.analysis == THERMAL ? 2 : 3;
  int axis, comp;
  case_axis(m, dir, axis, comp);
  const double jump = (double)(axis == 0 ? m.nx : m.ny);
  static const int FACE[2][2] = {{1, 2}, {2, 3}};
  auto dr = [](int k) { return -((k & 3) >> 1); };
  auto dc = [](int k) { return ((k & 3) == 1 || (k & 3) == 2) ? 1 : 0; };
  std::vector<double> out((size_t)nf * N, 0.0);
#pragma omp parallel for schedule(static)
  for (long n = 0; n < N; n++) {
    const long r = n % R, c = n / R;
    double f[3] = {0, 0, 0};
    for (int k = 0; k < 4; k++) {
      const long er = ((r - dr(k) - 1) % R + R) % R, ec = ((c - dc(k)) % C + C) % C;
      const bool boundary = axis == 0 ? ec == C - 1 : er == 0;
      const double px = dc(k), py = -dr(k);  // the node's corner in the pixel
      double g[2][2] = {{0, 0}, {0, 0}};       // [component][d/dx, d/dy]
      for (int j = 0; j < 4; j++) {
        const long node = ((er + 1 + dr(j)) % R + R) % R + ((ec + dc(j)) % C + C) % C * R;
        const int xj = dc(j), yj = -dr(j);
        const double dx = (xj ? 1.0 : -1.0) * (yj ? py : 1.0 - py), dy = (xj ? px : 1.0 - px) * (yj ? 1.0 : -1.0);
        const bool on_face = boundary && (FACE[axis][0] == j || FACE[axis][1] == j);
        for (int ci = 0; ci < nd; ci++) {
          const double v = x[node * nd + ci] + ((on_face && ci == comp) ? jump : 0.0);
          g[ci][0] += dx * v;
          g[ci][1] += dy * v;
        }
      }
      const int mat = m.elem_mat[er + ec * R];
      if (m.analysis == THERMAL) {
        f[0] += 0.25 * m.props[mat] * g[0][0];
        f[1] += 0.25 * m.props[mat] * g[0][1];
      } else {
        double D[3][3];
        plane_D(m, mat, D);
        const double exx = g[0][0], eyy = g[1][1], gxy = g[0][1] + g[1][0];
        for (int t = 0; t < 3; t++) f[t] += 0.25 * (D[t][0] * exx + D[t][1] * eyy + D[t][2] * gxy);
      }
    }
    for (int t = 0; t < nf; t++) out[(size_t)n * nf + t] = f[t];
  }
  return out;
}

void export_fields(const Model& m, int dir, const double* x, int block_index) {
  if (!m.sdf.empty()) {  // femhmg_thermal_3D.c:1113-1116 and its elastic / 2D counterparts
    SAY("WARNING: Field exportation not supported for scalar field input (.bin) yet.\n");
    return;
  }
  const std::string pre = m.nf_noext + "_";
  const std::string suf = "_" + std::to_string(dir) + ".bin";
  if (m.analysis == FLUID) {  // femhmg_fluid_3D.c:312-360, femhmg_fluid_2D.c:314-350
    const int D = m.dim2 ? 2 : 3;
    const uint8_t full = m.dim2 ? 15 : 255;
    std::vector<double> u(D * (size_t)m.N, 0.0), p(m.N, 0.0);
    for (long n = 0; n < m.N; n++) {
      const uint32_t id = m.dof_of_node[n];
      const uint8_t fk = m.fluid_keys[n];
      if (fk == full)
        for (int c = 0; c < D; c++) u[D * n + c] = x[D * (size_t)id + c];
      if (fk) p[n] = x[D * (size_t)m.nV + id];
    }
    write_bin(pre + "velocity" + suf, u.data(), u.size());
    write_bin(pre + "pressure" + suf, p.data(), p.size());
    return;
  }
  write_bin(pre + (m.analysis == THERMAL ? "temperature" : "displacement") + suf, x, m.ndof);
  int axis, comp;
  case_axis(m, dir, axis, comp);
  if (m.dim2) {  // femhmg_thermal_2D.c:423-596, femhmg_elastic_2D.c:908-1170
    const std::vector<double> f = fields_2d(m, dir, x);
    write_bin(pre + (m.analysis == THERMAL ? "flux" : "stress") + suf, f.data(), f.size());
    return;
  }
  const int nf = m.analysis == THERMAL ? 3 : 6;
  std::vector<double> field((size_t)nf * m.N);
  if (!cudapcgB200ComputeFields(block_index, axis, comp, (double)axis_len(m, axis), m.props, field.data())) {
    SAY("WARNING: field computation failed: %s\n", cudapcgB200LastError());
    return;
  }
  write_bin(pre + (m.analysis == THERMAL ? "flux" : "stress") + suf, field.data(), field.size());
}

// ---- .nf (femhmg.c:1456-1586) ---------------------------------------------------------
bool read_nf(Model& m, const char* fn) {
  FILE* f = fopen(fn, "r");
  if (!f) { fail(std::string("cannot open ") + fn); return false; }
  char tok[256];
  unsigned count = 0;
  const unsigned num_of_info = 12;
  int nx = -1, ny = -1, nz = -1;
  double tolbuf = 0;
  bool ok = true;
  for (int i = 0; i < 256; i++) m.props_keys[i] = -1;
  while (count < num_of_info && fscanf(f, "%255s", tok) == 1) {
    if (!strcmp(tok, "%type_of_analysis")) {
      if (fscanf(f, "%d", &m.analysis) != 1) break;
      count++;
      if (m.analysis < 0 || m.analysis > 2) { fail("provided analysis flag does not match any possible value"); ok = false; break; }
    } else if (!strcmp(tok, "%type_of_solver")) {
      int v; if (fscanf(f, "%d", &v) != 1) break;
      m.solver_flag = v; g_solver = v; count++;
    } else if (!strcmp(tok, "%voxel_size")) {
      if (fscanf(f, "%lf", &m.voxel) != 1) break;
      count++;
    } else if (!strcmp(tok, "%solver_tolerance")) {
      if (fscanf(f, "%lf", &tolbuf) != 1) break;
      m.tol = tolbuf; count++;
    } else if (!strcmp(tok, "%number_of_iterations")) {
      if (fscanf(f, "%u", &m.maxit) != 1) break;
      count++;
    } else if (!strcmp(tok, "%image_dimensions")) {
      if (fscanf(f, "%d %d %d", &nx, &ny, &nz) != 3) break;
      count++;
    } else if (!strcmp(tok, "%refinement")) {
      if (fscanf(f, "%u", &m.refinement) != 1) break;
      count++;
      if (m.refinement < 1) { fail("refinement must be >= 1"); ok = false; break; }
    } else if (!strcmp(tok, "%number_of_materials")) {
      if (fscanf(f, "%u", &m.nmat) != 1) break;
      count++;
      if (m.nmat > 256) { fail("too many materials"); ok = false; break; }
    } else if (!strcmp(tok, "%properties_of_materials")) {
      for (unsigned i = 0; i < m.nmat; i++) {
        int id = -1;
        if (m.analysis == ELASTIC) { if (fscanf(f, "%d %lf %lf", &id, &m.props[2 * i], &m.props[2 * i + 1]) != 3) break; }
        else if (m.analysis == THERMAL) { if (fscanf(f, "%d %lf", &id, &m.props[i]) != 2) break; }
        else { if (fscanf(f, "%d", &id) != 1) break; }
        count++;
        if (id < 0 || id > 255) { fail("material colour key must be 0..255"); ok = false; break; }
        m.props_keys[id] = (int)i;
      }
      if (!ok) break;
    } else if (!strcmp(tok, "%thermal_expansion")) {
      if (m.analysis == ELASTIC) {
        for (unsigned i = 0; i < m.nmat; i++) if (fscanf(f, "%lf", &m.alpha[i]) != 1) break;
        m.has_thermal_expansion = true;
      }
    } else if (!strcmp(tok, "%data_type")) {  // femhmg.c:1550-1561
      char buf[64]; if (fscanf(f, "%63s", buf) != 1) break;
      count++;
      m.data_type = (!strcmp(buf, "float64") || !strcmp(buf, "double")) ? 1 : 0;
    } else if (!strcmp(tok, "%xreduce_scale_factor")) {
      double v; if (fscanf(f, "%lf", &v) != 1) break;
      m.xreduce_stab = v;
      count++;
    }
  }
  fclose(f);
  if (!ok) return false;
  if (nx <= 0 || ny <= 0) { fail("%image_dimensions missing or invalid"); return false; }
  if (nz < 0) { fail("%image_dimensions missing or invalid"); return false; }
  m.dim2 = nz == 0;  // femhmg.c:1496-1504: zero layers make a 2D (pixel) model
  if (m.analysis < 0) { fail("%type_of_analysis missing"); return false; }
  if (m.nmat == 0) { fail("no materials"); return false; }
  if (m.refinement > 1) m.voxel /= m.refinement;
  // femhmg.c:1583-1584: the x-reduce stabilisation factor defaults to tol^2, or 1e-12 below 5e-7
  if (m.xreduce_stab < 0) m.xreduce_stab = m.tol >= 0.0000005 ? m.tol * m.tol : 0.000000000001;
  m.nx = (unsigned)nx * m.refinement; m.ny = (unsigned)ny * m.refinement; m.nz = m.dim2 ? 1u : (unsigned)nz * m.refinement;
  return true;
}

// ---- image (femhmg.c:1644-1758) -------------------------------------------------------
// The image's colour bytes (file order, x fastest), checked against the .nf material list.
bool read_colors(Model& m, const uint8_t* data, const char* raw) {
  const unsigned ref = m.refinement;
  m.frows = m.ny / ref; m.fcols = m.nx / ref; m.fslices = m.dim2 ? 1u : m.nz / ref;
  const size_t nvox_file = (size_t)m.frows * m.fcols * m.fslices;
  m.colors.resize(nvox_file);
  if (data) {
    memcpy(m.colors.data(), data, nvox_file);
  } else {
    FILE* f = fopen(raw, "rb");
    if (!f) { fail(std::string("cannot open image ") + raw); return false; }
    size_t got = fread(m.colors.data(), 1, nvox_file, f);
    fclose(f);
    if (got < nvox_file) { fail("reached end of image file before expected"); return false; }
  }
  m.N = (long)m.nx * m.ny * m.nz;
  bool seen[256] = {false};
  const uint8_t* c = m.colors.data();
  for (size_t i = 0; i < nvox_file; i++) seen[c[i]] = true;
  for (int v = 0; v < 256; v++)
    if (seen[v] && m.props_keys[v] < 0) { fail("image holds colour " + std::to_string(v) + " that the .nf does not list"); return false; }
  return true;
}

// Voxel material map in the model's order (row fastest, refined) from the colours.
void build_elem_mat(Model& m) {
  const unsigned ref = m.refinement, rows = m.frows, cols = m.fcols, slices = m.fslices;
  m.elem_mat.assign(m.N, 0);
  const size_t R = m.ny, C = m.nx;
  const uint8_t* src = m.colors.data();
#pragma omp parallel for schedule(static)
  for (long k = 0; k < (long)slices; k++)
    for (size_t i = 0; i < rows; i++)
      for (size_t j = 0; j < cols; j++) {
        const int mat = m.props_keys[src[(size_t)k * rows * cols + i * cols + j]];  // x fastest in the file
        const unsigned kref = m.dim2 ? 1u : ref;  // a 2D image is refined in its plane only
        for (unsigned kk = kref * k; kk < kref * (k + 1); kk++)
          for (unsigned ii = ref * i; ii < ref * (i + 1); ii++)
            for (unsigned jj = ref * j; jj < ref * (j + 1); jj++) m.elem_mat[ii + jj * R + (size_t)kk * R * C] = (uint16_t)mat;
      }
}

// Scalar density field (femhmg.c:1760-1835): the file holds float32 or float64 values (as
// %data_type says), x fastest; each value times its voxel's conductivity (thermal) or Young's
// modulus (elastic) is quantised to 16 bits between the smallest and largest product, and the
// properties are then normalised (thermal: one material of conductivity 1; elastic: E = 1,
// Poisson's ratios kept), so that voxel e's element matrix is scale_e times the normalised one.
// As the reference: the file must hold as many values as the refined model has voxels (only the
// image's count is used), the range pairs value i with the material of the model's voxel i, and
// a voxel's product reads the material at model index (row + col R + layer R C) x refinement.
bool read_density_field(Model& m, const char* fn) {
  const unsigned ref = m.refinement, rows = m.frows, cols = m.fcols, slices = m.fslices;
  const size_t R = m.ny, C = m.nx, N = (size_t)m.N, nfile = (size_t)rows * cols * slices;
  const size_t sz = m.data_type ? 8 : 4;
  const size_t lref = m.dim2 ? 1 : ref;  // a 2D image has one layer
  std::vector<unsigned char> raw(sz * N);
  FILE* f = fopen(fn, "rb");
  if (!f) { fail(std::string("failed to open ") + fn); return false; }
  const size_t got = fread(raw.data(), sz, N, f);
  fclose(f);
  if (got < N) { fail(std::string("failed to read the scalar density field from ") + fn); return false; }
  auto value = [&](size_t i) -> double {
    if (m.data_type) { double v; memcpy(&v, raw.data() + 8 * i, 8); return v; }
    float v; memcpy(&v, raw.data() + 4 * i, 4); return (double)v;
  };
  const int stride = m.analysis == ELASTIC ? 2 : 1;
  build_elem_mat(m);
  double vmax = value(0) * m.props[m.elem_mat[0] * stride], vmin = vmax;
  for (size_t i = 1; i < nfile; i++) {
    const double v = value(i) * m.props[m.elem_mat[i] * stride];
    vmax = v > vmax ? v : vmax;
    vmin = v < vmin ? v : vmin;
  }
  if (vmax == vmin) vmin = vmax - 1.0;
  const double dv = vmax - vmin;
  m.sdf_range[0] = vmin;
  m.sdf_range[1] = vmax;
  m.sdf.assign(N, 0);
  for (size_t k = 0; k < slices; k++)
    for (size_t i = 0; i < rows; i++)
      for (size_t j = 0; j < cols; j++) {
        const double v = value(j + i * cols + k * rows * cols) * m.props[m.elem_mat[(i + j * R + k * R * C) * ref] * stride];
        const uint16_t q = (uint16_t)(65535 * (v - vmin) / dv);
        for (size_t kk = lref * k; kk < lref * (k + 1); kk++)
          for (size_t ii = ref * i; ii < ref * (i + 1); ii++)
            for (size_t jj = ref * j; jj < ref * (j + 1); jj++) m.sdf[ii + jj * R + kk * R * C] = q;
      }
  if (m.analysis == THERMAL) {  // one material of conductivity 1 (femhmg.c:256-262)
    for (int c = 0; c < 256; c++) if (m.props_keys[c] >= 0) m.props_keys[c] = 0;
    m.nmat = 1;
    m.props[0] = 1.0;
    build_elem_mat(m);
  } else {
    for (unsigned j = 0; j < m.nmat; j++) m.props[2 * j] = 1.0;
  }
  return true;
}

// The host maps of a thermal / elastic model, for the paths that read them (one-by-one
// right-hand sides and tensor updates, coarse levels, EBE input, the model-array hooks).
bool ensure_host_maps(Model& m) {
  if (m.host_maps) return true;
  build_elem_mat(m);
  std::string err;
  if (!build_maps(m, err)) { fail(err); return false; }
  m.host_maps = true;
  return true;
}

// cudapcg model constructor (femhmg.c:54-85)
cudapcgFlag_t model_ctor(cudapcgModel_t** ptr, const void* data) {
  if (!data) return CUDAPCG_FALSE;
  const Model& m = *(const Model*)data;
  cudapcgModel_t* p = *ptr;
  p->name = (char*)malloc(m.nf_noext.size() + 1);
  strcpy(p->name, m.nf_noext.c_str());
  p->parStrategy_flag = (cudapcgFlag_t)g_par;
  p->poremap_flag = (cudapcgFlag_t)g_poremap;
  p->parametric_density_field_flag = m.sdf.empty() ? 0 : 1;  // femhmg.c:67
  p->nrows = m.ny; p->ncols = m.nx; p->nlayers = m.dim2 ? 0 : m.nz;
  p->nelem = (unsigned)m.N;
  p->nvars = (unsigned)m.ndof;
  p->nvarspernode = 3;
  p->nkeys = m.analysis == FLUID ? 1 : m.nmat;
  p->localmtxdim = m.dim2 ? (m.analysis == THERMAL ? 16 : (m.analysis == ELASTIC ? 64 : 144))
                          : (m.analysis == THERMAL ? 40 : (m.analysis == ELASTIC ? 576 : 1024));
  p->nporenodes = (unsigned)m.nV;
  p->nbordernodes = (unsigned)m.nB;
  p->nhmgvars = m.analysis == FLUID ? (unsigned)((m.dim2 ? 2 : 3) * m.nV) : (unsigned)m.ndof;
  return CUDAPCG_TRUE;
}

int pcg_flag_of(const Model& m) {
  if (m.dim2) return m.analysis == THERMAL ? CUDAPCG_THERMAL_2D : (m.analysis == ELASTIC ? CUDAPCG_ELASTIC_2D : CUDAPCG_FLUID_2D);
  return m.analysis == THERMAL ? CUDAPCG_THERMAL_3D : (m.analysis == ELASTIC ? CUDAPCG_ELASTIC_3D : CUDAPCG_FLUID_3D);
}

const char* DIR_STR[6] = {"X", "Y", "Z", "YZ (shear)", "XZ (shear)", "XY (shear)"};

// The model coarsened by 2 per axis for the recursive initial-guess search
// (femhmg.c:1844-1916): floor(n/2) voxels per axis (a 2D image keeps its one layer), voxel
// (r,c,l) takes the material of fine voxel (2r,2c,2l); same voxel size, materials and local
// matrices.  nullptr when an axis would vanish.
Model* coarse_copy(const Model& f) {
  if (f.nx < 2 || f.ny < 2 || (!f.dim2 && f.nz < 2)) return nullptr;
  Model* c = new Model();
  c->dim2 = f.dim2;
  c->analysis = f.analysis; c->solver_flag = f.solver_flag; c->voxel = f.voxel; c->tol = f.tol; c->maxit = f.maxit;
  c->refinement = f.refinement; c->nmat = f.nmat;
  memcpy(c->props, f.props, sizeof(f.props));
  memcpy(c->props_keys, f.props_keys, sizeof(f.props_keys));
  memcpy(c->alpha, f.alpha, sizeof(f.alpha));
  c->has_thermal_expansion = f.has_thermal_expansion;
  c->nf = f.nf; c->nf_noext = f.nf_noext; c->raw = f.raw;
  c->nd = f.nd; c->C_dim = f.C_dim;
  c->nx = f.nx / 2; c->ny = f.ny / 2; c->nz = f.dim2 ? 1u : f.nz / 2;
  c->N = (long)c->nx * c->ny * c->nz;
  c->elem_mat.assign(c->N, 0);
  const long fR = f.ny, fRC = (long)f.ny * f.nx, R = c->ny, RC = (long)c->ny * c->nx;
  for (long l = 0; l < (long)c->nz; l++)
    for (long col = 0; col < (long)c->nx; col++)
      for (long r = 0; r < R; r++) c->elem_mat[r + col * R + l * RC] = f.elem_mat[2 * r + 2 * col * fR + 2 * l * fRC];
  std::string err;
  if (!build_maps(*c, err)) { delete c; return nullptr; }
  c->host_maps = true;
  c->lcl = f.lcl; c->CB = f.CB; c->Kdense = f.Kdense;
  return c;
}

// coarse: a level of the recursive initial-guess search, which solves with CG or MINRES and the
// L2 stopping test whatever the main settings (femhmg.c:708-714)
bool setup_solver(Model& m, bool coarse = false) {
  if (!cudapcgInit((cudapcgFlag_t)pcg_flag_of(m), (cudapcgFlag_t)g_par)) { fail(std::string("cudapcgInit: ") + cudapcgB200LastError()); return false; }
  cudapcgSetHeaderString((char*)"    | ");
  cudapcgSetModelConstructorFcn(model_ctor);
  // femhmg.c:919-926: reduction of the 2-vector solvers, its scale h^2 / nelem and factor
  cudapcgSetXReduceMode((cudapcgFlag_t)g_xreduce);
  cudapcgSetXReduceScale((m.voxel * m.voxel) / (double)m.N);
  cudapcgSetReduceStabFactor(m.xreduce_stab);
  if (!cudapcgBuildModel(&m)) { fail(std::string("cudapcgBuildModel: ") + cudapcgB200LastError()); return false; }
  const int solver = coarse ? ((g_solver & 1) ? CUDAPCG_MINRES_SOLVER : CUDAPCG_CG_SOLVER) : g_solver;
  if (!cudapcgSetSolver((cudapcgFlag_t)solver)) { fail(std::string("cudapcgSetSolver: ") + cudapcgB200LastError()); return false; }
  cudapcgSetPreconditioner((cudapcgFlag_t)g_precond);
  cudapcgSetResNorm((cudapcgFlag_t)(coarse ? 0 : g_stopcrit));
  cudapcgSetNumTol(m.tol);
  cudapcgSetMaxIterations(m.maxit);
  cudapcgB200SetPrecision(g_precision);
  bool ok;
  if (m.analysis != FLUID) {
    // femhmg.c:1000-1004: node keys for NBN, the per-voxel material map for EBE; without host
    // maps the device builds the keys from the colours
    if (g_par == CUDAPCG_NBN && !m.host_maps && !m.dim2) {
      int lut[256];
      for (int c = 0; c < 256; c++) lut[c] = m.props_keys[c];
      ok = cudapcgB200SetImageColors(m.colors.data(), m.frows, m.fcols, m.fslices, m.refinement, lut);
    } else {
      ok = ensure_host_maps(m) && cudapcgSetImage(g_par == CUDAPCG_EBE ? m.elem_mat.data() : m.keys.data());
    }
  } else if (g_poremap == CUDAPCG_POREMAP_IMG) {
    // femhmg.c:962-965: the node->DOF map and every node's fluid key (image pore map)
    ok = ensure_host_maps(m) && cudapcgSetPeriodic2DOFMap(m.dof_of_node.data()) && cudapcgSetPoreMap(m.fluid_keys.data());
  } else if (!m.host_maps) {
    int lut[256];
    for (int c = 0; c < 256; c++) lut[c] = m.props_keys[c];
    unsigned nv = 0, nb = 0;
    ok = cudapcgB200SetPoreImageColors(m.colors.data(), m.frows, m.fcols, m.fslices, m.refinement, lut, &nv, &nb);
    if (ok && ((long)nv != m.nV || (long)nb != m.nB)) {
      fail("device DOF numbering disagrees with the host's counts");
      return false;
    }
  } else {
    ok = cudapcgSetPeriodic2DOFMap(m.dof_of_node.data()) && cudapcgSetPoreMap(m.border_keys.data()) &&
         cudapcgSetDOF2PeriodicMap(m.node_of_dof.data());
  }
  ok = ok && cudapcgSetLclMtxs(m.lcl.data()) && cudapcgAllocateArrays();
  if (ok && !m.sdf.empty()) ok = cudapcgSetParametricDensityField(m.sdf.data(), m.sdf_range[0], m.sdf_range[1]);  // femhmg.c:971-976
  if (!ok) { fail(std::string("model upload: ") + cudapcgB200LastError()); return false; }
  return true;
}

}  // namespace

// =======================================================================================
extern "C" {

logical hmgInit(char* data_filename, char* elem_filename, char* sdf_filename, uint8_t* data) {
  const auto t0 = std::chrono::steady_clock::now();
  hmgEnd();
  g_err.clear();
  if (!data_filename) { fail("no .nf file"); return 0; }
  SAY("Initializing femhmg...\n");
  Model* m = new Model();
  m->nf = data_filename;
  m->nf_noext = m->nf.size() > 3 ? m->nf.substr(0, m->nf.size() - 3) : m->nf;
  if (elem_filename) m->raw = elem_filename;
  if (!read_nf(*m, data_filename)) { delete m; return 0; }
  if (!data) {
    if (!elem_filename) { fail("no image"); delete m; return 0; }
    const size_t L = strlen(elem_filename);
    if (L < 4 || strcmp(elem_filename + L - 4, ".raw")) { fail(std::string("file ") + elem_filename + " is not in a valid format (.raw)"); delete m; return 0; }
  }
  m->nd = m->analysis == ELASTIC ? (m->dim2 ? 2 : 3) : 1;
  m->C_dim = (unsigned)(tensor_dim(*m) * tensor_dim(*m));
  if (!read_colors(*m, data, elem_filename)) { delete m; return 0; }
  if (m->dim2) {
    // 2D: the node keys (4 bits per pixel) or the Stokes DOF numbering are built on the host
    if (sdf_filename && m->analysis != FLUID && !read_density_field(*m, sdf_filename)) { delete m; return 0; }
    if (!ensure_host_maps(*m)) { delete m; return 0; }
  } else if (m->analysis == FLUID) {
    // the sizes of the DOF numbering here; the numbering itself on the device at upload
    // (cudapcgB200SetPoreImageColors), or on the host for the paths that read the maps
    build_elem_mat(*m);
    std::string err;
    if (!count_pore_nodes(*m, err)) { fail(err); delete m; return 0; }
  } else {
    // the node keys are built on the device from the colours (cudapcgB200SetImageColors)
    if (m->nmat > 4) { fail("more than 4 materials cannot be encoded in 16-bit node keys"); delete m; return 0; }
    m->ndof = m->N * m->nd;
    if (sdf_filename && !read_density_field(*m, sdf_filename)) { delete m; return 0; }
  }
  if (sdf_filename && m->analysis == FLUID) SAY("WARNING: Scalar density field input is not supported for permeability analysis.\n");
  build_local_matrices(*m);
  g_m = m;
  g_dir_set = 0;
  g_use_x0 = false; g_x0_file.clear(); g_export_x = false; g_export_fields = false;
  for (auto& v : g_x0_coarse) v.clear();
  g_have_coarse = false;
  const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  SAY("Done.(%.2e s)\n", t);
  return 1;
}

logical hmgEnd(void) {
  if (!g_m) return 0;
  delete g_m;
  g_m = nullptr;
  cudapcgEnd();
  return 1;
}

void hmgSetParallelStrategyFlag(uint8_t flag) { g_par = flag ? CUDAPCG_EBE : CUDAPCG_NBN; }
void hmgSetSolverFlag(uint8_t flag) { g_solver = flag; }
void hmgSetXReduceFlag(uint8_t flag) { g_xreduce = flag <= CUDAPCG_XREDUCE_FULL ? flag : CUDAPCG_XREDUCE_FULL; }
void hmgSetPreConditionerFlag(uint8_t flag) { g_precond = flag > 0; }
void hmgSetStoppingCriteria(uint8_t flag) { g_stopcrit = flag; }
logical hmgSetPoreMappingStrategy(uint8_t flag) {
  if (flag > CUDAPCG_POREMAP_NUM) return 1;  // femhmg.c:484: out-of-range flags are ignored
  g_poremap = flag;
  return 1;
}
void hmgExportX(logical flag) { g_export_x = flag > 0; }
void hmgImportX(char* file) {
  if (!g_m) return;
  g_x0_file = file ? file : "";
  g_use_x0 = true;
}
void hmgFindInitialGuesses(unsigned int nlevels) {
  g_recursions = (int)nlevels;
  for (auto& v : g_x0_coarse) v.clear();
  g_have_coarse = false;
  if (!nlevels || !g_m) return;
  Model& fine = *g_m;
  if (fine.analysis == FLUID) {  // femhmg.c:565-570
    SAY("WARNING: Initial guess estimation is not yet available for permeability analysis.\n");
    SAY("         Null initial guess will be considered (x0 = [0]).\n");
    return;
  }
  if (!fine.sdf.empty()) {  // femhmg.c:572-577 (a coarse level would need a coarsened field)
    SAY("WARNING: Initial guess estimation is not yet available for analyses with a scalar field input (.bin).\n");
    SAY("         Null initial guess will be considered (x0 = [0]).\n");
    return;
  }
  if (!ensure_host_maps(fine)) return;
  // coarse meshes: every second voxel of the finer level (femhmg.c:1844-1916)
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<Model*> levels{&fine};
  for (unsigned i = 0; i < nlevels; i++) {
    Model* c = coarse_copy(*levels.back());
    if (!c) {
      SAY("WARNING: the image cannot be coarsened %u times; using %u coarse levels.\n", nlevels, i);
      break;
    }
    levels.push_back(c);
  }
  SAY("Building coarse meshes...[%zu/%u] (%.2e s)\n", levels.size() - 1, nlevels,
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
  int dirs[6], nd = 0;
  if (g_dir_set) dirs[nd++] = g_dir;
  else { nd = load_case_count(fine); load_case_list(fine, dirs); }
  // from the coarsest level up: each level starts from the prolonged solution of the one below
  std::vector<double> prev[6];
  bool have_prev = false;
  for (size_t li = levels.size() - 1; li >= 1; li--) {
    Model& m = *levels[li];
    SAY("Computing initial guesses in coarse mesh %zu...\n", li);
    if (!setup_solver(m, true)) { cudapcgEnd(); break; }
    std::vector<double> rhs(m.ndof), x(m.ndof);
    std::vector<double> cur[6];
    for (int k = 0; k < nd; k++) {
      SAY("    ------------------------------------------------------\n    Finding initial guess on %s:\n    Mesh dimension: [%u,%u,%u] elements\n",
          DIR_STR[dirs[k]], m.nx, m.ny, m.nz);
      assemble_rhs(m, dirs[k], rhs.data());
      cudapcgSetRHS(rhs.data());
      if (have_prev && !prev[dirs[k]].empty()) cudapcgSetX0(prev[dirs[k]].data(), 1);
      else cudapcgSetX0(nullptr, 0);
      const bool found = cudapcgSolve(x.data()) != 0;
      if (!g_quiet) cudapcgPrintSolverMetrics();
      if (found) cur[dirs[k]] = x;  // femhmg.c:787-801: only a converged solution is passed up
    }
    cudapcgFreeArrays();
    cudapcgSetX0(nullptr, 0);
    cudapcgEnd();
    for (int d = 0; d < 6; d++) prev[d].swap(cur[d]);
    have_prev = true;
    if (li == 1) break;
  }
  for (size_t li = 1; li < levels.size(); li++) delete levels[li];
  if (have_prev) {
    for (int d = 0; d < 6; d++) g_x0_coarse[d].swap(prev[d]);
    g_have_coarse = true;
  }
  SAY("Done.(%.2e s)\n", std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
}
void hmgSetHomogenizationFlag(hmgFlag_t flag) {
  if (!g_m) return;
  const int maxdir = g_m->analysis == ELASTIC ? 5 : (g_m->dim2 ? 1 : 2);
  if (flag > maxdir) { g_dir_set = 0; return; }
  if (g_m->dim2 && g_m->analysis == ELASTIC && flag > 1 && flag != 5) { g_dir_set = 0; return; }  // femhmg.c:536-541
  g_dir_set = 1;
  g_dir = flag;
}

void hmgSolveHomogenization(void) {
  if (!g_m) return;
  Model& m = *g_m;
  if (!m.sdf.empty() && m.has_thermal_expansion) {
    fail("thermal expansion is not provided with a scalar density field");
    return;
  }
  const auto t_all = std::chrono::steady_clock::now();
  memset(&g_stats, 0, sizeof(g_stats));
  int dirs[6], nd = 0;
  if (g_dir_set) dirs[nd++] = g_dir;
  else { nd = load_case_count(m); load_case_list(m, dirs); }
  for (unsigned i = 0; i < m.C_dim; i++) m.C[i] = 0.0;
  if (m.analysis != FLUID && g_solver > CUDAPCG_MINRES3_SOLVER) {  // femhmg.c:852-856
    SAY("WARNING: CG2 and MINRES2 are only available for FLUID.\n");
    SAY("         Defaulting to %s.\n", g_solver == CUDAPCG_CG2_SOLVER ? "CG3" : "MINRES3");
    g_solver = g_solver == CUDAPCG_CG2_SOLVER ? CUDAPCG_CG3_SOLVER : CUDAPCG_MINRES3_SOLVER;
  }
  // the 2-vector solvers never form the solution: its exports have nothing to write
  const bool two_vector = g_solver >= CUDAPCG_CG2_SOLVER;
  if (two_vector && (g_export_fields || g_export_x))
    SAY("WARNING: the 2-vector solvers (CG2/MINRES2) reduce the solution on the fly; fields and x are not exported.\n");
  SAY("Running homogenization...\n");
  {
    const auto ts = std::chrono::steady_clock::now();
    if (!setup_solver(m)) return;
    g_stats.setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
  }
  std::vector<double> x, x0;
  g_stats.n_cases = nd;
  g_stats.ndof = (unsigned)m.ndof;
  // Block multi-RHS path: all load cases of the analysis advance together (one operator pass
  // per iteration for all of them).  Same per-case recurrence, stopping test and results.
  // (a scalar density field runs the one-by-one host path: right-hand sides and tensor terms
  // scaled per voxel on the host)
  const bool block = g_multirhs && !two_vector && m.sdf.empty() && !m.dim2 && ((m.analysis != FLUID && !(g_solver & 1) &&
                                     ((m.analysis == THERMAL && nd == 3) || (m.analysis == ELASTIC && (nd == 6 || nd == 3)))) ||
                                    (m.analysis == FLUID && (g_solver & 1) && nd == 3));
  if (block) {
    // right-hand sides and the effective-tensor volume term on the device
    // (cudapcgB200SolveLoadCases); x comes back only to be exported
    const bool want_x = g_export_x || g_export_fields;
    std::vector<std::vector<double>> xs(want_x ? nd : 0, std::vector<double>(m.ndof)), x0s(nd);
    std::vector<const double*> px0(nd, nullptr);
    std::vector<double*> px(nd, nullptr);
    int axis[6], comp[6];
    double jump[6], volume[36];
    for (int k = 0; k < nd; k++) {
      case_axis(m, dirs[k], axis[k], comp[k]);
      jump[k] = (double)axis_len(m, axis[k]);
      if (want_x) px[k] = xs[k].data();
      if (g_use_x0 && !g_x0_file.empty()) {
        const std::string fn = g_x0_file + "_" + std::to_string(dirs[k]) + ".bin";
        FILE* f = fopen(fn.c_str(), "rb");
        if (f) {
          x0s[k].assign(m.ndof, 0.0);
          if (fread(x0s[k].data(), sizeof(double), m.ndof, f) < (size_t)m.ndof) SAY("WARNING: Failed to read all %ld items from %s...", m.ndof, fn.c_str());
          fclose(f);
          px0[k] = x0s[k].data();
        }
      } else if (g_x0_user[dirs[k]]) {
        px0[k] = g_x0_user[dirs[k]];
      } else if (g_have_coarse && !g_x0_coarse[dirs[k]].empty()) {
        px0[k] = g_x0_coarse[dirs[k]].data();
      }
    }
    bool any_user = false;
    for (int k = 0; k < nd; k++) any_user = any_user || g_x0_user[dirs[k]];
    const int interp = (g_use_x0 && !g_x0_file.empty()) ? 0 : (any_user ? (g_x0_user_device ? 2 : 0) : (g_have_coarse ? 1 : 0));
    const unsigned ns = m.analysis == ELASTIC ? 6 : 3;
    SAY("    ------------------------------------------------------\n    Block solve of %d load cases (", nd);
    for (int k = 0; k < nd; k++) SAY("%s%s", k ? ", " : "", DIR_STR[dirs[k]]);
    SAY(")...\n");
    unsigned its[6] = {0};
    double res[6] = {0};
    const auto tc = std::chrono::steady_clock::now();
    const bool solved = cudapcgB200SolveLoadCases((unsigned)nd, axis, comp, jump, m.CB.data(), ns, px0.data(), interp, volume, px.data(), its, res);
    g_stats.solve_call_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - tc).count();
    if (!solved && cudapcgB200LastError()[0]) {
      fail(std::string("block solve: ") + cudapcgB200LastError());
      cudapcgEnd();
      return;
    }
    cudapcgB200Stats st;
    cudapcgB200GetStats(&st);
    for (int k = 0; k < nd; k++) {
      const int dir = dirs[k];
      g_stats.direction[k] = dir;
      g_stats.iterations[k] = its[k];
      g_stats.residual[k] = res[k];
      g_stats.solve_seconds[k] = (k == 0) ? st.solve_seconds + st.setup_seconds : 0.0;
      if (g_export_x) {
        const std::string fn = m.nf_noext + "_X_" + std::to_string(dir) + ".bin";
        FILE* f = fopen(fn.c_str(), "wb");
        if (f) { fwrite(xs[k].data(), sizeof(double), m.ndof, f); fclose(f); }
      }
      if (g_export_fields) export_fields(m, dir, xs[k].data(), k);
      const auto t = std::chrono::steady_clock::now();
      update_C_from_volume(m, dir, volume + ns * k);
      g_stats.update_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
    }
    g_stats.kernel_launches += st.kernel_launches;
    if (!g_quiet) cudapcgPrintSolverMetrics();
  }
  // One-by-one path: right-hand side, solution and tensor volume term stay on the device unless
  // x must come back to the host (-xo, -e: the solution files are written from it).
  const bool on_device = !g_export_x && !g_export_fields && m.sdf.empty() && !m.dim2;
  if (!block) {  // host vectors (and, for the host path, maps) of the one-by-one path
    if (!on_device && !ensure_host_maps(m)) { cudapcgEnd(); return; }
    m.rhs.assign(on_device ? 0 : m.ndof, 0.0);
    x.assign(on_device ? 3 : m.ndof, 0.0);  // 3: the 2-vector solvers' reduced sums
  }
  for (int k = 0; k < nd && !block; k++) {
    const int dir = dirs[k];
    SAY("    ------------------------------------------------------\n    Analysis on %s:\n", DIR_STR[dir]);
    auto t = std::chrono::steady_clock::now();
    int axis = dir, comp = 0;
    if (m.analysis != FLUID) case_axis(m, dir, axis, comp);
    if (on_device) {
      if (!cudapcgB200SetLoadCaseRHS(axis, comp, (double)axis_len(m, axis), m.CB.data())) {
        fail(std::string("right-hand side: ") + cudapcgB200LastError());
        cudapcgEnd();
        return;
      }
    } else {
      assemble_rhs(m, dir, m.rhs.data());
      cudapcgSetRHS(m.rhs.data());
    }
    g_stats.rhs_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
    if (g_use_x0 && !g_x0_file.empty()) {  // femhmg.c:1047-1067: <prefix>_<dir>.bin
      const std::string fn = g_x0_file + "_" + std::to_string(dir) + ".bin";
      FILE* f = fopen(fn.c_str(), "rb");
      if (!f) { SAY("    | Reading initial guess from %s...Failed!...\n", fn.c_str()); cudapcgSetX0(nullptr, 0); }
      else {
        x0.assign(m.ndof, 0.0);
        if (fread(x0.data(), sizeof(double), m.ndof, f) < (size_t)m.ndof) SAY("WARNING: Failed to read all %ld items from %s...", m.ndof, fn.c_str());
        fclose(f);
        cudapcgSetX0(x0.data(), 0);
      }
    } else if (g_x0_user[dir]) {
      if (g_x0_user_device) cudapcgB200SetX0Device(g_x0_user[dir]);
      else cudapcgSetX0((double*)g_x0_user[dir], 0);
    } else if (g_have_coarse) {  // femhmg.c:1048-1050: the recursive guess, prolonged
      if (!g_x0_coarse[dir].empty()) { SAY("    | Interpolating initial guess...\n"); cudapcgSetX0(g_x0_coarse[dir].data(), 1); }
      else cudapcgSetX0(nullptr, 0);
    } else {
      cudapcgSetX0(nullptr, 0);  // no guess for this case: not the previous case's
    }
    SAY("    Solving system of equations...\n");
    if (two_vector) cudapcgSetXReduceShift(dir <= 2 ? dir : 0);  // femhmg.c:1068
    const auto tc = std::chrono::steady_clock::now();
    cudapcgSolve(on_device && !two_vector ? nullptr : x.data());
    g_stats.solve_call_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - tc).count();
    if (!g_quiet) cudapcgPrintSolverMetrics();
    cudapcgB200Stats st;
    cudapcgB200GetStats(&st);
    g_stats.direction[k] = dir;
    g_stats.iterations[k] = st.iterations;
    g_stats.residual[k] = st.residual;
    g_stats.solve_seconds[k] = st.solve_seconds;
    g_stats.kernel_launches += st.kernel_launches;
    if (two_vector) {  // femhmg.c:1087-1094: the reduced sums are the column of C
      SAY("    Effective fields:\n");
      const int D = tensor_dim(m);  // 3, or 2 on a 2D image
      for (int jj = 0; jj < D; jj++) {
        SAY("        %.8e\n", x[jj]);
        m.C[jj * D + dir] = x[jj];
      }
      if (g_report) {
        char buf[512];
        snprintf(buf, sizeof(buf), "Analysis on %s: %u iterations, residual %.3e, solver time %.3e s\n", DIR_STR[dir], st.iterations, st.residual, st.solve_seconds);
        g_report_text += buf;
      }
      continue;
    }
    if (g_export_fields) export_fields(m, dir, x.data(), -1);
    if (g_export_x) {  // femhmg.c:1077-1084
      const std::string fn = m.nf_noext + "_X_" + std::to_string(dir) + ".bin";
      FILE* f = fopen(fn.c_str(), "wb");
      if (f) { fwrite(x.data(), sizeof(double), m.ndof, f); fclose(f); }
    }
    t = std::chrono::steady_clock::now();
    if (on_device) {  // the volume term reduced on the device, the face term here
      double volume[6];
      const unsigned ns = m.analysis == ELASTIC ? 6 : 3;
      if (!cudapcgB200VolumeTerm(m.CB.data(), ns, volume)) {
        fail(std::string("tensor update: ") + cudapcgB200LastError());
        cudapcgEnd();
        return;
      }
      update_C_from_volume(m, dir, volume);
    } else {
      update_C(m, dir, x.data());
    }
    g_stats.update_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
    if (g_report) {
      char buf[512];
      snprintf(buf, sizeof(buf), "Analysis on %s: %u iterations, residual %.3e, solver time %.3e s\n", DIR_STR[dir], st.iterations, st.residual, st.solve_seconds);
      g_report_text += buf;
    }
  }
  if (m.analysis == ELASTIC && m.has_thermal_expansion) {
    // femhmg.c:1121-1168: one more solve, under a unit temperature rise, after the load cases;
    // the effective expansion follows from its stress and the tensor just computed
    SAY("    ------------------------------------------------------\n    Thermal expansion analysis:\n");
    if (!ensure_host_maps(m)) { cudapcgEnd(); return; }
    std::vector<double> rhs(m.ndof);
    assemble_rhs_thermal_expansion(m, rhs.data());
    double volume[6];
    std::vector<double> xs(m.dim2 ? m.ndof : 0);  // 2D: the stress sums are taken on the host
    const bool ok = cudapcgSetRHS(rhs.data()) && cudapcgSetX0(nullptr, 0) &&
                    (cudapcgSolve(m.dim2 ? xs.data() : nullptr), true) &&
                    (m.dim2 || cudapcgB200VolumeTerm(m.CB.data(), 6, volume));
    if (!ok) { fail(std::string("thermal expansion: ") + cudapcgB200LastError()); cudapcgEnd(); return; }
    if (!g_quiet) cudapcgPrintSolverMetrics();
    if (m.dim2) update_thermal_expansion_2d(m, xs.data());
    else update_thermal_expansion(m, volume);
  }
  {
    const auto tt = std::chrono::steady_clock::now();
    cudapcgSetX0(nullptr, 0);
    cudapcgFreeArrays();
    cudapcgEnd();
    g_stats.teardown_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tt).count();
  }
  for (auto& p : g_x0_user) p = nullptr;  // used once
  g_stats.total_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_all).count();
  SAY("    ------------------------------------------------------\nDone.(%.2e s)\n", g_stats.total_seconds);
}

void hmgPrintModelData(void) {
  if (!g_m || g_quiet) return;
  const Model& m = *g_m;
  static const char* AN[6] = {"THERMAL_3D", "ELASTIC_3D", "FLUID_3D", "THERMAL_2D", "ELASTIC_2D", "FLUID_2D"};
  static const char* SO[6] = {"CG", "MINRES", "CG3", "MINRES3", "CG2", "MINRES2"};
  printf("*******************************************************\nMODEL DATA:\nAnalysis: %s\n", AN[m.analysis + (m.dim2 ? 3 : 0)]);
  printf("Number of voxels (x,y,z): [%u,%u,%u]\nNumber of voxels (total): %ld\n", m.nx, m.ny, m.nz, m.N);
  if (m.analysis == FLUID)
    printf("  | porosity: %05.2f%%\n  | within pores: %ld\n  | at interfaces: %ld\n", 100.0 * m.nporeelem / (double)m.N, m.nV, m.nB);
  printf("Number of DOFs: %ld\nNumber of materials: %u\nNumerical tolerance: %.3e\nMax iterations: %u\nSolver: %s%s\n",
         m.ndof, m.nmat, m.tol, m.maxit, g_precond ? "P" : "", SO[g_solver < 6 ? g_solver : 0]);
  if (g_solver >= CUDAPCG_CG2_SOLVER) printf("xreduce stab factor: %.2e\n", m.xreduce_stab);
  printf("Precision: %s\n*******************************************************\n", !g_precision ? "FP64" : (m.analysis == FLUID ? "FP64 (mixed precision is not used for Stokes)" : "mixed (FP32 fields, FP64 reductions)"));
}

void hmgPrintConstitutiveMtx(void) {
  if (!g_m) return;
  const Model& m = *g_m;
  static const char* NAME[3] = {"Thermal Conductivity", "Elasticity", "Permeability"};
  const int n = tensor_dim(m);
  printf("-------------------------------------------------------\nHomogenized Constitutive Matrix (%s):\n", NAME[m.analysis]);
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < n; j++) printf("  %.8e", m.C[i * n + j]);
    printf("\n");
  }
  printf("-------------------------------------------------------\n");
  if (m.analysis == ELASTIC && m.has_thermal_expansion) {  // femhmg_elastic_3D.c:1625-1631, femhmg_elastic_2D.c:754-759
    const double* a = m.thermal_expansion;
    printf("Effective thermal expansion:\n");
    if (m.dim2) printf("  %.8e  %.8e\n  %.8e  %.8e\n", a[0], a[2], a[2], a[1]);
    else printf("  %.8e  %.8e  %.8e\n  %.8e  %.8e  %.8e\n  %.8e  %.8e  %.8e\n", a[0], a[5], a[4], a[5], a[1], a[3], a[4], a[3], a[2]);
    printf("-------------------------------------------------------\n");
  }
}
var* hmgGetConstitutiveMtx(void) { return g_m ? g_m->C : nullptr; }
unsigned int hmgGetConstitutiveMtxDim(void) { return g_m ? g_m->C_dim : 0; }
var* hmgGetThermalExpansion(void) { return (g_m && g_m->analysis == ELASTIC && g_m->has_thermal_expansion) ? g_m->thermal_expansion : nullptr; }
unsigned int hmgGetThermalExpansionDim(void) { return hmgGetThermalExpansion() ? (g_m->dim2 ? 3 : 6) : 0; }  // femhmg.c:1341-1345
logical hmgSaveConstitutiveMtx(const char* filename) {
  if (!g_m) return 0;
  FILE* f = fopen(filename, "wb");
  if (!f) return 0;
  fwrite(g_m->C, sizeof(double), g_m->C_dim, f);
  if (hmgGetThermalExpansionDim()) fwrite(g_m->thermal_expansion, sizeof(double), hmgGetThermalExpansionDim(), f);  // femhmg.c:1362-1363
  fclose(f);
  return 1;
}
void hmgSaveFields(logical mustExport, logical) { g_export_fields = mustExport != 0; }
static int g_run_export_fields = 0;  // for the next chfemB200Run
void chfemB200SetExportFields(int on) { g_export_fields = on != 0; g_run_export_fields = on != 0; }
void hmgKeepTrackOfAnalysisReport(uint8_t flag) {
  g_report = flag != 0;
  if (g_report && g_m) g_report_text = "Neutral file: " + g_m->nf + "\nImage: " + g_m->raw + "\n";
}
uint8_t hmgPrintReport(const char* filename) {
  if (!g_report) return 0;
  if (!filename) { printf("%s", g_report_text.c_str()); return 1; }
  FILE* f = fopen(filename, "w");
  if (!f) return 0;
  fputs(g_report_text.c_str(), f);
  fclose(f);
  return 1;
}

// ---------------- extensions ----------------
void chfemB200SetPrecision(int mode) { g_precision = mode ? CHFEM_B200_PREC_MIXED : CHFEM_B200_PREC_FP64; }
void chfemB200SetMultiRHS(int on) { g_multirhs = on; }
void chfemB200SetQuiet(int quiet) {
  g_quiet = quiet;
  if (quiet) setenv("CHFEM_B200_QUIET", "1", 1); else unsetenv("CHFEM_B200_QUIET");
}
const char* chfemB200LastError(void) { return g_err.c_str(); }
int chfemB200GetSolveStats(chfemB200SolveStats* out) {
  if (!out) return 0;
  *out = g_stats;
  return 1;
}

int chfemB200SetInitialGuesses(int ncases, const double* const* x0, int on_device) {
  if (ncases < 0 || ncases > 6 || (ncases && !x0)) return 0;
  for (int k = 0; k < 6; k++) g_x0_user[k] = (k < ncases) ? x0[k] : nullptr;
  g_x0_user_device = on_device ? 1 : 0;
  return 1;
}

int chfemB200UpdateCFromVolume(int direction, const double* volume, double* C_out) {
  if (!g_m || !volume || !C_out) return 0;
  const int nd = load_case_count(*g_m);
  if (direction < 0 || direction >= nd) return 0;
  update_C_from_volume(*g_m, direction, volume);
  memcpy(C_out, g_m->C, sizeof(double) * g_m->C_dim);
  return 1;
}

static cudapcgB200BatchStats g_batch_stats;
int chfemB200LastBatchStats(cudapcgB200BatchStats* out) {
  if (!out) return 0;
  *out = g_batch_stats;
  return 1;
}

int chfemB200RunThermalBatch(unsigned int nsamples, const chfemB200ThermalSample* samples, double tol, unsigned int maxit,
                             int precision, double* C_out, unsigned int* iterations, double* solve_seconds) {
  g_err.clear();
  if (!nsamples || !samples || !C_out) { fail("chfemB200RunThermalBatch: null argument"); return 0; }
  for (unsigned s = 0; s < nsamples; s++) {
    const chfemB200ThermalSample& t = samples[s];
    if (!t.voxels || !t.nx || !t.ny || !t.nz) { fail("sample " + std::to_string(s) + ": empty image"); return 0; }
    if (t.nmat < 1 || t.nmat > 4) { fail("sample " + std::to_string(s) + ": 1 to 4 materials"); return 0; }
  }
  // per sample: voxel material map, node keys and element matrices (the host model layer)
  std::vector<Model> models(nsamples);
  std::vector<int> ok(nsamples, 1);
#pragma omp parallel for schedule(dynamic)
  for (long s = 0; s < (long)nsamples; s++) {
    const chfemB200ThermalSample& t = samples[s];
    Model& m = models[s];
    m.analysis = THERMAL; m.nd = 1; m.C_dim = 9; m.voxel = 1.0; m.refinement = 1; m.tol = tol; m.maxit = maxit;
    m.nx = t.nx; m.ny = t.ny; m.nz = t.nz; m.nmat = t.nmat;
    for (int c = 0; c < 256; c++) m.props_keys[c] = -1;
    for (unsigned k = 0; k < t.nmat; k++) { m.props_keys[t.colors[k]] = (int)k; m.props[k] = t.conductivity[k]; }
    std::string err;
    if (!read_colors(m, t.voxels, nullptr)) { ok[s] = 0; continue; }
    build_elem_mat(m);
    if (!build_maps(m, err)) { ok[s] = 0; continue; }
    m.host_maps = true;
    build_local_matrices(m);
  }
  for (unsigned s = 0; s < nsamples; s++)
    if (!ok[s]) { if (g_err.empty()) fail("sample " + std::to_string(s) + ": image holds a colour outside its list"); return 0; }
  std::vector<unsigned> dims(3 * nsamples), nmat(nsamples);
  std::vector<const uint16_t*> keys(nsamples);
  std::vector<const double*> K(nsamples), CB(nsamples);
  for (unsigned s = 0; s < nsamples; s++) {
    dims[3 * s] = models[s].ny; dims[3 * s + 1] = models[s].nx; dims[3 * s + 2] = models[s].nz;
    nmat[s] = models[s].nmat; keys[s] = models[s].keys.data(); K[s] = models[s].Kdense.data(); CB[s] = models[s].CB.data();
  }
  std::vector<double> moments(9 * (size_t)nsamples);
  cudapcgB200BatchStats& st = g_batch_stats;
  const int rc = cudapcgB200SolveThermalBatch(nsamples, dims.data(), keys.data(), nmat.data(), K.data(), CB.data(), tol, maxit,
                                              precision ? CHFEM_B200_MIXED : CHFEM_B200_FP64, 1, moments.data(), iterations,
                                              nullptr, &st);
  if (!rc) { fail(std::string("batch solve: ") + cudapcgB200BatchLastError()); return 0; }
  if (solve_seconds) *solve_seconds = st.setup_seconds + st.solve_seconds;
#pragma omp parallel for schedule(dynamic)
  for (long s = 0; s < (long)nsamples; s++) {
    Model& m = models[s];
    for (int dir = 0; dir < 3; dir++) update_C_from_volume(m, dir, moments.data() + 9 * s + 3 * dir);
    for (int t = 0; t < 9; t++) C_out[9 * s + t] = m.C[t];
  }
  return rc;
}

int chfemB200Run(const uint8_t* voxels, const char* nf, int direction, int solver, int precondition, int precision, int multirhs,
                 double* C_out) {
  if (!voxels || !nf || !C_out) { fail("chfemB200Run: null argument"); return 0; }
  g_solver = solver; g_precond = precondition > 0; g_precision = precision; g_multirhs = multirhs;
  const int export_fields = g_run_export_fields;
  g_run_export_fields = 0;
  if (!hmgInit((char*)nf, nullptr, nullptr, (uint8_t*)voxels)) return 0;
  g_export_fields = export_fields != 0;
  g_solver = solver;  // the .nf %type_of_solver is overridden by the caller, like chfem_wrapper.c:20-24
  if (direction < 6) hmgSetHomogenizationFlag((hmgFlag_t)direction);
  hmgPrintModelData();
  hmgSolveHomogenization();
  if (!g_err.empty()) return 0;
  const int n = tensor_dim(*g_m);
  memcpy(C_out, g_m->C, sizeof(double) * n * n);
  return n;
}

unsigned long long chfemB200ModelArraySize(int which) {
  if (!g_m || !ensure_host_maps(*g_m)) return 0;
  const Model& m = *g_m;
  switch (which) {
    case 0: return m.keys.size() * 2;
    case 1: return m.dof_of_node.size() * 4;
    case 2: return m.node_of_dof.size() * 4;
    case 3: return m.border_keys.size();
    case 4: return m.lcl.size() * 8;
    case 5: return m.rhs.size() * 8;
    case 6: return m.elem_mat.size() * 2;
    case 7: return m.CB.size() * 8;
    case 8: return m.sdf.size() * 2;
    case 9: return m.sdf.empty() ? 0 : 16;
  }
  return 0;
}
int chfemB200CopyModelArray(int which, void* dst, unsigned long long bytes) {
  if (!g_m || !dst) return 0;
  const Model& m = *g_m;
  const void* src = nullptr;
  switch (which) {
    case 0: src = m.keys.data(); break;
    case 1: src = m.dof_of_node.data(); break;
    case 2: src = m.node_of_dof.data(); break;
    case 3: src = m.border_keys.data(); break;
    case 4: src = m.lcl.data(); break;
    case 5: src = m.rhs.data(); break;
    case 6: src = m.elem_mat.data(); break;
    case 7: src = m.CB.data(); break;
    case 8: src = m.sdf.data(); break;
    case 9: src = m.sdf_range; break;  // min, max
    default: return 0;
  }
  const unsigned long long have = chfemB200ModelArraySize(which);
  memcpy(dst, src, bytes < have ? bytes : have);
  return 1;
}
int chfemB200AssembleRHS(int direction, double* dst) {
  if (!g_m || !dst || !ensure_host_maps(*g_m)) return 0;
  assemble_rhs(*g_m, direction, dst);
  return 1;
}
int chfemB200AssembleThermalExpansionRHS(double* dst) {
  if (!g_m || !dst || g_m->analysis != ELASTIC || !ensure_host_maps(*g_m)) return 0;
  assemble_rhs_thermal_expansion(*g_m, dst);
  return 1;
}
int chfemB200UpdateThermalExpansion(const double* x, const double* C, double* alpha_out) {
  if (!g_m || !x || !C || !alpha_out || g_m->analysis != ELASTIC || !ensure_host_maps(*g_m)) return 0;
  memcpy(g_m->C, C, sizeof(double) * g_m->C_dim);
  thermal_expansion_from_solution(*g_m, x);
  memcpy(alpha_out, g_m->thermal_expansion, sizeof(double) * (g_m->dim2 ? 3 : 6));
  return 1;
}
int chfemB200UpdateC(int direction, const double* x, double* C_out) {
  if (!g_m || !x || !ensure_host_maps(*g_m)) return 0;
  update_C(*g_m, direction, x);
  if (C_out) memcpy(C_out, g_m->C, sizeof(double) * g_m->C_dim);
  return 1;
}
int chfemB200ModelInfo(unsigned int* info) {
  if (!g_m || !info) return 0;
  const Model& m = *g_m;
  info[0] = m.nx; info[1] = m.ny; info[2] = m.nz; info[3] = (unsigned)m.N; info[4] = (unsigned)m.ndof;
  info[5] = (unsigned)m.nV; info[6] = (unsigned)m.nB; info[7] = m.nmat; info[8] = (unsigned)m.analysis;
  return 1;
}

}  // extern "C"
