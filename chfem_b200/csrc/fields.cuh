// fields.cuh -- exported fields of a solution: the nodal heat flux (thermal) or stress
// (elastic) that chfem writes with -e (chfem/src/femhmg/physical_phenomena/
// femhmg_thermal_3D.c:674-1111, femhmg_elastic_3D.c:1684-1760, :1800-2650).
//
// At each node, the field is the mean over the node's 8 voxels of the flux (k grad T) or stress
// (D(E, nu) B u) of that voxel evaluated at the node's own corner.  A voxel on the +axis
// boundary of the cell (last column for x, first row for y, first layer for z) sees the
// load case's macroscopic jump on its +axis face nodes.  The reference scatters each voxel's
// eight corner values into the nodes; here every node gathers its own eight, so there is no
// accumulation race and no atomic.
#pragma once
#include "common.cuh"
#include "loadcase.cuh"

namespace chfem {

struct FieldProps {
  double p[8];  // thermal: k per material; elastic: (E, nu) per material
};

// derivative of the trilinear shape function of local node j along axis i (0 x, 1 y, 2 z)
// at local point (px, py, pz); node j sits at (dcol(j), -drow(j), 1 - dlay(j)).
__device__ __forceinline__ double dshape(int j, int i, double px, double py, double pz) {
  const int xj = dcol(j), yj = -drow(j), zj = 1 - dlay(j);
  const double fx = xj ? px : 1.0 - px, fy = yj ? py : 1.0 - py, fz = zj ? pz : 1.0 - pz;
  const double sx = xj ? 1.0 : -1.0, sy = yj ? 1.0 : -1.0, sz = zj ? 1.0 : -1.0;
  return i == 0 ? sx * fy * fz : (i == 1 ? fx * sy * fz : fx * fy * sz);
}

// out[n * NF + f]: NF = 3 (thermal flux) or 6 (elastic stress, Voigt xx yy zz yz xz xy)
template <int ND>
__global__ void k_nodal_fields(const uint16_t* keys, const double* x, int R, int C, int L, int axis, int comp, double jump,
                               FieldProps props, double* out) {
  constexpr int NF = ND == 1 ? 3 : 6;
  const long N = (long)R * C * L;
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x) {
    const int rr = (int)(n % R), cc = (int)((n / R) % C), ll = (int)(n / ((long)R * C));
    const unsigned key = keys[n];
    double f[NF];
#pragma unroll
    for (int t = 0; t < NF; t++) f[t] = 0.0;
    for (int k = 0; k < 8; k++) {
      // the voxel in which this node is local node k, and this node's corner in it
      const int er = wrap(rr - drow(k) - 1, R), ec = wrap(cc - dcol(k), C), el = wrap(ll - dlay(k), L);
      const bool boundary = axis == 0 ? ec == C - 1 : (axis == 1 ? er == 0 : el == 0);
      const int mat = (key >> (2 * k)) & 3;
      const double px = dcol(k), py = -drow(k), pz = 1 - dlay(k);
      double g[ND][3];  // gradient of each component
#pragma unroll
      for (int ci = 0; ci < ND; ci++) g[ci][0] = g[ci][1] = g[ci][2] = 0.0;
      for (int j = 0; j < 8; j++) {
        const long node = (long)wrap(er + 1 + drow(j), R) + (long)wrap(ec + dcol(j), C) * R + (long)wrap(el + dlay(j), L) * R * C;
        bool on_face = false;
        if (boundary)
          for (int t = 0; t < 4; t++) on_face = on_face || face_node(axis, t) == j;
        const double d0 = dshape(j, 0, px, py, pz), d1 = dshape(j, 1, px, py, pz), d2 = dshape(j, 2, px, py, pz);
#pragma unroll
        for (int ci = 0; ci < ND; ci++) {
          const double v = x[node * ND + ci] + ((on_face && ci == comp) ? jump : 0.0);
          g[ci][0] += d0 * v;
          g[ci][1] += d1 * v;
          g[ci][2] += d2 * v;
        }
      }
      if constexpr (ND == 1) {
        const double kk = props.p[mat];
#pragma unroll
        for (int i = 0; i < 3; i++) f[i] += 0.125 * kk * g[0][i];
      } else {
        const double E = props.p[2 * mat], nu = props.p[2 * mat + 1];
        const double co = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
        const double exx = g[0][0], eyy = g[1][1], ezz = g[2][2];
        const double gyz = g[1][2] + g[2][1], gxz = g[0][2] + g[2][0], gxy = g[0][1] + g[1][0];
        const double sh = co * 0.5 * (1.0 - 2.0 * nu);
        f[0] += 0.125 * co * ((1.0 - nu) * exx + nu * eyy + nu * ezz);
        f[1] += 0.125 * co * (nu * exx + (1.0 - nu) * eyy + nu * ezz);
        f[2] += 0.125 * co * (nu * exx + nu * eyy + (1.0 - nu) * ezz);
        f[3] += 0.125 * sh * gyz;
        f[4] += 0.125 * sh * gxz;
        f[5] += 0.125 * sh * gxy;
      }
    }
#pragma unroll
    for (int t = 0; t < NF; t++) out[n * NF + t] = f[t];
  }
}

}  // namespace chfem
