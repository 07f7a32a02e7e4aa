// asm_table.cuh -- the operator row of a node assembled by neighbour for images of at most two
// materials: the table of per-material-configuration neighbour blocks and its lookup.
//
// The reference builds a node's row of the operator element by element: for each of the 8
// voxels around the node, the row block of the node in that voxel's element matrix times the
// voxel's 8 nodal values (chfem/src/femhmg/cudapcg/kernels/matrix_free.cu:410-459 elastic,
// :191-323 thermal), 64 (voxel, node) pairs of ND x ND blocks per node.  Summed by neighbour
// instead, the row is 27 blocks A(n, n+o) = sum over the voxels shared by n and n+o of
// K_mat(voxel)[local n, local n+o].  A neighbour shared through one voxel (corner) has 2
// possible blocks in a two-material image, one shared through 2 voxels (edge) 4, through 4
// (face) 16, the node itself (8 voxels) 256: 416 blocks in all, tabulated once per model (the
// sums taken in FP64 on the host) and held in shared memory.  Per node and right-hand side the
// operator is then 27 x ND x ND multiply-adds (243 elastic) instead of 64 x ND x ND (576), and
// 27 coefficient blocks are read instead of 64.
#pragma once
#include <algorithm>
#include <type_traits>
#include <utility>
#include "common.cuh"

namespace chfem {

// ---- the 2 x 2 x 2 voxels around a node --------------------------------------------------
// Position p of the voxel in which a node is local node e: bit 0 set when the voxel spans the
// node's row and the next row (rows {0,+1} relative to the node; clear: {-1,0}), bit 1 the same
// for columns, bit 2 for layers.
__host__ __device__ constexpr int asm_local(int dr, int dc, int dl) {
  return (dr == 0 ? (dc == 0 ? 0 : 1) : (dc == 1 ? 2 : 3)) + 4 * dl;
}
__host__ __device__ constexpr int asm_epos(int e) {
  return (drow(e) == -1 ? 1 : 0) | (dcol(e) == 0 ? 2 : 0) | (dlay(e) == 0 ? 4 : 0);
}
// local index of the node in the voxel at position p
__host__ __device__ constexpr int asm_eloc(int p) { return asm_local(-(p & 1), 1 - ((p >> 1) & 1), 1 - (p >> 2)); }
// one axis: a voxel whose position bit is b spans offsets {-1,0} (b = 0) or {0,+1} (b = 1)
__host__ __device__ constexpr bool asm_axis(int d, int b) { return d == 0 || (d == 1 && b == 1) || (d == -1 && b == 0); }
// neighbour offset o = (dr + 1) + 3 (dc + 1) + 9 (dl + 1), the numbering of pair_nbr
__host__ __device__ constexpr bool asm_reaches(int p, int o) {
  return asm_axis(o % 3 - 1, p & 1) && asm_axis((o / 3) % 3 - 1, (p >> 1) & 1) && asm_axis(o / 9 - 1, p >> 2);
}
__host__ __device__ constexpr int asm_count(int o) {
  int n = 0;
  for (int p = 0; p < 8; p++) n += asm_reaches(p, o) ? 1 : 0;
  return n;
}
// first table block of offset o; the blocks of o are its 2^count material configurations
__host__ __device__ constexpr int asm_base(int o) {
  int b = 0;
  for (int i = 0; i < o; i++) b += 1 << asm_count(i);
  return b;
}
constexpr int ASM_NBLK = asm_base(27);  // 416
// The Q1 conduction matrix couples no two nodes of a voxel that share an edge, so for one DOF
// per node the six face neighbours (reached only through such pairs) have a zero block.
template <int ND>
__host__ __device__ constexpr bool asm_used(int o) {
  return !(ND == 1 && ((o % 3 != 1) + ((o / 3) % 3 != 1) + (o / 9 != 1)) == 1);
}

// 8-bit material configuration of a node (bit p = material of the voxel at position p) from the
// 16-bit node key (2 bits per voxel, by local index; materials 0 and 1 only)
__host__ __device__ __forceinline__ unsigned asm_config(unsigned key) {
  unsigned m = 0;
#pragma unroll
  for (int e = 0; e < 8; e++) m |= ((key >> (2 * e)) & 1u) << asm_epos(e);
  return m;
}
// configuration index of offset O: the material bits of the voxels reaching O, in ascending
// position order, packed from bit 0; a run of consecutive positions moves as one shifted field
__host__ __device__ constexpr bool asm_run_start(int o, int p) { return asm_reaches(p, o) && (p == 0 || !asm_reaches(p - 1, o)); }
__host__ __device__ constexpr int asm_run_len(int o, int p) {
  int len = 0;
  while (p + len < 8 && asm_reaches(p + len, o)) len++;
  return len;
}
__host__ __device__ constexpr int asm_rank(int o, int p) {
  int j = 0;
  for (int i = 0; i < p; i++) j += asm_reaches(i, o) ? 1 : 0;
  return j;
}
template <int O, int P>
__host__ __device__ __forceinline__ unsigned asm_run(unsigned m) {
  if constexpr (asm_run_start(O, P)) {
    constexpr int len = asm_run_len(O, P), j = asm_rank(O, P);
    return (m >> (P - j)) & (((1u << len) - 1u) << j);
  } else {
    return 0u;
  }
}
template <int O, int... Ps>
__host__ __device__ __forceinline__ unsigned asm_variant_runs(unsigned m, std::integer_sequence<int, Ps...>) {
  return (asm_run<O, Ps>(m) | ...);
}
template <int O>
__host__ __device__ __forceinline__ unsigned asm_variant(unsigned m) {
  return asm_variant_runs<O>(m, std::make_integer_sequence<int, 8>{});
}

template <int ND, typename T, int NR>
struct AsmLayout {
  static constexpr int NV = NR * ND;
  // FP32 with an even number of right-hand sides: values and accumulators held as pairs of
  // right-hand sides, one packed FP32 FMA (sm_100) per pair, which has the rounding of two
  // scalar FMAs and half their issue slots
  static constexpr bool PAIRS = std::is_same<T, float>::value && NR % 2 == 0;
  using V = std::conditional_t<PAIRS, float2, T>;
  static constexpr int NW = PAIRS ? NR / 2 : NR;  // V per component
  // a point of the staged planes: [component][right-hand side], padded so that consecutive
  // lanes' points fall on distinct banks (an odd count of 8-byte pairs, or of words)
  static constexpr int PS = PAIRS ? ((NV / 2) % 2 ? NV : NV + 2) : (NV % 2 ? NV : NV + 1);
  // FP32 elastic blocks padded to 12 words: two 16-byte loads and one word
  static constexpr bool QUADS = std::is_same<T, float>::value && ND == 3;
  static constexpr int BS = ND == 1 ? 1 : (QUADS ? 12 : ND * ND);
};

// out += A(n, n+O) val for every right-hand side; val, out: [component][right-hand side (pairs)]
template <int ND, typename T, int O, typename V, int NW>
__device__ __forceinline__ void asm_block(const T* __restrict__ sT, unsigned m, const V (&val)[ND][NW], V (&out)[ND][NW]) {
  if constexpr (asm_used<ND>(O)) {
    constexpr int BS = ND == 1 ? 1 : ((std::is_same<T, float>::value && ND == 3) ? 12 : ND * ND);
    constexpr int kBase = asm_base(O);  // evaluated at compile time, not per node
    const T* tb = sT + (kBase + asm_variant<O>(m)) * BS;
    T blk[ND * ND];
    if constexpr (std::is_same<T, float>::value && ND == 3) {
      const float4 q0 = *reinterpret_cast<const float4*>(tb);
      const float4 q1 = *reinterpret_cast<const float4*>(tb + 4);
      blk[0] = q0.x; blk[1] = q0.y; blk[2] = q0.z; blk[3] = q0.w;
      blk[4] = q1.x; blk[5] = q1.y; blk[6] = q1.z; blk[7] = q1.w;
      blk[8] = tb[8];
    } else {
#pragma unroll
      for (int i = 0; i < ND * ND; i++) blk[i] = tb[i];
    }
#pragma unroll
    for (int ci = 0; ci < ND; ci++)
#pragma unroll
      for (int cj = 0; cj < ND; cj++) {
        const T kv = blk[ci * ND + cj];
#pragma unroll
        for (int w = 0; w < NW; w++) {
          if constexpr (std::is_same<V, float2>::value) out[ci][w] = __ffma2_rn(make_float2(kv, kv), val[cj][w], out[ci][w]);
          else out[ci][w] = fma(kv, val[cj][w], out[ci][w]);
        }
      }
  }
}

// After the blocks the table holds the inverse Jacobi diagonal of each of the 256 node
// configurations (ND values each): the Jacobi preconditioner's M^-1 of a node from its
// configuration alone (the diagonal of its centre block, matrix_free.cu:167-188 and :388-408
// sum it from the 8 voxels' element-matrix diagonals).
constexpr int ASM_NCFG = 256;
__host__ __device__ constexpr int asm_table_words(int nd, int bs) { return ASM_NBLK * bs + ASM_NCFG * nd; }

// Host: the 416 assembled blocks of a model from its dense element matrices Kd [nmat][8ND][8ND]
// (row-major), summed in FP64; block (o, v) at (asm_base(o) + v) * bs; then the inverse
// diagonals at ASM_NBLK * bs + m * nd.
inline void asm_build_table(int nd, int nmat, const double* Kd, int bs, double* tab) {
  const int ED = 8 * nd;
  for (int i = 0; i < asm_table_words(nd, bs); i++) tab[i] = 0.0;
  for (int m = 0; m < ASM_NCFG; m++)
    for (int c = 0; c < nd; c++) {
      double d = 0.0;
      for (int p = 0; p < 8; p++) {
        const int e = asm_eloc(p), mat = std::min((m >> p) & 1, nmat - 1);
        d += Kd[(size_t)mat * ED * ED + (size_t)(e * nd + c) * ED + e * nd + c];
      }
      tab[ASM_NBLK * bs + m * nd + c] = 1.0 / d;
    }
  for (int o = 0; o < 27; o++) {
    const int dr = o % 3 - 1, dc = (o / 3) % 3 - 1, dl = o / 9 - 1;
    const int cnt = asm_count(o);
    for (int v = 0; v < (1 << cnt); v++) {
      double* blk = tab + (size_t)(asm_base(o) + v) * bs;
      int j = 0;
      for (int p = 0; p < 8; p++) {
        if (!asm_reaches(p, o)) continue;
        const int mat = std::min((v >> j) & 1, nmat - 1);
        j++;
        const int e = asm_eloc(p);
        const int b = asm_local(drow(e) + dr, dcol(e) + dc, dlay(e) + dl);
        const double* K = Kd + (size_t)mat * ED * ED;
        for (int ci = 0; ci < nd; ci++)
          for (int cj = 0; cj < nd; cj++) blk[ci * nd + cj] += K[(e * nd + ci) * ED + b * nd + cj];
      }
    }
  }
}

}  // namespace chfem
