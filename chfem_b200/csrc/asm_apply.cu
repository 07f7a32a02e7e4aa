// asm_apply.cu -- launches of the assembled-stencil block operator (stencil_asm.cuh) for every
// (dof per node, precision, block size) the block solver runs.
#include "asm_apply.h"
#include "stencil_asm.cuh"

namespace chfem {

namespace {
// The launched form: synchronous staging with an L2 bulk prefetch of the next step's planes, the
// table in shared memory, and registers capped so that two CTAs fit on an SM (measured on the
// elastic 128^3 six-case pass: 0.329 ms against 0.369 without the prefetch; asynchronous
// cp.async staging at one CTA per SM 0.447 ms, the table read through L1 0.378 ms; a 4-slot
// plane ring with one barrier per layer, which fits two CTAs per SM only at 32 x 6 or 32 x 7
// nodes, 0.356 and 0.362 ms against 0.336 at 32 x 8: the fewer warps cost more than the
// barrier saves).
// (FP64 elastic planes of 19 doubles per node leave room for one CTA per SM: no cap there.)
template <int ND, typename T, int NR, int TC, int ZB, int RING = ZB + 2>
constexpr auto asm_kernel = k_asm_apply<ND, T, NR, TC, ZB, (ND == 3 && sizeof(T) == 8) ? 1 : 2, RING>;

template <int ND, typename T, int NR, int TC, int ZB, int RING = ZB + 2>
int ctas_of(int R, int C, int L, int num_sms) {
  const size_t smem = asm_smem_bytes<ND, T, NR, TC, ZB, RING>();
  static int per_sm = 0;  // per instantiation: the attribute is set and the occupancy asked once
  if (!per_sm) {
    if (cudaFuncSetAttribute(asm_kernel<ND, T, NR, TC, ZB, RING>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, asm_kernel<ND, T, NR, TC, ZB, RING>, TE_TR * TC, smem) != cudaSuccess || per_sm < 1)
      per_sm = 1;
  }
  const long work = (long)((R + TE_TR - 1) / TE_TR) * ((C + TC - 1) / TC) * L;
  return (int)std::max(1L, std::min((long)per_sm * num_sms, work / TE_MIN_RUN));
}
template <int ND, typename T, int NR, int TC, int ZB, int RING = ZB + 2>
cudaError_t launch(const BlkArgs<ND, T>& a, const T* tab, int nb, cudaStream_t st) {
  asm_kernel<ND, T, NR, TC, ZB, RING><<<nb, dim3(TE_TR, TC), asm_smem_bytes<ND, T, NR, TC, ZB, RING>(), st>>>(a, tab);
  return cudaGetLastError();
}
}  // namespace

// FP32 elastic, six load cases: the tile variants; FP64 elastic: 32 x 8, one layer per thread
// (its planes of 19 doubles per node leave no room for a fourth); thermal: 32 x 8, two layers.
template <int ND, typename T, int NR>
int asm_block_ctas(int R, int C, int L, int num_sms, int tile) {
  if constexpr (ND == 3 && NR == 6 && std::is_same<T, float>::value) {
    switch (tile) {
      case ASM_TILE_8x1: return ctas_of<ND, T, NR, 8, 1>(R, C, L, num_sms);
      case ASM_TILE_8x2: return ctas_of<ND, T, NR, 8, 2>(R, C, L, num_sms);
      case ASM_TILE_4x2: return ctas_of<ND, T, NR, 4, 2>(R, C, L, num_sms);
      case ASM_TILE_6x1_RING4: return ctas_of<ND, T, NR, 6, 1, 4>(R, C, L, num_sms);
      case ASM_TILE_7x1_RING4: return ctas_of<ND, T, NR, 7, 1, 4>(R, C, L, num_sms);
      default: return ctas_of<ND, T, NR, 6, 2>(R, C, L, num_sms);
    }
  } else if constexpr (ND == 1) {
    return ctas_of<ND, T, NR, 8, 2>(R, C, L, num_sms);
  } else {
    return ctas_of<ND, T, NR, 8, 1>(R, C, L, num_sms);
  }
}

template <int ND, typename T, int NR>
cudaError_t asm_block_launch(const BlkArgs<ND, T>& a, const T* tab, int nb, int tile, cudaStream_t st) {
  if constexpr (ND == 3 && NR == 6 && std::is_same<T, float>::value) {
    switch (tile) {
      case ASM_TILE_8x1: return launch<ND, T, NR, 8, 1>(a, tab, nb, st);
      case ASM_TILE_8x2: return launch<ND, T, NR, 8, 2>(a, tab, nb, st);
      case ASM_TILE_4x2: return launch<ND, T, NR, 4, 2>(a, tab, nb, st);
      case ASM_TILE_6x1_RING4: return launch<ND, T, NR, 6, 1, 4>(a, tab, nb, st);
      case ASM_TILE_7x1_RING4: return launch<ND, T, NR, 7, 1, 4>(a, tab, nb, st);
      default: return launch<ND, T, NR, 6, 2>(a, tab, nb, st);
    }
  } else if constexpr (ND == 1) {
    return launch<ND, T, NR, 8, 2>(a, tab, nb, st);
  } else {
    return launch<ND, T, NR, 8, 1>(a, tab, nb, st);
  }
}

template <int ND, typename T, int MODE>
int asm_te_ctas(int R, int C, int L, int num_sms) {
  static int per_sm = 0;
  const size_t smem = te_asm_smem_bytes<ND, T>();
  if (!per_sm) {
    if (cudaFuncSetAttribute(k_te_apply<ND, T, MODE, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_te_apply<ND, T, MODE, true>, TE_NT, smem) != cudaSuccess || per_sm < 1)
      per_sm = 1;
  }
  const long work = (long)((R + TE_TR - 1) / TE_TR) * ((C + TE_TC - 1) / TE_TC) * L;
  return (int)std::max(1L, std::min((long)per_sm * num_sms, work / TE_MIN_RUN));
}
template <int ND, typename T, int MODE>
cudaError_t asm_te_launch(const TeArgs<ND, T>& a, const T* tab, int nb, cudaStream_t st) {
  k_te_apply<ND, T, MODE, true><<<nb, dim3(TE_TR, TE_TC), te_asm_smem_bytes<ND, T>(), st>>>(a, tab);
  return cudaGetLastError();
}
#define CHFEM_ASM_TE_INSTANTIATE(ND, T, MODE)                 \
  template int asm_te_ctas<ND, T, MODE>(int, int, int, int); \
  template cudaError_t asm_te_launch<ND, T, MODE>(const TeArgs<ND, T>&, const T*, int, cudaStream_t);
CHFEM_ASM_TE_INSTANTIATE(1, float, TE_PLAIN)
CHFEM_ASM_TE_INSTANTIATE(1, float, TE_PCG)
CHFEM_ASM_TE_INSTANTIATE(1, float, TE_MR)
CHFEM_ASM_TE_INSTANTIATE(1, double, TE_PLAIN)
CHFEM_ASM_TE_INSTANTIATE(1, double, TE_PCG)
CHFEM_ASM_TE_INSTANTIATE(1, double, TE_MR)
CHFEM_ASM_TE_INSTANTIATE(3, float, TE_PLAIN)
CHFEM_ASM_TE_INSTANTIATE(3, float, TE_PCG)
CHFEM_ASM_TE_INSTANTIATE(3, float, TE_MR)
CHFEM_ASM_TE_INSTANTIATE(3, double, TE_PLAIN)
CHFEM_ASM_TE_INSTANTIATE(3, double, TE_PCG)
CHFEM_ASM_TE_INSTANTIATE(3, double, TE_MR)
CHFEM_ASM_TE_INSTANTIATE(1, float, TE_DIRDOT)
CHFEM_ASM_TE_INSTANTIATE(1, float, TE_UPD)
CHFEM_ASM_TE_INSTANTIATE(1, double, TE_DIRDOT)
CHFEM_ASM_TE_INSTANTIATE(1, double, TE_UPD)
CHFEM_ASM_TE_INSTANTIATE(3, float, TE_DIRDOT)
CHFEM_ASM_TE_INSTANTIATE(3, float, TE_UPD)
CHFEM_ASM_TE_INSTANTIATE(3, double, TE_DIRDOT)
CHFEM_ASM_TE_INSTANTIATE(3, double, TE_UPD)

#define CHFEM_ASM_INSTANTIATE(ND, T, NR)                                              \
  template int asm_block_ctas<ND, T, NR>(int, int, int, int, int);                    \
  template cudaError_t asm_block_launch<ND, T, NR>(const BlkArgs<ND, T>&, const T*, int, int, cudaStream_t);
CHFEM_ASM_INSTANTIATE(1, float, 3)
CHFEM_ASM_INSTANTIATE(1, double, 3)
CHFEM_ASM_INSTANTIATE(3, float, 6)
CHFEM_ASM_INSTANTIATE(3, double, 6)
CHFEM_ASM_INSTANTIATE(3, float, 3)
CHFEM_ASM_INSTANTIATE(3, double, 3)

}  // namespace chfem
