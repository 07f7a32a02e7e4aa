// asm_apply.h -- host entry of the assembled-stencil block operator (stencil_asm.cuh), compiled in
// its own translation unit (asm_apply.cu).
#pragma once
#include <cuda_runtime.h>
#include "stencil_block.cuh"
#include "stencil_te.cuh"

namespace chfem {

// Tile of the FP32 elastic six-case pass: column tile of 32 x TC nodes, ZB layers per thread;
// _RING4: a 4-slot plane ring (the next plane staged during the arithmetic, one barrier a layer).
enum AsmTile : int { ASM_TILE_8x1 = 0, ASM_TILE_6x2 = 1, ASM_TILE_8x2 = 2, ASM_TILE_4x2 = 3, ASM_TILE_6x1_RING4 = 4,
                     ASM_TILE_7x1_RING4 = 5 };

// CTAs of one pass on an R x C x L model: as many as fit on the GPU at once, at least
// TE_MIN_RUN layers of work each.
template <int ND, typename T, int NR>
int asm_block_ctas(int R, int C, int L, int num_sms, int tile);
// One block PCG operator pass (contract of k_blk_apply) on nb CTAs; tab: the model's 416
// assembled blocks in the layout of AsmLayout<ND, T, NR>.
template <int ND, typename T, int NR>
cudaError_t asm_block_launch(const BlkArgs<ND, T>& a, const T* tab, int nb, int tile, cudaStream_t st);

// The single right-hand-side operator pass k_te_apply<ND, T, MODE> with the assembled blocks
// (asm_table.cuh): CTAs as many as fit at once (at least TE_MIN_RUN layers each), and one launch.
template <int ND, typename T, int MODE>
int asm_te_ctas(int R, int C, int L, int num_sms);
template <int ND, typename T, int MODE>
cudaError_t asm_te_launch(const TeArgs<ND, T>& a, const T* tab, int nb, cudaStream_t st);

}  // namespace chfem
