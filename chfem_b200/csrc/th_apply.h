// th_apply.h -- host entry of the thermal operator pass for cubic-symmetric conduction matrices
// (stencil_th.cuh), compiled in its own translation unit (th_apply.cu).
#pragma once
#include <cuda_runtime.h>
#include "stencil_te.cuh"

namespace chfem {

// The pass's table (th_table_words() values, FP64) from the dense 8 x 8 element matrices of
// nmat <= 4 materials (Kd[m][8][8]); false when a matrix lacks the structure the pass relies on
// (one diagonal value, zero between edge neighbours, one face-diagonal and one body-diagonal
// value, to 1e-12 of the diagonal).
bool th_build_table(int nmat, const double* Kd, double* tab);
int th_table_words();

// CTAs of one pass (as many as fit on the GPU at once, at least TE_MIN_RUN layers each) and one
// launch, with the contract of k_te_apply<1, T, MODE>.
template <typename T, int MODE>
int th_ctas(int R, int C, int L, int num_sms);
template <typename T, int MODE>
cudaError_t th_launch(const TeArgs<1, T>& a, const T* tab, int nb, cudaStream_t st);

}  // namespace chfem
