// th_apply.cu -- launches of the thermal operator pass of stencil_th.cuh, and its table.
#include <algorithm>
#include <cmath>
#include "th_apply.h"
#include "stencil_th.cuh"

namespace chfem {

namespace {
constexpr int TH_TC = 8;  // 32 x 8 node columns per CTA
template <typename T, int MODE>
constexpr auto th_kernel = k_th_apply<T, MODE, TH_TC>;
int pair_kind(int a, int b) { return (drow(a) != drow(b)) + (dcol(a) != dcol(b)) + (dlay(a) != dlay(b)); }
}  // namespace

int th_table_words() { return TH_WORDS; }

bool th_build_table(int nmat, const double* Kd, double* tab) {
  if (nmat < 1 || nmat > 4) return false;
  for (int i = 0; i < TH_WORDS; i++) tab[i] = 0.0;
  double d[4] = {0, 0, 0, 0};
  for (int m = 0; m < nmat; m++) {
    const double* K = Kd + (size_t)m * 64;
    const double dm = K[0];
    if (!(std::fabs(dm) > 0.0)) return false;
    double f = 0.0, c = 0.0;
    for (int b = 1; b < 8; b++) {
      if (pair_kind(0, b) == 2 && f == 0.0) f = K[b];
      if (pair_kind(0, b) == 3) c = K[b];
    }
    const double tol = 1e-12 * std::fabs(dm);
    for (int a = 0; a < 8; a++)
      for (int b = 0; b < 8; b++) {
        const int n = pair_kind(a, b);
        const double want = n == 0 ? dm : (n == 1 ? 0.0 : (n == 2 ? f : c));
        if (std::fabs(K[8 * a + b] - want) > tol) return false;
      }
    d[m] = dm;
    tab[2 * m] = f;
    tab[2 * m + 1] = c;
  }
  for (int n3 = 0; n3 <= 8; n3++)
    for (int n2 = 0; n2 + n3 <= 8; n2++)
      for (int n1 = 0; n1 + n2 + n3 <= 8; n1++) {
        const int n0 = 8 - n1 - n2 - n3;
        const double D = n0 * d[0] + n1 * d[1] + n2 * d[2] + n3 * d[3];
        const int idx = n1 + 9 * n2 + 81 * n3;
        tab[TH_DIAG + idx] = D;
        tab[TH_INV + idx] = 1.0 / D;
      }
  return true;
}

template <typename T, int MODE>
int th_ctas(int R, int C, int L, int num_sms) {
  static int per_sm = 0;  // per instantiation: the attribute is set and the occupancy asked once
  const size_t smem = th_smem_bytes<T, TH_TC>();
  if (!per_sm) {
    if (cudaFuncSetAttribute(th_kernel<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, th_kernel<T, MODE>, TE_TR * TH_TC, smem) != cudaSuccess || per_sm < 1)
      per_sm = 1;
  }
  const long work = (long)((R + TE_TR - 1) / TE_TR) * ((C + TH_TC - 1) / TH_TC) * L;
  return (int)std::max(1L, std::min((long)per_sm * num_sms, work / TE_MIN_RUN));
}

template <typename T, int MODE>
cudaError_t th_launch(const TeArgs<1, T>& a, const T* tab, int nb, cudaStream_t st) {
  th_kernel<T, MODE><<<nb, dim3(TE_TR, TH_TC), th_smem_bytes<T, TH_TC>(), st>>>(a, tab);
  return cudaGetLastError();
}

#define CHFEM_TH_INSTANTIATE(T, MODE)                \
  template int th_ctas<T, MODE>(int, int, int, int); \
  template cudaError_t th_launch<T, MODE>(const TeArgs<1, T>&, const T*, int, cudaStream_t);
CHFEM_TH_INSTANTIATE(float, TE_PLAIN)
CHFEM_TH_INSTANTIATE(float, TE_PCG)
CHFEM_TH_INSTANTIATE(float, TE_MR)
CHFEM_TH_INSTANTIATE(float, TE_DIRDOT)
CHFEM_TH_INSTANTIATE(float, TE_UPD)
CHFEM_TH_INSTANTIATE(double, TE_PLAIN)
CHFEM_TH_INSTANTIATE(double, TE_PCG)
CHFEM_TH_INSTANTIATE(double, TE_MR)
CHFEM_TH_INSTANTIATE(double, TE_DIRDOT)
CHFEM_TH_INSTANTIATE(double, TE_UPD)

}  // namespace chfem
