// One-electron integral kernels of the classes with la <= 2 (see one_electron_impl.cuh).
#include "one_electron_impl.cuh"

namespace lai {

int launch_one_e_l012(int la, int lb, int op, const OneEArgs& g, const int2* pairs, int n, cudaStream_t s) {
#define LAI_1E_CASE(A, B) \
  if (la == A && lb == B) return launch_op<A, B>(op, g, pairs, n, s);
  LAI_1E_CASE(0, 0) LAI_1E_CASE(1, 0) LAI_1E_CASE(1, 1) LAI_1E_CASE(2, 0) LAI_1E_CASE(2, 1) LAI_1E_CASE(2, 2)
#undef LAI_1E_CASE
  return -1;
}

}  // namespace lai
