// One-electron integral kernels of the classes with la = 4 (see one_electron_impl.cuh).
#include "one_electron_impl.cuh"

namespace lai {

int launch_one_e_l4(int la, int lb, int op, const OneEArgs& g, const int2* pairs, int n, cudaStream_t s) {
#define LAI_1E_CASE(A, B) \
  if (la == A && lb == B) return launch_op<A, B>(op, g, pairs, n, s);
  LAI_1E_CASE(4, 0) LAI_1E_CASE(4, 1) LAI_1E_CASE(4, 2) LAI_1E_CASE(4, 3) LAI_1E_CASE(4, 4)
#undef LAI_1E_CASE
  return -1;
}

}  // namespace lai
