// One-electron integral kernels of the classes with la = 3 (see one_electron_impl.cuh).
#include "one_electron_impl.cuh"

namespace lai {

int launch_one_e_l3(int la, int lb, int op, const OneEArgs& g, const int2* pairs, int n, cudaStream_t s) {
#define LAI_1E_CASE(A, B) \
  if (la == A && lb == B) return launch_op<A, B>(op, g, pairs, n, s);
  LAI_1E_CASE(3, 0) LAI_1E_CASE(3, 1) LAI_1E_CASE(3, 2) LAI_1E_CASE(3, 3)
#undef LAI_1E_CASE
  return -1;
}

}  // namespace lai
