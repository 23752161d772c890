// Instantiations of the three-/two-centre integral kernel (eri3c_impl.cuh),
// bra shells with l_a <= 1.
#include "eri3c_impl.cuh"

namespace lai {

int launch_eri3c_l01(int la, int lb, int lp, const Eri3cArgs& g, cudaStream_t s) {
#define X(a, b, p) \
  if (la == a && lb == b && lp == p) return launch_eri3c_cls<a, b, p>(g, s);
  X(0, 0, 0) X(0, 0, 1) X(0, 0, 2) X(0, 0, 3) X(0, 0, 4) \
  X(1, 0, 0) X(1, 0, 1) X(1, 0, 2) X(1, 0, 3) X(1, 0, 4) \
  X(1, 1, 0) X(1, 1, 1) X(1, 1, 2) X(1, 1, 3) X(1, 1, 4)
#undef X
  return -1;
}

}  // namespace lai
