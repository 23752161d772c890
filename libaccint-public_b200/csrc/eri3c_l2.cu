// Instantiations of the three-/two-centre integral kernel (eri3c_impl.cuh),
// bra shells with l_a = 2.
#include "eri3c_impl.cuh"

namespace lai {

int launch_eri3c_l2(int la, int lb, int lp, const Eri3cArgs& g, cudaStream_t s) {
#define X(a, b, p) \
  if (la == a && lb == b && lp == p) return launch_eri3c_cls<a, b, p>(g, s);
  X(2, 0, 0) X(2, 0, 1) X(2, 0, 2) X(2, 0, 3) X(2, 0, 4) \
  X(2, 1, 0) X(2, 1, 1) X(2, 1, 2) X(2, 1, 3) X(2, 1, 4) \
  X(2, 2, 0) X(2, 2, 1) X(2, 2, 2) X(2, 2, 3) X(2, 2, 4)
#undef X
  return -1;
}

}  // namespace lai
