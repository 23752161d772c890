// Instantiations of the three-/two-centre integral kernel (eri3c_impl.cuh),
// bra shells with l_a = 4.
#include "eri3c_impl.cuh"

namespace lai {

int launch_eri3c_l4(int la, int lb, int lp, const Eri3cArgs& g, cudaStream_t s) {
#define X(a, b, p) \
  if (la == a && lb == b && lp == p) return launch_eri3c_cls<a, b, p>(g, s);
  X(4, 0, 0) X(4, 0, 1) X(4, 0, 2) X(4, 0, 3) X(4, 0, 4)
#undef X
  return -1;
}

}  // namespace lai
