// Dispatch of the thread-per-quartet gradient kernels (eri_grad_small.cuh) over
// the classes they cover: the canonical (la,lb|lc,ld) with l <= 2 whose Cartesian
// block has at most 54 components (the rest run on the warp kernel of
// eri_grad.cu).  The kernels are instantiated in eri_grad_small_i*.cu.
#include "eri_grad_small.cuh"

namespace lai {
namespace grad_small {

#define LAI_GRAD_SMALL_CLASSES(X) \
  X(0, 0, 0, 0) X(1, 0, 0, 0) X(1, 0, 1, 0) X(1, 1, 0, 0) X(1, 1, 1, 0) X(2, 0, 0, 0) \
  X(2, 0, 1, 0) X(2, 0, 1, 1) X(2, 0, 2, 0) X(2, 1, 0, 0) X(2, 1, 1, 0) X(2, 2, 0, 0)

#define X(a, b, c, d)                                                                              \
  extern template int launch<a, b, c, d>(const QuartetBlock&, const GradSmallArgs&, const RysTablesView&, \
                                         cudaStream_t, int);
LAI_GRAD_SMALL_CLASSES(X)
#undef X

using Launcher = int (*)(const QuartetBlock&, const GradSmallArgs&, const RysTablesView&, cudaStream_t, int);

Launcher find(int la, int lb, int lc, int ld) {
#define X(a, b, c, d) \
  if (la == a && lb == b && lc == c && ld == d) return &launch<a, b, c, d>;
  LAI_GRAD_SMALL_CLASSES(X)
#undef X
  return nullptr;
}

}  // namespace grad_small

bool grad_small_supported(int la, int lb, int lc, int ld) { return grad_small::find(la, lb, lc, ld) != nullptr; }

int launch_grad_small(const QuartetBlock& blk, const double* D, int nbf, const int* shell_atom, double* grad,
                      double prim_eps, const RysTablesView& tab, cudaStream_t stream, int num_sms) {
  const auto f = grad_small::find(blk.bra.la, blk.bra.lb, blk.ket.la, blk.ket.lb);
  if (!f) return -1;
  grad_small::GradSmallArgs ga{D, nbf, shell_atom, grad, prim_eps};
  return f(blk, ga, tab, stream, num_sms);
}

}  // namespace lai
