// Instantiations of the warp-per-quartet kernel (eri_warpq_impl.cuh): f classes (part 2).
#include <algorithm>

#include "eri_warpq_impl.cuh"

namespace lai {

#define LAI_WARPQ_CLASSES(X) \
  X(3, 1, 2, 1) X(3, 1, 2, 2) X(3, 1, 3, 0) X(3, 1, 3, 1) \
  X(3, 2, 0, 0) X(3, 2, 1, 0) X(3, 2, 1, 1) X(3, 2, 2, 0)

int launch_warpq_f1(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                    int num_sms, bool fp32) {
  const int la = blk.bra.la, lb = blk.bra.lb, lc = blk.ket.la, ld = blk.ket.lb;
#define X(a, b, c, d) \
  if (la == a && lb == b && lc == c && ld == d) return launch_warpq_cls<a, b, c, d, true>(blk, args, tab, stream, num_sms, fp32);
  LAI_WARPQ_CLASSES(X)
#undef X
  return -1;
}

bool warpq_supported_f1(int la, int lb, int lc, int ld) {
#define X(a, b, c, d) \
  if (la == a && lb == b && lc == c && ld == d) return true;
  LAI_WARPQ_CLASSES(X)
#undef X
  return false;
}

}  // namespace lai
