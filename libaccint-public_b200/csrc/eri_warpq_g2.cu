// Instantiations of the warp-per-quartet kernel (eri_warpq_impl.cuh): g classes (part 3).
#include <algorithm>

#include "eri_warpq_impl.cuh"

namespace lai {

#define LAI_WARPQ_CLASSES(X) \
  X(4, 2, 0, 0) X(4, 2, 1, 0) X(4, 2, 1, 1) X(4, 2, 2, 0) \
  X(4, 2, 2, 1) X(4, 2, 3, 0) X(4, 2, 4, 0)

int launch_warpq_g2(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                    int num_sms, bool fp32) {
  (void)fp32;  // g classes: FP64 only
  const int la = blk.bra.la, lb = blk.bra.lb, lc = blk.ket.la, ld = blk.ket.lb;
#define X(a, b, c, d) \
  if (la == a && lb == b && lc == c && ld == d) return launch_warpq_cls<a, b, c, d, false>(blk, args, tab, stream, num_sms, fp32);
  LAI_WARPQ_CLASSES(X)
#undef X
  return -1;
}

bool warpq_supported_g2(int la, int lb, int lc, int ld) {
#define X(a, b, c, d) \
  if (la == a && lb == b && lc == c && ld == d) return true;
  LAI_WARPQ_CLASSES(X)
#undef X
  return false;
}

}  // namespace lai
