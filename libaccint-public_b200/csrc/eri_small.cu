// Dispatch of the thread-per-quartet small-class kernels (eri_small_impl.cuh);
// the kernels themselves are instantiated in eri_small_i*.cu.
#include <cuda_runtime.h>

#include "eri_kernels.h"

namespace lai {
namespace small_detail {
template <int LA, int LB, int LC, int LD>
int launch_one(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
               cudaStream_t stream, bool fp32, int num_sms, LaunchTune tune);
}  // namespace small_detail

#define LAI_SMALL_CLASSES(X) \
  X(0, 0, 0, 0) X(1, 0, 0, 0) X(1, 0, 1, 0) X(1, 1, 0, 0) X(1, 1, 1, 0) X(2, 0, 0, 0) \
  X(2, 0, 1, 0) X(2, 0, 2, 0) X(2, 1, 0, 0) X(2, 2, 0, 0) X(3, 0, 0, 0) X(3, 0, 1, 0)   \
  X(3, 1, 0, 0) X(4, 0, 0, 0) X(1, 1, 1, 1) X(2, 0, 1, 1) X(2, 1, 1, 0) X(2, 1, 2, 0) X(2, 2, 1, 0)

bool small_class_supported(int la, int lb, int lc, int ld) {
#define X(a, b, c, d) if (la == a && lb == b && lc == c && ld == d) return true;
  LAI_SMALL_CLASSES(X)
#undef X
  return false;
}

int launch_small(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
                 cudaStream_t stream, bool fp32, int num_sms, LaunchTune tune) {
  const int la = blk.bra.la, lb = blk.bra.lb, lc = blk.ket.la, ld = blk.ket.lb;
#define X(a, b, c, d) \
  if (la == a && lb == b && lc == c && ld == d) return small_detail::launch_one<a, b, c, d>(blk, args, tab, stream, fp32, num_sms, tune);
  LAI_SMALL_CLASSES(X)
#undef X
  return 0;
}

}  // namespace lai
