// Dispatch of the warp-per-quartet kernel over its instantiation groups
// (eri_warpq_<group>.cu, compiled in parallel).
#include "eri_kernels.h"
#include "eri_warpq_impl.cuh"

namespace lai {

// classes where the warp-per-quartet kernel beat the tiled kernel ((dd|dp): 59 ms
// tiled, 14 ms warp-per-quartet in a (H2O)64/cc-pVDZ build)
#define LAI_WARPQ_PREFERRED(W) \
  W(2, 2, 1, 1) W(2, 2, 2, 1) W(2, 2, 2, 2) W(3, 0, 1, 1) W(3, 0, 2, 0) W(3, 0, 2, 1) W(3, 0, 2, 2) W(3, 0, 3, 0) \
  W(3, 1, 1, 0) W(3, 1, 1, 1) W(3, 1, 2, 0) W(3, 1, 3, 0) W(3, 2, 0, 0) W(3, 2, 1, 0) \
  W(3, 2, 2, 0) W(3, 2, 3, 0) W(3, 3, 0, 0) W(3, 3, 1, 0) W(4, 0, 1, 0) W(4, 0, 1, 1) \
  W(4, 0, 2, 0) W(4, 0, 2, 1) W(4, 0, 2, 2) W(4, 0, 3, 0) W(4, 0, 3, 1) W(4, 0, 3, 2) \
  W(4, 0, 4, 0) W(4, 1, 0, 0) W(4, 1, 1, 0) W(4, 1, 1, 1) W(4, 1, 2, 0) W(4, 1, 2, 1) \
  W(4, 1, 3, 0) W(4, 1, 3, 1) W(4, 1, 4, 0) W(4, 2, 0, 0) W(4, 2, 1, 0) W(4, 3, 0, 0) \
  W(4, 3, 1, 0) W(4, 4, 0, 0) W(4, 4, 1, 0)

int launch_warpq_d(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                    int num_sms, bool fp32);
int launch_warpq_f0(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                    int num_sms, bool fp32);
int launch_warpq_f1(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                    int num_sms, bool fp32);
int launch_warpq_f2(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                    int num_sms, bool fp32);
int launch_warpq_g0(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                    int num_sms, bool fp32);
int launch_warpq_g1(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                    int num_sms, bool fp32);
int launch_warpq_g2(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                    int num_sms, bool fp32);
int launch_warpq_g3(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                    int num_sms, bool fp32);

bool warpq_supported_d(int la, int lb, int lc, int ld);
bool warpq_supported_f0(int la, int lb, int lc, int ld);
bool warpq_supported_f1(int la, int lb, int lc, int ld);
bool warpq_supported_f2(int la, int lb, int lc, int ld);
bool warpq_supported_g0(int la, int lb, int lc, int ld);
bool warpq_supported_g1(int la, int lb, int lc, int ld);
bool warpq_supported_g2(int la, int lb, int lc, int ld);
bool warpq_supported_g3(int la, int lb, int lc, int ld);

cudaError_t warpq_launch_error() { return warpq_last_error(); }

int launch_warpq(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                 int num_sms, bool fp32) {
  if (args.mode != MODE_JK) return -1;
  if (blk.total - blk.t_begin <= 0) return 0;
  int rc;
  if ((rc = launch_warpq_d(blk, args, tab, stream, num_sms, fp32)) != -1) return rc;
  if ((rc = launch_warpq_f0(blk, args, tab, stream, num_sms, fp32)) != -1) return rc;
  if ((rc = launch_warpq_f1(blk, args, tab, stream, num_sms, fp32)) != -1) return rc;
  if ((rc = launch_warpq_f2(blk, args, tab, stream, num_sms, fp32)) != -1) return rc;
  if ((rc = launch_warpq_g0(blk, args, tab, stream, num_sms, fp32)) != -1) return rc;
  if ((rc = launch_warpq_g1(blk, args, tab, stream, num_sms, fp32)) != -1) return rc;
  if ((rc = launch_warpq_g2(blk, args, tab, stream, num_sms, fp32)) != -1) return rc;
  if ((rc = launch_warpq_g3(blk, args, tab, stream, num_sms, fp32)) != -1) return rc;
  return -1;
}

bool warpq_class_supported(int la, int lb, int lc, int ld) {
  return warpq_supported_d(la, lb, lc, ld) ||
         warpq_supported_f0(la, lb, lc, ld) ||
         warpq_supported_f1(la, lb, lc, ld) ||
         warpq_supported_f2(la, lb, lc, ld) ||
         warpq_supported_g0(la, lb, lc, ld) ||
         warpq_supported_g1(la, lb, lc, ld) ||
         warpq_supported_g2(la, lb, lc, ld) ||
         warpq_supported_g3(la, lb, lc, ld);
}

// Default kernel family per class: the warp-per-quartet kernel where it measured
// faster than the tiled one on B200 ((H2O)64/cc-pVDZ, C12H26/cc-pVTZ,
// (H2O)2/cc-pVQZ builds), the bra-sliced kernel for its classes, else tiled.
int default_kernel(int la, int lb, int lc, int ld) {
  if (sliced_class_supported(la, lb, lc, ld)) return KERNEL_SLICED;
  if (!warpq_class_supported(la, lb, lc, ld)) return KERNEL_TILED;
#define W(a, b, c, d) \
  if (la == a && lb == b && lc == c && ld == d) return KERNEL_WARPQ;
  LAI_WARPQ_PREFERRED(W)
#undef W
  return KERNEL_TILED;
}

}  // namespace lai
