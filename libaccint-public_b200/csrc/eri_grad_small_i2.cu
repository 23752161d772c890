// Explicit instantiations of the thread-per-quartet gradient kernels (part 3
// of 3; split so nvcc compiles the classes in parallel).
#include "eri_grad_small.cuh"

namespace lai {
namespace grad_small {

#define X(a, b, c, d)                                                                                \
  template int launch<a, b, c, d>(const QuartetBlock&, const GradSmallArgs&, const RysTablesView&, \
                                  cudaStream_t, int);
X(2, 0, 2, 0) X(2, 1, 0, 0) X(2, 1, 1, 0) X(2, 2, 0, 0)
#undef X

}  // namespace grad_small
}  // namespace lai
