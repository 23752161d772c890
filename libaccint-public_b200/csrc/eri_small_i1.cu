// Explicit instantiations of the small-class kernels (part 2 of 6; split so
// nvcc compiles the classes in parallel).
#include "eri_small_impl.cuh"

namespace lai {
namespace small_detail {

template int launch_one<1, 0, 0, 0>(const QuartetBlock&, const JKArgs&, const RysTablesView&,
                                   cudaStream_t, bool, int, LaunchTune);
template int launch_one<2, 0, 2, 0>(const QuartetBlock&, const JKArgs&, const RysTablesView&,
                                   cudaStream_t, bool, int, LaunchTune);
template int launch_one<4, 0, 0, 0>(const QuartetBlock&, const JKArgs&, const RysTablesView&,
                                   cudaStream_t, bool, int, LaunchTune);

}  // namespace small_detail
}  // namespace lai
