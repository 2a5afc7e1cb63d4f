// Explicit instantiations of the small-LU launchers, single precision (compiled
// separately so the variants build in parallel).
#include "small_lu_kernels.cuh"

namespace mb200 {
MB200_INSTANTIATE_SMALL(float, 64, 2)
MB200_INSTANTIATE_SMALL(float, 64, 4)
}  // namespace mb200
