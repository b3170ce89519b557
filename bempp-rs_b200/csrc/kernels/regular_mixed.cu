// Mixed-precision regular quadrature (FP32 far pairs, FP64 near pairs).
#include "launch.h"

namespace bempp_b200 {

cudaError_t launch_regular_dp0_mixed(const CellSet&, const CellSet&, const RegularRule&,
                                     const RegularArgs&, cudaStream_t) {
  return cudaErrorNotSupported;
}

cudaError_t launch_regular_scatter_mixed(const CellSet&, const SpaceTiles&, const CellSet&,
                                         const SpaceTiles&, const RegularRule&,
                                         const RegularArgs&, cudaStream_t) {
  return cudaErrorNotSupported;
}

}  // namespace bempp_b200
