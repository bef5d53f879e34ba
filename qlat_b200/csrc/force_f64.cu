// force_f64.cu -- double instantiation of the gauge force kernels.
#include "force_impl.cuh"

namespace qgb
{
template cudaError_t launch_force<double>(const Geo&, ForceMode, const ForceArgs&, int, cudaStream_t);
template cudaError_t launch_corners<double>(const Geo&, const void*, void*, cudaStream_t);
template cudaError_t launch_force_batch<double>(long, int, const long*, const ChainInfo*, bool, ForceMode,
                                              const ForceArgs&, cudaStream_t, int);
}  // namespace qgb
