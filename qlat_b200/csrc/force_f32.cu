// force_f32.cu -- float instantiation of the gauge force kernels.
#include "force_impl.cuh"

namespace qgb
{
template cudaError_t launch_force<float>(const Geo&, ForceMode, const ForceArgs&, int, cudaStream_t);
template cudaError_t launch_corners<float>(const Geo&, const void*, void*, cudaStream_t);
template cudaError_t launch_force_batch<float>(long, int, const long*, const ChainInfo*, bool, ForceMode,
                                              const ForceArgs&, cudaStream_t, int);
}  // namespace qgb
