// st_zpass_k6.cu -- fast-path instantiations for K classes 16, 20, 24, 32.
#include "st_zpass_fast.cuh"

namespace st {
namespace zfast {
template cudaError_t launch_b2g_kw<16, 2>(const LaunchSet&, int, int, size_t);
template cudaError_t launch_b2g_kw<20, 2>(const LaunchSet&, int, int, size_t);
template cudaError_t launch_b2g_kw<24, 2>(const LaunchSet&, int, int, size_t);
template cudaError_t launch_b2g_kw<32, 2>(const LaunchSet&, int, int, size_t);
}  // namespace zfast
}  // namespace st
