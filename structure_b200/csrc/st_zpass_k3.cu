// st_zpass_k3.cu -- fast-path instantiations for K classes 7, 8.
#include "st_zpass_fast.cuh"

namespace st {
namespace zfast {
template cudaError_t launch_b2g_kw<7, 8>(const LaunchSet&, int, int, size_t);
template cudaError_t launch_b2g_kw<8, 8>(const LaunchSet&, int, int, size_t);
}  // namespace zfast
}  // namespace st
