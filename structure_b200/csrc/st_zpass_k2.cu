// st_zpass_k2.cu -- fast-path instantiations for K classes 5, 6.
#include "st_zpass_fast.cuh"

namespace st {
namespace zfast {
template cudaError_t launch_b2g_kw<5, 8>(const LaunchSet&, int, int, size_t);
template cudaError_t launch_b2g_kw<6, 8>(const LaunchSet&, int, int, size_t);
}  // namespace zfast
}  // namespace st
