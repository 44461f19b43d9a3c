// st_zpass_k5.cu -- fast-path instantiations for K classes 11, 12.
#include "st_zpass_fast.cuh"

namespace st {
namespace zfast {
template cudaError_t launch_b2g_kw<11, 8>(const LaunchSet&, int, int, size_t);
template cudaError_t launch_b2g_kw<12, 8>(const LaunchSet&, int, int, size_t);
}  // namespace zfast
}  // namespace st
