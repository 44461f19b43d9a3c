// st_zpass_k4.cu -- fast-path instantiations for K classes 9, 10.
#include "st_zpass_fast.cuh"

namespace st {
namespace zfast {
template cudaError_t launch_b2g_kw<9, 8>(const LaunchSet&, int, int, size_t);
template cudaError_t launch_b2g_kw<10, 8>(const LaunchSet&, int, int, size_t);
}  // namespace zfast
}  // namespace st
