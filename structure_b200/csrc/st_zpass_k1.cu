// st_zpass_k1.cu -- fast-path instantiations for K classes 1, 2, 3, 4.
#include "st_zpass_fast.cuh"

namespace st {
namespace zfast {
template cudaError_t launch_b2g_kw<1, 8>(const LaunchSet&, int, int, size_t);
template cudaError_t launch_b2g_kw<2, 8>(const LaunchSet&, int, int, size_t);
template cudaError_t launch_b2g_kw<3, 8>(const LaunchSet&, int, int, size_t);
template cudaError_t launch_b2g_kw<4, 8>(const LaunchSet&, int, int, size_t);

size_t zlayout_total(int KT, int K, int T, int nw32, int mode) {
  return zlayout(KT, K, T, nw32, mode).total;
}
}  // namespace zfast
}  // namespace st
