// st_zpass_ind.cu -- instantiations of the individual-lane Z pass (K classes
// 1..8) and the kernel that builds its individual-major genotype copy.
#include "st_zpass_ind.cuh"

namespace st {

cudaError_t launch_zpass_ind(const LaunchSet& ls, int KT, int flags) {
  switch (KT) {
#define ST_ICASE(k) case k: return zind::launch_ind_kt<k>(ls, flags);
    ST_ICASE(1) ST_ICASE(2) ST_ICASE(3) ST_ICASE(4) ST_ICASE(5) ST_ICASE(6) ST_ICASE(7)
    ST_ICASE(8)
#undef ST_ICASE
  }
  return cudaErrorInvalidValue;
}

namespace {
// One output word per thread: individual 32*blk + lane, loci 64*w4 + 16*q + j.
__global__ void build_g2t_kernel(const uint32_t* __restrict__ g2, int wpr, int N, int L, int nlw4,
                                 uint32_t* __restrict__ g2t, size_t nwords) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nwords) return;
  const int q = (int)(t & 3), lane = (int)((t >> 2) & 31);
  const size_t rest = t >> 7;
  const int w4 = (int)(rest % (size_t)nlw4);
  const int blk = (int)(rest / (size_t)nlw4);
  const int i = blk * 32 + lane;
  uint32_t word = 0u;
  for (int j = 0; j < 16; j++) {
    const int l = w4 * 64 + q * 16 + j;
    const uint32_t code = (i < N && l < L) ? (g2[(size_t)l * wpr + (i >> 4)] >> (2 * (i & 15))) & 3u : 3u;
    word |= code << (2 * j);
  }
  g2t[t] = word;
}
}  // namespace

cudaError_t launch_build_g2t(const uint32_t* g2, int wpr, int N, int L, uint32_t* g2t,
                             cudaStream_t s) {
  const int nlw4 = (L + 63) / 64;
  const size_t nwords = (size_t)((N + 31) / 32) * nlw4 * 128;
  build_g2t_kernel<<<(unsigned)((nwords + 255) / 256), 256, 0, s>>>(g2, wpr, N, L, nlw4, g2t, nwords);
  return cudaGetLastError();
}

}  // namespace st
