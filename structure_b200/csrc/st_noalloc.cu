// st_noalloc.cu -- st_update_z_noalloc: the biallelic Z pass with counts and
// ln P(D), for callers that cannot allocate device memory.
//
// Who needs it: a host program that owns every device allocation itself --
// a memory-pool allocator that forbids outside cudaMalloc, a caller that
// runs under a fixed device-memory budget, or code on a path where an
// allocation would synchronise the device -- still wants one Z update on
// buffers it already holds.  The chain API (st_chain_create) allocates the
// per-CTA count partials for each chain; this entry point instead keeps
// them in one file-scope device array of fixed size, so a call allocates
// nothing: no cudaMalloc, no cudaFree, no allocating library routine.
//
// Limits and sharing:
//  * The array holds kScratchBytes (ST_NOALLOC_SCRATCH_BYTES, 32 MiB) on
//    every GPU that loads the library, until the process exits.  A problem
//    whose partials need more is rejected with ST_ERR_ADMISSION.
//  * Every call on a device uses the same array, and it keeps what the last
//    call left.  The call itself rewrites the header (chain descriptor, the
//    done counter of the last-CTA protocol, the error word) and clears the two
//    count histograms the Z pass adds into, all of which must start at zero;
//    the ln P(D) partials are written before they are read.
//    Two calls whose kernels overlap on the GPU (different streams, or
//    different host threads without ordering) race on the array.
//  * The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; that may
//    load this library's device code.  Make the first call before any stream
//    capture.  The cached address belongs to the device's context: after a
//    cudaDeviceReset the library has to be loaded again.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "stgpu.h"
#include "st_kernels.h"
#include "st_types.h"

namespace st {
namespace {

constexpr size_t kScratchBytes = ST_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;
constexpr int kClasses[] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 16, 20, 24, 32};

// One array per device that loads the library.  Host code must not pass the
// name to a kernel: on the host it is only a stand-in for the symbol.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_dev[kMaxDevices];  // device address of g_scratch, per device

// Header at the start of the array, rewritten by every call.
struct Head {
  ChainDev chain;
  int prefix[4];
  unsigned ctr[kCtrCount];
  int rep;
  int err;
};

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

int k_class(int K) {
  for (int k : kClasses)
    if (k >= K) return k;
  return 0;
}

// Copies the Z pass's histograms into the caller's layouts:
// n_out[l][k][a] = npart[k][a][l], m_out[i][k] = mpart[i][k].
__global__ void noalloc_sum_kernel(const Head* head, const int32_t* npart, const int32_t* mpart,
                                   const double* stats, int32_t* n_out, int32_t* m_out,
                                   double* like_out, int32_t* err_out) {
  const ChainDev& h = head->chain;
  const int L = h.L, K = h.K, N = h.N;
  const size_t nn = (size_t)K * 2 * L, nm = (size_t)N * K;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < nn + nm; j += stride) {
    if (j < nn) {
      const size_t l = j % L, ka = j / L;
      n_out[l * (size_t)K * 2 + ka] = npart[j];
    } else {
      m_out[j - nn] = mpart[j - nn];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (like_out) *like_out = stats[kStLike];
    if (err_out) *err_out = head->err;
  }
}

// Device address of g_scratch on `device` (which is current), looked up once.
int scratch_addr(int device, void** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_dev[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return ST_ERR_CUDA;
    g_scratch_dev[device] = p;
  }
  *out = g_scratch_dev[device];
  return ST_OK;
}

int run(int device, const uint32_t* g2, int wpr, int N, int L, int K, const float* Q,
        const float* P, uint64_t seed, int rep, int32_t* n_out, int32_t* m_out,
        double* like_out, int32_t* err_out, cudaStream_t stream, size_t* scratch_bytes) {
  const int KT = k_class(K);
  int T, W, R;
  default_zpass_tile(N, L, K, &T, &W, &R);   // the tile a chain of this shape gets
  const int nchunks = (N + T - 1) / T;
  const int lblocks = (L + 32 * W - 1) / (32 * W);
  const int ngroups = (lblocks + R - 1) / R;
  const size_t ntiles = (size_t)nchunks * ngroups;

  // scratch layout: head | stats | likepart | n histogram | m histogram
  const size_t o_stats = align256(sizeof(Head));
  const size_t o_like = o_stats + align256(sizeof(double) * kStSize);
  const size_t o_n = o_like + align256(sizeof(double) * ntiles);
  const size_t nbytes = sizeof(int32_t) * (size_t)K * 2 * L;
  const size_t mbytes = sizeof(int32_t) * (size_t)N * K;
  const size_t o_m = o_n + align256(nbytes);
  const size_t need = o_m + align256(mbytes);
  if (scratch_bytes) *scratch_bytes = need;
  if (need > kScratchBytes) return ST_ERR_ADMISSION;

  void* base = nullptr;
  int rc = scratch_addr(device, &base);
  if (rc != ST_OK) return rc;
  unsigned char* s = static_cast<unsigned char*>(base);

  Head hd;
  memset(&hd, 0, sizeof hd);  // zero done counters, error word, unused pointers
  ChainDev& h = hd.chain;
  h.N = N; h.L = L; h.K = K; h.A = 2;
  h.G = 1;
  while (h.G < K) h.G <<= 1;
  h.layout = kLayoutB2G; h.wpr = wpr; h.Leff = L;
  h.numboxes = 1; h.metrofreq = 1;
  {
    // seed32 of the chain seed, as st_chain_create derives it (splitmix64,
    // Steele, Lea & Flood 2014; low word)
    uint64_t z = seed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    h.key = (uint32_t)z;
  }
  h.tileT = T; h.tileW = W; h.tileR = R;
  h.nchunks = nchunks; h.ngroups = ngroups;
  h.cnt_chunks = 1; h.cnt_groups = 1;
  h.g2 = g2;
  h.Q = const_cast<float*>(Q);
  h.P = const_cast<float*>(P);
  h.npart = reinterpret_cast<int32_t*>(s + o_n);
  h.mpart = reinterpret_cast<int32_t*>(s + o_m);
  h.stats = reinterpret_cast<double*>(s + o_stats);
  h.likepart = reinterpret_cast<double*>(s + o_like);
  Head* dhead = reinterpret_cast<Head*>(s);
  h.ctr = dhead->ctr;
  h.rep = &dhead->rep;
  h.err = &dhead->err;
  hd.rep = rep;

  // pageable source: the call returns once the bytes are staged
  if (cudaMemcpyAsync(dhead, &hd, sizeof hd, cudaMemcpyHostToDevice, stream) != cudaSuccess)
    return ST_ERR_CUDA;
  // the Z pass adds into the histograms: they must start at zero
  if (cudaMemsetAsync(s + o_n, 0, nbytes, stream) != cudaSuccess ||
      cudaMemsetAsync(s + o_m, 0, mbytes, stream) != cudaSuccess)
    return ST_ERR_CUDA;

  LaunchSet ls;
  ls.chains = &dhead->chain;
  ls.prefix = dhead->prefix;
  ls.nchains = 1;
  ls.total_ctas = (int)ntiles;
  ls.stream = stream;
  const size_t smem = zpass_b2g_smem(KT, K, T, W, kZNormal);
  if (launch_zpass_b2g(ls, KT, W, kZNormal, like_out ? kZfLikeAlways : 0, smem) != cudaSuccess)
    return ST_ERR_CUDA;

  const size_t total = (size_t)K * 2 * L + (size_t)N * K;
  size_t blocks = (total + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  noalloc_sum_kernel<<<(unsigned)blocks, 256, 0, stream>>>(
      dhead, h.npart, h.mpart, h.stats, n_out, m_out, like_out, err_out);
  return cudaGetLastError() == cudaSuccess ? ST_OK : ST_ERR_CUDA;
}

}  // namespace
}  // namespace st

extern "C" int st_update_z_noalloc(int device, const uint32_t* g2, int32_t wpr,
                                   int32_t num_inds, int32_t num_loci, int32_t maxpops,
                                   const float* Q, const float* P, uint64_t seed, int32_t rep,
                                   int32_t* n_out, int32_t* m_out, double* like_out,
                                   int32_t* err_out, void* cuda_stream, size_t* scratch_bytes) {
  if (scratch_bytes) *scratch_bytes = 0;
  if (!g2 || !Q || !P || !n_out || !m_out) return ST_ERR_ARG;
  if (num_inds < 1 || num_loci < 1 || rep < 0) return ST_ERR_ARG;
  if (maxpops < 1 || maxpops > st::kMaxPops) return ST_ERR_ARG;
  if (wpr < (num_inds + 15) / 16) return ST_ERR_ARG;
  if (device < 0 || device >= st::kMaxDevices) return ST_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return ST_ERR_NODEVICE;
  }
  if (device >= ndev) return ST_ERR_ARG;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return ST_ERR_CUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return ST_ERR_CUDA;
  const int rc = st::run(device, g2, wpr, num_inds, num_loci, maxpops, Q, P, seed, rep, n_out,
                         m_out, like_out, err_out, static_cast<cudaStream_t>(cuda_stream),
                         scratch_bytes);
  if (prev != device) cudaSetDevice(prev);
  return rc;
}
