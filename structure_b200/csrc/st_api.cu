// st_api.cu -- the C ABI (include/stgpu.h): contexts with HBM admission,
// genotype upload and packing, chain state, the per-update entry points, the
// fused sweep and the batched sweep.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <map>
#include <mutex>
#include <unordered_map>
#include <cuda_runtime.h>
#include "stgpu.h"
#include "st_kernels.h"

using namespace st;

struct st_ctx {
  int device = 0;
  size_t budget = 0, in_use = 0;
  cudaStream_t stream = nullptr;       // launch stream (own or caller's)
  cudaStream_t own = nullptr;
  std::string err;
  int64_t launches = 0;
  bool profile = false;
  struct Ev { cudaEvent_t a, b; int kind; };
  std::vector<Ev> evs;
  double prof_ms[ST_K_COUNT] = {0};
  int64_t prof_n[ST_K_COUNT] = {0};
  // device blocks of destroyed chains / data sets kept for reuse: creating
  // chains of a shape seen before then needs no cudaMalloc (whose cost swings
  // by tens of ms when the driver must map fresh memory)
  std::multimap<size_t, void*> cache;   // size -> block
  size_t cached = 0;
  std::unordered_map<void*, size_t> live;   // block -> size, for ctx_free
};

struct st_data {
  st_ctx* ctx = nullptr;
  int N = 0, L = 0, A = 1, layout = kLayoutU8, wpr = 0, Leff = 0;
  uint32_t* g2 = nullptr;
  uint8_t* g8 = nullptr;
  int32_t* numalleles = nullptr;
  int32_t* popflags = nullptr;
  std::vector<int32_t> na_h;
  std::vector<int32_t> popflags_h, population_h;   // population empty: no POPDATA
  std::vector<int32_t> location_h;                 // empty: no location data
  std::vector<int64_t> cnt_h;    // [L][A] allele copies observed
  std::vector<int64_t> tot_h;    // [L] non-missing copies
  // the initial eps of the data set's chains (src/Init.c:173-240) for one
  // (FREQSCORR, LAMBDA), on the device: [L][A]
  double* eps0 = nullptr;
  int eps0_fc = -1;
  double eps0_lambda = 0.0;
  size_t bytes = 0;
  int chains = 0;
};

struct st_chain {
  st_ctx* ctx = nullptr;
  st_data* data = nullptr;
  st_model model{};
  ChainDev h{};
  ChainDev* d_chain = nullptr;
  int* d_prefix = nullptr;
  std::vector<void*> allocs;
  size_t bytes = 0;
  int host_rep = 0;
  bool fast = false;
  int KT = 0;
  size_t zsmem = 0;
  double* d_injected = nullptr;
  size_t injected_n = 0;
  int tile_min_t = 0;      // Z-pass tiles the scratch was sized for: T >= tile_min_t,
  int tile_min_r = 1;      // R >= tile_min_r (fast path; the autotuner stays inside)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;
  bool timed = false;
  GradArgs mcur{}, mprop{};   // Langevin move: current and proposed Q passes
};

// Chains of one K capacity class: a contiguous slice of the batch table,
// advanced by one Z-pass launch per step.
struct ZGroup {
  int first = 0, n = 0;    // slice of the batch table
  int KT = 0, W = 8;
  size_t zsmem = 0;
  int tz = 0;              // CTAs of the slice
  bool same = false;       // one data set and tile for the whole slice (kZfInterleave)
};

struct st_batch {
  st_ctx* ctx = nullptr;
  std::vector<st_chain*> chains;   // sorted by K class
  ChainDev* d_table = nullptr;
  int* d_pz = nullptr;     // prefix: Z pass (restarting at 0 in every group)
  int* d_pl = nullptr;     // prefix: locus kernel (over d_table_l)
  ChainDev* d_table_l = nullptr;   // the table in the locus kernel's CTA order
  int* d_pi = nullptr;     // prefix: individual kernel
  int tz = 0, tl = 0, ti = 0;
  std::vector<ZGroup> zg;  // fast path: one Z launch per K class
  int G = 1;
  bool fast = false;
  bool graphs = true;                          // replay captured sweeps
  cudaGraphExec_t gx[2] = {nullptr, nullptr};  // [Gibbs sweep, Metropolis sweep]
  int glaunches[2] = {0, 0};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<ChainDev> table;             // host copies of the device tables
  std::vector<ChainDev> table_l;
  std::vector<int> pz, pl, pi;
  std::vector<cudaStream_t> aux;           // one per K class (several classes only)
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
};

namespace {

constexpr int kBlockLoc = 256;
constexpr int kBlockInd = 256;
constexpr int kBlockCol = 256;
const int kFastK[] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 16, 20, 24, 32};

int seterr(st_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

int cuda_check(st_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return ST_OK;
  return seterr(ctx, ST_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}
#define ST_CUDA(ctx, call)                                            \
  do {                                                                \
    int _r = cuda_check((ctx), (call), #call);                        \
    if (_r != ST_OK) return _r;                                       \
  } while (0)

constexpr size_t kCacheMax = (size_t)8 << 30;   // bytes kept for reuse per context

void ctx_release_cache(st_ctx* ctx) {
  for (auto& kv : ctx->cache) cudaFree(kv.second);
  ctx->cache.clear();
  ctx->cached = 0;
}

// Device memory for a chain, data set or gradient workspace, under the
// context's admission budget; a cached block of a fitting size (at most a
// quarter larger) is reused before cudaMalloc is called.
int ctx_alloc(st_ctx* ctx, size_t bytes, void** p, std::vector<void*>* track, size_t* acc) {
  *p = nullptr;
  if (bytes == 0) return ST_OK;
  if (ctx->in_use + bytes > ctx->budget)
    return seterr(ctx, ST_ERR_ADMISSION,
                  "admission: %zu bytes requested, %zu of %zu in use", bytes, ctx->in_use,
                  ctx->budget);
  size_t got = bytes;
  auto it = ctx->cache.lower_bound(bytes);
  if (it != ctx->cache.end() && it->first <= bytes + bytes / 4) {
    got = it->first;
    *p = it->second;
    ctx->cached -= got;
    ctx->cache.erase(it);
  } else {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess && ctx->cached) {   // give the cache back and try again
      cudaGetLastError();
      ctx_release_cache(ctx);
      e = cudaMalloc(p, bytes);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      *p = nullptr;
      return seterr(ctx, ST_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
  }
  ctx->live[*p] = got;
  ctx->in_use += got;
  if (track) track->push_back(*p);
  if (acc) *acc += got;
  return ST_OK;
}

// Returns a block from ctx_alloc.  The caller has synchronised whatever may
// still use it; the block goes to the cache (or back to the driver when the
// cache is full).
void ctx_free(st_ctx* ctx, void* p) {
  if (!p) return;
  auto it = ctx->live.find(p);
  if (it == ctx->live.end()) return;
  const size_t n = it->second;
  ctx->live.erase(it);
  ctx->in_use -= n;
  if (ctx->cached + n <= kCacheMax) {
    ctx->cache.emplace(n, p);
    ctx->cached += n;
  } else {
    cudaFree(p);
  }
}

int pow2_at_least(int k) {
  int g = 1;
  while (g < k) g <<= 1;
  return g;
}

int fast_kt(int K) {
  for (int k : kFastK)
    if (k >= K) return k;
  return 0;
}

// Bracket one launch with events when profiling; always count it.
struct Bracket {
  st_ctx* ctx;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  Bracket(st_ctx* c, int k) : ctx(c), kind(k) {
    ctx->launches++;
    if (ctx->profile) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, ctx->stream);
    }
  }
  ~Bracket() {
    if (ctx->profile) {
      cudaEventRecord(b, ctx->stream);
      ctx->evs.push_back({a, b, kind});
    }
  }
};

LaunchSet single(st_chain* c, int ctas) {
  LaunchSet ls;
  ls.chains = c->d_chain;
  ls.prefix = c->d_prefix;
  ls.nchains = 1;
  ls.total_ctas = ctas;
  ls.stream = c->ctx->stream;
  return ls;
}

int upload_chain(st_chain* c) {
  return cuda_check(c->ctx, cudaMemcpyAsync(c->d_chain, &c->h, sizeof(ChainDev),
                                            cudaMemcpyHostToDevice, c->ctx->stream),
                    "upload chain");
}

int set_rep(st_chain* c, int rep) {
  c->host_rep = rep;
  return cuda_check(c->ctx, cudaMemcpyAsync(c->h.rep, &c->host_rep, sizeof(int),
                                            cudaMemcpyHostToDevice, c->ctx->stream),
                    "set rep");
}

// Z-pass tiling heuristic: W warps of 32 loci, T individuals per chunk (a
// multiple of 16), R locus blocks per CTA.  Shared memory is kept under
// 72 KB so three 256-thread CTAs fit on an SM where the K class allows.
size_t zpass_smem_all(int KT, int K, int T, int W) {
  size_t s = 0;
  for (int mode : {kZNormal, kZMetro, kZInit, kZRecount, kZLike})
    s = std::max(s, zpass_b2g_smem(KT, K, T, W, mode));
  return s;
}

void choose_tile(const st_model* m, int N, int L, int K, int* T, int* W, int* R) {
  const int KT = fast_kt(K);
  int w = zpass_b2g_width(KT);
  int t = m->tile_t > 0 ? m->tile_t : 256;
  t = (t + 15) & ~15;
  const int np = (N + 15) & ~15;
  if (t > np) t = np;
  if (m->tile_t <= 0) {
    // three CTAs per SM (72 KB each) if a tile of >= 128 individuals fits,
    // else two (112 KB each; 226 KB with the per-CTA reserve) rather than
    // tiles so small that the per-lane allele table is rebuilt every few
    // rows (the wide classes' tables and Q rows take the most)
    auto fits = [&](int tt, size_t b) { return zpass_smem_all(KT, K, tt, w) <= b; };
    int t3 = t;
    while (t3 > 128 && !fits(t3, 72 * 1024)) t3 -= 16;
    if (fits(t3, 72 * 1024)) {
      t = t3;
    } else {
      while (t > 32 && !fits(t, 112 * 1024)) t -= 16;
    }
  }
  while (t > 16 && zpass_smem_all(KT, K, t, w) > 200 * 1024) t -= 16;
  int r = m->tile_r;
  if (r <= 0) {
    const long lblocks = (L + 32 * w - 1) / (32 * w);
    const long nch = (N + t - 1) / t;
    const long target = 148L * 3 * 2;
    r = (int)std::max(1L, (lblocks * nch) / target);
    if (r > 64) r = 64;
  }
  *T = t;
  *W = w;
  *R = r;
}

int zpass(st_chain* c, int mode, int flags) {
  Bracket br(c->ctx, mode == kZMetro ? ST_K_METRO : (mode == kZNormal ? ST_K_ZPASS : ST_K_OTHER));
  st_ctx* ctx = c->ctx;
  if (mode == kZNormal || mode == kZInit || mode == kZRecount) {
    ST_CUDA(ctx, cudaMemsetAsync(c->h.npart, 0, sizeof(int32_t) * (size_t)c->h.K * c->h.A * c->h.L, ctx->stream));
    ST_CUDA(ctx, cudaMemsetAsync(c->h.mpart, 0, sizeof(int32_t) * (size_t)c->h.N * c->h.K, ctx->stream));
  }
  if (c->fast) {
    LaunchSet ls = single(c, ctas_zpass_b2g(c->h));
    return cuda_check(c->ctx, launch_zpass_b2g(ls, c->KT, c->h.tileW, mode, flags, c->zsmem),
                      "zpass_b2g");
  }
  if (mode == kZMetro)
    ST_CUDA(ctx, cudaMemsetAsync(c->h.ldpart, 0, sizeof(double) * (size_t)c->h.N, ctx->stream));
  if (c->model.precision == 1) flags |= kZfF64;
  LaunchSet ls = single(c, ctas_zpass_u8(c->h, 256));
  return cuda_check(ctx, launch_zpass_u8(ls, mode, flags), "zpass_u8");
}

int locus(st_chain* c, int stages) {
  Bracket br(c->ctx, ST_K_LOCUS);
  LaunchSet ls = single(c, ctas_locus(c->h, kBlockLoc));
  return cuda_check(c->ctx, launch_locus(ls, stages, kBlockLoc), "locus");
}

int ind(st_chain* c, int mode, int stages) {
  Bracket br(c->ctx, ST_K_IND);
  LaunchSet ls = single(c, ctas_ind(c->h, kBlockInd));
  return cuda_check(c->ctx, launch_ind(ls, c->h.G, mode, stages, kBlockInd), "ind");
}

int check_model(st_ctx* ctx, const st_model* m) {
  if (m->maxpops < 1 || m->maxpops > kMaxPops)
    return seterr(ctx, ST_ERR_UNSUPPORTED, "MAXPOPS=%d outside 1..%d", m->maxpops, kMaxPops);
  if (m->noadmix && m->mala)
    return seterr(ctx, ST_ERR_UNSUPPORTED, "the Langevin move needs the admixture model");
  if (m->noadmix && m->admburnin >= m->burnin)
    return seterr(ctx, ST_ERR_ARG, "ADMBURNIN must finish before BURNIN (src/Util.c:70)");
  if (m->linkage) return seterr(ctx, ST_ERR_UNSUPPORTED, "LINKAGE=1 is not on the GPU path");
  if (m->usepopinfo && (m->gensback < 0 || m->gensback > 7))
    return seterr(ctx, ST_ERR_UNSUPPORTED, "GENSBACK must be in 0..7");
  if (m->usepopinfo && (m->migrprior < 0.0 || m->migrprior > 1.0))
    return seterr(ctx, ST_ERR_ARG, "MIGRPRIOR must be in [0, 1] (src/Init.c:22-26)");
  if (m->usepopinfo && m->mala)
    return seterr(ctx, ST_ERR_UNSUPPORTED, "the Langevin move does not combine with USEPOPINFO");
  if (m->locprior && m->noadmix && m->maxpops < 2)
    return seterr(ctx, ST_ERR_UNSUPPORTED, "LOCPRIOR with NOADMIX needs MAXPOPS >= 2");
  if (m->locprior && m->mala)
    return seterr(ctx, ST_ERR_UNSUPPORTED, "the Langevin move does not combine with LOCPRIOR");
  if (m->locprior && (m->maxlocprior <= 0.0 || m->locpriorstep <= 0.0 || m->locpriorinit <= 0.0 ||
                      m->locpriorinit >= m->maxlocprior))
    return seterr(ctx, ST_ERR_ARG, "LOCPRIORINIT must be in (0, MAXLOCPRIOR), LOCPRIORSTEP > 0");
  if (m->recessivealleles)
    return seterr(ctx, ST_ERR_UNSUPPORTED, "RECESSIVEALLELES=1 is not on the GPU path");
  if (m->freqscorr && (m->fpriormean <= 0 || m->fpriorsd <= 0))
    return seterr(ctx, ST_ERR_ARG, "FPRIORMEAN/FPRIORSD must be positive");
  if (m->burnin < 0 || m->numreps < 0) return seterr(ctx, ST_ERR_ARG, "negative BURNIN/NUMREPS");
  if (m->ancestdist && m->numboxes < 1) return seterr(ctx, ST_ERR_ARG, "NUMBOXES < 1");
  if (m->precision != 0 && m->precision != 1) return seterr(ctx, ST_ERR_ARG, "precision must be 0 or 1");
  if (m->mala && (m->maxpops > kGradMaxK || m->precision != 0))
    return seterr(ctx, ST_ERR_UNSUPPORTED, "the Langevin move needs K <= %d and FP32", kGradMaxK);
  if (m->mala_target < 0 || m->mala_target >= 1000)
    return seterr(ctx, ST_ERR_ARG, "mala_target must be in 0..999 (acceptance x 1000)");
  return ST_OK;
}

}  // namespace

// The Z-pass tile a chain of this shape gets by default (st_model tile fields
// zero), for callers without a chain (st_update_z_noalloc).
void st::default_zpass_tile(int N, int L, int K, int* T, int* W, int* R) {
  st_model m{};
  st_model_defaults(&m);
  m.tile_t = m.tile_w = m.tile_r = 0;
  choose_tile(&m, N, L, K, T, W, R);
}

// ===========================================================================
// context
// ===========================================================================
extern "C" int st_version(void) { return STGPU_VERSION; }

extern "C" int st_ctx_create(int device, size_t hbm_budget, st_ctx** out) {
  if (!out) return ST_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return ST_ERR_NODEVICE;
  }
  if (device < 0 || device >= n) return ST_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return ST_ERR_CUDA;
  st_ctx* ctx = new st_ctx();
  ctx->device = device;
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  const size_t reserve = (size_t)2 << 30;
  ctx->budget = hbm_budget ? hbm_budget : (fr > reserve ? fr - reserve : fr / 2);
  if (cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return ST_ERR_CUDA;
  }
  ctx->stream = ctx->own;
  *out = ctx;
  return ST_OK;
}

extern "C" int st_ctx_destroy(st_ctx* ctx) {
  if (!ctx) return ST_ERR_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& e : ctx->evs) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
  ctx_release_cache(ctx);
  cudaStreamDestroy(ctx->own);
  delete ctx;
  return ST_OK;
}

extern "C" int st_ctx_set_stream(st_ctx* ctx, void* stream) {
  if (!ctx) return ST_ERR_ARG;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own;
  return ST_OK;
}

extern "C" int st_ctx_profile(st_ctx* ctx, int enable) {
  if (!ctx) return ST_ERR_ARG;
  ctx->profile = enable != 0;
  return ST_OK;
}

extern "C" int st_ctx_profile_read(st_ctx* ctx, double* ms, int64_t* n) {
  if (!ctx) return ST_ERR_ARG;
  cudaSetDevice(ctx->device);
  ST_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (auto& e : ctx->evs) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, e.a, e.b) == cudaSuccess) {
      ctx->prof_ms[e.kind] += t;
      ctx->prof_n[e.kind] += 1;
    }
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  cudaGetLastError();
  ctx->evs.clear();
  for (int k = 0; k < ST_K_COUNT; k++) {
    if (ms) ms[k] = ctx->prof_ms[k];
    if (n) n[k] = ctx->prof_n[k];
    ctx->prof_ms[k] = 0.0;
    ctx->prof_n[k] = 0;
  }
  return ST_OK;
}

extern "C" int64_t st_ctx_launches(const st_ctx* ctx) { return ctx ? ctx->launches : -1; }

extern "C" const char* st_last_error(const st_ctx* ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}

extern "C" int st_ctx_memory(const st_ctx* ctx, size_t* in_use, size_t* budget) {
  if (!ctx) return ST_ERR_ARG;
  if (in_use) *in_use = ctx->in_use;
  if (budget) *budget = ctx->budget;
  return ST_OK;
}

// ===========================================================================
// data
// Allele counts of each locus of 2-bit packed data, 16 genotypes per word,
// on the device after the upload: one warp per locus row.  With lo / hi the
// low / high bit of every code, popcounts give the number of codes 1
// (lo & ~hi), 2 (hi & ~lo) and 3 = missing (lo & hi); padding genotypes of
// the last word are masked off.  Feeds the initial eps (Init.c:173-240).
namespace {
__global__ void count_b2g_kernel(const uint32_t* __restrict__ g2, int N, int L, int wpr, int A,
                                 long long* __restrict__ cnt, long long* __restrict__ tot) {
  const int l = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (l >= L) return;   // warp-uniform
  const uint32_t tail = (N & 15) ? (0x55555555u >> (2 * (16 - (N & 15)))) : 0x55555555u;
  const uint32_t* row = g2 + (size_t)l * wpr;
  unsigned n1 = 0, n2 = 0, n3 = 0;
  for (int w = lane; w < wpr; w += 32) {
    const uint32_t valid = w == wpr - 1 ? tail : 0x55555555u;
    const uint32_t x = row[w];
    const uint32_t lo = x & valid, hi = (x >> 1) & valid;
    n1 += __popc(lo & ~hi);
    n2 += __popc(hi & ~lo);
    n3 += __popc(lo & hi);
  }
  n1 = __reduce_add_sync(0xffffffffu, n1);
  n2 = __reduce_add_sync(0xffffffffu, n2);
  n3 = __reduce_add_sync(0xffffffffu, n3);
  if (lane == 0) {
    const long long n0 = (long long)N - n1 - n2 - n3;
    tot[l] = 2 * (n0 + n1 + n2);
    cnt[(size_t)l * A] = 2 * n0 + n1;
    if (A > 1) cnt[(size_t)l * A + 1] = 2 * (long long)n2 + n1;
  }
}

// Runs count_b2g_kernel on the uploaded words and reads the counts back.
int count_b2g_device(st_ctx* ctx, const uint32_t* g2, int N, int L, int wpr, int A,
                     int64_t* cnt_h, int64_t* tot_h) {
  void* p = nullptr;
  size_t scratch = 0;
  const size_t ncnt = (size_t)L * A;
  int rc = ctx_alloc(ctx, sizeof(long long) * (ncnt + L), &p, nullptr, &scratch);
  if (rc) return rc;
  long long* cnt = (long long*)p;
  long long* tot = cnt + ncnt;
  cudaStream_t s = ctx->stream;
  const int block = 256;
  const unsigned grid = (unsigned)(((size_t)L * 32 + block - 1) / block);
  {
    Bracket br(ctx, ST_K_OTHER);
    count_b2g_kernel<<<grid, block, 0, s>>>(g2, N, L, wpr, A, cnt, tot);
  }
  rc = cuda_check(ctx, cudaGetLastError(), "count alleles");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(cnt_h, cnt, sizeof(long long) * ncnt,
                                                cudaMemcpyDeviceToHost, s), "read counts");
  if (!rc) rc = cuda_check(ctx, cudaMemcpyAsync(tot_h, tot, sizeof(long long) * L,
                                                cudaMemcpyDeviceToHost, s), "read totals");
  if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(s), "count alleles");
  ctx_free(ctx, p);
  return rc;
}
}  // namespace

// ===========================================================================
extern "C" int st_data_upload(st_ctx* ctx, const st_data_desc* d, st_data** out) {
  if (!ctx || !d || !out) return ST_ERR_ARG;
  *out = nullptr;
  cudaSetDevice(ctx->device);
  if (d->lines != 2) return seterr(ctx, ST_ERR_UNSUPPORTED, "LINES=%d: only diploid data", d->lines);
  if (d->num_inds < 1 || d->num_loci < 1 || !d->num_alleles)
    return seterr(ctx, ST_ERR_ARG, "empty data set or missing num_alleles");
  if (!d->geno && !d->packed) return seterr(ctx, ST_ERR_ARG, "need geno or packed");
  const int N = d->num_inds, L = d->num_loci;
  st_data* s = new st_data();
  s->ctx = ctx;
  s->N = N;
  s->L = L;
  s->na_h.assign(d->num_alleles, d->num_alleles + L);
  int A = 1;
  for (int l = 0; l < L; l++) {
    if (s->na_h[l] < 0 || s->na_h[l] > 254) {
      delete s;
      return seterr(ctx, ST_ERR_ARG, "num_alleles[%d]=%d out of range", l, d->num_alleles[l]);
    }
    A = std::max(A, s->na_h[l]);
    if (s->na_h[l] > 0) s->Leff++;
  }
  if (A > kMaxAlleles) {
    delete s;
    return seterr(ctx, ST_ERR_UNSUPPORTED, "%d alleles at a locus (limit %d)", A, kMaxAlleles);
  }
  s->A = A;
  s->cnt_h.assign((size_t)L * A, 0);
  s->tot_h.assign(L, 0);

  // decide the layout and validate the genotypes
  bool b2g_ok = A <= 2;
  if (d->geno) {
    for (int i = 0; i < N; i++)
      for (int l = 0; l < L; l++) {
        int a0 = d->geno[((size_t)i * 2) * L + l], a1 = d->geno[((size_t)i * 2 + 1) * L + l];
        for (int a : {a0, a1}) {
          if (a >= 0) {
            if (a >= s->na_h[l]) {
              delete s;
              return seterr(ctx, ST_ERR_ARG, "allele %d >= num_alleles[%d]=%d", a, l, s->na_h[l]);
            }
            s->cnt_h[(size_t)l * A + a]++;
            s->tot_h[l]++;
          } else if (a != kUnassigned) {
            delete s;
            return seterr(ctx, ST_ERR_ARG, "genotype value %d: expected 0..k-1 or -9", a);
          }
        }
        if ((a0 < 0) != (a1 < 0)) b2g_ok = false;
        if (a0 >= 0 && a1 >= 0 && a0 > a1) b2g_ok = false;
      }
  } else {
    if (A > 2) {
      delete s;
      return seterr(ctx, ST_ERR_ARG, "packed genotypes need <= 2 alleles per locus");
    }
    // allele counts: on the device once the words are there (below)
  }
  int layout = d->layout;
  if (layout == ST_LAYOUT_AUTO) layout = b2g_ok ? ST_LAYOUT_B2G : ST_LAYOUT_U8;
  if (layout == ST_LAYOUT_B2G && !b2g_ok) {
    delete s;
    return seterr(ctx, ST_ERR_ARG, "data not representable at 2 bits/genotype (multi-allelic, "
                  "half-missing or non-canonical heterozygote)");
  }
  if (layout == ST_LAYOUT_U8 && !d->geno) {
    delete s;
    return seterr(ctx, ST_ERR_ARG, "U8 layout needs geno");
  }
  s->layout = layout == ST_LAYOUT_B2G ? kLayoutB2G : kLayoutU8;

  int rc;
  void* p;
  rc = ctx_alloc(ctx, sizeof(int32_t) * L, &p, nullptr, &s->bytes);
  if (rc) { delete s; return rc; }
  s->numalleles = (int32_t*)p;
  rc = ctx_alloc(ctx, sizeof(int32_t) * N, &p, nullptr, &s->bytes);
  if (rc) { ctx_free(ctx, s->numalleles); delete s; return rc; }
  s->popflags = (int32_t*)p;
  cudaMemcpy(s->numalleles, s->na_h.data(), sizeof(int32_t) * L, cudaMemcpyHostToDevice);
  std::vector<int32_t> pf(N, 0);
  if (d->popflags) pf.assign(d->popflags, d->popflags + N);
  cudaMemcpy(s->popflags, pf.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice);
  s->popflags_h = pf;
  if (d->population) s->population_h.assign(d->population, d->population + N);
  if (d->location) {
    for (int i = 0; i < N; i++)
      if (d->location[i] < 0) {
        ctx_free(ctx, s->numalleles);
        ctx_free(ctx, s->popflags);
        delete s;
        // src/Util.c:241-246
        return seterr(ctx, ST_ERR_ARG, "individual %d has negative location %d", i, d->location[i]);
      }
    s->location_h.assign(d->location, d->location + N);
  }

  if (s->layout == kLayoutB2G) {
    const int wpr = (N + 15) / 16;
    s->wpr = wpr;
    std::vector<uint32_t> words;
    const uint32_t* src = d->packed;
    if (!src) {
      words.assign((size_t)L * wpr, 0xFFFFFFFFu);
      for (int l = 0; l < L; l++)
        for (int i = 0; i < N; i++) {
          int a0 = d->geno[((size_t)i * 2) * L + l], a1 = d->geno[((size_t)i * 2 + 1) * L + l];
          uint32_t g = (a0 < 0) ? 3u : (uint32_t)(a0 + a1);
          uint32_t& w = words[(size_t)l * wpr + (i >> 4)];
          w &= ~(3u << (2 * (i & 15)));
          w |= g << (2 * (i & 15));
        }
      src = words.data();
    }
    rc = ctx_alloc(ctx, sizeof(uint32_t) * (size_t)L * wpr, &p, nullptr, &s->bytes);
    if (rc) { st_data_destroy(s); return rc; }
    s->g2 = (uint32_t*)p;
    rc = cuda_check(ctx, cudaMemcpy(s->g2, src, sizeof(uint32_t) * (size_t)L * wpr,
                                    cudaMemcpyHostToDevice), "upload packed");
    if (!rc && d->packed)
      rc = count_b2g_device(ctx, s->g2, N, L, wpr, A, s->cnt_h.data(), s->tot_h.data());
    if (rc) { st_data_destroy(s); return rc; }
  } else {
    const size_t n = (size_t)N * 2 * L;
    rc = ctx_alloc(ctx, n, &p, nullptr, &s->bytes);
    if (rc) { st_data_destroy(s); return rc; }
    s->g8 = (uint8_t*)p;
    // stage the int32 genotypes through a temporary device buffer in slices
    const size_t slice = (size_t)1 << 26;
    int32_t* tmp = nullptr;
    rc = cuda_check(ctx, cudaMalloc(&tmp, sizeof(int32_t) * std::min(n, slice)), "staging");
    if (rc) { st_data_destroy(s); return rc; }
    for (size_t off = 0; off < n; off += slice) {
      size_t m = std::min(slice, n - off);
      cudaMemcpy(tmp, d->geno + off, sizeof(int32_t) * m, cudaMemcpyHostToDevice);
      launch_pack_u8(tmp, s->g8 + off, m, 0);
      ctx->launches++;
    }
    cudaDeviceSynchronize();
    cudaFree(tmp);
    rc = cuda_check(ctx, cudaGetLastError(), "pack genotypes");
    if (rc) { st_data_destroy(s); return rc; }
  }
  *out = s;
  return ST_OK;
}

extern "C" int st_data_destroy(st_data* s) {
  if (!s) return ST_ERR_ARG;
  if (s->chains > 0) return seterr(s->ctx, ST_ERR_STATE, "data still used by %d chains", s->chains);
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  for (void* p : {(void*)s->g2, (void*)s->g8, (void*)s->numalleles, (void*)s->popflags,
                  (void*)s->eps0})
    ctx_free(s->ctx, p);
  delete s;
  return ST_OK;
}

extern "C" int st_data_layout(const st_data* s) {
  if (!s) return ST_ERR_ARG;
  return s->layout == kLayoutB2G ? ST_LAYOUT_B2G : ST_LAYOUT_U8;
}

// ===========================================================================
// model / chain
// ===========================================================================
extern "C" int st_model_defaults(st_model* m) {
  if (!m) return ST_ERR_ARG;
  memset(m, 0, sizeof(*m));
  // src/params.c:571-670 PresetValues
  m->maxpops = 2;
  m->burnin = 10000;
  m->admburnin = 2500;   // src/params.c:610 (BURNIN/4 of the preset BURNIN)
  m->gensback = 2;       // src/params.c:627
  m->migrprior = 0.05;   // src/params.c:629
  m->updatelocprior = 1; // src/params.c:660-667
  m->locpriorinit = 1.0;
  m->maxlocprior = 20.0;
  m->locpriorstep = 0.1;
  m->numreps = 20000;
  m->freqscorr = 1;
  m->onefst = 0;
  m->inferalpha = 1;
  m->popalphas = 0;
  m->inferlambda = 0;
  m->unifprioralpha = 1;
  m->computeprob = 1;
  m->pfrompopflagonly = 0;
  m->ancestdist = 0;
  m->numboxes = 1000;
  m->metrofreq = 20;
  m->alpha = 1.0;
  m->alphamax = 10.0;
  m->alphapropsd = 0.05;
  m->alphapriora = 1.0;
  m->alphapriorb = 2.0;
  m->lambda = 1.0;
  m->fpriormean = 0.1;
  m->fpriorsd = 0.1;
  return ST_OK;
}

extern "C" int st_chain_create(st_ctx* ctx, st_data* data, const st_model* model, uint64_t seed,
                               st_chain** out) {
  if (!ctx || !data || !model || !out) return ST_ERR_ARG;
  *out = nullptr;
  cudaSetDevice(ctx->device);
  int rc = check_model(ctx, model);
  if (rc) return rc;
  const int N = data->N, L = data->L, K = model->maxpops, A = data->A;
  st_chain* c = new st_chain();
  c->ctx = ctx;
  c->data = data;
  c->model = *model;
  ChainDev& h = c->h;
  h.N = N; h.L = L; h.K = K; h.A = A; h.G = pow2_at_least(K);
  h.layout = data->layout; h.wpr = data->wpr; h.Leff = data->Leff;
  h.freqscorr = model->freqscorr; h.onefst = model->onefst; h.inferalpha = model->inferalpha;
  h.popalphas = model->popalphas; h.unifprioralpha = model->unifprioralpha;
  h.inferlambda = model->inferlambda; h.popspecificlambda = model->popspecificlambda;
  h.noadmix = model->noadmix; h.admburnin = model->admburnin;
  h.usepopinfo = model->usepopinfo; h.gensback = model->gensback; h.migrprior = model->migrprior;
  h.alpha_n = N;
  // USEPOPINFO flags as src/Init.c:15-70 CheckPopPriors leaves them: everybody
  // without a POPFLAG column, then nobody whose population is outside 1..K
  std::vector<int32_t> pflag, pop1, initpop;
  if (model->usepopinfo) {
    if (data->population_h.empty()) {
      delete c;
      return seterr(ctx, ST_ERR_ARG, "USEPOPINFO needs population data (st_data_desc.population)");
    }
    pop1 = data->population_h;
    pflag.resize(N);
    int unflagged = 0;
    for (int i = 0; i < N; i++) {
      pflag[i] = model->popflag_given ? data->popflags_h[i] : 1;
      if (pflag[i] && (pop1[i] < 1 || pop1[i] > K)) pflag[i] = 0;
      if (!pflag[i]) unflagged++;
    }
    h.alpha_n = unflagged;
    if (model->inferalpha && !model->noadmix && unflagged == 0) {   // NOALPHA
      h.inferalpha = 0;
      h.noalpha = 1;
    }
    initpop.resize(N);
    for (int i = 0; i < N; i++) initpop[i] = (pop1[i] >= 1 && pop1[i] <= K) ? pop1[i] - 1 : -1;
    popinfo_plan(N, L, &h.pi_lchunks, &h.pi_lchunk_len);
  }
  // LOCPRIOR: locations numbered in increasing order of their ids
  // (src/Util.c:237-275 GetNumLocations), individuals grouped by location
  std::vector<int32_t> myloc, loc_start, loc_inds;
  if (model->locprior) {
    if (data->location_h.empty()) {
      delete c;
      return seterr(ctx, ST_ERR_ARG, "LOCPRIOR needs location data (st_data_desc.location)");
    }
    std::vector<int32_t> ids(data->location_h);
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    h.nloc = (int)ids.size();
    myloc.resize(N);
    loc_start.assign(h.nloc + 1, 0);
    for (int i = 0; i < N; i++) {
      myloc[i] = (int32_t)(std::lower_bound(ids.begin(), ids.end(), data->location_h[i]) - ids.begin());
      loc_start[myloc[i] + 1]++;
    }
    for (int l = 0; l < h.nloc; l++) loc_start[l + 1] += loc_start[l];
    loc_inds.resize(N);
    std::vector<int32_t> fill(loc_start.begin(), loc_start.end() - 1);
    for (int i = 0; i < N; i++) loc_inds[fill[myloc[i]]++] = i;
    h.locprior = 1;
    h.lp_admix = model->noadmix ? 0 : 1;
    h.updatelocprior = model->updatelocprior ? 1 : 0;
    h.locpriorstep = model->locpriorstep;
    h.maxlocprior = model->maxlocprior;
    h.lp_len = model->noadmix ? 1 + K * (h.nloc + 1) : 1;
    // with admixture UpdateAlphaLocPrior replaces UpdateAlpha whatever
    // INFERALPHA says (src/structure.c:577-590)
    if (h.lp_admix) h.inferalpha = 0;
  }
  const size_t arows = h.lp_admix ? (size_t)h.nloc + 1 : 1;
  h.computeprob = model->computeprob; h.pfrompopflagonly = model->pfrompopflagonly;
  h.ancestdist = model->ancestdist; h.numboxes = model->numboxes > 0 ? model->numboxes : 1;
  h.metrofreq = model->metrofreq; h.burnin = model->burnin;
  h.alphamax = model->alphamax; h.alphapropsd = model->alphapropsd;
  h.alphapriora = model->alphapriora; h.alphapriorb = model->alphapriorb;
  h.fpriormean = model->fpriormean; h.fpriorsd = model->fpriorsd;
  h.invsqrtnuminds = pow((double)N, -0.5);    // src/Updates/UpdateEpsilon.c:80
  {
    // splitmix64 (Steele, Lea & Flood 2014): seed32 = low word
    uint64_t z = seed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    h.key = (uint32_t)z;
  }
  h.g2 = data->g2; h.g8 = data->g8; h.numalleles = data->numalleles; h.popflags = data->popflags;
  h.loc_tpl = locus_lanes(L, K, A);

  c->fast = data->layout == kLayoutB2G && model->precision == 0 && fast_kt(K) > 0;
  if (data->layout == kLayoutB2G && !c->fast) {
    delete c;
    return seterr(ctx, ST_ERR_UNSUPPORTED, "FP64 Z arithmetic needs U8 data (ST_LAYOUT_U8)");
  }
  if (c->fast) {
    c->KT = fast_kt(K);
    int T, W, R;
    choose_tile(model, N, L, K, &T, &W, &R);
    h.tileT = T; h.tileW = W; h.tileR = R;
    h.nchunks = (N + T - 1) / T;
    const int lblocks = (L + 32 * W - 1) / (32 * W);
    h.ngroups = (lblocks + R - 1) / R;
    c->zsmem = zpass_smem_all(c->KT, K, T, W);
  } else {
    h.tileT = N; h.tileW = 8; h.tileR = 1;
    h.nchunks = 1;
    h.ngroups = 1;
  }
  h.cnt_chunks = 1;
  h.cnt_groups = 1;

  const size_t NK = (size_t)N * K, LKA = (size_t)L * K * A, LA = (size_t)L * A;
  int zctas = c->fast ? ctas_zpass_b2g(h) : ctas_zpass_u8(h, 256);
  if (c->fast) {
    // room for the autotuner's smaller tiles (st_batch_autotune): T down to
    // half the chosen one at the chosen R
    c->tile_min_t = std::max(16, (h.tileT / 2 + 15) & ~15);
    c->tile_min_r = h.tileR;
    ChainDev hs = h;
    hs.nchunks = (N + c->tile_min_t - 1) / c->tile_min_t;
    zctas = std::max(zctas, ctas_zpass_b2g(hs));
  }
  ChainDev hw = h;
  hw.G = 32;  // scratch sized for the widest group a batch may impose
  const int nred = std::max(ctas_locus(hw, kBlockLoc) * K, ctas_ind(hw, kBlockInd) * (K + 1));
  struct Buf { void** p; size_t bytes; };
  void *Q, *logQ, *TQ, *lTQ, *P, *logP, *eps, *F, *alpha, *lambda, *Z = nullptr, *npart, *mpart,
      *ldpart, *QSum, *PSum, *SumEps, *FstSum, *sumAlpha, *sumlambda, *AD = nullptr, *stats,
      *likepart, *redpart, *ctr, *rep, *err, *chain, *prefix;
  std::vector<Buf> bufs = {
      {&Q, NK * 4}, {&logQ, NK * 4}, {&TQ, NK * 4}, {&lTQ, NK * 4}, {&P, LKA * 4},
      {&logP, LKA * 4}, {&eps, LA * 8}, {&F, (size_t)K * 8}, {&alpha, arows * K * 8},
      {&lambda, (size_t)K * 8}, {&npart, LKA * 4},
      {&mpart, NK * 4}, {&ldpart, (size_t)h.ngroups * N * 8},
      {&QSum, NK * 8}, {&PSum, LKA * 8}, {&SumEps, LA * 8}, {&FstSum, (size_t)K * 8},
      {&sumAlpha, arows * K * 8}, {&sumlambda, (size_t)K * 8}, {&stats, (size_t)kStSize * 8},
      {&likepart, (size_t)zctas * 8}, {&redpart, (size_t)nred * 8},
      {&ctr, (size_t)kCtrCount * 4}, {&rep, 4}, {&err, 4}, {&chain, sizeof(ChainDev)},
      {&prefix, 16}};
  if (model->store_z) bufs.push_back({&Z, (size_t)N * 2 * L});
  void *pi_flag = nullptr, *pi_pop = nullptr, *pi_init = nullptr, *pi_use = nullptr,
       *pi_part = nullptr;
  if (model->usepopinfo) {
    const size_t KG = (size_t)K * (model->gensback + 1);
    for (Buf b : std::vector<Buf>{{&pi_flag, (size_t)N * 4}, {&pi_pop, (size_t)N * 4},
                                  {&pi_init, (size_t)N * 4}, {&pi_use, (size_t)N * KG * 8},
                                  {&pi_part, (size_t)h.pi_lchunks * N * KG * 8}})
      bufs.push_back(b);
  } else if (model->startatpopinfo && !data->population_h.empty()) {
    // STARTATPOPINFO (src/Init.c:412-413,74-117 InitFromGeogPop): copies of
    // individuals with a population in 1..K start there, the others at random
    initpop.resize(N);
    for (int i = 0; i < N; i++) {
      const int p = data->population_h[i];
      initpop[i] = (p >= 1 && p <= K) ? p - 1 : -1;
    }
    bufs.push_back({&pi_init, (size_t)N * 4});
  }
  void *lp_myloc = nullptr, *lp_start = nullptr, *lp_inds = nullptr, *lp_p = nullptr,
       *lp_sum = nullptr;
  if (model->locprior)
    for (Buf b : std::vector<Buf>{{&lp_myloc, (size_t)N * 4}, {&lp_start, (size_t)(h.nloc + 1) * 4},
                                  {&lp_inds, (size_t)N * 4}, {&lp_p, (size_t)h.lp_len * 8},
                                  {&lp_sum, (size_t)h.lp_len * 8}})
      bufs.push_back(b);
  void* napart = nullptr;
  if (model->noadmix) {
    noadmix_plan(N, L, &h.na_lchunks, &h.na_lchunk_len);
    bufs.push_back({&napart, (size_t)h.na_lchunks * NK * 8});
  }
  void *mQp = nullptr, *mG = nullptr, *mGp = nullptr, *mLL = nullptr, *mLLp = nullptr,
       *mTh = nullptr, *mThp = nullptr, *mEps = nullptr, *mgq = nullptr, *mll = nullptr,
       *mbp = nullptr;
  if (model->mala) {
    if (!c->fast || A != 2) {
      delete c;
      return seterr(ctx, ST_ERR_UNSUPPORTED, "the Langevin move needs biallelic 2-bit data");
    }
    GradArgs& g = c->mcur;
    g.N = N; g.L = L; g.K = K; g.wpr = data->wpr; g.g2 = data->g2;
    grad_plan(N, L, &g);
    for (Buf b : std::vector<Buf>{{&mQp, NK * 4}, {&mG, NK * 4}, {&mGp, NK * 4}, {&mLL, (size_t)N * 8},
                                  {&mLLp, (size_t)N * 8}, {&mTh, NK * 8}, {&mThp, NK * 8},
                                  {&mEps, (size_t)N * 4}, {&mgq, (size_t)g.lchunks * NK * 4},
                                  {&mll, (size_t)g.lchunks * N * 8}, {&mbp, (size_t)g.nblocks_q * 8}})
      bufs.push_back(b);
  }
  if (model->ancestdist) bufs.push_back({&AD, NK * (size_t)h.numboxes * 4});
  // one device allocation per chain, carved into 256-byte aligned arrays
  // (a few dozen cudaMalloc calls would dominate the chain's creation time)
  size_t arena = 0;
  for (auto& b : bufs) arena += (b.bytes + 255) & ~(size_t)255;
  void* base = nullptr;
  rc = ctx_alloc(ctx, arena, &base, &c->allocs, &c->bytes);
  if (rc) { st_chain_destroy(c); return rc; }
  {
    char* at = (char*)base;
    for (auto& b : bufs) {
      *b.p = b.bytes ? (void*)at : nullptr;
      at += (b.bytes + 255) & ~(size_t)255;
    }
  }
  h.Q = (float*)Q; h.logQ = (float*)logQ; h.TestQ = (float*)TQ; h.logTestQ = (float*)lTQ;
  h.P = (float*)P; h.logP = (float*)logP; h.eps = (double*)eps; h.F = (double*)F;
  h.alpha = (double*)alpha; h.lambda = (double*)lambda; h.Z = (uint8_t*)Z;
  h.npart = (int32_t*)npart; h.mpart = (int32_t*)mpart; h.ldpart = (double*)ldpart;
  h.QSum = (double*)QSum; h.PSum = (double*)PSum; h.SumEps = (double*)SumEps;
  h.FstSum = (double*)FstSum; h.sumAlpha = (double*)sumAlpha; h.sumlambda = (double*)sumlambda;
  h.AncestDist = (int32_t*)AD; h.stats = (double*)stats; h.likepart = (double*)likepart;
  h.redpart = (double*)redpart; h.ctr = (unsigned*)ctr; h.rep = (int*)rep; h.err = (int*)err;
  c->d_chain = (ChainDev*)chain;
  c->d_prefix = (int*)prefix;
  data->chains++;
  h.napart = (double*)napart;
  if (model->locprior) {
    h.myloc = (const int32_t*)lp_myloc;
    h.loc_start = (const int32_t*)lp_start;
    h.loc_inds = (const int32_t*)lp_inds;
    h.locp = (double*)lp_p;
    h.sumlocp = (double*)lp_sum;
  }
  if (!initpop.empty()) h.initpop = (const int32_t*)pi_init;
  if (model->usepopinfo) {
    h.popflags = (int32_t*)pi_flag;
    h.population = (const int32_t*)pi_pop;
    h.usepop = (double*)pi_use;
    h.pipart = (double*)pi_part;
  }
  h.mala = model->mala ? 1 : 0;
  h.mala_target = (model->mala_target > 0 ? model->mala_target : 574) / 1000.0f;
  if (model->mala) {
    h.mQp = (float*)mQp; h.mG = (float*)mG; h.mGp = (float*)mGp; h.mLL = (double*)mLL;
    h.mLLp = (double*)mLLp; h.mTh = (double*)mTh; h.mThp = (double*)mThp; h.mEps = (float*)mEps;
    GradArgs& g = c->mcur;
    g.P = h.P; g.Q = h.Q; g.gqpart = mgq; g.llpart = (double*)mll; g.blockpart = (double*)mbp;
    g.dq = h.mG; g.ll_ind = h.mLL;
    c->mprop = g;
    c->mprop.Q = h.mQp; c->mprop.dq = h.mGp; c->mprop.ll_ind = h.mLLp;
  }

  // ---- Initialization (src/Init.c:329-444, src/structure.c:51-58) ---------
  cudaStream_t s = ctx->stream;
  const int fc = model->freqscorr ? 1 : 0;
  if (!data->eps0 || data->eps0_fc != fc || data->eps0_lambda != model->lambda) {
    // src/Init.c:173-240 InitFreqPriors, once per data set and prior; a chain
    // created earlier may still be reading the previous values
    std::vector<double> ev(LA, 0.0);
    for (int l = 0; l < L; l++)
      for (int a = 0; a < data->na_h[l]; a++)
        ev[(size_t)l * A + a] = fc
            ? (((double)model->lambda + (double)data->cnt_h[(size_t)l * A + a]) /
               ((double)data->na_h[l] * (double)model->lambda + (double)data->tot_h[l]))
            : model->lambda;
    rc = cuda_check(ctx, cudaStreamSynchronize(s), "chain init");
    if (!rc && !data->eps0) rc = ctx_alloc(ctx, LA * 8, (void**)&data->eps0, nullptr, &data->bytes);
    if (!rc)
      rc = cuda_check(ctx, cudaMemcpyAsync(data->eps0, ev.data(), LA * 8, cudaMemcpyHostToDevice, s),
                      "initial eps");
    if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(s), "initial eps");
    if (rc) { st_chain_destroy(c); return rc; }
    data->eps0_fc = fc;
    data->eps0_lambda = model->lambda;
  }
  cudaMemsetAsync(h.P, 0, LKA * 4, s);
  cudaMemsetAsync(h.logP, 0, LKA * 4, s);
  cudaMemsetAsync(h.TestQ, 0, NK * 4, s);
  cudaMemsetAsync(h.logTestQ, 0, NK * 4, s);
  cudaMemsetAsync(h.QSum, 0, NK * 8, s);
  cudaMemsetAsync(h.PSum, 0, LKA * 8, s);
  cudaMemsetAsync(h.SumEps, 0, LA * 8, s);
  cudaMemsetAsync(h.FstSum, 0, K * 8, s);
  cudaMemsetAsync(h.sumAlpha, 0, arows * K * 8, s);
  cudaMemsetAsync(h.sumlambda, 0, K * 8, s);
  cudaMemsetAsync(h.stats, 0, kStSize * 8, s);
  cudaMemsetAsync(h.ctr, 0, kCtrCount * 4, s);
  cudaMemsetAsync(h.rep, 0, 4, s);
  cudaMemsetAsync(h.err, 0, 4, s);
  cudaMemsetAsync(h.ldpart, 0, (size_t)h.ngroups * N * 8, s);
  if (h.AncestDist) cudaMemsetAsync(h.AncestDist, 0, NK * (size_t)h.numboxes * 4, s);
  std::vector<float> e0;
  if (h.mala) {
    // first Langevin step ~ the posterior scale of a logit with 2L copies;
    // adapted per individual during burn-in
    e0.assign(N, (float)(1.0 / sqrt(2.0 * L + 1.0)));
    cudaMemcpyAsync(h.mEps, e0.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s);
  }
  std::vector<double> lpv;
  if (h.locprior) {
    // LocPrior = 1/K everywhere, r = LOCPRIORINIT (src/Init.c:359-368)
    lpv.assign(h.lp_len, 1.0 / K);
    lpv[0] = model->locpriorinit;
    cudaMemcpyAsync(lp_myloc, myloc.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(lp_start, loc_start.data(), (size_t)(h.nloc + 1) * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(lp_inds, loc_inds.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(lp_p, lpv.data(), (size_t)h.lp_len * 8, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(lp_sum, 0, (size_t)h.lp_len * 8, s);
  }
  if (!initpop.empty())
    cudaMemcpyAsync(pi_init, initpop.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s);
  if (h.usepopinfo) {
    cudaMemcpyAsync(pi_flag, pflag.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(pi_pop, pop1.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(pi_use, 0, (size_t)N * K * (h.gensback + 1) * 8, s);
  }
  // descriptor, prefix, Q = 1/K, eps, F, alpha = ALPHA for every location row
  // (src/Init.c:350-368), lambda: one kernel, no host copy to wait on
  rc = cuda_check(ctx,
                  launch_init_chain(h, c->d_chain, c->d_prefix, data->eps0, (int)arows,
                                    (float)(1.0 / K), (float)log(1.0 / K),
                                    fc ? model->fpriormean : 0.5, model->alpha, model->lambda, s),
                  "chain init");
  if (!rc) rc = zpass(c, kZInit, model->store_z ? kZfStoreZ : 0);
  if (!rc) rc = cuda_check(ctx, cudaGetLastError(), "chain init");
  if (rc) { st_chain_destroy(c); return rc; }
  cudaEventCreate(&c->ev0);
  cudaEventCreate(&c->ev1);
  *out = c;
  return ST_OK;
}

extern "C" int st_chain_destroy(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  cudaSetDevice(c->ctx->device);
  cudaStreamSynchronize(c->ctx->stream);
  for (void* p : c->allocs) ctx_free(c->ctx, p);
  if (c->d_injected) ctx_free(c->ctx, c->d_injected);
  if (c->h.N) c->data->chains--;
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  delete c;
  return ST_OK;
}

// ===========================================================================
// per-update entry points
// ===========================================================================
extern "C" int st_update_p(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  cudaSetDevice(c->ctx->device);
  return locus(c, kLocP);
}

extern "C" int st_update_eps(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  if (!c->h.freqscorr) return seterr(c->ctx, ST_ERR_STATE, "UpdateEpsilon needs FREQSCORR=1");
  cudaSetDevice(c->ctx->device);
  return locus(c, kLocEps);
}

extern "C" int st_update_fst(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  if (!c->h.freqscorr) return seterr(c->ctx, ST_ERR_STATE, "UpdateFst needs FREQSCORR=1");
  cudaSetDevice(c->ctx->device);
  return locus(c, kLocFst);
}

// NOADMIX schedule (src/Updates/UpdateQ.c:738-745, UpdateAlpha.c:204): the
// one-population update from sweep ADMBURNIN+1 (or BURNIN+1), admixture Gibbs
// before it; alpha moves only before sweep ADMBURNIN (or BURNIN+1).
static bool noadmix_q(const ChainDev& h, int rep) {
  // "don't use ADMBURNIN with LOCPRIOR models" (src/Updates/UpdateQ.c:731)
  return h.noadmix && (rep > h.admburnin || rep > h.burnin || h.locprior);
}
static bool alpha_moves(const ChainDev& h, int rep) {
  return !(h.noadmix && (rep >= h.admburnin || rep > h.burnin));
}

static int popinfo_step(st_chain* c) {
  Bracket br(c->ctx, ST_K_IND);
  c->ctx->launches++;   // two kernels
  return cuda_check(c->ctx, launch_popinfo(c->h, c->d_chain, c->ctx->stream), "popinfo");
}

static int update_q_impl(st_chain* c, int stages) {
  const int rep = c->host_rep;
  // USEPOPINFO individuals first (src/Updates/UpdateQ.c:734-736), then the
  // others by the model's own update, which leaves the flagged ones alone
  if (c->h.usepopinfo)
    if (int rc = popinfo_step(c)) return rc;
  if (!alpha_moves(c->h, rep)) stages &= ~kIndAlpha;
  if (noadmix_q(c->h, rep)) {
    {
      Bracket br(c->ctx, ST_K_IND);
      c->ctx->launches++;   // two kernels
      int rc = cuda_check(c->ctx, launch_noadmix(c->h, c->d_chain, c->ctx->stream), "noadmix");
      if (rc) return rc;
    }
    return ind(c, kIndNone, stages);
  }
  if (!c->h.noadmix && c->h.metrofreq > 0 && rep % c->h.metrofreq == 0) {
    int rc = ind(c, kIndPropose, 0);
    if (!rc) rc = zpass(c, kZMetro, 0);
    if (!rc) rc = ind(c, kIndAccept, stages);
    return rc;
  }
  return ind(c, kIndGibbs, stages);
}

extern "C" int st_update_q(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  cudaSetDevice(c->ctx->device);
  return update_q_impl(c, 0);
}

extern "C" int st_update_z(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  cudaSetDevice(c->ctx->device);
  return zpass(c, kZNormal, c->model.store_z ? kZfStoreZ : 0);
}

static int alpha_locprior_step(st_chain* c);

extern "C" int st_update_alpha(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  cudaSetDevice(c->ctx->device);
  if (c->h.lp_admix) return alpha_locprior_step(c);   // UpdateAlphaLocPrior
  if (!c->h.inferalpha) return seterr(c->ctx, ST_ERR_STATE, "UpdateAlpha needs INFERALPHA=1");
  return ind(c, kIndNone, kIndAlpha);
}

extern "C" int st_collect(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  cudaSetDevice(c->ctx->device);
  int rc = ST_OK;
  if (c->h.computeprob) rc = zpass(c, kZLike, kZfLikeAlways);
  if (rc) return rc;
  Bracket br(c->ctx, ST_K_OTHER);
  LaunchSet ls = single(c, ctas_collect(c->h, kBlockCol));
  return cuda_check(c->ctx, launch_collect(ls, kBlockCol), "collect");
}

// CalcLike (src/CalcLike.c:387-426): ln P(D|Q,P) of the chain's current
// state, sums untouched.
extern "C" int st_calc_like(st_chain* c, double* like) {
  if (!c || !like) return ST_ERR_ARG;
  cudaSetDevice(c->ctx->device);
  if (int rc = zpass(c, kZLike, kZfLikeAlways)) return rc;
  ST_CUDA(c->ctx, cudaMemcpyAsync(like, c->h.stats + kStLike, sizeof(double), cudaMemcpyDeviceToHost,
                                  c->ctx->stream));
  ST_CUDA(c->ctx, cudaStreamSynchronize(c->ctx->stream));
  return ST_OK;
}

extern "C" int st_update_z_injected(st_chain* c, const double* u, size_t n, int precision) {
  if (!c || !u) return ST_ERR_ARG;
  if (c->fast || c->h.layout != kLayoutU8)
    return seterr(c->ctx, ST_ERR_STATE, "injected uniforms need U8 data (ST_LAYOUT_U8)");
  if (n != (size_t)c->h.N * c->h.L * 2)
    return seterr(c->ctx, ST_ERR_ARG, "need N*L*2 = %zu uniforms", (size_t)c->h.N * c->h.L * 2);
  if (precision != 32 && precision != 64) return seterr(c->ctx, ST_ERR_ARG, "precision 32 or 64");
  cudaSetDevice(c->ctx->device);
  if (c->injected_n != n) {
    if (c->d_injected) {
      cudaStreamSynchronize(c->ctx->stream);
      ctx_free(c->ctx, c->d_injected);
    }
    c->d_injected = nullptr;
    c->injected_n = 0;
    void* p;
    int rc = ctx_alloc(c->ctx, n * 8, &p, nullptr, nullptr);
    if (rc) return rc;
    c->d_injected = (double*)p;
    c->injected_n = n;
  }
  ST_CUDA(c->ctx, cudaMemcpyAsync(c->d_injected, u, n * 8, cudaMemcpyHostToDevice, c->ctx->stream));
  c->h.injected = c->d_injected;
  int rc = upload_chain(c);
  if (rc) return rc;
  const int saved = c->model.precision;
  c->model.precision = 0;
  int flags = kZfInjected | (c->model.store_z ? kZfStoreZ : 0) | (precision == 64 ? kZfF64 : 0);
  rc = zpass(c, kZNormal, flags);
  c->model.precision = saved;
  return rc;
}

// Injected-array parity modes of UpdateP and UpdateQMetro (st_injected.cu).
// The caller's array goes to the chain's injected buffer (grown on demand,
// shared with st_update_z_injected), plus N ints of draw counts for the
// Metropolis step.
static int injected_buffer(st_chain* c, size_t doubles, size_t ints) {
  const size_t n = doubles + (ints + 1) / 2;
  if (c->injected_n >= n && c->d_injected) return ST_OK;
  if (c->d_injected) {
    cudaStreamSynchronize(c->ctx->stream);
    ctx_free(c->ctx, c->d_injected);
  }
  c->d_injected = nullptr;
  c->injected_n = 0;
  void* p;
  if (int rc = ctx_alloc(c->ctx, n * 8, &p, nullptr, nullptr)) return rc;
  c->d_injected = (double*)p;
  c->injected_n = n;
  return ST_OK;
}

extern "C" int st_update_p_injected(st_chain* c, const double* u, size_t n) {
  if (!c || !u) return ST_ERR_ARG;
  const size_t need = (size_t)c->h.L * c->h.K * c->h.A * 64;
  if (n != need)
    return seterr(c->ctx, ST_ERR_ARG, "need L*K*MAXALLELES*64 = %zu uniforms", need);
  cudaSetDevice(c->ctx->device);
  if (int rc = injected_buffer(c, n, 0)) return rc;
  ST_CUDA(c->ctx, cudaMemcpyAsync(c->d_injected, u, n * 8, cudaMemcpyHostToDevice, c->ctx->stream));
  Bracket br(c->ctx, ST_K_OTHER);
  return cuda_check(c->ctx, launch_inj_p(c->h, c->d_chain, c->d_injected, c->ctx->stream),
                    "injected UpdateP");
}

extern "C" int st_update_q_metro_injected(st_chain* c, const double* u, size_t n) {
  if (!c || !u) return ST_ERR_ARG;
  const size_t need = (size_t)c->h.N * 64;
  if (n != need) return seterr(c->ctx, ST_ERR_ARG, "need NUMINDS*64 = %zu uniforms", need);
  if (c->h.noadmix)
    return seterr(c->ctx, ST_ERR_STATE, "NOADMIX chains have no Metropolis Q update");
  cudaSetDevice(c->ctx->device);
  if (int rc = injected_buffer(c, n, (size_t)c->h.N)) return rc;
  st_ctx* ctx = c->ctx;
  int* taken = reinterpret_cast<int*>(c->d_injected + n);
  ST_CUDA(ctx, cudaMemcpyAsync(c->d_injected, u, n * 8, cudaMemcpyHostToDevice, ctx->stream));
  {
    Bracket br(ctx, ST_K_IND);
    ST_CUDA(ctx, launch_inj_metro_propose(c->h, c->d_chain, c->d_injected, taken, ctx->stream));
  }
  if (int rc = zpass(c, kZMetro, 0)) return rc;
  Bracket br(ctx, ST_K_IND);
  return cuda_check(ctx, launch_inj_metro_accept(c->h, c->d_chain, c->d_injected, taken,
                                                 ctx->stream),
                    "injected UpdateQMetro");
}

// ===========================================================================
// sweeps
// ===========================================================================
// UpdateLambda / UpdatePopLambda (src/Updates/UpdateLambda.c:8-102).
static int lambda_step(st_chain* c) {
  Bracket br(c->ctx, ST_K_OTHER);
  LaunchSet ls = single(c, ctas_lambda(c->h, 256));
  return cuda_check(c->ctx, launch_lambda(ls, 256), "lambda");
}

extern "C" int st_update_lambda(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  if (!c->h.inferlambda) return seterr(c->ctx, ST_ERR_STATE, "UpdateLambda needs INFERLAMBDA=1");
  cudaSetDevice(c->ctx->device);
  return lambda_step(c);
}

// One Langevin move on every Q_i (Z summed out, P fixed): four kernels of the
// gradient pass and two per-individual kernels.
static int mala_step(st_chain* c) {
  Bracket br(c->ctx, ST_K_OTHER);
  c->ctx->launches += 5;   // 6 kernels, the bracket counted one
  GradArgs a = c->mcur, b = c->mprop;
  a.stream = b.stream = c->ctx->stream;
  return cuda_check(c->ctx, launch_mala_step(a, b, c->d_chain), "mala");
}

extern "C" int st_update_q_mala(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  if (!c->h.mala) return seterr(c->ctx, ST_ERR_STATE, "chain created without the Langevin move");
  cudaSetDevice(c->ctx->device);
  if (c->h.K < 2) return ST_OK;
  return mala_step(c);
}

// UpdateLocPrior after the Q update (src/structure.c:535-537; with
// UPDATELOCPRIOR=0 the kernels only add the sums) and, with admixture,
// UpdateAlphaLocPrior in place of UpdateAlpha (src/structure.c:577-590).
static int locprior_step(st_chain* c) {
  Bracket br(c->ctx, ST_K_OTHER);
  if (c->h.noadmix) c->ctx->launches++;   // two kernels
  return cuda_check(c->ctx, launch_locprior(c->h, c->d_chain, c->ctx->stream), "locprior");
}
static int alpha_locprior_step(st_chain* c) {
  Bracket br(c->ctx, ST_K_OTHER);
  c->ctx->launches++;   // two kernels
  return cuda_check(c->ctx, launch_alpha_locprior(c->h, c->d_chain, c->ctx->stream),
                    "alpha locprior");
}

extern "C" int st_update_locprior(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  if (!c->h.locprior) return seterr(c->ctx, ST_ERR_STATE, "UpdateLocPrior needs LOCPRIOR=1");
  cudaSetDevice(c->ctx->device);
  return locprior_step(c);
}

static int sweep_once(st_chain* c) {
  const int zflags = (c->h.computeprob ? kZfLikeIfCollect : 0) | kZfCollect | kZfAdvance |
                     (c->model.store_z ? kZfStoreZ : 0);
  // with INFERLAMBDA, lambda is updated between P and eps (src/structure.c:586-599)
  int rc = c->h.inferlambda ? locus(c, kLocP) : locus(c, kLocP | kLocEps | kLocFst | kLocCollect);
  if (!rc && c->h.inferlambda) rc = lambda_step(c);
  if (!rc && c->h.inferlambda) rc = locus(c, kLocEps | kLocFst | kLocCollect);
  if (!rc) rc = update_q_impl(c, kIndAlpha | kIndCollect);
  if (!rc && c->h.locprior) rc = locprior_step(c);
  if (!rc && c->h.lp_admix) rc = alpha_locprior_step(c);
  if (!rc && c->h.mala && c->h.K > 1) rc = mala_step(c);
  if (!rc) rc = zpass(c, kZNormal, zflags);
  if (!rc) c->host_rep++;
  return rc;
}

extern "C" int st_sweep(st_chain* c, int nsweeps) {
  if (!c || nsweeps < 0) return ST_ERR_ARG;
  cudaSetDevice(c->ctx->device);
  cudaEventRecord(c->ev0, c->ctx->stream);
  for (int s = 0; s < nsweeps; s++) {
    int rc = sweep_once(c);
    if (rc) return rc;
  }
  cudaEventRecord(c->ev1, c->ctx->stream);
  c->timed = true;
  return ST_OK;
}

extern "C" int st_run(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  int todo = c->model.burnin + c->model.numreps - c->host_rep;
  if (todo <= 0) return ST_OK;
  int rc = st_sweep(c, todo);
  if (rc) return rc;
  return st_sync(c);
}

extern "C" int st_sync(st_chain* c) {
  if (!c) return ST_ERR_ARG;
  cudaSetDevice(c->ctx->device);
  ST_CUDA(c->ctx, cudaStreamSynchronize(c->ctx->stream));
  int e = 0;
  ST_CUDA(c->ctx, cudaMemcpy(&e, c->h.err, 4, cudaMemcpyDeviceToHost));
  if (c->timed) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->ev0, c->ev1) == cudaSuccess) c->last_ms = ms;
    cudaGetLastError();
    c->timed = false;
  }
  if (e) return seterr(c->ctx, ST_ERR_DEVICE, "device error word 0x%x", e);
  return ST_OK;
}

extern "C" int st_get_timing(st_chain* c, double* ms) {
  if (!c || !ms) return ST_ERR_ARG;
  *ms = c->last_ms;
  return ST_OK;
}

// ===========================================================================
// state
// ===========================================================================
extern "C" size_t st_field_bytes(st_chain* c, int f) {
  if (!c) return 0;
  const ChainDev& h = c->h;
  const size_t NK = (size_t)h.N * h.K, LKA = (size_t)h.L * h.K * h.A, LA = (size_t)h.L * h.A;
  switch (f) {
    case ST_F_Q: case ST_F_LOGQ: case ST_F_TESTQ: case ST_F_LOGTESTQ: return NK * 4;
    case ST_F_P: case ST_F_LOGP: return LKA * 4;
    case ST_F_EPS: case ST_F_SUMEPS: return LA * 8;
    case ST_F_F: case ST_F_LAMBDA: case ST_F_FSTSUM: case ST_F_SUMLAMBDA: return (size_t)h.K * 8;
    case ST_F_ALPHA: case ST_F_SUMALPHA:
      return (size_t)h.K * (h.lp_admix ? h.nloc + 1 : 1) * 8;
    case ST_F_Z: return (size_t)h.N * 2 * h.L;
    case ST_F_N: return LKA * 4;
    case ST_F_M: return NK * 4;
    case ST_F_LOGDIFF: return (size_t)h.N * 8;
    case ST_F_QSUM: return NK * 8;
    case ST_F_PSUM: return LKA * 8;
    case ST_F_ANCESTDIST: return NK * (size_t)h.numboxes * 4;
    case ST_F_STATS: return (size_t)kStSize * 8;
    case ST_F_REP: case ST_F_ERR: return 4;
    case ST_F_DIMS: return 32;
    case ST_F_MALA_EPS: return h.mala ? (size_t)h.N * 4 : 0;
    case ST_F_USEPOPPROBS: return h.usepopinfo ? (size_t)h.N * h.K * (h.gensback + 1) * 8 : 0;
    case ST_F_LOCPRIOR: case ST_F_SUMLOCPRIOR: return h.locprior ? (size_t)h.lp_len * 8 : 0;
    case ST_F_MYLOC: return h.locprior ? (size_t)h.N * 4 : 0;
  }
  return 0;
}

static void* field_ptr(st_chain* c, int f) {
  ChainDev& h = c->h;
  switch (f) {
    case ST_F_Q: return h.Q;
    case ST_F_LOGQ: return h.logQ;
    case ST_F_TESTQ: return h.TestQ;
    case ST_F_LOGTESTQ: return h.logTestQ;
    case ST_F_P: return h.P;
    case ST_F_LOGP: return h.logP;
    case ST_F_EPS: return h.eps;
    case ST_F_F: return h.F;
    case ST_F_ALPHA: return h.alpha;
    case ST_F_LAMBDA: return h.lambda;
    case ST_F_Z: return h.Z;
    case ST_F_QSUM: return h.QSum;
    case ST_F_PSUM: return h.PSum;
    case ST_F_SUMEPS: return h.SumEps;
    case ST_F_FSTSUM: return h.FstSum;
    case ST_F_SUMALPHA: return h.sumAlpha;
    case ST_F_SUMLAMBDA: return h.sumlambda;
    case ST_F_ANCESTDIST: return h.AncestDist;
    case ST_F_STATS: return h.stats;
    case ST_F_ERR: return h.err;
    case ST_F_MALA_EPS: return h.mEps;
    case ST_F_USEPOPPROBS: return h.usepop;
    case ST_F_LOCPRIOR: return h.locp;
    case ST_F_SUMLOCPRIOR: return h.sumlocp;
    case ST_F_MYLOC: return (void*)h.myloc;
  }
  return nullptr;
}

extern "C" int st_get_state(st_chain* c, int f, void* host, size_t bytes) {
  if (!c || !host) return ST_ERR_ARG;
  const size_t need = st_field_bytes(c, f);
  if (need == 0 || bytes != need)
    return seterr(c->ctx, ST_ERR_ARG, "field %d: %zu bytes given, %zu expected", f, bytes, need);
  cudaSetDevice(c->ctx->device);
  cudaStream_t s = c->ctx->stream;
  ST_CUDA(c->ctx, cudaStreamSynchronize(s));
  const ChainDev& h = c->h;
  if (f == ST_F_REP) { memcpy(host, &c->host_rep, 4); return ST_OK; }
  if (f == ST_F_DIMS) {
    int32_t d[8] = {h.N, h.L, h.K, h.A, h.layout, h.G, h.nchunks, h.ngroups};
    memcpy(host, d, 32);
    return ST_OK;
  }
  if (f == ST_F_N) {
    const size_t LKA = (size_t)h.L * h.K * h.A;
    std::vector<int32_t> part((size_t)h.cnt_chunks * LKA);
    ST_CUDA(c->ctx, cudaMemcpy(part.data(), h.npart, part.size() * 4, cudaMemcpyDeviceToHost));
    int32_t* o = (int32_t*)host;
    memset(o, 0, bytes);
    for (int cc = 0; cc < h.cnt_chunks; cc++)
      for (int k = 0; k < h.K; k++)
        for (int a = 0; a < h.A; a++)
          for (int l = 0; l < h.L; l++)
            o[((size_t)l * h.K + k) * h.A + a] +=
                part[(((size_t)cc * h.K + k) * h.A + a) * h.L + l];
    return ST_OK;
  }
  if (f == ST_F_M) {
    const size_t NK = (size_t)h.N * h.K;
    std::vector<int32_t> part((size_t)h.cnt_groups * NK);
    ST_CUDA(c->ctx, cudaMemcpy(part.data(), h.mpart, part.size() * 4, cudaMemcpyDeviceToHost));
    int32_t* o = (int32_t*)host;
    memset(o, 0, bytes);
    for (int g = 0; g < h.cnt_groups; g++)
      for (size_t j = 0; j < NK; j++) o[j] += part[(size_t)g * NK + j];
    return ST_OK;
  }
  if (f == ST_F_LOGDIFF) {
    std::vector<double> part((size_t)h.ngroups * h.N);
    ST_CUDA(c->ctx, cudaMemcpy(part.data(), h.ldpart, part.size() * 8, cudaMemcpyDeviceToHost));
    double* o = (double*)host;
    for (int i = 0; i < h.N; i++) {
      double s2 = 0.0;
      for (int g = 0; g < h.ngroups; g++) s2 += part[(size_t)g * h.N + i];
      o[i] = s2;
    }
    return ST_OK;
  }
  void* p = field_ptr(c, f);
  if (!p) return seterr(c->ctx, ST_ERR_STATE, "field %d not held (store_z / ancestdist off?)", f);
  ST_CUDA(c->ctx, cudaMemcpy(host, p, bytes, cudaMemcpyDeviceToHost));
  return ST_OK;
}

extern "C" int st_set_state(st_chain* c, int f, const void* host, size_t bytes) {
  if (!c || !host) return ST_ERR_ARG;
  const size_t need = st_field_bytes(c, f);
  if (need == 0 || bytes != need)
    return seterr(c->ctx, ST_ERR_ARG, "field %d: %zu bytes given, %zu expected", f, bytes, need);
  cudaSetDevice(c->ctx->device);
  cudaStream_t s = c->ctx->stream;
  ChainDev& h = c->h;
  if (f == ST_F_REP) return set_rep(c, *(const int32_t*)host);
  if (f == ST_F_DIMS || f == ST_F_LOGDIFF || f == ST_F_MYLOC)
    return seterr(c->ctx, ST_ERR_ARG, "field %d is read-only", f);
  if (f == ST_F_N || f == ST_F_M) {
    // counts become partial slice 0; the other slices are cleared
    if (f == ST_F_N) {
      const size_t LKA = (size_t)h.L * h.K * h.A;
      std::vector<int32_t> part((size_t)h.cnt_chunks * LKA, 0);
      const int32_t* in = (const int32_t*)host;
      for (int k = 0; k < h.K; k++)
        for (int a = 0; a < h.A; a++)
          for (int l = 0; l < h.L; l++)
            part[((size_t)k * h.A + a) * h.L + l] = in[((size_t)l * h.K + k) * h.A + a];
      ST_CUDA(c->ctx, cudaMemcpy(h.npart, part.data(), part.size() * 4, cudaMemcpyHostToDevice));
    } else {
      const size_t NK = (size_t)h.N * h.K;
      std::vector<int32_t> part((size_t)h.cnt_groups * NK, 0);
      memcpy(part.data(), host, NK * 4);
      ST_CUDA(c->ctx, cudaMemcpy(h.mpart, part.data(), part.size() * 4, cudaMemcpyHostToDevice));
    }
    return ST_OK;
  }
  void* p = field_ptr(c, f);
  if (!p) return seterr(c->ctx, ST_ERR_STATE, "field %d not held (store_z / ancestdist off?)", f);
  ST_CUDA(c->ctx, cudaMemcpyAsync(p, host, bytes, cudaMemcpyHostToDevice, s));
  if (f == ST_F_Q || f == ST_F_P || f == ST_F_TESTQ) {
    // keep the log companion consistent
    const size_t n = bytes / 4;
    std::vector<float> lg(n);
    const float* v = (const float*)host;
    for (size_t j = 0; j < n; j++) lg[j] = (float)log((double)v[j]);
    void* lp = f == ST_F_Q ? (void*)h.logQ : (f == ST_F_P ? (void*)h.logP : (void*)h.logTestQ);
    ST_CUDA(c->ctx, cudaMemcpyAsync(lp, lg.data(), bytes, cudaMemcpyHostToDevice, s));
    ST_CUDA(c->ctx, cudaStreamSynchronize(s));
  }
  if (f == ST_F_Z) {
    // counts follow Z (the reference's GetNumFromPops / GetNumLociPop)
    int rc = zpass(c, kZRecount, 0);
    if (rc) return rc;
  }
  ST_CUDA(c->ctx, cudaStreamSynchronize(s));
  return ST_OK;
}

// ===========================================================================
// batches
// ===========================================================================

// ---------------------------------------------------------------------------
// Batch launch layout: per-chain CTA prefixes of the three kernels and, on
// the fast path, one Z launch per K class (ZGroup).  The host copies are kept
// in the batch so the autotuner can rebuild them after changing tiles.
// ---------------------------------------------------------------------------
static int batch_layout(st_batch* b, bool keep_groups) {
  const int n = (int)b->chains.size();
  b->table.assign(n, ChainDev{});
  b->pz.assign(n, 0);
  b->pl.assign(n, 0);
  b->pi.assign(n, 0);
  b->tz = b->tl = b->ti = 0;
  if (!keep_groups) b->zg.clear();
  for (ZGroup& g : b->zg) { g.tz = 0; g.zsmem = 0; g.n = 0; }
  size_t gi = 0;
  for (int j = 0; j < n; j++) {
    st_chain* c = b->chains[j];
    b->table[j] = c->h;
    b->table[j].G = b->G;   // every chain's kernels index their groups by the batch-wide G
    if (b->fast) {
      if (!keep_groups && (b->zg.empty() || b->zg.back().KT != c->KT)) {
        ZGroup g;
        g.first = j;
        g.KT = c->KT;
        g.W = c->h.tileW;
        b->zg.push_back(g);
      }
      while (gi + 1 < b->zg.size() && j >= b->zg[gi + 1].first) gi++;
      ZGroup& g = keep_groups ? b->zg[gi] : b->zg.back();
      if (c->h.tileW != g.W)
        return seterr(b->ctx, ST_ERR_ARG, "chains of one K class must share the Z-pass width");
      b->pz[j] = g.tz;
      g.tz += ctas_zpass_b2g(b->table[j]);
      g.zsmem = std::max(g.zsmem, c->zsmem);
      g.n++;
    } else {
      b->pz[j] = b->tz;
      b->tz += ctas_zpass_u8(b->table[j], 256);
    }
    b->pi[j] = b->ti;
    b->ti += ctas_ind(b->table[j], kBlockInd);
  }
  for (ZGroup& g : b->zg) {
    const ChainDev& h0 = b->table[g.first];
    g.same = g.n > 1;
    for (int j = g.first + 1; j < g.first + g.n; j++) {
      const ChainDev& h = b->table[j];
      g.same = g.same && h.g2 == h0.g2 && h.N == h0.N && h.L == h0.L && h.wpr == h0.wpr &&
               h.tileT == h0.tileT && h.tileR == h0.tileR && h.nchunks == h0.nchunks &&
               h.ngroups == h0.ngroups;
    }
  }
  // locus kernel: chains whose CTAs take longest first (longest-processing-
  // time order), so a batch of uneven K does not end on a tail of its slowest
  // chain's CTAs; a CTA's time is about its lanes' serial gamma draws
  std::vector<int> order(n);
  for (int j = 0; j < n; j++) order[j] = j;
  auto lane_draws = [&](int j) {
    const ChainDev& h = b->table[j];
    const int tpl = h.loc_tpl;
    if (tpl <= 1) return (long)h.K * h.A;
    int J = 1;
    while (J * 2 * h.K <= tpl && J * 2 <= 32) J *= 2;
    const int kslots = tpl / J;
    return (long)((h.K + kslots - 1) / kslots) * ((h.A + J - 1) / J);
  };
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return lane_draws(x) > lane_draws(y); });
  b->table_l.resize(n);
  for (int q = 0; q < n; q++) {
    const int j = order[q];
    b->table_l[q] = b->table[j];
    b->pl[q] = b->tl;
    b->tl += ctas_locus(b->table[j], kBlockLoc);
  }
  return ST_OK;
}

static void batch_upload(st_batch* b) {
  const int n = (int)b->chains.size();
  cudaMemcpy(b->d_table, b->table.data(), sizeof(ChainDev) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(b->d_pz, b->pz.data(), 4 * n, cudaMemcpyHostToDevice);
  cudaMemcpy(b->d_pl, b->pl.data(), 4 * n, cudaMemcpyHostToDevice);
  cudaMemcpy(b->d_table_l, b->table_l.data(), sizeof(ChainDev) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(b->d_pi, b->pi.data(), 4 * n, cudaMemcpyHostToDevice);
}

// Z-pass tile (T individuals per chunk, R locus blocks per CTA) of one chain;
// false when the chain's scratch was not sized for it.
static bool set_tile(st_chain* c, int T, int R) {
  ChainDev& h = c->h;
  if (!c->fast || T < c->tile_min_t || R < c->tile_min_r || (T & 15)) return false;
  const size_t smem = zpass_smem_all(c->KT, h.K, T, h.tileW);
  if (smem > 200 * 1024) return false;
  h.tileT = T;
  h.tileR = R;
  h.nchunks = (h.N + T - 1) / T;
  const int lblocks = (h.L + 32 * h.tileW - 1) / (32 * h.tileW);
  h.ngroups = (lblocks + R - 1) / R;
  c->zsmem = smem;
  return true;
}

static bool apply_group_tile(st_batch* b, const ZGroup& g, int T, int R) {
  for (int j = g.first; j < g.first + g.n; j++) {
    st_chain* c = b->chains[j];
    const int t0 = c->h.tileT, r0 = c->h.tileR;
    if (!set_tile(c, std::min(T, (c->h.N + 15) & ~15), R)) {
      set_tile(c, t0, r0);
      for (int q = g.first; q < j; q++) set_tile(b->chains[q], b->table[q].tileT, b->table[q].tileR);
      return false;
    }
  }
  for (int j = g.first; j < g.first + g.n; j++) upload_chain(b->chains[j]);
  return true;
}

// In-process cache of tuned tiles, keyed by the K class and the shapes of the
// group's chains.
struct TileKey {
  int KT;
  std::vector<int64_t> shapes;
  bool operator<(const TileKey& o) const {
    return KT != o.KT ? KT < o.KT : shapes < o.shapes;
  }
};
static std::mutex g_tile_mu;
static std::map<TileKey, std::pair<int, int>> g_tile_cache;

static TileKey tile_key(st_batch* b, const ZGroup& g) {
  TileKey k{g.KT, {}};
  for (int j = g.first; j < g.first + g.n; j++)
    k.shapes.push_back(((int64_t)b->chains[j]->h.N << 32) | (uint32_t)b->chains[j]->h.L);
  return k;
}

static bool tile_cache_get(st_batch* b, const ZGroup& g, int* T, int* R) {
  for (int j = g.first; j < g.first + g.n; j++)
    if (b->chains[j]->model.tile_t > 0 || b->chains[j]->model.tile_r > 0) return false;
  std::lock_guard<std::mutex> lk(g_tile_mu);
  auto it = g_tile_cache.find(tile_key(b, g));
  if (it == g_tile_cache.end()) return false;
  *T = it->second.first;
  *R = it->second.second;
  return true;
}

extern "C" int st_batch_create(st_ctx* ctx, st_chain** chains, int n, st_batch** out) {
  if (!ctx || !chains || n < 1 || !out) return ST_ERR_ARG;
  *out = nullptr;
  for (int j = 0; j < n; j++)
    if (!chains[j]) return ST_ERR_ARG;
  cudaSetDevice(ctx->device);
  st_batch* b = new st_batch();
  b->ctx = ctx;
  b->chains.assign(chains, chains + n);
  // one Z launch per K class: keep each class contiguous in the table
  std::stable_sort(b->chains.begin(), b->chains.end(),
                   [](const st_chain* a, const st_chain* c) { return a->KT < c->KT; });
  st_chain* c0 = b->chains[0];
  b->fast = c0->fast;
  int G = 1;
  for (st_chain* c : b->chains) {
    if (c->ctx != ctx || c->fast != b->fast || c->h.metrofreq != c0->h.metrofreq ||
        c->host_rep != c0->host_rep || c->model.store_z != c0->model.store_z ||
        c->model.precision != c0->model.precision ||
        c->h.computeprob != c0->h.computeprob || c->h.noadmix != c0->h.noadmix ||
        (c0->h.noadmix && (c->h.admburnin != c0->h.admburnin || c->h.burnin != c0->h.burnin ||
                           c->h.locprior != c0->h.locprior))) {
      delete b;
      return seterr(ctx, ST_ERR_ARG,
                    "batched chains must share the context, data path, METROFREQ, COMPUTEPROB, "
                    "NOADMIX schedule, sweep counter and Z storage");
    }
    G = std::max(G, c->h.G);
  }
  b->G = G;
  if (int rc = batch_layout(b, false)) {
    delete b;
    return rc;
  }
  auto alloc = [&](void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    return e == cudaSuccess ? ST_OK : seterr(ctx, ST_ERR_NOMEM, "batch table");
  };
  if (alloc((void**)&b->d_table, sizeof(ChainDev) * n) || alloc((void**)&b->d_pz, 4 * n) ||
      alloc((void**)&b->d_pl, 4 * n) || alloc((void**)&b->d_pi, 4 * n) ||
      alloc((void**)&b->d_table_l, sizeof(ChainDev) * n)) {
    st_batch_destroy(b);
    return ST_ERR_NOMEM;
  }
  // tiles the autotuner found for the same shapes earlier in this process
  if (b->fast) {
    bool changed = false;
    for (ZGroup& g : b->zg) {
      int T, R;
      if (tile_cache_get(b, g, &T, &R)) changed = apply_group_tile(b, g, T, R) || changed;
    }
    if (changed) batch_layout(b, false);
  }
  batch_upload(b);
  cudaEventCreate(&b->ev0);
  cudaEventCreate(&b->ev1);
  if (b->fast && b->zg.size() > 1) {
    cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    for (size_t gi = 0; gi < b->zg.size(); gi++) {
      cudaStream_t as = nullptr;
      cudaEvent_t ev = nullptr;
      if (cudaStreamCreateWithFlags(&as, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        st_batch_destroy(b);
        return seterr(ctx, ST_ERR_CUDA, "batch streams");
      }
      b->aux.push_back(as);
      b->ev_join.push_back(ev);
    }
  }
  *out = b;
  return ST_OK;
}

// Z-pass tile autotuner: for each K class of the batch, times candidate
// tiles (T individuals per chunk x R locus blocks per CTA) on the batch's own
// chains and data with the sweep's Z pass (counts on, no ln P(D), no
// advance), keeps the fastest, and remembers it for batches of the same
// shapes created later in the process.  Draws and counts do not depend on
// the tile (Philox counters are per genotype, counts are exact), so a tuned
// batch samples the same chain; only the order of the FP64 ln P(D) partial
// sums changes.  The counts of the last Z pass are saved and restored around
// the trials.
extern "C" int st_batch_autotune(st_batch* b, int reps) {
  if (!b) return ST_ERR_ARG;
  if (!b->fast) return ST_OK;   // the generic path has one tile shape
  st_ctx* ctx = b->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  if (reps < 1) reps = 3;
  ST_CUDA(ctx, cudaStreamSynchronize(s));
  size_t total = 0;
  for (st_chain* c : b->chains)
    total += ((size_t)c->h.K * c->h.A * c->h.L + (size_t)c->h.N * c->h.K) * 4;
  char* scratch = nullptr;
  ST_CUDA(ctx, cudaMalloc((void**)&scratch, total));
  auto copy_counts = [&](bool save) {
    char* at = scratch;
    for (st_chain* c : b->chains) {
      const size_t nb = (size_t)c->h.K * c->h.A * c->h.L * 4, mb = (size_t)c->h.N * c->h.K * 4;
      cudaMemcpyAsync(save ? at : (void*)c->h.npart, save ? (void*)c->h.npart : at, nb,
                      cudaMemcpyDeviceToDevice, s);
      at += nb;
      cudaMemcpyAsync(save ? at : (void*)c->h.mpart, save ? (void*)c->h.mpart : at, mb,
                      cudaMemcpyDeviceToDevice, s);
      at += mb;
    }
  };
  copy_counts(true);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = ST_OK;
  for (size_t gi = 0; gi < b->zg.size() && rc == ST_OK; gi++) {
    ZGroup& g = b->zg[gi];
    st_chain* c0 = b->chains[g.first];
    const int T0 = c0->h.tileT, R0 = c0->h.tileR;
    std::vector<std::pair<int, int>> cand;
    for (int tm : {2, 3, 4, 5, 6, 8})
      for (int rm : {1, 2, 4, 8}) {
        const std::pair<int, int> tr{((T0 * tm / 4) + 15) & ~15, R0 * rm};
        if (std::find(cand.begin(), cand.end(), tr) == cand.end()) cand.push_back(tr);
      }
    double best = 1e300;
    int bT = T0, bR = R0;
    for (const auto& tr : cand) {
      if (!apply_group_tile(b, g, tr.first, tr.second)) continue;
      batch_layout(b, true);
      batch_upload(b);
      LaunchSet lg{b->d_table + g.first, b->d_pz + g.first, g.n, g.tz, s};
      double ms_sum = 0.0;
      for (int r = 0; r <= reps && rc == ST_OK; r++) {
        for (int j = g.first; j < g.first + g.n; j++) {
          const ChainDev& h = b->chains[j]->h;
          cudaMemsetAsync(h.npart, 0, (size_t)h.K * h.A * h.L * 4, s);
          cudaMemsetAsync(h.mpart, 0, (size_t)h.N * h.K * 4, s);
        }
        cudaEventRecord(e0, s);
        cudaError_t e = launch_zpass_b2g(lg, g.KT, g.W, kZNormal, g.same ? kZfInterleave : 0,
                                         g.zsmem);
        cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) rc = cuda_check(ctx, e, "autotune");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r > 0) ms_sum += ms;
      }
      if (rc == ST_OK && ms_sum < best) {
        best = ms_sum;
        bT = tr.first;
        bR = tr.second;
      }
    }
    apply_group_tile(b, g, bT, bR);
    std::lock_guard<std::mutex> lk(g_tile_mu);
    g_tile_cache[tile_key(b, g)] = {bT, bR};
  }
  batch_layout(b, true);
  batch_upload(b);
  copy_counts(false);
  cudaStreamSynchronize(s);
  cudaFree(scratch);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (int j = 0; j < 2; j++)   // launch shapes changed: capture the sweeps again
    if (b->gx[j]) {
      cudaGraphExecDestroy(b->gx[j]);
      b->gx[j] = nullptr;
    }
  return rc;
}

extern "C" int st_batch_destroy(st_batch* b) {
  if (!b) return ST_ERR_ARG;
  cudaSetDevice(b->ctx->device);
  for (void* p : {(void*)b->d_table, (void*)b->d_pz, (void*)b->d_pl, (void*)b->d_pi,
                  (void*)b->d_table_l})
    if (p) cudaFree(p);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  for (cudaGraphExec_t x : b->gx)
    if (x) cudaGraphExecDestroy(x);
  for (cudaStream_t as : b->aux) cudaStreamDestroy(as);
  for (cudaEvent_t ev : b->ev_join) cudaEventDestroy(ev);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  delete b;
  return ST_OK;
}

// The launches of one batched sweep in src/structure.c:497-685 order: P, eps
// and F (locus kernel); Q and alpha (individual kernel, with the Metropolis
// data pass on METROFREQ sweeps); the Z pass with counts and ln P(D).  The
// sweep index lives on the device, so the sequence depends on the host only
// through `metro`.
static int enqueue_batch_sweep(st_batch* b, bool metro) {
  st_ctx* ctx = b->ctx;
  const int n = (int)b->chains.size();
  st_chain* c0 = b->chains[0];
  cudaStream_t s = ctx->stream;
  LaunchSet lz{b->d_table, b->d_pz, n, b->tz, s};
  // one fast Z launch per K class over its slice of the table
  // one fast Z launch per K class; with several classes they run side by side
  // on forked streams (independent chains), so one class's tail overlaps the next
  auto zfast = [&](int mode, int flags) -> int {
    const bool fork = b->zg.size() > 1 && !b->aux.empty();
    if (fork) ST_CUDA(ctx, cudaEventRecord(b->ev_fork, s));
    for (size_t gi = 0; gi < b->zg.size(); gi++) {
      const ZGroup& g = b->zg[gi];
      cudaStream_t gs = fork ? b->aux[gi] : s;
      if (fork) ST_CUDA(ctx, cudaStreamWaitEvent(gs, b->ev_fork, 0));
      LaunchSet lg{b->d_table + g.first, b->d_pz + g.first, g.n, g.tz, gs};
      ST_CUDA(ctx, launch_zpass_b2g(lg, g.KT, g.W, mode, flags | (g.same ? kZfInterleave : 0),
                                    g.zsmem));
      if (fork) ST_CUDA(ctx, cudaEventRecord(b->ev_join[gi], gs));
    }
    if (fork)
      for (size_t gi = 0; gi < b->zg.size(); gi++)
        ST_CUDA(ctx, cudaStreamWaitEvent(s, b->ev_join[gi], 0));
    ctx->launches += (int64_t)b->zg.size() - 1;   // the bracket counted one
    return ST_OK;
  };
  LaunchSet ll{b->d_table_l, b->d_pl, n, b->tl, s};
  LaunchSet li{b->d_table, b->d_pi, n, b->ti, s};
  const int zflags = (c0->h.computeprob ? kZfLikeIfCollect : 0) | kZfCollect | kZfAdvance |
                     (c0->model.store_z ? kZfStoreZ : 0);
  bool lam = false;
  for (st_chain* c : b->chains) lam = lam || c->h.inferlambda;
  {
    Bracket br(ctx, ST_K_LOCUS);
    ST_CUDA(ctx, launch_locus(ll, lam ? kLocP : kLocP | kLocEps | kLocFst | kLocCollect, kBlockLoc));
  }
  if (lam) {
    for (st_chain* c : b->chains)
      if (c->h.inferlambda)
        if (int rc = lambda_step(c)) return rc;
    Bracket br(ctx, ST_K_LOCUS);
    ST_CUDA(ctx, launch_locus(ll, kLocEps | kLocFst | kLocCollect, kBlockLoc));
  }
  for (st_chain* c : b->chains)
    if (c->h.usepopinfo)
      if (int rc = popinfo_step(c)) return rc;
  if (metro) {
    {
      Bracket br(ctx, ST_K_IND);
      ST_CUDA(ctx, launch_ind(li, b->G, kIndPropose, 0, kBlockInd));
    }
    if (!b->fast)
      for (st_chain* c : b->chains)
        ST_CUDA(ctx, cudaMemsetAsync(c->h.ldpart, 0, sizeof(double) * c->h.N, s));
    {
      Bracket br(ctx, ST_K_METRO);
      if (b->fast) {
        if (int rc = zfast(kZMetro, 0)) return rc;
      } else {
        ST_CUDA(ctx, launch_zpass_u8(lz, kZMetro, c0->model.precision ? kZfF64 : 0));
      }
    }
    Bracket br(ctx, ST_K_IND);
    ST_CUDA(ctx, launch_ind(li, b->G, kIndAccept, kIndAlpha | kIndCollect, kBlockInd));
  } else {
    // NOADMIX batches share the schedule (checked at st_batch_create)
    const int rep = c0->host_rep;
    const int astage = alpha_moves(c0->h, rep) ? kIndAlpha : 0;
    if (noadmix_q(c0->h, rep)) {
      for (st_chain* c : b->chains) {
        Bracket br(ctx, ST_K_IND);
        ctx->launches++;   // two kernels
        ST_CUDA(ctx, launch_noadmix(c->h, c->d_chain, s));
      }
      Bracket br(ctx, ST_K_IND);
      ST_CUDA(ctx, launch_ind(li, b->G, kIndNone, astage | kIndCollect, kBlockInd));
    } else {
      Bracket br(ctx, ST_K_IND);
      ST_CUDA(ctx, launch_ind(li, b->G, kIndGibbs, astage | kIndCollect, kBlockInd));
    }
  }
  for (st_chain* c : b->chains) {
    if (c->h.locprior)
      if (int rc = locprior_step(c)) return rc;
    if (c->h.lp_admix)
      if (int rc = alpha_locprior_step(c)) return rc;
  }
  for (st_chain* c : b->chains)
    if (c->h.mala && c->h.K > 1)
      if (int rc = mala_step(c)) return rc;
  {   // the Z pass adds into cleared histograms: one kernel for every chain
    Bracket br(ctx, ST_K_OTHER);
    ST_CUDA(ctx, launch_clear_counts(b->d_table, n, s));
  }
  {
    Bracket br(ctx, ST_K_ZPASS);
    if (b->fast) {
      if (int rc = zfast(kZNormal, zflags)) return rc;
    } else {
      ST_CUDA(ctx, launch_zpass_u8(lz, kZNormal, zflags | (c0->model.precision ? kZfF64 : 0)));
    }
  }
  return ST_OK;
}

// Captures the sweep of kind `metro` into a CUDA graph on first use.  Returns
// false (and leaves graphs off for this batch) when capture is not possible.
static bool batch_graph(st_batch* b, bool metro) {
  st_ctx* ctx = b->ctx;
  const int j = metro ? 1 : 0;
  if (b->gx[j]) return true;
  cudaStream_t s = ctx->stream;
  const int64_t l0 = ctx->launches;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const int rc = enqueue_batch_sweep(b, metro);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  ctx->launches = l0;
  if (rc != ST_OK || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return false;
  }
  cudaGraphExec_t x = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&x, g, 0);
  size_t nodes = 0;
  cudaGraphGetNodes(g, nullptr, &nodes);
  std::vector<cudaGraphNode_t> list(nodes);
  int kernels = 0;
  if (nodes && cudaGraphGetNodes(g, list.data(), &nodes) == cudaSuccess)
    for (cudaGraphNode_t nd : list) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) kernels++;
    }
  cudaGraphDestroy(g);
  if (ei != cudaSuccess || !x) {
    cudaGetLastError();
    return false;
  }
  b->gx[j] = x;
  b->glaunches[j] = kernels;
  return true;
}

extern "C" int st_batch_graphs(st_batch* b, int enable) {
  if (!b) return ST_ERR_ARG;
  b->graphs = enable != 0;
  return ST_OK;
}

extern "C" int st_batch_sweep(st_batch* b, int nsweeps) {
  if (!b || nsweeps < 0) return ST_ERR_ARG;
  st_ctx* ctx = b->ctx;
  cudaSetDevice(ctx->device);
  st_chain* c0 = b->chains[0];
  cudaStream_t s = ctx->stream;
  // graphs replay the same launches; per-launch profiling events need the
  // direct path, and the legacy default stream cannot be captured
  const bool graphs = b->graphs && !ctx->profile && s != nullptr && !c0->h.noadmix;
  cudaEventRecord(b->ev0, s);
  for (int sw = 0; sw < nsweeps; sw++) {
    const int rep = c0->host_rep;
    const bool metro = !c0->h.noadmix && c0->h.metrofreq > 0 && rep % c0->h.metrofreq == 0;
    if (graphs && batch_graph(b, metro)) {
      ST_CUDA(ctx, cudaGraphLaunch(b->gx[metro ? 1 : 0], s));
      ctx->launches += b->glaunches[metro ? 1 : 0];
    } else {
      if (graphs) b->graphs = false;
      if (int rc = enqueue_batch_sweep(b, metro)) return rc;
    }
    for (st_chain* c : b->chains) c->host_rep++;
  }
  cudaEventRecord(b->ev1, s);
  return ST_OK;
}

// ===========================================================================
// gradient of ln P(D|Q,P) w.r.t. softmax logits
// ===========================================================================
struct st_grad {
  st_ctx* ctx = nullptr;
  st_data* data = nullptr;
  int K = 0;
  bool fp64 = false;
  GradArgs a{};
  std::vector<void*> allocs;
  size_t bytes = 0;
};

extern "C" int st_grad_create(st_ctx* ctx, st_data* data, int maxpops, int precision,
                              st_grad** out) {
  if (!ctx || !data || !out) return ST_ERR_ARG;
  *out = nullptr;
  if (precision != 32 && precision != 64)
    return seterr(ctx, ST_ERR_ARG, "precision must be 32 or 64");
  if (data->layout != kLayoutB2G || data->A != 2)
    return seterr(ctx, ST_ERR_UNSUPPORTED, "the gradient needs biallelic 2-bit data");
  if (grad_kclass(maxpops) == 0)
    return seterr(ctx, ST_ERR_UNSUPPORTED, "the gradient supports K = 1..%d", kGradMaxK);
  cudaSetDevice(ctx->device);
  st_grad* g = new st_grad();
  g->ctx = ctx;
  g->data = data;
  g->K = maxpops;
  g->fp64 = precision == 64;
  GradArgs& a = g->a;
  a.N = data->N; a.L = data->L; a.K = maxpops; a.wpr = data->wpr; a.g2 = data->g2;
  grad_plan(a.N, a.L, &a);
  const size_t es = g->fp64 ? 8 : 4;
  const size_t NK = (size_t)a.N * a.K, LK2 = (size_t)a.L * a.K * 2;
  struct { void** p; size_t b; } req[] = {
      {&a.Q, NK * es}, {&a.P, LK2 * es}, {&a.gqpart, (size_t)a.lchunks * NK * es},
      {(void**)&a.llpart, (size_t)a.lchunks * a.N * 8}, {&a.gppart, (size_t)a.ichunks * LK2 * es},
      {(void**)&a.blockpart, (size_t)a.nblocks_q * 8}};
  for (auto& r : req) {
    int rc = ctx_alloc(ctx, r.b, r.p, &g->allocs, &g->bytes);
    if (rc) {
      for (void* p : g->allocs) ctx_free(ctx, p);
      delete g;
      return rc;
    }
  }
  *out = g;
  return ST_OK;
}

extern "C" int st_grad_destroy(st_grad* g) {
  if (!g) return ST_ERR_ARG;
  cudaSetDevice(g->ctx->device);
  cudaStreamSynchronize(g->ctx->stream);
  for (void* p : g->allocs) ctx_free(g->ctx, p);
  delete g;
  return ST_OK;
}

extern "C" int st_loglik_grad(st_grad* g, const void* q_logits, const void* p_logits, void* dq,
                              void* dp, double* loglik, double* ll_ind) {
  if (!g || !q_logits || !p_logits || !dq || !dp) return ST_ERR_ARG;
  st_ctx* ctx = g->ctx;
  cudaSetDevice(ctx->device);
  GradArgs a = g->a;
  a.qlog = q_logits;
  a.plog = p_logits;
  a.dq = dq;
  a.dp = dp;
  a.loglik = loglik;
  a.ll_ind = ll_ind;
  a.stream = ctx->stream;
  Bracket br(ctx, ST_K_OTHER);
  ctx->launches += 4 + (loglik ? 1 : 0);   // softmax, 2 passes, 2 finishes (+ total)
  return cuda_check(ctx, launch_loglik_grad(a, g->fp64), "loglik_grad");
}

// ===========================================================================
// checkpoint / resume
// ===========================================================================
// File: "STGPUCK1", then int32 {version, N, L, K, A, layout, ngroups, host_rep,
// store_z, ancestdist, numboxes, mala}, uint32 key, the st_model as created,
// then every device array of the chain in the order of ckpt_fields() as
// (uint64 byte count, bytes).  Philox draws are keyed by (seed, sweep, update,
// element), so a chain loaded at sweep s continues exactly as the saved one.
namespace {

constexpr char kCkptMagic[8] = {'S', 'T', 'G', 'P', 'U', 'C', 'K', '1'};
constexpr int32_t kCkptVersion = 2;   // 1 also held the Metropolis scratch (ldpart)

struct CkField { void* p; size_t bytes; };

// alpha values held: K, or K per row (global + locations) under LOCPRIOR
size_t arow_n(const ChainDev& h) { return (size_t)h.K * (h.lp_admix ? h.nloc + 1 : 1); }

std::vector<CkField> ckpt_fields(st_chain* c) {
  ChainDev& h = c->h;
  const size_t NK = (size_t)h.N * h.K, LKA = (size_t)h.L * h.K * h.A, LA = (size_t)h.L * h.A;
  std::vector<CkField> f = {
      {h.Q, NK * 4}, {h.logQ, NK * 4}, {h.TestQ, NK * 4}, {h.logTestQ, NK * 4},
      {h.P, LKA * 4}, {h.logP, LKA * 4}, {h.eps, LA * 8}, {h.F, (size_t)h.K * 8},
      {h.alpha, arow_n(h) * 8}, {h.lambda, (size_t)h.K * 8}, {h.npart, LKA * 4},
      {h.mpart, NK * 4}, {h.QSum, NK * 8},
      {h.PSum, LKA * 8}, {h.SumEps, LA * 8}, {h.FstSum, (size_t)h.K * 8},
      {h.sumAlpha, arow_n(h) * 8}, {h.sumlambda, (size_t)h.K * 8},
      {h.stats, (size_t)kStSize * 8}, {h.err, 4}};
  if (h.Z) f.push_back({h.Z, (size_t)h.N * 2 * h.L});
  if (h.AncestDist) f.push_back({h.AncestDist, NK * (size_t)h.numboxes * 4});
  if (h.mala) f.push_back({h.mEps, (size_t)h.N * 4});
  if (h.usepopinfo) f.push_back({h.usepop, (size_t)h.N * h.K * (h.gensback + 1) * 8});
  if (h.locprior) {
    f.push_back({h.locp, (size_t)h.lp_len * 8});
    f.push_back({h.sumlocp, (size_t)h.lp_len * 8});
  }
  return f;
}

void ckpt_header(st_chain* c, int32_t hdr[12]) {
  const ChainDev& h = c->h;
  const int32_t v[12] = {kCkptVersion, h.N, h.L, h.K, h.A, h.layout, h.ngroups, c->host_rep,
                         h.Z != nullptr, h.AncestDist != nullptr, h.numboxes, h.mala};
  memcpy(hdr, v, sizeof v);
}

}  // namespace

extern "C" int st_chain_save(st_chain* c, const char* path) {
  if (!c || !path) return ST_ERR_ARG;
  st_ctx* ctx = c->ctx;
  cudaSetDevice(ctx->device);
  ST_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  FILE* f = fopen(path, "wb");
  if (!f) return seterr(ctx, ST_ERR_ARG, "cannot open %s for writing", path);
  int32_t hdr[12];
  ckpt_header(c, hdr);
  bool ok = fwrite(kCkptMagic, 1, 8, f) == 8 && fwrite(hdr, 4, 12, f) == 12 &&
            fwrite(&c->h.key, 4, 1, f) == 1 && fwrite(&c->model, sizeof(st_model), 1, f) == 1;
  std::vector<char> buf;
  for (const CkField& fl : ckpt_fields(c)) {
    if (!ok) break;
    buf.resize(fl.bytes);
    if (cudaMemcpy(buf.data(), fl.p, fl.bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
      fclose(f);
      return seterr(ctx, ST_ERR_CUDA, "checkpoint read-back failed");
    }
    const uint64_t n = fl.bytes;
    ok = fwrite(&n, 8, 1, f) == 1 && fwrite(buf.data(), 1, fl.bytes, f) == fl.bytes;
  }
  if (fclose(f) != 0) ok = false;
  return ok ? ST_OK : seterr(ctx, ST_ERR_ARG, "writing %s failed", path);
}

// The options a checkpoint must share with the chain it is loaded into: every
// st_model field except the Z-pass tile (draws do not depend on it) and
// NUMREPS (only where st_run stops).  Field by field, so struct padding in the
// file never matters.
static bool same_model(const st_model& a, const st_model& b) {
#define ST_SAME(f) (a.f == b.f)
  return ST_SAME(maxpops) && ST_SAME(burnin) && ST_SAME(noadmix) && ST_SAME(linkage) &&
         ST_SAME(usepopinfo) && ST_SAME(locprior) && ST_SAME(freqscorr) && ST_SAME(onefst) &&
         ST_SAME(inferalpha) && ST_SAME(popalphas) && ST_SAME(inferlambda) &&
         ST_SAME(popspecificlambda) && ST_SAME(unifprioralpha) && ST_SAME(computeprob) &&
         ST_SAME(pfrompopflagonly) && ST_SAME(ancestdist) && ST_SAME(numboxes) &&
         ST_SAME(metrofreq) && ST_SAME(recessivealleles) && ST_SAME(alpha) &&
         ST_SAME(alphamax) && ST_SAME(alphapropsd) && ST_SAME(alphapriora) &&
         ST_SAME(alphapriorb) && ST_SAME(lambda) && ST_SAME(fpriormean) && ST_SAME(fpriorsd) &&
         ST_SAME(store_z) && ST_SAME(precision) && ST_SAME(mala) && ST_SAME(mala_target) &&
         ST_SAME(admburnin) && ST_SAME(gensback) && ST_SAME(popflag_given) &&
         ST_SAME(updatelocprior) && ST_SAME(startatpopinfo) && ST_SAME(migrprior) &&
         ST_SAME(locpriorinit) && ST_SAME(maxlocprior) && ST_SAME(locpriorstep);
#undef ST_SAME
}

extern "C" int st_chain_load(st_chain* c, const char* path) {
  if (!c || !path) return ST_ERR_ARG;
  st_ctx* ctx = c->ctx;
  cudaSetDevice(ctx->device);
  FILE* f = fopen(path, "rb");
  if (!f) return seterr(ctx, ST_ERR_ARG, "cannot open %s", path);
  char magic[8];
  int32_t hdr[12], mine[12];
  uint32_t key = 0;
  st_model model;
  bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, kCkptMagic, 8) == 0 &&
            fread(hdr, 4, 12, f) == 12 && fread(&key, 4, 1, f) == 1 &&
            fread(&model, sizeof(st_model), 1, f) == 1;
  ckpt_header(c, mine);
  if (ok && hdr[0] != kCkptVersion) {
    fclose(f);
    return seterr(ctx, ST_ERR_STATE, "%s has checkpoint format %d; this library reads %d", path,
                  hdr[0], kCkptVersion);
  }
  // the chain must have been created on the same data with the same shape;
  // the sweep counter (slot 7) is what the file restores, and the Z-pass
  // locus grouping (slot 6) may differ (tiles are chosen per chain or batch
  // and nothing saved depends on them)
  for (int j = 0; ok && j < 12; j++)
    if (j != 7 && j != 6 && hdr[j] != mine[j]) ok = false;
  if (!ok) {
    fclose(f);
    return seterr(ctx, ST_ERR_STATE, "%s is not a checkpoint of a chain of this shape", path);
  }
  if (!same_model(model, c->model)) {
    fclose(f);
    return seterr(ctx, ST_ERR_STATE,
                  "%s was saved by a chain with other model options (st_model)", path);
  }
  // every field is read and size-checked before any of the chain's device
  // memory is written, so a truncated or mismatched file leaves it unchanged
  const std::vector<CkField> fields = ckpt_fields(c);
  std::vector<std::vector<char>> bufs(fields.size());
  for (size_t j = 0; ok && j < fields.size(); j++) {
    uint64_t n = 0;
    if (fread(&n, 8, 1, f) != 1 || n != fields[j].bytes) { ok = false; break; }
    bufs[j].resize(fields[j].bytes);
    if (fread(bufs[j].data(), 1, fields[j].bytes, f) != fields[j].bytes) ok = false;
  }
  char extra;
  if (ok && fread(&extra, 1, 1, f) != 0) ok = false;   // trailing bytes: another layout
  fclose(f);
  if (!ok) return seterr(ctx, ST_ERR_STATE, "%s is truncated or of another chain", path);
  ST_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (size_t j = 0; j < fields.size(); j++)
    if (cudaMemcpy(fields[j].p, bufs[j].data(), fields[j].bytes, cudaMemcpyHostToDevice) !=
        cudaSuccess)
      return seterr(ctx, ST_ERR_CUDA, "checkpoint upload failed");
  c->h.key = key;
  c->h.cnt_chunks = 1;
  c->h.cnt_groups = 1;
  int rc = upload_chain(c);
  if (!rc) rc = set_rep(c, hdr[7]);
  if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "checkpoint load");
  return rc;
}
