/*
 * noalloc.cu — a solve entry point that allocates no device memory.
 *
 * Some callers cannot let a library allocate: a framework that owns every
 * byte of device memory through its own caching allocator or a fixed arena
 * (a foreign cudaMalloc takes memory outside its budget and cudaFree
 * synchronises the whole device), or a latency-bound service loop where the
 * implicit synchronisation of cudaMalloc/cudaFree is not acceptable.
 * adds_sssp_noalloc serves them: the caller passes the graph and the output
 * as device arrays it already owns, and all the engine's working memory
 * (bucket page pool, page tables, bucket counters, split-row ring, control
 * block) comes from one file-scope device array of fixed size declared
 * below.  The array exists on every GPU that loads this library, from the
 * moment the library's code is loaded on it until the process exits.
 *
 * Limits: n <= ADDS_NOALLOC_MAX_N vertices, m <= ADDS_NOALLOC_MAX_M edges;
 * larger graphs are rejected with ADDS_ERR_UNSUPPORTED.  Because the page
 * pool cannot grow, a graph within the limits whose queues still outgrow
 * the pool reports ADDS_ERR_WL_OVERFLOW (the allocating entry point
 * adds_sssp would regrow and rerun instead).
 *
 * Every call uses the same array.  It keeps whatever the previous call left
 * there, so each call first clears the state that must start at zero.  Calls
 * whose work overlaps on the GPU (two streams, or two host threads) share
 * that memory and race; issue them one after another.
 */
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include "../../include/adds.h"
#include "adds_internal.h"

/* engine.cu */
cudaError_t adds_engine_prepare(bool flt, int block, int *max_blocks_per_sm);
cudaError_t adds_engine_launch_init(const EngParams &P, unsigned max_n, cudaStream_t st);
cudaError_t adds_engine_launch_solve(const EngParams &P, int block, cudaStream_t st);
cudaError_t adds_engine_launch_reset(unsigned long long *fq, unsigned fq_cells,
                                     unsigned pool_pages, unsigned *hub_seq, unsigned hub_cells,
                                     cudaStream_t st);
void adds_set_last_error(const char *msg);

namespace {

/* layout of the scratch array (byte offsets) */
constexpr unsigned kPoolPages = 1536;              /* 1536 x 4096 entries x 8 B = 48 MiB */
constexpr unsigned kFqCells = 2048;                /* power of two >= kPoolPages        */
constexpr unsigned kPtnLog2 = 11;                  /* page-table ring per slot           */
constexpr unsigned kHubCells = 1u << ADDS_HUB_RING_LOG2;
constexpr size_t kOffG = 0;                                        /* GlobalCtl  */
constexpr size_t kOffQd = 4096;                                    /* QueryDesc  */
constexpr size_t kOffCtl = kOffQd + 256;                           /* QueryCtl   */
constexpr size_t kOffSum = kOffCtl + 256;                          /* weight sum */
constexpr size_t kOffSlots = 8192;                                 /* 2*NB slots */
constexpr size_t kOffPgen = kOffSlots + 2 * ADDS_NB * sizeof(SlotCtr);
constexpr size_t kOffPcons = kOffPgen + kPoolPages * 4;
constexpr size_t kOffFq = (kOffPcons + kPoolPages * 4 + 255) & ~size_t(255);
constexpr size_t kOffHubSeq = kOffFq + kFqCells * 8;
constexpr size_t kOffHub = (kOffHubSeq + kHubCells * 4 + 255) & ~size_t(255);
constexpr size_t kOffPt = kOffHub + (size_t)kHubCells * sizeof(HubChunk);
constexpr size_t kPtWords = (size_t)2 * ADDS_NB << kPtnLog2;
constexpr size_t kOffPool = (kOffPt + kPtWords * 8 + 4095) & ~size_t(4095);
constexpr size_t kEnd = kOffPool + (size_t)kPoolPages * ADDS_PAGE * 8;
static_assert(sizeof(GlobalCtl) <= kOffQd, "control block does not fit");
static_assert(sizeof(QueryDesc) <= 256 && sizeof(QueryCtl) <= 256, "descriptor does not fit");
static_assert(kEnd <= ADDS_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the array");

}  // namespace

/* The engine's working memory for adds_sssp_noalloc.  In host code this
 * name is only a handle for the runtime: its device address is obtained
 * with cudaGetSymbolAddress (once per device) and handed to the kernels. */
static __device__ __align__(256) unsigned char g_noalloc_scratch[ADDS_NOALLOC_SCRATCH_BYTES];

namespace {

__global__ void na_setup(GlobalCtl *g, QueryDesc *qd, QueryDesc desc, unsigned pool_pages,
                         double *wsum) {
  /* clear-to-zero state was memset by the host; set the rest */
  g->fq_tail = pool_pages;
  *qd = desc;
  *wsum = 0.0;
}

/* mean of evenly spaced weights (the delta heuristic needs the scale) */
__global__ void na_sample(const uint2 *edges, unsigned long long m, int is_float, unsigned ns,
                          double *out) {
  double acc = 0;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x) {
    const unsigned long long e = (unsigned long long)((double)i * (double)m / (double)ns);
    const unsigned x = edges[e < m ? e : m - 1].y;
    acc += is_float ? (double)__uint_as_float(x) : (double)x;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, o);
  if ((threadIdx.x & 31u) == 0u) atomicAdd(out, acc);
}

struct DevState {
  unsigned char *base = nullptr; /* device address of g_noalloc_scratch */
  int ctas = 0;
};
DevState g_dev[64];

}  // namespace

extern "C" int adds_sssp_noalloc(uint32_t n, uint64_t m, const uint32_t *row_start,
                                 const uint32_t *edges, adds_wtype wt, uint32_t src,
                                 uint32_t *dist, void *stream) {
  if (!row_start || (m && !edges) || !dist || n == 0 || src >= n ||
      (wt != ADDS_I32 && wt != ADDS_F32))
    return ADDS_ERR_INVALID;
  if (n > ADDS_NOALLOC_MAX_N || m > ADDS_NOALLOC_MAX_M) {
    adds_set_last_error("graph exceeds the no-allocation limits "
                        "(n <= ADDS_NOALLOC_MAX_N, m <= ADDS_NOALLOC_MAX_M)");
    return ADDS_ERR_UNSUPPORTED;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return ADDS_ERR_NO_DEVICE;
  }
  DevState &D = g_dev[dev];
  cudaStream_t st = (cudaStream_t)stream;
  const bool flt = wt == ADDS_F32;
  const int block = 256;
#define NA_CK(x)                                  \
  do {                                            \
    cudaError_t _e = (x);                         \
    if (_e != cudaSuccess) {                      \
      char _m[200];                               \
      snprintf(_m, sizeof _m, "%s: %s", #x, cudaGetErrorString(_e)); \
      adds_set_last_error(_m);                    \
      cudaGetLastError();                         \
      return ADDS_ERR_CUDA;                       \
    }                                             \
  } while (0)
  if (!D.base) {
    /* once per device, with that device current: the scratch array's
     * device address, and how many solver CTAs fit */
    void *p = nullptr;
    NA_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    int bps_i = 0, bps_f = 0, sms = 0;
    NA_CK(adds_engine_prepare(false, block, &bps_i));
    NA_CK(adds_engine_prepare(true, block, &bps_f));
    NA_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int bps = bps_i < bps_f ? bps_i : bps_f;
    if (bps < 1) return ADDS_ERR_UNSUPPORTED;
    D.ctas = bps * sms;
    D.base = (unsigned char *)p;
  }
  unsigned char *B = D.base;
  GlobalCtl *g = (GlobalCtl *)(B + kOffG);
  QueryDesc *qd = (QueryDesc *)(B + kOffQd);
  QueryCtl *ctl = (QueryCtl *)(B + kOffCtl);
  double *wsum = (double *)(B + kOffSum);
  SlotCtr *slots = (SlotCtr *)(B + kOffSlots);
  unsigned *pgen = (unsigned *)(B + kOffPgen);
  unsigned *pcons = (unsigned *)(B + kOffPcons);
  unsigned long long *fq = (unsigned long long *)(B + kOffFq);
  unsigned *hub_seq = (unsigned *)(B + kOffHubSeq);
  HubChunk *hub = (HubChunk *)(B + kOffHub);
  unsigned long long *pt = (unsigned long long *)(B + kOffPt);
  unsigned long long *pool = (unsigned long long *)(B + kOffPool);

  /* the delta heuristic of the allocating path: bucket width from the mean
   * weight and the mean degree */
  const unsigned ns = (unsigned)(m < (1u << 16) ? m : (1u << 16));
  double sum = 0.0;
  NA_CK(cudaMemsetAsync(wsum, 0, 8, st));
  if (ns) {
    na_sample<<<64, 256, 0, st>>>((const uint2 *)edges, m, flt, ns, wsum);
    NA_CK(cudaGetLastError());
    NA_CK(cudaMemcpyAsync(&sum, wsum, 8, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
  }
  const double avg_w = ns ? sum / ns : 1.0;
  const double deg = (double)m / n > 1.0 ? (double)m / n : 1.0;
  const double aw = avg_w > 1e-30 ? avg_w : 1.0;
  const float scale = (float)(65536.0 / aw);
  const double dk = flt ? 8.0 * 65536.0 / deg : 8.0 * (avg_w > 1.0 ? avg_w : 1.0) / deg;
  int shift = 0;
  while (shift < 31 && (double)(1u << (shift + 1)) <= dk * 1.41421356) ++shift;

  /* clear the state that must start at zero (the array keeps the previous
   * call's contents) */
  NA_CK(cudaMemsetAsync(pool, 0, (size_t)kPoolPages * ADDS_PAGE * 8, st));
  NA_CK(cudaMemsetAsync(g, 0, sizeof(GlobalCtl), st));
  NA_CK(cudaMemsetAsync(ctl, 0, sizeof(QueryCtl), st));
  NA_CK(cudaMemsetAsync(slots, 0, 2 * ADDS_NB * sizeof(SlotCtr), st));
  NA_CK(cudaMemsetAsync(pgen, 0, kPoolPages * 4, st));
  NA_CK(cudaMemsetAsync(pcons, 0, kPoolPages * 4, st));
  NA_CK(cudaMemsetAsync(pt, 0xFF, kPtWords * 8, st));
  NA_CK(adds_engine_launch_reset(fq, kFqCells, kPoolPages, hub_seq, kHubCells, st));
  QueryDesc desc;
  memset(&desc, 0, sizeof desc);
  desc.row = row_start;
  desc.edges = (const uint2 *)edges;
  desc.split = nullptr; /* the weight-sorted copy would need memory */
  desc.dist = dist;
  desc.n = n;
  desc.src = src;
  desc.scale = scale;
  desc.ptn_log2 = kPtnLog2;
  desc.pt = pt;
  desc.slots = slots;
  desc.ctl = ctl;
  desc.shift0 = (unsigned)shift;
  desc.graph_id = 0;
  na_setup<<<1, 1, 0, st>>>(g, qd, desc, kPoolPages, wsum);
  NA_CK(cudaGetLastError());

  EngParams P;
  memset(&P, 0, sizeof P);
  P.qs = qd;
  P.nq = 1;
  P.nctas = (unsigned)D.ctas;
  P.g = g;
  P.pool = pool;
  P.pgen = pgen;
  P.pcons = pcons;
  P.fq = fq;
  P.fq_mask = kFqCells - 1u;
  P.pool_pages = kPoolPages;
  P.hub = hub;
  P.hub_seq = hub_seq;
  P.timeout_ns = 20000ull * 1000000ull;
  P.alloc_wait_ns = 200ull * 1000000ull;
  P.window = 2;
  P.batch_max = block;
  P.hub_threshold = 16384;
  P.hub_chunk = 4096;
  P.strict_order = 1;
  P.adapt = 0;
  P.is_float = flt ? 1u : 0u;
  P.single_src = 0xFFFFFFFFu;
  P.local_max = block;
  P.local_max_hungry = block / 8;
  P.block = block;
  P.greed = 4;
  NA_CK(adds_engine_launch_init(P, n, st));
  NA_CK(adds_engine_launch_solve(P, block, st));
  unsigned err[2] = {0, 0};
  NA_CK(cudaMemcpyAsync(err, &g->err, 8, cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
#undef NA_CK
  if (err[0] == ADDS_DEV_OK) return ADDS_OK;
  char msg[120];
  snprintf(msg, sizeof msg, "device error %u at wait site %u", err[0], err[1]);
  adds_set_last_error(msg);
  return (err[0] == ADDS_DEV_OVERFLOW || err[0] == ADDS_DEV_HUB_OVERFLOW) ? ADDS_ERR_WL_OVERFLOW
                                                                          : ADDS_ERR_DEVICE_TIMEOUT;
}
