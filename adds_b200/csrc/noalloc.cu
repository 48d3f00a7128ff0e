/*
 * noalloc.cu — a solve entry point that allocates no device memory.
 *
 * Some callers cannot let a library allocate: a framework that owns every
 * byte of device memory through its own caching allocator or a fixed arena
 * (a foreign cudaMalloc takes memory outside its budget and cudaFree
 * synchronises the whole device), or a latency-bound service loop where the
 * implicit synchronisation of cudaMalloc/cudaFree is not acceptable.
 * adds_sssp_noalloc serves them: the caller passes the graph and the output
 * as device arrays it already owns, and all the working memory of the phase
 * engine (bucket page pool, page tables, list tails, split-row records,
 * control block) comes from one file-scope device array of fixed size
 * declared below.  The array exists on every GPU that loads this library, from the
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
 *
 * The caller's arrays are validated on the device before the solver reads
 * them (row offsets, dst < n, weights), as the allocating path validates a
 * graph when it builds it; a failed check returns ADDS_ERR_FORMAT and the
 * solver never touches the arrays.  The bucket width is derived on the
 * device from a weight sample, so a call waits for the GPU once, at its end.
 */
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include "../../include/adds.h"
#include "adds_internal.h"
#include "phase_internal.h"

void adds_set_last_error(const char *msg);

namespace {

/* layout of the scratch array (byte offsets) */
constexpr unsigned kVariant = 0;        /* phase kernel: 256 threads, 4 CTAs per SM   */
constexpr unsigned kHubThreshold = 512; /* rows longer than this are split          */
constexpr unsigned kPtnLog2 = 11;       /* page-table ring per list (>= kPages + 2) */
constexpr unsigned kPages = 1792;       /* 1792 pages x 4096 entries x 8 B = 56 MiB */
constexpr unsigned kHubCap = 4u * (ADDS_NOALLOC_MAX_M / kHubThreshold) + 4096u;
constexpr size_t kOffG = 0;                                        /* PhGlobal     */
constexpr size_t kOffGrp = 4096;                                   /* PhGroup      */
constexpr size_t kOffQd = kOffGrp + 16384;                         /* PhQuery      */
constexpr size_t kOffSum = kOffQd + 256;                           /* weight sum   */
constexpr size_t kOffPt = kOffSum + 256;
constexpr size_t kPtBytes = ((size_t)PH_NLIST << kPtnLog2) * 8;
constexpr size_t kOffHub = (kOffPt + kPtBytes + 255) & ~size_t(255);
constexpr size_t kOffHubSeq = kOffHub + (size_t)kHubCap * sizeof(PhHub);
constexpr size_t kOffPool = (kOffHubSeq + (size_t)kHubCap * 4 + 4095) & ~size_t(4095);
constexpr size_t kEnd = kOffPool + (size_t)kPages * PH_PAGE * 8;
static_assert(sizeof(PhGlobal) <= kOffGrp, "control block does not fit");
static_assert(sizeof(PhGroup) <= kOffQd - kOffGrp, "group state does not fit");
static_assert(sizeof(PhQuery) <= 256, "descriptor does not fit");
static_assert((1u << kPtnLog2) >= kPages + 2u, "page-table ring smaller than the pool");
static_assert(kEnd <= ADDS_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the array");

}  // namespace

/* The engine's working memory for adds_sssp_noalloc.  In host code this
 * name is only a handle for the runtime: its device address is obtained
 * with cudaGetSymbolAddress (once per device) and handed to the kernels. */
static __device__ __align__(256) unsigned char g_noalloc_scratch[ADDS_NOALLOC_SCRATCH_BYTES];

namespace {

/* Failed-check bits of the validation word (the allocating path checks the
 * same properties when it builds a graph, api.cu k_check_rows /
 * k_pack_edges). */
enum : unsigned { BAD_DST = 1u, BAD_FLOAT_W = 2u, BAD_INT_W = 4u, BAD_ROWS = 8u };

/* Validation of the caller's arrays, and the mean of evenly spaced weights
 * (the bucket width needs it).  Rows: row[0] == 0, row[n] == m, offsets
 * non-decreasing; edges: dst < n, int weights in [0, INT32_MAX], float
 * weights not negative and not NaN (-0.0 is accepted: it sums like +0.0).
 * Nothing is read past row[n] or edges[m-1]. */
__global__ void na_check(const unsigned *row, const uint2 *edges, unsigned n,
                         unsigned long long m, int is_float, unsigned ns, double *wsum,
                         unsigned *bad) {
  const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  const unsigned long long nth = (unsigned long long)gridDim.x * blockDim.x;
  unsigned b = 0u;
  if (tid == 0 && (row[0] != 0u || (unsigned long long)row[n] != m)) b |= BAD_ROWS;
  for (unsigned long long v = tid; v < n; v += nth) {
    const unsigned a = row[v], e = row[v + 1];
    if (e < a || (unsigned long long)e > m) b |= BAD_ROWS;
  }
  for (unsigned long long i = tid; i < m; i += nth) {
    const uint2 x = edges[i];
    if (x.x >= n) b |= BAD_DST;
    if (is_float) {
      if (x.y != 0x80000000u && x.y > 0x7F800000u) b |= BAD_FLOAT_W;
    } else if (x.y > 0x7FFFFFFFu) {
      b |= BAD_INT_W;
    }
  }
  double acc = 0;
  for (unsigned long long i = tid; i < ns; i += nth) {
    const unsigned long long e = (unsigned long long)((double)i * (double)m / (double)ns);
    const unsigned x = edges[e < m ? e : m - 1].y;
    acc += is_float ? (double)__uint_as_float(x & 0x7FFFFFFFu) : (double)x;
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc += __shfl_down_sync(0xFFFFFFFFu, acc, o);
    b |= __shfl_down_sync(0xFFFFFFFFu, b, o);
  }
  if ((threadIdx.x & 31u) == 0u) {
    if (acc != 0.0) atomicAdd(wsum, acc);
    if (b) atomicOr(bad, b);
  }
}

/* The solve's descriptor, with the bucket width worked out here from the
 * sampled mean weight so the host never waits for it: delta ~ 4 x mean
 * weight / mean degree key units (the allocating path's starting point,
 * api.cu auto_shift), shift = nearest integer to log2(delta) in [0, 31];
 * float keys are dist * 2^16 / mean weight (api.cu auto_scale).  Arrays
 * that failed validation set the error word instead, and the solver exits
 * at its first decision without touching them. */
__global__ void na_setup(PhQuery *qd, PhQuery desc, int is_float, const double *wsum,
                         unsigned ns, const unsigned *bad, PhGlobal *g) {
  const double avg_w = ns ? *wsum / ns : 1.0;
  const double deg = (double)desc.m / desc.n > 1.0 ? (double)desc.m / desc.n : 1.0;
  const double aw = avg_w > 1e-30 ? avg_w : 1.0;
  const double dk = is_float ? 4.0 * 65536.0 / deg : 4.0 * (avg_w > 1.0 ? avg_w : 1.0) / deg;
  unsigned shift = 0;
  while (shift < 31u && (double)(1ull << shift) * 1.4142135623730951 <= dk) ++shift;
  desc.shift = shift;
  desc.scale = (float)(65536.0 / aw);
  *qd = desc;
  if (*bad != 0u) {
    g->err = PH_ERR_INPUT;
    g->err_where = *bad;
  }
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
    NA_CK(adds_phase_prepare(false, kVariant, &bps_i));
    NA_CK(adds_phase_prepare(true, kVariant, &bps_f));
    NA_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int bps = bps_i < bps_f ? bps_i : bps_f;
    if (bps < 1) return ADDS_ERR_UNSUPPORTED;
    D.ctas = bps * sms;
    D.base = (unsigned char *)p;
  }
  unsigned char *B = D.base;
  PhGlobal *g = (PhGlobal *)(B + kOffG);
  PhGroup *grp = (PhGroup *)(B + kOffGrp);
  PhQuery *qd = (PhQuery *)(B + kOffQd);
  double *wsum = (double *)(B + kOffSum);
  unsigned *bad = (unsigned *)(B + kOffSum + 8);
  unsigned long long *pt = (unsigned long long *)(B + kOffPt);
  PhHub *hub = (PhHub *)(B + kOffHub);
  unsigned *hub_seq = (unsigned *)(B + kOffHubSeq);
  unsigned long long *pool = (unsigned long long *)(B + kOffPool);

  /* clear the state that must start at zero (the array keeps the previous
   * call's contents): group barrier and lists, statistics and error word,
   * weight sum and validation word, page-table tags, split-row record
   * sequence words.  Pool pages are always written before they are read. */
  NA_CK(cudaMemsetAsync(g, 0, sizeof(PhGlobal), st));
  NA_CK(cudaMemsetAsync(grp, 0, sizeof(PhGroup), st));
  NA_CK(cudaMemsetAsync(wsum, 0, 16, st));
  NA_CK(cudaMemsetAsync(pt, 0xFF, kPtBytes, st));
  NA_CK(cudaMemsetAsync(hub_seq, 0, (size_t)kHubCap * 4, st));
  /* the caller's arrays are checked on the device before the solver reads
   * them, and the bucket width is worked out there too */
  const unsigned ns = (unsigned)(m < (1u << 16) ? m : (1u << 16));
  na_check<<<2 * 148, 256, 0, st>>>(row_start, (const uint2 *)edges, n, m, flt, ns, wsum, bad);
  NA_CK(cudaGetLastError());
  PhQuery desc;
  memset(&desc, 0, sizeof desc);
  desc.row = row_start;
  desc.edges = (const uint2 *)edges;
  desc.split = nullptr; /* the weight-sorted copy would need memory */
  desc.dist = dist;
  desc.n = n;
  desc.src = src;
  desc.m = m;
  na_setup<<<1, 1, 0, st>>>(qd, desc, flt, wsum, ns, bad, g);
  NA_CK(cudaGetLastError());

  PhParams P;
  memset(&P, 0, sizeof P);
  P.qs = qd;
  P.order = nullptr;
  P.nq = 1;
  P.groups = 1;
  P.gsize = (unsigned)D.ctas;
  P.grp = grp;
  P.g = g;
  P.pool = pool;
  P.pages_per_group = kPages;
  P.pt = pt;
  P.ptn_log2 = kPtnLog2;
  P.hub = hub;
  P.hub_seq = hub_seq;
  P.hub_cap = kHubCap;
  P.hub_threshold = kHubThreshold;
  P.hub_chunk = kHubThreshold;
  P.solo_max = 1024;
  P.adapt = 0u;
  P.lh_adapt = 1u;
  P.dense_shift = 6u;
  P.is_float = flt ? 1u : 0u;
  P.single_src = 0xFFFFFFFFu;
  P.timeout_ns = 20000ull * 1000000ull;
  NA_CK(adds_phase_launch(P, kVariant, st));
  unsigned err[2] = {0, 0};
  NA_CK(cudaMemcpyAsync(err, &g->err, 8, cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
#undef NA_CK
  if (err[0] == 0u) return ADDS_OK;
  char msg[160];
  if (err[0] == PH_ERR_INPUT) {
    snprintf(msg, sizeof msg, "invalid graph arrays:%s%s%s%s",
             (err[1] & BAD_ROWS) ? " row offsets" : "", (err[1] & BAD_DST) ? " dst >= n" : "",
             (err[1] & BAD_FLOAT_W) ? " negative or NaN float weight" : "",
             (err[1] & BAD_INT_W) ? " negative int weight" : "");
    adds_set_last_error(msg);
    return ADDS_ERR_FORMAT;
  }
  snprintf(msg, sizeof msg, "device error %u at wait site %u", err[0], err[1]);
  adds_set_last_error(msg);
  if (err[0] == PH_ERR_OVERFLOW || err[0] == PH_ERR_HUB_OVERFLOW) return ADDS_ERR_WL_OVERFLOW;
  if (err[0] == PH_ERR_MAPPING) return ADDS_ERR_CUDA;
  return ADDS_ERR_DEVICE_TIMEOUT;
}
