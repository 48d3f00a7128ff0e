/*
 * diag.cu — the relaxation ceiling of one graph on this GPU.
 *
 * Measures what one pass over every edge costs in the memory system alone,
 * with the distances of a finished solve resident: (0) streaming each edge's
 * {dst, w} and its source's distance (12 bytes per edge), (1) the same plus
 * the random 4-byte gather of dist[dst] and the comparison a relaxation
 * makes, (2) the same plus a min-reduction on every edge whose comparison
 * succeeds (none do on final distances, so (2) also shows the cost of the
 * branch), (3) a min-reduction on every edge with no gather.  The engines
 * relax edges this way, so (1) bounds any push-based schedule: it is the
 * figure behind the roofline discussion.  No counterpart in the reference.
 */
#include <cuda_runtime.h>

#include <vector>

#include "../../include/adds.h"
#include "adds_internal.h"

void adds_graph_internal(const adds_graph *g, const unsigned **row, const uint2 **edges,
                         uint32_t *n, uint64_t *m, int *device);
void adds_set_last_error(const char *msg);

namespace {

/* the source distance of every edge (a one-time layout for the pass) */
__global__ void k_edge_src_dist(const unsigned *row, const unsigned *dist, unsigned n,
                                unsigned *edu) {
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const unsigned d = dist[v];
    for (unsigned e = row[v]; e < row[v + 1]; ++e) edu[e] = d;
  }
}

template <int MODE>
__global__ void k_pass(const uint2 *edges, const unsigned *edu, unsigned *dist,
                       unsigned long long m, unsigned long long *sink) {
  constexpr int U = 4;
  unsigned long long acc = 0;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x * U;
  for (unsigned long long i0 = (unsigned long long)blockIdx.x * blockDim.x * U + threadIdx.x;
       i0 < m; i0 += stride) {
    uint2 e[U];
    unsigned du[U];
    bool ok[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned long long i = i0 + (unsigned long long)u * blockDim.x;
      ok[u] = i < m;
      if (ok[u]) {
        e[u] = __ldg(edges + i);
        du[u] = __ldg(edu + i);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!ok[u]) continue;
      const unsigned nd = du[u] + e[u].y; /* the int sum; a float sum costs the same */
      if (MODE == 0) acc += e[u].x ^ nd;
      if (MODE == 1) acc += nd < __ldcg(dist + e[u].x);
      if (MODE == 2) {
        if (nd < __ldcg(dist + e[u].x))
          asm volatile("red.relaxed.gpu.global.min.u32 [%0], %1;" ::"l"(dist + e[u].x), "r"(nd)
                       : "memory");
      }
      if (MODE == 3)
        asm volatile("red.relaxed.gpu.global.min.u32 [%0], %1;" ::"l"(dist + e[u].x), "r"(nd)
                     : "memory");
    }
  }
  if (acc == 0xFFFFFFFFFFFFFFFFull) atomicAdd(sink, acc); /* keeps the loads alive */
}

}  // namespace

extern "C" int adds_diag_relax_pass(adds_graph *g, uint32_t src, double ms_out[4]) {
  if (!g || !ms_out) return ADDS_ERR_INVALID;
  const unsigned *row;
  const uint2 *edges;
  uint32_t n;
  uint64_t m;
  int dev;
  adds_graph_internal(g, &row, &edges, &n, &m, &dev);
  if (src >= n) return ADDS_ERR_INVALID;
  if (cudaSetDevice(dev) != cudaSuccess) return ADDS_ERR_CUDA;
  /* the final distances of one solve from src */
  unsigned *dist = nullptr, *scratch = nullptr, *edu = nullptr;
  unsigned long long *sink = nullptr;
  int rc = ADDS_OK;
  cudaEvent_t a = nullptr, z = nullptr;
  if (cudaMalloc(&dist, (size_t)n * 4) != cudaSuccess ||
      cudaMalloc(&scratch, (size_t)n * 4) != cudaSuccess ||
      cudaMalloc(&edu, (m ? m : 1) * 4) != cudaSuccess || cudaMalloc(&sink, 8) != cudaSuccess ||
      cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&z) != cudaSuccess) {
    cudaGetLastError();
    rc = ADDS_ERR_OOM;
  }
  if (!rc) rc = adds_sssp(g, src, dist, nullptr, nullptr);
  if (!rc) {
    k_edge_src_dist<<<592, 256>>>(row, dist, n, edu);
    const int blocks = 148 * 8, threads = 256;
    for (int mode = 0; mode < 4 && !rc; ++mode) {
      float best = 1e30f;
      for (int r = 0; r < 4; ++r) {
        cudaMemcpy(scratch, dist, (size_t)n * 4, cudaMemcpyDeviceToDevice);
        cudaEventRecord(a);
        switch (mode) {
          case 0: k_pass<0><<<blocks, threads>>>(edges, edu, scratch, m, sink); break;
          case 1: k_pass<1><<<blocks, threads>>>(edges, edu, scratch, m, sink); break;
          case 2: k_pass<2><<<blocks, threads>>>(edges, edu, scratch, m, sink); break;
          default: k_pass<3><<<blocks, threads>>>(edges, edu, scratch, m, sink); break;
        }
        cudaEventRecord(z);
        if (cudaEventSynchronize(z) != cudaSuccess) {
          rc = ADDS_ERR_CUDA;
          break;
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, a, z);
        if (r > 0 && ms < best) best = ms; /* the first round warms up */
      }
      ms_out[mode] = best;
    }
    if (!rc && cudaGetLastError() != cudaSuccess) rc = ADDS_ERR_CUDA;
  }
  if (a) cudaEventDestroy(a);
  if (z) cudaEventDestroy(z);
  cudaFree(dist);
  cudaFree(scratch);
  cudaFree(edu);
  cudaFree(sink);
  return rc;
}
