/*
 * gen.cu — seeded synthetic graph generators on the GPU.
 *
 * The reference measures on SuiteSparse / DIMACS / SNAP .gr files named in
 * graph_list_int / graph_list_float; those files are not available, so the
 * benchmarks run on seeded synthetic graphs of the shapes the engine is
 * specified on (R-MAT, road-like grid with local shortcuts, Erdos-Renyi,
 * plain grid).  Every random draw is a pure function of (seed, stream,
 * index) through a splitmix64-style mixer, so adds_b200/graphs.py computes
 * bit-identical graphs with numpy.  Pipeline: one 64-bit key (src<<32|dst)
 * per candidate edge (invalid ones = ~0), radix sort, unique, CSR offsets,
 * weights hashed from (src, dst) so they do not depend on draw order.
 */
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/adds.h"
#include "adds_internal.h"

namespace adds_gen {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
/* H(seed, stream, i): the only source of randomness */
__host__ __device__ __forceinline__ uint64_t H(uint64_t seed, uint64_t stream, uint64_t i) {
  const uint64_t s = mix64(seed + 0x9E3779B97F4A7C15ull * (stream + 1ull));
  return mix64(s ^ (i * 0xD1B54A32D192ED03ull + 0x8CB92BA72F3D8DD7ull));
}
__host__ __device__ __forceinline__ uint32_t mulshift(uint64_t r, uint32_t n) {
  return (uint32_t)(((r >> 32) * (uint64_t)n) >> 32);
}

enum : uint64_t { S_WEIGHT = 1000, S_SC_U = 2000, S_SC_OFF = 2001, S_ER_S = 3000, S_ER_D = 3001 };

__global__ void rmat_keys(uint64_t *keys, uint64_t ndraw, int scale, double a, double ab,
                          double abc, uint64_t seed) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ndraw;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s = 0, d = 0;
    for (int l = 0; l < scale; ++l) {
      const uint64_t r = H(seed, 1ull + (uint64_t)l, i);
      const double u = (double)(r >> 11) * 0x1.0p-53;
      const uint32_t q = u < a ? 0u : (u < ab ? 1u : (u < abc ? 2u : 3u));
      const int bit = scale - 1 - l;
      s |= (q >> 1) << bit;
      d |= (q & 1u) << bit;
    }
    keys[i] = (s == d) ? ~0ull : (((uint64_t)s << 32) | d);
  }
}

__global__ void er_keys(uint64_t *keys, uint64_t ndraw, uint32_t n, uint64_t seed) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ndraw;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = mulshift(H(seed, S_ER_S, i), n);
    const uint32_t d = mulshift(H(seed, S_ER_D, i), n);
    keys[i] = (s == d) ? ~0ull : (((uint64_t)s << 32) | d);
  }
}

/* grid: 4 directed neighbour edges per vertex (out of range = invalid),
 * then 2 keys per shortcut pair */
__global__ void grid_keys(uint64_t *keys, uint32_t sx, uint32_t sy, uint64_t npairs,
                          const int2 *offs, uint32_t noff, uint64_t seed) {
  const uint64_t n = (uint64_t)sx * sy;
  const uint64_t total = 4ull * n + 2ull * npairs;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t key = ~0ull;
    if (i < 4ull * n) {
      const uint32_t v = (uint32_t)(i >> 2), dir = (uint32_t)(i & 3u);
      const uint32_t x = v % sx, y = v / sx;
      int nx = (int)x, ny = (int)y;
      if (dir == 0) nx += 1; else if (dir == 1) nx -= 1; else if (dir == 2) ny += 1; else ny -= 1;
      if (nx >= 0 && ny >= 0 && nx < (int)sx && ny < (int)sy)
        key = ((uint64_t)v << 32) | ((uint32_t)ny * sx + (uint32_t)nx);
    } else {
      const uint64_t j = (i - 4ull * n) >> 1;
      const uint32_t u = mulshift(H(seed, S_SC_U, j), (uint32_t)n);
      const int2 o = offs[mulshift(H(seed, S_SC_OFF, j), noff)];
      const int x = (int)(u % sx) + o.x, y = (int)(u / sx) + o.y;
      if (x >= 0 && y >= 0 && x < (int)sx && y < (int)sy) {
        const uint32_t v = (uint32_t)y * sx + (uint32_t)x;
        key = ((i - 4ull * n) & 1ull) ? (((uint64_t)v << 32) | u) : (((uint64_t)u << 32) | v);
      }
    }
    keys[i] = key;
  }
}

/* row offsets from sorted unique keys; edges with hashed weights */
__global__ void build_csr(const uint64_t *keys, uint64_t m, uint32_t n, unsigned *row,
                          uint2 *edges, int is_float, double w_lo, double w_hi, uint64_t seed) {
  const uint32_t ilo = (uint32_t)w_lo;
  const uint64_t span = (uint64_t)((int64_t)w_hi - (int64_t)w_lo + 1);
  const float flo = (float)w_lo, fspan = (float)(w_hi - w_lo);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    /* row[v] = i for every v in (src(i-1), src(i)], src(-1) = -1, src(m) = n */
    const int64_t s = (i < m) ? (int64_t)(keys[i] >> 32) : (int64_t)n;
    const int64_t sprev = (i == 0) ? -1 : (int64_t)(keys[i - 1] >> 32);
    for (int64_t v = sprev + 1; v <= s; ++v) row[v] = (unsigned)i;
    if (i < m) {
      const uint32_t d = (uint32_t)keys[i];
      const uint64_t r = H(seed, S_WEIGHT, keys[i]);
      uint32_t wb;
      if (is_float) {
        const float u = (float)(uint32_t)(r >> 40) * 0x1.0p-24f;
        wb = __float_as_uint(__fadd_rn(flo, __fmul_rn(fspan, u)));
      } else {
        wb = ilo + (uint32_t)(((r >> 32) * span) >> 32);
      }
      edges[i] = make_uint2(d, wb);
    }
  }
}

}  // namespace adds_gen

/* Builds device CSR for spec; returns arrays allocated with cudaMalloc. */
extern "C++" int adds_gen_build(const adds_gen_spec *sp, unsigned **row_out, uint2 **edges_out,
                                uint32_t *n_out, uint64_t *m_out, cudaStream_t st) {
  using namespace adds_gen;
  uint64_t ndraw = 0;
  uint32_t n = 0;
  int2 *d_offs = nullptr;
  uint32_t noff = 0;
  uint64_t npairs = 0;
  if (sp->kind == 0) {
    if (sp->scale < 1 || sp->scale > 30 || sp->edge_factor < 1) return ADDS_ERR_INVALID;
    n = 1u << sp->scale;
    ndraw = (uint64_t)sp->edge_factor << sp->scale;
  } else if (sp->kind == 2) {
    if (sp->n < 2 || sp->edge_factor < 1) return ADDS_ERR_INVALID;
    n = sp->n;
    ndraw = (uint64_t)sp->edge_factor * n;
  } else if (sp->kind == 1 || sp->kind == 3) {
    if (sp->side_x < 1 || sp->side_y < 1) return ADDS_ERR_INVALID;
    const uint64_t nn = (uint64_t)sp->side_x * sp->side_y;
    if (nn >= (1ull << 31)) return ADDS_ERR_INVALID;
    n = (uint32_t)nn;
    const uint64_t egrid = 2ull * (sp->side_x - 1) * sp->side_y + 2ull * sp->side_x * (sp->side_y - 1);
    if (sp->kind == 1 && sp->shortcut_frac > 0.0) {
      npairs = (uint64_t)(sp->shortcut_frac * (double)egrid + 0.5);
      const int R = sp->shortcut_radius > 1 ? (sp->shortcut_radius < 63 ? sp->shortcut_radius : 63) : 8;
      int2 offs_h[4 * 64 * 64];
      for (int dy = -R; dy <= R; ++dy)
        for (int dx = -R; dx <= R; ++dx) {
          const int dd = (dx < 0 ? -dx : dx) + (dy < 0 ? -dy : dy);
          if (dd >= 2 && dd <= R && noff < 4 * 64 * 64) offs_h[noff++] = make_int2(dx, dy);
        }
      if (cudaMalloc(&d_offs, noff * sizeof(int2)) != cudaSuccess) return ADDS_ERR_OOM;
      cudaMemcpyAsync(d_offs, offs_h, noff * sizeof(int2), cudaMemcpyHostToDevice, st);
      cudaStreamSynchronize(st);
    }
    ndraw = 4ull * n + 2ull * npairs;
  } else {
    return ADDS_ERR_INVALID;
  }
  uint64_t *keys = nullptr, *keys2 = nullptr;
  int rc = ADDS_OK;
  void *tmp = nullptr;
  size_t tmp_bytes = 0, tmp2 = 0;
  int *d_nsel = nullptr;
  unsigned *row = nullptr;
  uint2 *edges = nullptr;
  uint64_t m = 0;
  int nsel_h = 0;
  if (ndraw >= (1ull << 31)) { rc = ADDS_ERR_UNSUPPORTED; goto done; } /* cub int offsets */
  if (cudaMalloc(&keys, ndraw * 8) != cudaSuccess || cudaMalloc(&keys2, ndraw * 8) != cudaSuccess) {
    rc = ADDS_ERR_OOM;
    goto done;
  }
  if (sp->kind == 0)
    rmat_keys<<<4 * 148, 256, 0, st>>>(keys, ndraw, sp->scale, sp->a, sp->a + sp->b,
                                       sp->a + sp->b + sp->c, sp->seed);
  else if (sp->kind == 2)
    er_keys<<<4 * 148, 256, 0, st>>>(keys, ndraw, n, sp->seed);
  else
    grid_keys<<<4 * 148, 256, 0, st>>>(keys, sp->side_x, sp->side_y, npairs, d_offs, noff, sp->seed);
  /* sort (invalid keys are ~0 and sort last; keep all 64 bits unless R-MAT) */
  cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, keys, keys2, (int)ndraw, 0, 64, st);
  cub::DeviceSelect::Unique(nullptr, tmp2, keys2, keys, d_nsel, (int)ndraw, st);
  if (tmp2 > tmp_bytes) tmp_bytes = tmp2;
  if (cudaMalloc(&tmp, tmp_bytes) != cudaSuccess || cudaMalloc(&d_nsel, sizeof(int)) != cudaSuccess) {
    rc = ADDS_ERR_OOM;
    goto done;
  }
  cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, keys, keys2, (int)ndraw, 0, 64, st);
  cub::DeviceSelect::Unique(tmp, tmp_bytes, keys2, keys, d_nsel, (int)ndraw, st);
  cudaMemcpyAsync(&nsel_h, d_nsel, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) { rc = ADDS_ERR_CUDA; goto done; }
  m = (uint64_t)nsel_h;
  if (m > 0) {
    uint64_t last = 0;
    cudaMemcpy(&last, keys + (m - 1), 8, cudaMemcpyDeviceToHost);
    if (last == ~0ull) --m; /* drop the invalid-key run */
  }
  if (cudaMalloc(&row, ((size_t)n + 1) * 4) != cudaSuccess ||
      cudaMalloc(&edges, (m + ADDS_EDGE_PAD) * sizeof(uint2)) != cudaSuccess ||
      cudaMemsetAsync(edges + m, 0, ADDS_EDGE_PAD * sizeof(uint2), st) != cudaSuccess) {
    rc = ADDS_ERR_OOM;
    goto done;
  }
  build_csr<<<4 * 148, 256, 0, st>>>(keys, m, n, row, edges, sp->wtype == ADDS_F32, sp->w_lo,
                                     sp->w_hi, sp->seed);
  if (cudaStreamSynchronize(st) != cudaSuccess) { rc = ADDS_ERR_CUDA; goto done; }
  *row_out = row;
  *edges_out = edges;
  row = nullptr;
  edges = nullptr;
  *n_out = n;
  *m_out = m;
done:
  if (row) cudaFree(row);
  if (edges) cudaFree(edges);
  if (keys) cudaFree(keys);
  if (keys2) cudaFree(keys2);
  if (tmp) cudaFree(tmp);
  if (d_nsel) cudaFree(d_nsel);
  if (d_offs) cudaFree(d_offs);
  return rc;
}
