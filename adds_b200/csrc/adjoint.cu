/*
 * adjoint.cu — dL/dw of batched SSSP distances (float graphs).
 *
 * No reference counterpart: the reference only computes distances.  With
 * d(t) = fold of fl(d + w) along the shortest path, the (sub)gradient taken
 * along the shortest-path tree is dd(t)/dw_e = 1 if e lies on the tree path
 * to t.  So with lambda[v] = dL/dd[v] + sum over tree children c of
 * lambda[c], dL/dw_pred(v) = lambda[v].
 *
 * Determinism:
 *   - pred(v) = the tight in-edge e=(u->v), fl(d[u]+w_e) == d[v] with
 *     d[u] < d[v], of smallest CSR index (64-bit atomicMin on e<<32|u);
 *     vertices reached only through zero-gap tight edges (d[u] == d[v])
 *     get their parent in breadth-first rounds from already-treed vertices,
 *     again smallest index first, so the tree never has a cycle;
 *   - lambda[x] = seed[x] + lambda of x's children summed in x's CSR edge
 *     order, computed by the last child to finish ("last arriver
 *     continues" up the tree): no float atomics, fixed summation order;
 *   - grad[e] sums the queries of a graph in query order.
 * The CPU oracle's adjoint (oracle_adjoint in oracle/oracle.c) follows the
 * same orders, so the gradient is bit-exact against it.
 */
#include <cuda_runtime.h>
#include <string.h>

#include <vector>

#include "../../include/adds.h"
#include "adds_internal.h"

struct adds_graph;
struct adds_batch;
int adds_batch_internal(adds_batch *b, cudaStream_t *st, unsigned *nq,
                        std::vector<adds_graph *> **qgraph, std::vector<uint32_t> **srcs,
                        std::vector<adds_graph *> **ugraph, std::vector<unsigned> **qgid,
                        unsigned **dist_all, std::vector<size_t> **dist_off, void ***adj);
void adds_graph_internal(const adds_graph *g, const unsigned **row, const uint2 **edges,
                         uint32_t *n, uint64_t *m, int *device);

#define NO_PRED 0xFFFFFFFFFFFFFFFFull
#define NO_ROUND 0xFFFFFFFFu

struct AdjQ {
  const unsigned *row;
  const uint2 *edges;
  const float *dist;
  const float *seed; /* dL/d dist */
  unsigned long long *pred;
  float *lam;
  unsigned *cnt;
  unsigned *pend;
  unsigned *round;
  unsigned n;
  unsigned src;
};

struct AdjG { /* one distinct graph and the queries that use it */
  const uint2 *edges;
  float *grad;
  unsigned m;
  unsigned q_begin, q_end; /* into the query-index list */
};

namespace adj {

__global__ void k_init(const AdjQ *qs) {
  const AdjQ &q = qs[blockIdx.y];
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < q.n; v += gridDim.x * blockDim.x) {
    q.pred[v] = NO_PRED;
    q.cnt[v] = 0u;
    q.lam[v] = 0.f;
    q.round[v] = (v == q.src) ? 0u : NO_ROUND;
  }
}

/* strict tight edges: d[u] < d[v] and fl(d[u] + w) == d[v] */
__global__ void k_pred_strict(const AdjQ *qs) {
  const AdjQ &q = qs[blockIdx.y];
  for (unsigned u = blockIdx.x * blockDim.x + threadIdx.x; u < q.n; u += gridDim.x * blockDim.x) {
    const float du = q.dist[u];
    if (__float_as_uint(du) == ADDS_INF_F32_BITSV) continue;
    const unsigned e1 = q.row[u + 1];
    for (unsigned e = q.row[u]; e < e1; ++e) {
      const uint2 ed = q.edges[e];
      if (ed.x == q.src) continue;
      const float dv = q.dist[ed.x];
      if (du < dv && __fadd_rn(du, __uint_as_float(ed.y)) == dv)
        atomicMin(&q.pred[ed.x], ((unsigned long long)e << 32) | u);
    }
  }
}

/* round 0 marks; count reached vertices left without a parent */
__global__ void k_mark0(const AdjQ *qs, unsigned *orphans) {
  const AdjQ &q = qs[blockIdx.y];
  unsigned c = 0;
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < q.n; v += gridDim.x * blockDim.x) {
    if (q.pred[v] != NO_PRED) q.round[v] = 0u;
    else if (v != q.src && __float_as_uint(q.dist[v]) != ADDS_INF_F32_BITSV) ++c;
  }
  if (c) atomicAdd(orphans, c);
}

/* breadth-first round r over zero-gap tight edges */
__global__ void k_pred_zero(const AdjQ *qs, unsigned r, unsigned *changed) {
  const AdjQ &q = qs[blockIdx.y];
  for (unsigned u = blockIdx.x * blockDim.x + threadIdx.x; u < q.n; u += gridDim.x * blockDim.x) {
    if (q.round[u] >= r) continue; /* u must be in the tree before round r */
    const float du = q.dist[u];
    const unsigned e1 = q.row[u + 1];
    for (unsigned e = q.row[u]; e < e1; ++e) {
      const uint2 ed = q.edges[e];
      if (ed.x == q.src) continue;
      if (q.round[ed.x] < r) continue; /* already in the tree */
      const float dv = q.dist[ed.x];
      if (du == dv && __fadd_rn(du, __uint_as_float(ed.y)) == dv) {
        atomicMin(&q.pred[ed.x], ((unsigned long long)e << 32) | u);
        atomicMin(&q.round[ed.x], r);
        *changed = 1u;
      }
    }
  }
}

__global__ void k_children(const AdjQ *qs) {
  const AdjQ &q = qs[blockIdx.y];
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < q.n; v += gridDim.x * blockDim.x) {
    const unsigned long long p = q.pred[v];
    if (p != NO_PRED) atomicAdd(&q.cnt[(unsigned)p], 1u);
  }
}

__global__ void k_copy_pend(const AdjQ *qs) {
  const AdjQ &q = qs[blockIdx.y];
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < q.n; v += gridDim.x * blockDim.x)
    q.pend[v] = q.cnt[v];
}

/* lambda of x from its seed and its children, in x's CSR edge order */
__device__ __forceinline__ float gather_lambda(const AdjQ &q, unsigned x) {
  float acc = q.seed ? __ldcg(q.seed + x) : 0.f;
  const unsigned e1 = q.row[x + 1];
  for (unsigned e = q.row[x]; e < e1; ++e) {
    const unsigned v = q.edges[e].x;
    const unsigned long long p = __ldcg(&q.pred[v]);
    if ((unsigned)(p >> 32) == e && p != NO_PRED) acc = __fadd_rn(acc, __ldcg(q.lam + v));
  }
  return acc;
}

/* every leaf of the tree starts a walk; the last child to finish carries
 * on with its parent */
__global__ void k_walk(const AdjQ *qs) {
  const AdjQ &q = qs[blockIdx.y];
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < q.n; v += gridDim.x * blockDim.x) {
    if (q.cnt[v] != 0u) continue;
    if (__float_as_uint(q.dist[v]) == ADDS_INF_F32_BITSV) continue;
    unsigned x = v;
    for (unsigned hops = 0; hops <= q.n; ++hops) {
      const float l = gather_lambda(q, x);
      __stcg(q.lam + x, l);
      const unsigned long long p = __ldcg(&q.pred[x]);
      if (p == NO_PRED) break; /* the source (or an unreached root) */
      const unsigned parent = (unsigned)p;
      __threadfence();
      if (atomicSub(&q.pend[parent], 1u) != 1u) break; /* siblings still running */
      __threadfence();
      x = parent;
    }
  }
}

/* grad[e] (+)= sum over the graph's queries, in query order, of lambda at
 * dst(e) when e is that vertex's tree edge */
__global__ void k_grad(const AdjG *gs, const AdjQ *qs, const unsigned *qidx, int accumulate) {
  const AdjG &g = gs[blockIdx.y];
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < g.m; e += gridDim.x * blockDim.x) {
    const unsigned v = g.edges[e].x;
    float acc = 0.f;
    for (unsigned i = g.q_begin; i < g.q_end; ++i) {
      const AdjQ &q = qs[qidx[i]];
      const unsigned long long p = q.pred[v];
      if (p != NO_PRED && (unsigned)(p >> 32) == e) acc = __fadd_rn(acc, q.lam[v]);
    }
    g.grad[e] = accumulate ? __fadd_rn(g.grad[e], acc) : acc;
  }
}

}  // namespace adj

/* scratch kept with the batch between backward calls */
struct AdjScratch {
  size_t cap_vertices = 0;
  void *mem = nullptr;
  AdjQ *d_qs = nullptr;
  AdjG *d_gs = nullptr;
  unsigned *d_qidx = nullptr;
  unsigned *d_flag = nullptr;
  size_t nq = 0, ng = 0;
};

void adds_adjoint_free(void *p) {
  AdjScratch *s = (AdjScratch *)p;
  if (!s) return;
  if (s->mem) cudaFree(s->mem);
  if (s->d_qs) cudaFree(s->d_qs);
  if (s->d_gs) cudaFree(s->d_gs);
  if (s->d_qidx) cudaFree(s->d_qidx);
  if (s->d_flag) cudaFree(s->d_flag);
  delete s;
}

static int adj_fail(cudaError_t e) {
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? ADDS_ERR_OOM : ADDS_ERR_CUDA;
}
#define CKA(x)                                  \
  do {                                          \
    cudaError_t _e = (x);                       \
    if (_e != cudaSuccess) return adj_fail(_e); \
  } while (0)

/* Core: queries (row, edges, n, src, dist, seed) + graphs (edges, m, grad,
 * query list) -> gradient. */
static int run_adjoint(AdjScratch *S, std::vector<AdjQ> &qh, std::vector<AdjG> &gh,
                       const std::vector<unsigned> &qidx, int accumulate, cudaStream_t st) {
  size_t need = 0;
  unsigned max_n = 0;
  for (auto &q : qh) {
    need += ((size_t)q.n + 31) & ~(size_t)31;
    if (q.n > max_n) max_n = q.n;
  }
  if (need > S->cap_vertices) {
    if (S->mem) cudaFree(S->mem);
    S->mem = nullptr;
    CKA(cudaMalloc(&S->mem, need * 24));
    S->cap_vertices = need;
  }
  if (qh.size() != S->nq) {
    if (S->d_qs) cudaFree(S->d_qs);
    S->d_qs = nullptr;
    CKA(cudaMalloc(&S->d_qs, qh.size() * sizeof(AdjQ)));
    S->nq = qh.size();
  }
  if (gh.size() != S->ng) {
    if (S->d_gs) cudaFree(S->d_gs);
    if (S->d_qidx) cudaFree(S->d_qidx);
    S->d_gs = nullptr;
    S->d_qidx = nullptr;
    CKA(cudaMalloc(&S->d_gs, gh.size() * sizeof(AdjG)));
    CKA(cudaMalloc(&S->d_qidx, qidx.size() * sizeof(unsigned)));
    S->ng = gh.size();
  }
  if (!S->d_flag) CKA(cudaMalloc(&S->d_flag, 8));
  /* carve: pred u64 | lam f32 | cnt | pend | round */
  unsigned long long *pred = (unsigned long long *)S->mem;
  float *lam = (float *)(pred + need);
  unsigned *cnt = (unsigned *)(lam + need);
  unsigned *pend = cnt + need;
  unsigned *round = pend + need;
  size_t off = 0;
  for (auto &q : qh) {
    q.pred = pred + off;
    q.lam = lam + off;
    q.cnt = cnt + off;
    q.pend = pend + off;
    q.round = round + off;
    off += ((size_t)q.n + 31) & ~(size_t)31;
  }
  CKA(cudaMemcpyAsync(S->d_qs, qh.data(), qh.size() * sizeof(AdjQ), cudaMemcpyHostToDevice, st));
  CKA(cudaMemcpyAsync(S->d_gs, gh.data(), gh.size() * sizeof(AdjG), cudaMemcpyHostToDevice, st));
  CKA(cudaMemcpyAsync(S->d_qidx, qidx.data(), qidx.size() * sizeof(unsigned),
                      cudaMemcpyHostToDevice, st));
  unsigned bx = (max_n + 255u) / 256u;
  if (bx > 592u) bx = 592u;
  if (bx == 0u) bx = 1u;
  const dim3 grid(bx, (unsigned)qh.size());
  adj::k_init<<<grid, 256, 0, st>>>(S->d_qs);
  adj::k_pred_strict<<<grid, 256, 0, st>>>(S->d_qs);
  CKA(cudaMemsetAsync(S->d_flag, 0, 8, st));
  adj::k_mark0<<<grid, 256, 0, st>>>(S->d_qs, S->d_flag);
  unsigned orphans = 0;
  CKA(cudaMemcpyAsync(&orphans, S->d_flag, 4, cudaMemcpyDeviceToHost, st));
  CKA(cudaStreamSynchronize(st));
  for (unsigned r = 1; orphans && r <= max_n; ++r) { /* zero-gap ties only */
    unsigned changed = 0;
    CKA(cudaMemsetAsync(S->d_flag, 0, 4, st));
    adj::k_pred_zero<<<grid, 256, 0, st>>>(S->d_qs, r, S->d_flag);
    CKA(cudaMemcpyAsync(&changed, S->d_flag, 4, cudaMemcpyDeviceToHost, st));
    CKA(cudaStreamSynchronize(st));
    if (!changed) break;
  }
  adj::k_children<<<grid, 256, 0, st>>>(S->d_qs);
  adj::k_copy_pend<<<grid, 256, 0, st>>>(S->d_qs);
  adj::k_walk<<<grid, 256, 0, st>>>(S->d_qs);
  unsigned max_m = 0;
  for (auto &g : gh)
    if (g.m > max_m) max_m = g.m;
  unsigned gx = (max_m + 255u) / 256u;
  if (gx > 592u) gx = 592u;
  if (gx == 0u) gx = 1u;
  adj::k_grad<<<dim3(gx, (unsigned)gh.size()), 256, 0, st>>>(S->d_gs, S->d_qs, S->d_qidx, accumulate);
  CKA(cudaGetLastError());
  CKA(cudaStreamSynchronize(st));
  return ADDS_OK;
}

extern "C" int adds_batch_backward(adds_batch *b, const float *const *grad_dist,
                                   float *const *grad_w) {
  if (!b || !grad_dist || !grad_w) return ADDS_ERR_INVALID;
  cudaStream_t st;
  unsigned nq;
  std::vector<adds_graph *> *qgraph, *ugraph;
  std::vector<uint32_t> *srcs;
  std::vector<unsigned> *qgid;
  unsigned *dist_all;
  std::vector<size_t> *dist_off;
  void **adjp;
  adds_batch_internal(b, &st, &nq, &qgraph, &srcs, &ugraph, &qgid, &dist_all, &dist_off, &adjp);
  const unsigned *row;
  const uint2 *edges;
  uint32_t n;
  uint64_t m;
  int dev;
  adds_graph_internal((*qgraph)[0], &row, &edges, &n, &m, &dev);
  CKA(cudaSetDevice(dev));
  std::vector<AdjQ> qh(nq);
  for (unsigned i = 0; i < nq; ++i) {
    adds_graph_internal((*qgraph)[i], &row, &edges, &n, &m, &dev);
    AdjQ q;
    memset(&q, 0, sizeof q);
    q.row = row;
    q.edges = edges;
    q.dist = (const float *)(dist_all + (*dist_off)[i]);
    q.seed = grad_dist[i];
    q.n = n;
    q.src = (*srcs)[i];
    qh[i] = q;
  }
  std::vector<AdjG> gh(ugraph->size());
  std::vector<unsigned> qidx;
  for (size_t gi = 0; gi < ugraph->size(); ++gi) {
    adds_graph_internal((*ugraph)[gi], &row, &edges, &n, &m, &dev);
    if (!grad_w[gi]) return ADDS_ERR_INVALID;
    AdjG g;
    g.edges = edges;
    g.m = (unsigned)m;
    g.grad = grad_w[gi];
    g.q_begin = (unsigned)qidx.size();
    for (unsigned i = 0; i < nq; ++i)
      if ((*qgid)[i] == gi) qidx.push_back(i);
    g.q_end = (unsigned)qidx.size();
    gh[gi] = g;
  }
  if (!*adjp) *adjp = new AdjScratch();
  return run_adjoint((AdjScratch *)*adjp, qh, gh, qidx, 1, st);
}

extern "C" int adds_sssp_backward(adds_graph *g, uint32_t ns, const uint32_t *srcs, const float *dist,
                                  const float *grad_dist, float *grad_w, const adds_opts *opts) {
  if (!g || !srcs || !dist || !grad_w || ns == 0) return ADDS_ERR_INVALID;
  const unsigned *row;
  const uint2 *edges;
  uint32_t n;
  uint64_t m;
  int dev;
  adds_graph_internal(g, &row, &edges, &n, &m, &dev);
  for (uint32_t i = 0; i < ns; ++i)
    if (srcs[i] >= n) return ADDS_ERR_INVALID;
  CKA(cudaSetDevice(dev));
  cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : 0;
  std::vector<AdjQ> qh(ns);
  std::vector<unsigned> qidx(ns);
  for (uint32_t i = 0; i < ns; ++i) {
    AdjQ q;
    memset(&q, 0, sizeof q);
    q.row = row;
    q.edges = edges;
    q.dist = dist + (size_t)i * n;
    q.seed = grad_dist ? grad_dist + (size_t)i * n : nullptr;
    q.n = n;
    q.src = srcs[i];
    qh[i] = q;
    qidx[i] = i;
  }
  std::vector<AdjG> gh(1);
  gh[0].edges = edges;
  gh[0].m = (unsigned)m;
  gh[0].grad = grad_w;
  gh[0].q_begin = 0;
  gh[0].q_end = ns;
  AdjScratch S;
  const int rc = run_adjoint(&S, qh, gh, qidx, 0, st);
  if (S.mem) cudaFree(S.mem);
  if (S.d_qs) cudaFree(S.d_qs);
  if (S.d_gs) cudaFree(S.d_gs);
  if (S.d_qidx) cudaFree(S.d_qidx);
  if (S.d_flag) cudaFree(S.d_flag);
  return rc;
}
