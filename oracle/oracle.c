/*
 * oracle.c — CPU restatement of the reference SSSP path.  TEST
 * INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline may call it, as the checker or the timed CPU arm; the product
 * (libadds.so) never links or calls it.
 *
 * What it restates (reference files; Galois itself is not vendored, it is
 * cloned at commit 38cd91cf by build_all.sh:45-64 and absent here):
 *   - serial Dijkstra, the reference's gold standard (run_all.sh:93-107 with
 *     -algo=dijkstra -t 1; cpu_sssp_int.patch:50-64 MinHeap loop);
 *   - Galois delta-stepping, the reference's CPU comparison
 *     (cpu_sssp_int.patch:17-46: buckets keyed dist >> shift, chunks of 64
 *     items, skip an item whose node improved since it was pushed, push when
 *     atomicMin lowered the distance; float: bucket (unsigned)(dist/div),
 *     cpu_sssp_float.patch:13,23,267-279), bulk-synchronous over pthreads;
 *   - relaxation arithmetic of the GPU path (ads_int/kernel.cu:112-121):
 *     int new = d[u] + w as 32-bit (both operands < 2^31, so no wrap),
 *     accepted iff new < d[v] with INF = INT32_MAX; float new = fl(d[u]+w)
 *     in IEEE single precision, accepted iff new < d[v] with INF = FLT_MAX.
 *   - the adjoint rule of the engine's backward pass (tie-broken predecessor
 *     tree, lambda summed in CSR child order, queries in order).
 * Compiled with -ffp-contract=off so float sums are single IEEE adds.
 */
#define _GNU_SOURCE
#include <float.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define INF_I32 0x7FFFFFFFu

/* ---------------- binary heap of (key, vertex) ---------------- */
typedef struct {
  uint64_t *key;
  uint32_t *v;
  size_t n, cap;
} heap_t;

static int heap_push(heap_t *h, uint64_t k, uint32_t v) {
  if (h->n == h->cap) {
    size_t nc = h->cap ? h->cap * 2 : 1024;
    uint64_t *nk = realloc(h->key, nc * sizeof *nk);
    if (!nk) return -1;
    h->key = nk;
    uint32_t *nv = realloc(h->v, nc * sizeof *nv);
    if (!nv) return -1;
    h->v = nv;
    h->cap = nc;
  }
  size_t i = h->n++;
  while (i) {
    size_t p = (i - 1) / 2;
    if (h->key[p] <= k) break;
    h->key[i] = h->key[p];
    h->v[i] = h->v[p];
    i = p;
  }
  h->key[i] = k;
  h->v[i] = v;
  return 0;
}

static void heap_pop(heap_t *h, uint64_t *k, uint32_t *v) {
  *k = h->key[0];
  *v = h->v[0];
  uint64_t lk = h->key[--h->n];
  uint32_t lv = h->v[h->n];
  size_t i = 0;
  for (;;) {
    size_t c = 2 * i + 1;
    if (c >= h->n) break;
    if (c + 1 < h->n && h->key[c + 1] < h->key[c]) ++c;
    if (h->key[c] >= lk) break;
    h->key[i] = h->key[c];
    h->v[i] = h->v[c];
    i = c;
  }
  h->key[i] = lk;
  h->v[i] = lv;
}

static void heap_free(heap_t *h) {
  free(h->key);
  free(h->v);
}

/* dist words are 32-bit; for non-negative floats the bit pattern orders
 * like the value, so one heap serves both types (key = bits). */
static float f_of(uint32_t b) {
  float f;
  memcpy(&f, &b, 4);
  return f;
}
static uint32_t b_of(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  return b;
}

/* Serial Dijkstra.  is_float selects the fold; dist receives 32-bit words.
 * work = vertices settled (the Galois dj work count). */
int oracle_dijkstra(uint32_t n, const uint64_t *row, const uint32_t *dst, const uint32_t *w,
                    uint32_t src, int is_float, uint32_t *dist, uint64_t *work) {
  if (src >= n) return -1;
  const uint32_t inf = is_float ? b_of(FLT_MAX) : INF_I32;
  for (uint32_t v = 0; v < n; ++v) dist[v] = inf;
  dist[src] = 0;
  heap_t h = {0};
  if (heap_push(&h, 0, src)) return -2;
  uint64_t wk = 0;
  while (h.n) {
    uint64_t k;
    uint32_t u;
    heap_pop(&h, &k, &u);
    if ((uint32_t)k != dist[u]) continue; /* stale */
    ++wk;
    const uint32_t du = dist[u];
    for (uint64_t e = row[u]; e < row[u + 1]; ++e) {
      const uint32_t v = dst[e];
      uint32_t nd;
      if (is_float) {
        volatile float s = f_of(du) + f_of(w[e]);
        nd = b_of(s);
      } else {
        nd = du + w[e];
      }
      if (nd < dist[v]) {
        dist[v] = nd;
        if (heap_push(&h, nd, v)) {
          heap_free(&h);
          return -2;
        }
      }
    }
  }
  heap_free(&h);
  if (work) *work = wk;
  return 0;
}

/* float64 Dijkstra on double weights (finite-difference reference). */
int oracle_dijkstra_f64(uint32_t n, const uint64_t *row, const uint32_t *dst, const double *w,
                        uint32_t src, double *dist) {
  if (src >= n) return -1;
  for (uint32_t v = 0; v < n; ++v) dist[v] = 1e300;
  dist[src] = 0;
  heap_t h = {0};
  uint64_t key;
  memcpy(&key, &dist[src], 8);
  if (heap_push(&h, key, src)) return -2;
  while (h.n) {
    uint64_t k;
    uint32_t u;
    heap_pop(&h, &k, &u);
    double du;
    memcpy(&du, &k, 8);
    if (du != dist[u]) continue;
    for (uint64_t e = row[u]; e < row[u + 1]; ++e) {
      const uint32_t v = dst[e];
      const double nd = du + w[e];
      if (nd < dist[v]) {
        dist[v] = nd;
        memcpy(&key, &nd, 8); /* non-negative doubles order like their bits */
        if (heap_push(&h, key, v)) {
          heap_free(&h);
          return -2;
        }
      }
    }
  }
  heap_free(&h);
  return 0;
}

/* ---------------- parallel delta-stepping (CPU baseline) ----------------
 * Same bucket function and item rule as the Galois OBIM loop the reference
 * compares against (cpu_sssp_int.patch:17-46: bucket = dist >> shift, or
 * (unsigned)(dist/div) for float; an item whose node improved since it was
 * pushed is skipped; push when the atomic min lowered the distance), run
 * bulk-synchronously: all threads drain the lowest non-empty bucket from a
 * shared frontier (claimed in chunks of 64), pushing into thread-local
 * buckets, until that bucket stays empty; then the next bucket. */
#define CHUNK 64

typedef struct {
  uint32_t *v, *d;
  size_t n, cap;
} ivec_t;

typedef struct {
  ivec_t *b;
  size_t nb;
} tbk_t;

typedef struct {
  uint32_t n;
  const uint64_t *row;
  const uint32_t *dst;
  const uint32_t *w;
  int is_float;
  uint32_t shift;
  float div;
  _Atomic uint32_t *dist;
  int nthreads;
  tbk_t *tb;
  pthread_barrier_t bar;
  uint32_t *fv, *fd;
  size_t fcap, ftotal;
  size_t *cnt, *off;
  _Atomic size_t next;
  _Atomic size_t minb;
  size_t cur;
  int done;
  _Atomic int failed;
  _Atomic uint64_t work;
} ds_t;

static size_t prio(const ds_t *s, uint32_t d) {
  if (s->is_float) {
    const float q = f_of(d) / s->div;
    return q >= 4294967295.0f ? 4294967295u : (size_t)(uint32_t)q;
  }
  return d >> s->shift;
}

static int ivec_push(ivec_t *x, uint32_t v, uint32_t d) {
  if (x->n == x->cap) {
    size_t nc = x->cap ? x->cap * 2 : 256;
    uint32_t *nv = realloc(x->v, nc * 4), *nd;
    if (!nv) return -1;
    x->v = nv;
    nd = realloc(x->d, nc * 4);
    if (!nd) return -1;
    x->d = nd;
    x->cap = nc;
  }
  x->v[x->n] = v;
  x->d[x->n] = d;
  ++x->n;
  return 0;
}

static int tb_push(tbk_t *t, size_t b, uint32_t v, uint32_t d) {
  if (b >= t->nb) {
    size_t nn = t->nb ? t->nb : 64;
    while (nn <= b) nn *= 2;
    ivec_t *nb = realloc(t->b, nn * sizeof *nb);
    if (!nb) return -1;
    memset(nb + t->nb, 0, (nn - t->nb) * sizeof *nb);
    t->b = nb;
    t->nb = nn;
  }
  return ivec_push(&t->b[b], v, d);
}

typedef struct {
  ds_t *s;
  int tid;
} targ_t;

static void *ds_worker(void *arg) {
  ds_t *s = ((targ_t *)arg)->s;
  const int tid = ((targ_t *)arg)->tid;
  tbk_t *my = &s->tb[tid];
  for (;;) {
    /* lowest non-empty bucket over all threads */
    size_t lo = SIZE_MAX;
    for (size_t b = s->cur; b < my->nb; ++b)
      if (my->b[b].n) {
        lo = b;
        break;
      }
    size_t cur = atomic_load(&s->minb);
    while (lo < cur && !atomic_compare_exchange_weak(&s->minb, &cur, lo)) {
    }
    pthread_barrier_wait(&s->bar);
    if (tid == 0) {
      s->cur = atomic_load(&s->minb);
      s->done = s->cur == SIZE_MAX || atomic_load(&s->failed);
      atomic_store(&s->minb, SIZE_MAX);
    }
    pthread_barrier_wait(&s->bar);
    if (s->done) break;
    const size_t b = s->cur;
    for (;;) { /* phases of bucket b until it stays empty */
      s->cnt[tid] = (b < my->nb) ? my->b[b].n : 0;
      pthread_barrier_wait(&s->bar);
      if (tid == 0) {
        size_t t = 0;
        for (int i = 0; i < s->nthreads; ++i) {
          s->off[i] = t;
          t += s->cnt[i];
        }
        s->ftotal = t;
        if (t > s->fcap) {
          size_t nc = t + t / 2 + 1024;
          uint32_t *nv = realloc(s->fv, nc * 4), *nd = NULL;
          if (nv) {
            s->fv = nv;
            nd = realloc(s->fd, nc * 4);
          }
          if (!nv || !nd) {
            atomic_store(&s->failed, 1);
            s->ftotal = 0;
          } else {
            s->fd = nd;
            s->fcap = nc;
          }
        }
        atomic_store(&s->next, 0);
      }
      pthread_barrier_wait(&s->bar);
      const size_t total = s->ftotal;
      if (total == 0) break;
      if (s->cnt[tid]) {
        memcpy(s->fv + s->off[tid], my->b[b].v, s->cnt[tid] * 4);
        memcpy(s->fd + s->off[tid], my->b[b].d, s->cnt[tid] * 4);
        my->b[b].n = 0;
      }
      pthread_barrier_wait(&s->bar);
      uint64_t wk = 0;
      for (;;) {
        const size_t i0 = atomic_fetch_add(&s->next, CHUNK);
        if (i0 >= total) break;
        const size_t i1 = i0 + CHUNK < total ? i0 + CHUNK : total;
        for (size_t i = i0; i < i1; ++i) {
          const uint32_t u = s->fv[i];
          const uint32_t du = atomic_load_explicit(&s->dist[u], memory_order_relaxed);
          if (du < s->fd[i]) continue; /* improved since it was pushed */
          ++wk;
          for (uint64_t e = s->row[u]; e < s->row[u + 1]; ++e) {
            const uint32_t v = s->dst[e];
            uint32_t nd;
            if (s->is_float) {
              volatile float sum = f_of(du) + f_of(s->w[e]);
              nd = b_of(sum);
            } else {
              nd = du + s->w[e];
            }
            uint32_t old = atomic_load_explicit(&s->dist[v], memory_order_relaxed);
            while (nd < old && !atomic_compare_exchange_weak_explicit(
                                   &s->dist[v], &old, nd, memory_order_relaxed,
                                   memory_order_relaxed)) {
            }
            if (nd < old) {
              size_t nb = prio(s, nd);
              if (nb < b) nb = b;
              if (tb_push(my, nb, v, nd)) atomic_store(&s->failed, 1);
            }
          }
        }
      }
      atomic_fetch_add(&s->work, wk);
      pthread_barrier_wait(&s->bar);
    }
  }
  return NULL;
}

/* Parallel delta-stepping.  Returns 0; ms = wall time of the solve (graph
 * already in memory); work = items processed (Galois WORK_COUNT). */
int oracle_delta_step(uint32_t n, const uint64_t *row, const uint32_t *dst, const uint32_t *w,
                      uint32_t src, int is_float, uint32_t shift, float div, int nthreads,
                      uint32_t *dist_out, uint64_t *work, double *ms) {
  if (src >= n || nthreads < 1) return -1;
  if (is_float && !(div > 0.f)) return -1;
  ds_t s;
  memset(&s, 0, sizeof s);
  s.n = n;
  s.row = row;
  s.dst = dst;
  s.w = w;
  s.is_float = is_float;
  s.shift = shift;
  s.div = div;
  s.dist = (_Atomic uint32_t *)dist_out;
  s.nthreads = nthreads;
  s.tb = calloc((size_t)nthreads, sizeof(tbk_t));
  s.cnt = calloc((size_t)nthreads, sizeof(size_t));
  s.off = calloc((size_t)nthreads, sizeof(size_t));
  pthread_t *th = malloc(sizeof(pthread_t) * (size_t)nthreads);
  targ_t *ta = malloc(sizeof(targ_t) * (size_t)nthreads);
  if (!s.tb || !s.cnt || !s.off || !th || !ta) return -2;
  pthread_barrier_init(&s.bar, NULL, (unsigned)nthreads);
  atomic_store(&s.minb, SIZE_MAX);
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  const uint32_t inf = is_float ? b_of(FLT_MAX) : INF_I32;
  for (uint32_t v = 0; v < n; ++v) atomic_store_explicit(&s.dist[v], inf, memory_order_relaxed);
  atomic_store(&s.dist[src], 0u);
  if (tb_push(&s.tb[0], prio(&s, 0), src, 0)) return -2;
  for (int i = 0; i < nthreads; ++i) {
    ta[i].s = &s;
    ta[i].tid = i;
    pthread_create(&th[i], NULL, ds_worker, &ta[i]);
  }
  for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
  clock_gettime(CLOCK_MONOTONIC, &t1);
  for (int i = 0; i < nthreads; ++i) {
    for (size_t b = 0; b < s.tb[i].nb; ++b) {
      free(s.tb[i].b[b].v);
      free(s.tb[i].b[b].d);
    }
    free(s.tb[i].b);
  }
  free(s.tb);
  free(s.cnt);
  free(s.off);
  free(s.fv);
  free(s.fd);
  free(th);
  free(ta);
  pthread_barrier_destroy(&s.bar);
  if (work) *work = atomic_load(&s.work);
  if (ms) *ms = (t1.tv_sec - t0.tv_sec) * 1e3 + (t1.tv_nsec - t0.tv_nsec) * 1e-6;
  return atomic_load(&s.failed) ? -2 : 0;
}

/* ---------------- adjoint reference ---------------- */
#define NO_PRED UINT64_MAX
#define NO_ROUND UINT32_MAX

typedef struct {
  float d;
  uint32_t r;
  uint32_t v;
} ord_t;

static int ord_cmp(const void *a, const void *b) { /* children before parents */
  const ord_t *x = a, *y = b;
  if (x->d != y->d) return x->d > y->d ? -1 : 1;
  if (x->r != y->r) return x->r > y->r ? -1 : 1;
  return x->v < y->v ? -1 : (x->v > y->v);
}

/* Predecessor tree of one solve: strict tight in-edge of smallest index,
 * zero-gap ties resolved in breadth-first rounds.  pred[v] = e<<32 | u. */
static void build_pred(uint32_t n, const uint64_t *row, const uint32_t *dst, const float *w,
                       uint32_t src, const float *d, uint64_t *pred, uint32_t *round) {
  for (uint32_t v = 0; v < n; ++v) {
    pred[v] = NO_PRED;
    round[v] = v == src ? 0 : NO_ROUND;
  }
  for (uint32_t u = 0; u < n; ++u) {
    if (d[u] == FLT_MAX) continue;
    for (uint64_t e = row[u]; e < row[u + 1]; ++e) {
      const uint32_t v = dst[e];
      if (v == src) continue;
      volatile float s = d[u] + w[e];
      if (d[u] < d[v] && s == d[v]) {
        const uint64_t k = (e << 32) | u;
        if (k < pred[v]) pred[v] = k;
      }
    }
  }
  size_t orphans = 0;
  for (uint32_t v = 0; v < n; ++v) {
    if (pred[v] != NO_PRED) round[v] = 0;
    else if (v != src && d[v] != FLT_MAX) ++orphans;
  }
  for (uint32_t r = 1; orphans && r <= n; ++r) {
    int changed = 0;
    for (uint32_t u = 0; u < n; ++u) {
      if (round[u] >= r) continue;
      for (uint64_t e = row[u]; e < row[u + 1]; ++e) {
        const uint32_t v = dst[e];
        if (v == src || round[v] < r) continue;
        volatile float s = d[u] + w[e];
        if (d[u] == d[v] && s == d[v]) {
          const uint64_t k = (e << 32) | u;
          if (k < pred[v]) pred[v] = k;
          if (r < round[v]) round[v] = r;
          changed = 1;
        }
      }
    }
    if (!changed) break;
  }
}

/* grad[e] = sum over solves (in order) of lambda_s[dst(e)] where e is the
 * tree edge of dst(e); lambda_s[x] = seed_s[x] + sum of children's lambda in
 * x's CSR edge order.  dist/seed: [ns][n]; grad: [m], overwritten.
 * pred_out (optional): [ns][n]. */
int oracle_adjoint(uint32_t n, uint64_t m, const uint64_t *row, const uint32_t *dst, const float *w,
                   uint32_t ns, const uint32_t *srcs, const float *dist, const float *seed,
                   float *grad, uint64_t *pred_out) {
  uint64_t *pred = malloc((size_t)n * 8 * ns);
  uint32_t *round = malloc((size_t)n * 4);
  float *lam = malloc((size_t)n * 4 * ns);
  ord_t *ord = malloc((size_t)n * sizeof(ord_t));
  if (!pred || !round || !lam || !ord) {
    free(pred);
    free(round);
    free(lam);
    free(ord);
    return -2;
  }
  for (uint32_t s = 0; s < ns; ++s) {
    const float *d = dist + (size_t)s * n;
    const float *sd = seed ? seed + (size_t)s * n : NULL;
    uint64_t *p = pred + (size_t)s * n;
    float *l = lam + (size_t)s * n;
    build_pred(n, row, dst, w, srcs[s], d, p, round);
    size_t k = 0;
    for (uint32_t v = 0; v < n; ++v) {
      l[v] = 0.f;
      if (d[v] != FLT_MAX) {
        ord[k].d = d[v];
        ord[k].r = round[v];
        ord[k].v = v;
        ++k;
      }
    }
    qsort(ord, k, sizeof(ord_t), ord_cmp);
    for (size_t i = 0; i < k; ++i) {
      const uint32_t x = ord[i].v;
      volatile float acc = sd ? sd[x] : 0.f;
      for (uint64_t e = row[x]; e < row[x + 1]; ++e) {
        const uint32_t c = dst[e];
        if (p[c] != NO_PRED && (p[c] >> 32) == e) acc = acc + l[c];
      }
      l[x] = acc;
    }
  }
  for (uint64_t e = 0; e < m; ++e) {
    const uint32_t v = dst[e];
    volatile float acc = 0.f;
    for (uint32_t s = 0; s < ns; ++s) {
      const uint64_t pv = pred[(size_t)s * n + v];
      if (pv != NO_PRED && (pv >> 32) == e) acc = acc + lam[(size_t)s * n + v];
    }
    grad[e] = acc;
  }
  if (pred_out) memcpy(pred_out, pred, (size_t)n * 8 * ns);
  free(pred);
  free(round);
  free(lam);
  free(ord);
  return 0;
}
