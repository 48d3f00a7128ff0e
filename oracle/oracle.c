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
 *     (cpu_sssp_int.patch:17-46: OBIM buckets keyed dist >> shift, chunks of
 *     64 items, skip an item whose node improved since it was pushed, push
 *     when atomicMin lowered the distance; float: bucket (unsigned)(dist/div),
 *     cpu_sssp_float.patch:13,23,267-279) with std threads;
 *   - relaxation arithmetic of the GPU path (ads_int/kernel.cu:112-121):
 *     int new = d[u] + w as 32-bit (both operands < 2^31, so no wrap),
 *     accepted iff new < d[v] with INF = INT32_MAX; float new = fl(d[u]+w)
 *     in IEEE single precision, accepted iff new < d[v] with INF = FLT_MAX.
 *   - the adjoint rule of the engine's backward pass (tie-broken predecessor
 *     tree, lambda summed in CSR child order, queries in order).
 * Compiled with -ffp-contract=off so float sums are single IEEE adds.
 */
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

/* ---------------- Galois-style parallel delta-stepping ---------------- */
#define CHUNK 64

typedef struct chunk {
  struct chunk *next;
  uint32_t n;
  uint32_t node[CHUNK];
  uint32_t dist[CHUNK];
} chunk_t;

typedef struct {
  uint32_t n;
  const uint64_t *row;
  const uint32_t *dst;
  const uint32_t *w;
  int is_float;
  uint32_t shift;
  float div;
  _Atomic uint32_t *dist;
  pthread_mutex_t lock;
  chunk_t **bucket; /* bucket lists, index = priority */
  size_t nbucket;
  size_t cur;        /* lowest possibly non-empty bucket */
  _Atomic int64_t outstanding;
  _Atomic uint64_t work;
  _Atomic int failed;
} ds_t;

static size_t prio(const ds_t *s, uint32_t d) {
  if (s->is_float) {
    const float q = f_of(d) / s->div;
    return q >= 4294967295.0f ? 4294967295u : (size_t)(uint32_t)q;
  }
  return d >> s->shift;
}

static int publish(ds_t *s, chunk_t *c, size_t b) {
  pthread_mutex_lock(&s->lock);
  if (b >= s->nbucket) {
    size_t nn = s->nbucket ? s->nbucket : 1024;
    while (nn <= b) nn *= 2;
    chunk_t **nb = realloc(s->bucket, nn * sizeof *nb);
    if (!nb) {
      pthread_mutex_unlock(&s->lock);
      return -1;
    }
    memset(nb + s->nbucket, 0, (nn - s->nbucket) * sizeof *nb);
    s->bucket = nb;
    s->nbucket = nn;
  }
  c->next = s->bucket[b];
  s->bucket[b] = c;
  if (b < s->cur) s->cur = b;
  pthread_mutex_unlock(&s->lock);
  return 0;
}

static chunk_t *take(ds_t *s) {
  chunk_t *c = NULL;
  pthread_mutex_lock(&s->lock);
  while (s->cur < s->nbucket && !s->bucket[s->cur]) ++s->cur;
  if (s->cur < s->nbucket) {
    c = s->bucket[s->cur];
    s->bucket[s->cur] = c->next;
  }
  pthread_mutex_unlock(&s->lock);
  return c;
}

#define OPEN 8 /* per-thread open chunks, keyed by bucket */

typedef struct {
  ds_t *s;
} targ_t;

static void *ds_worker(void *arg) {
  ds_t *s = ((targ_t *)arg)->s;
  chunk_t *open[OPEN] = {0};
  size_t openb[OPEN] = {0};
  int idle = 0;
  while (!atomic_load(&s->failed)) {
    chunk_t *c = take(s);
    if (!c) {
      /* nothing global: publish local partial chunks, then check for the end */
      int had = 0;
      for (int i = 0; i < OPEN; ++i)
        if (open[i]) {
          if (publish(s, open[i], openb[i])) atomic_store(&s->failed, 1);
          open[i] = NULL;
          had = 1;
        }
      if (had) continue;
      if (atomic_load(&s->outstanding) == 0) break;
      if (++idle > 64) {
        struct timespec ts = {0, 1000};
        nanosleep(&ts, NULL);
      }
      continue;
    }
    idle = 0;
    int64_t pushed = 0;
    for (uint32_t i = 0; i < c->n; ++i) {
      const uint32_t u = c->node[i];
      const uint32_t du = atomic_load_explicit(&s->dist[u], memory_order_relaxed);
      if (du < c->dist[i]) continue; /* WLEmptyWork: node improved since push */
      atomic_fetch_add_explicit(&s->work, 1, memory_order_relaxed);
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
        while (nd < old &&
               !atomic_compare_exchange_weak_explicit(&s->dist[v], &old, nd, memory_order_relaxed,
                                                      memory_order_relaxed)) {
        }
        if (nd < old) { /* pushWrap */
          const size_t b = prio(s, nd);
          int slot = -1;
          for (int k = 0; k < OPEN; ++k)
            if (open[k] && openb[k] == b) slot = k;
          if (slot < 0) {
            for (int k = 0; k < OPEN; ++k)
              if (!open[k]) slot = k;
            if (slot < 0) { /* evict one open chunk (count its items first) */
              slot = 0;
              atomic_fetch_add(&s->outstanding, pushed);
              pushed = 0;
              if (publish(s, open[0], openb[0])) atomic_store(&s->failed, 1);
              open[0] = NULL;
            }
            open[slot] = calloc(1, sizeof(chunk_t));
            if (!open[slot]) {
              atomic_store(&s->failed, 1);
              break;
            }
            openb[slot] = b;
          }
          chunk_t *oc = open[slot];
          oc->node[oc->n] = v;
          oc->dist[oc->n] = nd;
          ++oc->n;
          ++pushed;
          if (oc->n == CHUNK) {
            atomic_fetch_add(&s->outstanding, pushed);
            pushed = 0;
            if (publish(s, oc, b)) atomic_store(&s->failed, 1);
            open[slot] = NULL;
          }
        }
      }
    }
    /* new items are counted before this chunk's own items are retired */
    atomic_fetch_add(&s->outstanding, pushed - (int64_t)c->n);
    free(c);
  }
  for (int i = 0; i < OPEN; ++i) free(open[i]);
  return NULL;
}

/* Multithreaded delta-stepping.  Returns 0; ms = wall time of the solve
 * (graph already in memory); work = items processed (Galois WORK_COUNT). */
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
  pthread_mutex_init(&s.lock, NULL);
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  const uint32_t inf = is_float ? b_of(FLT_MAX) : INF_I32;
  for (uint32_t v = 0; v < n; ++v) atomic_store_explicit(&s.dist[v], inf, memory_order_relaxed);
  atomic_store(&s.dist[src], 0u);
  chunk_t *c0 = calloc(1, sizeof(chunk_t));
  if (!c0) return -2;
  c0->node[0] = src;
  c0->dist[0] = 0;
  c0->n = 1;
  atomic_store(&s.outstanding, 1);
  if (publish(&s, c0, 0)) return -2;
  pthread_t *th = malloc(sizeof(pthread_t) * (size_t)nthreads);
  targ_t ta = {&s};
  for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], NULL, ds_worker, &ta);
  for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
  clock_gettime(CLOCK_MONOTONIC, &t1);
  free(th);
  for (size_t b = 0; b < s.nbucket; ++b)
    while (s.bucket[b]) {
      chunk_t *c = s.bucket[b];
      s.bucket[b] = c->next;
      free(c);
    }
  free(s.bucket);
  pthread_mutex_destroy(&s.lock);
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
