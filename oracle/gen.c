/*
 * gen.c — host twins of the seeded graph generators, for the CPU arms of the
 * benchmark.  TEST / MEASUREMENT INFRASTRUCTURE ONLY: bench.py's reference
 * arm builds its input graph here so that it loads nothing but the oracle
 * library; the product never links or calls this file.
 *
 * Every random draw is H(seed, stream, index) through the same
 * splitmix64-style mixer as the GPU generator and adds_b200/graphs.py, so the
 * three produce the identical CSR for the same spec: one 64-bit key
 * (src << 32 | dst) per candidate edge, self-loops and out-of-range draws
 * dropped, keys sorted and made unique, weights hashed from the key.
 * Keys are sorted with a multithreaded LSD radix sort (8-bit digits; digits
 * that are equal in every key are skipped).
 * Compiled with -ffp-contract=off: the float weight lo + span * u is two
 * IEEE single-precision roundings, as on the GPU.
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static uint64_t H(uint64_t seed, uint64_t stream, uint64_t i) {
  const uint64_t s = mix64(seed + 0x9E3779B97F4A7C15ull * (stream + 1ull));
  return mix64(s ^ (i * 0xD1B54A32D192ED03ull + 0x8CB92BA72F3D8DD7ull));
}
static uint32_t mulshift(uint64_t r, uint32_t n) {
  return (uint32_t)(((r >> 32) * (uint64_t)n) >> 32);
}
enum { S_WEIGHT = 1000, S_SC_U = 2000, S_SC_OFF = 2001 };

#define MAXT 256

/* ---------------- fork-join over [0, n) ---------------- */
typedef struct {
  void (*fn)(void *ctx, int t, uint64_t lo, uint64_t hi);
  void *ctx;
  int t, nt;
  uint64_t n;
} job_t;

static void *job_run(void *p) {
  job_t *j = (job_t *)p;
  const uint64_t lo = j->n * (uint64_t)j->t / (uint64_t)j->nt;
  const uint64_t hi = j->n * (uint64_t)(j->t + 1) / (uint64_t)j->nt;
  j->fn(j->ctx, j->t, lo, hi);
  return NULL;
}

static void par_for(int nt, uint64_t n, void (*fn)(void *, int, uint64_t, uint64_t), void *ctx) {
  pthread_t th[MAXT];
  job_t jb[MAXT];
  int started[MAXT];
  for (int t = 0; t < nt; ++t) {
    jb[t] = (job_t){fn, ctx, t, nt, n};
    started[t] = t > 0 && pthread_create(&th[t], NULL, job_run, &jb[t]) == 0;
  }
  job_run(&jb[0]);
  for (int t = 1; t < nt; ++t) {
    if (started[t])
      pthread_join(th[t], NULL);
    else
      job_run(&jb[t]); /* no thread: run it here */
  }
}

/* ---------------- key generation ---------------- */
typedef struct {
  uint64_t *keys;
  uint64_t *cnt; /* valid keys per thread */
  int scale;
  double a, ab, abc;
  uint64_t seed;
  /* grid */
  uint32_t sx, sy;
  uint64_t n4, npairs;
  const int32_t *offs;
  uint32_t noff;
} kgen_t;

/* each thread writes its valid keys to the front of its own range */
static void rmat_part(void *p, int t, uint64_t lo, uint64_t hi) {
  kgen_t *g = (kgen_t *)p;
  uint64_t w = lo;
  for (uint64_t i = lo; i < hi; ++i) {
    uint32_t s = 0, d = 0;
    for (int l = 0; l < g->scale; ++l) {
      const uint64_t r = H(g->seed, 1ull + (uint64_t)l, i);
      const double u = (double)(r >> 11) * 0x1.0p-53;
      const uint32_t q = u < g->a ? 0u : (u < g->ab ? 1u : (u < g->abc ? 2u : 3u));
      const int bit = g->scale - 1 - l;
      s |= (q >> 1) << bit;
      d |= (q & 1u) << bit;
    }
    if (s != d) g->keys[w++] = ((uint64_t)s << 32) | d;
  }
  g->cnt[t] = w - lo;
}

static void grid_part(void *p, int t, uint64_t lo, uint64_t hi) {
  kgen_t *g = (kgen_t *)p;
  const uint32_t sx = g->sx, sy = g->sy;
  const uint32_t n = sx * sy;
  uint64_t w = lo;
  for (uint64_t i = lo; i < hi; ++i) {
    if (i < g->n4) {
      const uint32_t v = (uint32_t)(i >> 2), dir = (uint32_t)(i & 3u);
      int nx = (int)(v % sx), ny = (int)(v / sx);
      if (dir == 0) nx += 1; else if (dir == 1) nx -= 1; else if (dir == 2) ny += 1; else ny -= 1;
      if (nx >= 0 && ny >= 0 && nx < (int)sx && ny < (int)sy)
        g->keys[w++] = ((uint64_t)v << 32) | ((uint32_t)ny * sx + (uint32_t)nx);
    } else {
      const uint64_t j = (i - g->n4) >> 1;
      const uint32_t u = mulshift(H(g->seed, S_SC_U, j), n);
      const uint32_t k = mulshift(H(g->seed, S_SC_OFF, j), g->noff);
      const int x = (int)(u % sx) + g->offs[2 * k], y = (int)(u / sx) + g->offs[2 * k + 1];
      if (x >= 0 && y >= 0 && x < (int)sx && y < (int)sy) {
        const uint32_t v = (uint32_t)y * sx + (uint32_t)x;
        g->keys[w++] = ((i - g->n4) & 1ull) ? (((uint64_t)v << 32) | u) : (((uint64_t)u << 32) | v);
      }
    }
  }
  g->cnt[t] = w - lo;
}

/* ---------------- parallel LSD radix sort ---------------- */
typedef struct {
  uint64_t *src, *dst;
  uint64_t (*hist)[256]; /* [thread][digit] -> counts, then offsets */
  int shift;
} rs_t;

static void rs_count(void *p, int t, uint64_t lo, uint64_t hi) {
  rs_t *r = (rs_t *)p;
  uint64_t *h = r->hist[t];
  memset(h, 0, 256 * sizeof *h);
  for (uint64_t i = lo; i < hi; ++i) ++h[(r->src[i] >> r->shift) & 0xFFu];
}
static void rs_scatter(void *p, int t, uint64_t lo, uint64_t hi) {
  rs_t *r = (rs_t *)p;
  uint64_t *h = r->hist[t];
  for (uint64_t i = lo; i < hi; ++i) {
    const uint64_t k = r->src[i];
    r->dst[h[(k >> r->shift) & 0xFFu]++] = k;
  }
}

/* sorts keys[0, n) in place (tmp: n scratch words) */
static void radix_sort(uint64_t *keys, uint64_t *tmp, uint64_t n, int nt) {
  uint64_t or_all = 0, and_all = ~0ull;
  for (uint64_t i = 0; i < n; ++i) {
    or_all |= keys[i];
    and_all &= keys[i];
  }
  uint64_t (*hist)[256] = malloc((size_t)nt * sizeof *hist);
  if (!hist) abort();
  uint64_t *src = keys, *dst = tmp;
  for (int shift = 0; shift < 64; shift += 8) {
    if ((((or_all ^ and_all) >> shift) & 0xFFu) == 0) continue; /* digit constant */
    rs_t r = {src, dst, hist, shift};
    par_for(nt, n, rs_count, &r);
    uint64_t off = 0;
    for (int d = 0; d < 256; ++d)
      for (int t = 0; t < nt; ++t) {
        const uint64_t c = hist[t][d];
        hist[t][d] = off;
        off += c;
      }
    par_for(nt, n, rs_scatter, &r);
    uint64_t *x = src;
    src = dst;
    dst = x;
  }
  if (src != keys) memcpy(keys, src, n * sizeof *keys);
  free(hist);
}

/* ---------------- CSR from sorted unique keys ---------------- */
typedef struct {
  const uint64_t *keys;
  uint64_t m;
  uint32_t n;
  uint64_t *row;
  uint32_t *dst, *w;
  int is_float;
  double w_lo, w_hi;
  uint64_t seed;
} csr_t;

static void csr_part(void *p, int t, uint64_t lo, uint64_t hi) {
  (void)t;
  csr_t *c = (csr_t *)p;
  const uint32_t ilo = (uint32_t)c->w_lo;
  const uint64_t span = (uint64_t)((int64_t)c->w_hi - (int64_t)c->w_lo + 1);
  const float flo = (float)c->w_lo, fspan = (float)(c->w_hi - c->w_lo);
  for (uint64_t i = lo; i < hi; ++i) {
    /* row[v] = i for every v in (src(i-1), src(i)] (src(-1) = -1, src(m) = n) */
    const int64_t s = (i < c->m) ? (int64_t)(c->keys[i] >> 32) : (int64_t)c->n;
    const int64_t sp = (i == 0) ? -1 : (int64_t)(c->keys[i - 1] >> 32);
    for (int64_t v = sp + 1; v <= s; ++v) c->row[v] = i;
    if (i < c->m) {
      const uint64_t r = H(c->seed, S_WEIGHT, c->keys[i]);
      uint32_t wb;
      if (c->is_float) {
        const float u = (float)(uint32_t)(r >> 40) * 0x1.0p-24f;
        const float x = flo + fspan * u;
        memcpy(&wb, &x, 4);
      } else {
        wb = ilo + (uint32_t)(((r >> 32) * span) >> 32);
      }
      c->dst[i] = (uint32_t)c->keys[i];
      c->w[i] = wb;
    }
  }
}

/* compacts each thread's valid keys, sorts, drops duplicates; returns m */
static uint64_t finish_keys(uint64_t *keys, uint64_t *tmp, uint64_t ndraw, const uint64_t *cnt,
                            int nt) {
  uint64_t m = 0;
  for (int t = 0; t < nt; ++t) {
    const uint64_t lo = ndraw * (uint64_t)t / (uint64_t)nt;
    memmove(keys + m, keys + lo, cnt[t] * sizeof *keys);
    m += cnt[t];
  }
  radix_sort(keys, tmp, m, nt);
  uint64_t u = 0;
  for (uint64_t i = 0; i < m; ++i)
    if (i == 0 || keys[i] != keys[i - 1]) keys[u++] = keys[i];
  return u;
}

static int build(kgen_t *g, void (*part)(void *, int, uint64_t, uint64_t), uint64_t ndraw,
                 uint32_t n, int wtype, double w_lo, double w_hi, uint64_t seed, int threads,
                 uint64_t *row, uint32_t *dst, uint32_t *w, uint64_t cap, uint64_t *m_out) {
  const int nt = threads < 1 ? 1 : (threads > MAXT ? MAXT : threads);
  uint64_t *keys = malloc(ndraw * sizeof *keys), *tmp = malloc(ndraw * sizeof *tmp);
  uint64_t cnt[MAXT];
  if (!keys || !tmp) {
    free(keys);
    free(tmp);
    return -4;
  }
  g->keys = keys;
  g->cnt = cnt;
  par_for(nt, ndraw, part, g);
  const uint64_t m = finish_keys(keys, tmp, ndraw, cnt, nt);
  free(tmp);
  if (m > cap) {
    free(keys);
    return -1;
  }
  csr_t c = {keys, m, n, row, dst, w, wtype == 1, w_lo, w_hi, seed};
  par_for(nt, m + 1, csr_part, &c);
  free(keys);
  *m_out = m;
  return 0;
}

/* R-MAT: edge_factor * 2^scale draws (the GPU generator's rmat_keys).
 * row: 2^scale + 1 entries; dst, w: cap >= edge_factor * 2^scale entries. */
int oracle_gen_rmat(int scale, int edge_factor, double a, double b, double c, int wtype,
                    double w_lo, double w_hi, uint64_t seed, int threads, uint64_t *row,
                    uint32_t *dst, uint32_t *w, uint64_t cap, uint64_t *m_out) {
  if (scale < 1 || scale > 30 || edge_factor < 1) return -1;
  kgen_t g;
  memset(&g, 0, sizeof g);
  g.scale = scale;
  g.a = a;
  g.ab = a + b;
  g.abc = a + b + c;
  g.seed = seed;
  return build(&g, rmat_part, (uint64_t)edge_factor << scale, 1u << scale, wtype, w_lo, w_hi,
               seed, threads, row, dst, w, cap, m_out);
}

/* 4-neighbour grid plus shortcut pairs to a vertex at Manhattan distance
 * 2..radius (the GPU generator's grid_keys).  row: sx*sy + 1 entries;
 * dst, w: cap >= 4*sx*sy + 2*npairs entries, npairs = round(frac * grid edges). */
int oracle_gen_grid(uint32_t sx, uint32_t sy, double frac, int radius, int wtype, double w_lo,
                    double w_hi, uint64_t seed, int threads, uint64_t *row, uint32_t *dst,
                    uint32_t *w, uint64_t cap, uint64_t *m_out) {
  if (sx < 1 || sy < 1 || (uint64_t)sx * sy >= (1ull << 31)) return -1;
  const uint64_t n = (uint64_t)sx * sy;
  const uint64_t egrid = 2ull * (sx - 1) * sy + 2ull * sx * (sy - 1);
  kgen_t g;
  memset(&g, 0, sizeof g);
  static int32_t offs[2 * 4 * 64 * 64];
  uint32_t noff = 0;
  if (frac > 0.0) {
    g.npairs = (uint64_t)(frac * (double)egrid + 0.5);
    const int R = radius > 1 ? (radius < 63 ? radius : 63) : 8;
    for (int dy = -R; dy <= R; ++dy)
      for (int dx = -R; dx <= R; ++dx) {
        const int dd = (dx < 0 ? -dx : dx) + (dy < 0 ? -dy : dy);
        if (dd >= 2 && dd <= R && noff < 4 * 64 * 64) {
          offs[2 * noff] = dx;
          offs[2 * noff + 1] = dy;
          ++noff;
        }
      }
  }
  g.sx = sx;
  g.sy = sy;
  g.n4 = 4ull * n;
  g.offs = offs;
  g.noff = noff;
  g.seed = seed;
  return build(&g, grid_part, 4ull * n + 2ull * g.npairs, (uint32_t)n, wtype, w_lo, w_hi, seed,
               threads, row, dst, w, cap, m_out);
}
