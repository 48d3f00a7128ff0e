/*
 * engine.cu — persistent asynchronous delta-stepping SSSP for sm_100a.
 *
 * Behavioural source: ADDS (ads_int/kernel.cu:30-128 workers,
 * ads_int/wl.h:192-1972 worklist + manager).  What is kept:
 *   - 32 circular distance buckets per solve, bucket = clip(dist >> shift
 *     relative to the lowest live bucket, 0, 31) (wl.h:1958-1972);
 *   - several consecutive buckets may be processed at once (the reference's
 *     concur_bag, wl.h:1398-1510), the lowest is retired only once it is
 *     empty and none of its entries is still being processed (wl.h:714-724);
 *   - relax = new = d[u] + w, accept if d[v] > new, atomic minimum, push
 *     (kernel.cu:112-121; here the minimum is a fire-and-forget reduction
 *     and the push follows the comparison with the gathered d[v], as the
 *     reference's int kernel pushes whatever its atomicMin returned,
 *     kernel.cu:78-82); float uses the IEEE bit order of non-negative
 *     floats for the 32-bit minimum instead of the reference's 64-bit CAS
 *     (ads_float/csr_graph.h:58-70); rows longer than a threshold are split
 *     across workers (wl.h:1638-1696, here across the whole grid).
 * What is new: no manager block and no CDP.  One cooperative launch of
 * CTAs that pop whole batches from the bucket queues with a CAS, expand the
 * batch edge-balanced over the CTA, stage pushes in shared memory and flush
 * them with one reservation per bucket.  Queue entries are (vertex, pushed
 * distance) pairs; an entry whose vertex has since improved is dropped.
 * Termination is a per-query count of live entries.  Every wait is bounded
 * by a device deadline and reports ADDS_DEV_TIMEOUT instead of hanging.
 */
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "adds_internal.h"

namespace cg = cooperative_groups;

namespace adds {

/* ------------------------------------------------------------------------ */
/* memory-model helpers (PTX ISA: ld/st .relaxed.gpu, globaltimer)           */
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned long long ld_rlx64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned ld_rlx32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned ld_acq32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_rlx64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_rlx32(unsigned *p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_rel32(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
/* fire-and-forget atomic minimum (no result, so the thread does not wait) */
__device__ __forceinline__ void red_min(unsigned *p, unsigned v) {
  asm volatile("red.relaxed.gpu.global.min.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

/* where a wait gave up (GlobalCtl::err_where) */
enum : unsigned {
  W_ALLOC = 1, W_PT = 2, W_ENTRY = 3, W_HUB_PUB = 4, W_HUB_POP = 5, W_IDLE = 6,
  W_SPAN = 7, W_INIT = 8
};

__device__ __forceinline__ void raise_err(GlobalCtl *g, unsigned code, unsigned where) {
  if (atomicCAS(&g->err, 0u, code) == 0u) st_rlx32(&g->err_where, where);
}

/* Bounded wait: call once per spin iteration; false = give up. */
struct Waiter {
  unsigned long long deadline;
  unsigned it;
  unsigned code; /* error raised when the deadline passes */
  __device__ __forceinline__ bool spin(GlobalCtl *g, unsigned where) {
    ++it;
    if ((it & 15u) == 0u) {
      if (ld_rlx32(&g->err) != 0u) return false;
      if (gtimer() > deadline) {
        raise_err(g, code, where);
        return false;
      }
    }
    __nanosleep(it < 64 ? 20 : 200);
    return true;
  }
};

#define PAGE_MASK (ADDS_PAGE - 1u)
#define PI_BAD 0xFFFFFFFFu /* page-info sentinel: phys | phase << 31 */

/* ------------------------------------------------------------------------ */
/* page pool                                                                  */

/* Pops a free page (MPMC ticket queue).  Replaces alloc_manager
 * (wl.h:488-622), which pre-mapped pages ahead of each bag from one warp. */
__device__ unsigned alloc_page(const EngParams &P, unsigned long long deadline) {
  GlobalCtl *g = P.g;
  const unsigned long long t = atomicAdd(&g->fq_head, 1ull);
  unsigned long long *cell = &P.fq[t & P.fq_mask];
  const unsigned long long give_up = gtimer() + P.alloc_wait_ns;
  /* no page back within alloc_wait_ns means the pool is exhausted */
  Waiter w{deadline < give_up ? deadline : give_up, 0,
           deadline < give_up ? (unsigned)ADDS_DEV_TIMEOUT : (unsigned)ADDS_DEV_OVERFLOW};
  for (;;) {
    const unsigned long long e = ld_rlx64(cell);
    if ((unsigned)e == (unsigned)t) {
      const unsigned phys = (unsigned)(e >> 32);
      const unsigned gen = atomicAdd(&P.pgen[phys], 1u) + 1u;
      return phys | ((gen & 1u) << 31);
    }
    if (!w.spin(g, W_ALLOC)) return PI_BAD;
  }
}

__device__ void free_page(const EngParams &P, unsigned phys) {
  atomicExch(&P.pcons[phys], 0u);
  __threadfence();
  const unsigned long long t = atomicAdd(&P.g->fq_tail, 1ull);
  st_rlx64(&P.fq[t & P.fq_mask], ((unsigned long long)phys << 32) | (unsigned)t);
}

/* Marks cnt entries of page pi consumed and returns the count before; the
 * caller frees the page (consume_end) when that completes it.  The two
 * halves are split so that the wait for the count overlaps other work. */
__device__ __forceinline__ unsigned consume_begin(const EngParams &P, unsigned pi, unsigned cnt) {
  if (pi == PI_BAD || cnt == 0) return 0u;
  return atomicAdd(&P.pcons[pi & 0x7FFFFFFFu], cnt);
}
__device__ __forceinline__ void consume_end(const EngParams &P, unsigned pi, unsigned cnt,
                                            unsigned old) {
  if (pi == PI_BAD || cnt == 0) return;
  if (old + cnt == ADDS_PAGE) free_page(P, pi & 0x7FFFFFFFu);
}

__device__ __forceinline__ unsigned long long *pt_cell(const QueryDesc &d, unsigned s,
                                                       unsigned long long vp) {
  return d.pt + (((unsigned long long)s << d.ptn_log2) |
                 (vp & ((1ull << d.ptn_log2) - 1ull)));
}

/* Waits until virtual page vp of slot s is mapped (translate_write_ptr,
 * wl.h:1874-1900, resolved from an HBM page table; `cvp`/`cpi` are the
 * CTA's cached mapping for the slot, checked and refreshed here). */
__device__ unsigned pt_wait(const EngParams &P, const QueryDesc &d, unsigned s,
                            unsigned long long vp, unsigned long long deadline,
                            unsigned long long *cvp, unsigned *cpi) {
  if (*cvp == vp) return *cpi;
  unsigned long long *cell = pt_cell(d, s, vp);
  Waiter w{deadline, 0, ADDS_DEV_TIMEOUT};
  for (;;) {
    const unsigned long long e = ld_rlx64(cell);
    if ((unsigned)e == (unsigned)vp) {
      *cvp = vp;
      *cpi = (unsigned)(e >> 32);
      return *cpi;
    }
    if (!w.spin(P.g, W_PT)) return PI_BAD;
  }
}

/* Reserves c entries at the tail of slot s; maps the (at most two) pages the
 * range touches.  The reservation that contains a page's first entry
 * allocates it; others wait for the mapping.  Replaces push_work's
 * reservation + translate (wl.h:1902-1928). */
__device__ bool slot_reserve(const EngParams &P, const QueryDesc &d, unsigned s,
                             unsigned c, unsigned long long deadline,
                             unsigned long long *pbase, unsigned *pp0, unsigned *pp1,
                             unsigned long long *cvp, unsigned *cpi) {
  SlotCtr *sc = d.slots + s;
  /* span of live entries the page-table ring must cover.  head is read
   * together with the reservation (one round trip): a head older than the
   * reservation only makes the span look longer, so the check stays safe.
   * Claimers may also have moved head past this (still unwritten) range,
   * whose entries they then wait for: head > base + c is legal and means a
   * short span; the unsigned difference must not wrap into a spurious
   * overflow. */
  const unsigned long long head = ld_rlx64(&sc->head);
  const unsigned long long base = atomicAdd(&sc->tail, (unsigned long long)c);
  *pbase = base;
  *pp0 = *pp1 = PI_BAD;
  const unsigned long long ptn = 1ull << d.ptn_log2;
  const unsigned long long end = base + c;
  if (end > head && end - head > (ptn - 3ull) * ADDS_PAGE) {
    raise_err(P.g, ADDS_DEV_OVERFLOW, W_SPAN);
    return false;
  }
  const unsigned long long vp0 = base >> ADDS_PAGE_LOG2;
  const unsigned long long vp1 = (base + c - 1) >> ADDS_PAGE_LOG2;
  for (unsigned long long vp = vp0; vp <= vp1; ++vp) {
    unsigned pi;
    if ((vp << ADDS_PAGE_LOG2) >= base) {
      pi = alloc_page(P, deadline);
      if (pi == PI_BAD) return false;
      st_rlx64(pt_cell(d, s, vp), ((unsigned long long)pi << 32) | (unsigned)vp);
      *cvp = vp;
      *cpi = pi;
    } else {
      pi = pt_wait(P, d, s, vp, deadline, cvp, cpi);
      if (pi == PI_BAD) return false;
    }
    if (vp == vp0) *pp0 = pi; else *pp1 = pi;
  }
  if (vp1 == vp0) *pp1 = *pp0;
  return true;
}

__device__ __forceinline__ unsigned long long *entry_ptr(const EngParams &P, unsigned pi,
                                                         unsigned long long idx) {
  return P.pool + ((((unsigned long long)(pi & 0x7FFFFFFFu)) << ADDS_PAGE_LOG2) |
                   (idx & PAGE_MASK));
}
__device__ __forceinline__ unsigned long long make_entry(unsigned v, unsigned d,
                                                         unsigned pi) {
  return ((unsigned long long)d << 32) | (v & 0x7FFFFFFFu) | (pi & 0x80000000u);
}

/* ------------------------------------------------------------------------ */
/* bucket mapping (dist_to_bag_id_int, wl.h:1958-1972)                        */
template <bool FLT>
__device__ __forceinline__ unsigned dist_key(unsigned d, float scale) {
  if (FLT) return __float2uint_rz(__fmul_rn(__uint_as_float(d), scale));
  return d;
}
__device__ __forceinline__ unsigned bucket_slot(unsigned key, unsigned shift,
                                                unsigned base_b, unsigned base_key) {
  const unsigned kk = key >> shift;
  const unsigned off = kk > base_key ? min(kk - base_key, (unsigned)ADDS_NB - 1u) : 0u;
  return (base_b + off) & (ADDS_NB - 1u);
}

/* ------------------------------------------------------------------------ */
/* shared memory of one CTA                                                   */
#define NSLOT (2 * ADDS_NB) /* light buckets [0, NB), heavy lists [NB, 2NB) */

template <int BLOCK>
struct Smem {
  static constexpr int U = 4;               /* edges per thread per round    */
  static constexpr int SB = 2 * BLOCK * U;  /* staged pushes                 */
  unsigned it_rb[BLOCK];                    /* first edge of each item       */
  unsigned it_du[BLOCK];                    /* distance used for the item    */
  unsigned it_off[BLOCK];                   /* exclusive scan of degrees     */
  unsigned loc_v[BLOCK];                    /* own pushes kept for next batch */
  unsigned loc_d[BLOCK];
  unsigned pb_v[SB];
  unsigned pb_d[SB];
  unsigned short pb_rank[SB];
  unsigned char pb_s[SB];
  unsigned long long bbase[NSLOT];
  unsigned bp0[NSLOT];
  unsigned bp1[NSLOT];
  unsigned hist[NSLOT];
  unsigned gcnt[NSLOT];                     /* per-slot entries sent to HBM  */
  unsigned wsum[BLOCK / 32];
  /* batch descriptor written by the acquiring warp */
  unsigned long long h;
  unsigned status, q, slot, k;
  unsigned pi0, pi1;
  unsigned base_b, base_key, shift;
  unsigned pcnt, total_edges, hub_chunks;
  unsigned cur_q, idle, hungry;
  unsigned loc_k, loc_slot, keep_slot;
  unsigned hub_u, ptc_q, done_late;
  unsigned win; /* the batch's window of buckets (adapted on the device) */
  /* descriptor of query qd_q, copied once per change of query, so that a
   * batch reads its pointers from shared memory instead of HBM */
  QueryDesc qd;
  unsigned qd_q;
  /* page-table cache: last (virtual page -> page info) seen per slot of
   * query ptc_q.  A claimed or reserved entry keeps its page mapped, so a
   * hit on the same virtual page is always current. */
  unsigned long long ptc_vp[NSLOT];
  unsigned ptc_pi[NSLOT];
};

enum : unsigned { ST_WORK = 0, ST_HUB = 1, ST_IDLE = 2, ST_EXIT = 3, ST_LOCAL = 4, ST_HEAVY = 5 };

/* claim up to ~avail/nctas entries of one slot: inflight first (so the
 * bucket is never seen empty and drained while entries are held), then the
 * avail count, then the head index.  Returns the count, 0 if none. */
__device__ __forceinline__ unsigned claim(SlotCtr *sc, long long av, const EngParams &P,
                                          unsigned long long *h0) {
  /* CTAs expected to share one query's bucket: all of them for a single
   * solve, fewer as the batch has more queries */
  const unsigned per_q = (P.nctas >> P.greed) / P.nq;
  const long long share = (long long)(per_q ? per_q : 1u);
  long long want = (av + share - 1) / share;
  if (want > (long long)P.batch_max) want = P.batch_max;
  if (want < 1) want = 1;
  atomicAdd(&sc->inflight, (unsigned long long)want);
  const long long old =
      (long long)atomicAdd((unsigned long long *)&sc->avail, (unsigned long long)(-want));
  long long got = old < want ? old : want;
  if (got < 0) got = 0;
  if (got < want) {
    atomicAdd((unsigned long long *)&sc->avail, (unsigned long long)(want - got));
    atomicAdd(&sc->inflight, (unsigned long long)(got - want));
  }
  if (got > 0) *h0 = atomicAdd(&sc->head, (unsigned long long)got);
  return (unsigned)got;
}

/* ------------------------------------------------------------------------ */
/* Acquire a batch (warp 0).  Replaces the assign manager + get_global
 * mailbox handshake (wl.h:851-1527, 1698-1853).  Per query, the lowest live
 * bucket goes through two phases: L, its vertices are popped and their
 * light edges relaxed (buckets up to window-1 above it may run too), and
 * H, once its light queue is empty and drained, the heavy-edge lists of the
 * vertices it settled are expanded.  When both are empty and drained the
 * bucket retires and the next non-empty one becomes the base. */
template <int BLOCK>
__device__ void acquire(const EngParams &P, Smem<BLOCK> &S,
                        unsigned long long deadline) {
  const unsigned lane = threadIdx.x & 31u;
  GlobalCtl *g = P.g;
  /* independent control words are loaded together: a batch's acquisition
   * is a chain of memory round trips, each one on a wave front's path */
  const unsigned err0 = ld_rlx32(&g->err);
  const unsigned rem0 = ld_rlx32(&g->remaining);
  const unsigned hungry0 = P.adapt ? ld_rlx32(&g->hungry) : 0u;
  unsigned long long hh0 = 0ull, ht0 = 0ull;
  if (lane == 0) {
    hh0 = ld_rlx64(&g->hub_head);
    ht0 = ld_rlx64(&g->hub_tail);
  }
  if (err0 != 0u || rem0 == 0u) {
    if (lane == 0) S.status = ST_EXIT;
    return;
  }
  /* 1. split-row chunks first: they belong to vertices already popped */
  {
    unsigned long long ticket = ~0ull;
    if (lane == 0) {
      unsigned long long hh = hh0;
      for (int tries = 0; tries < 4; ++tries) {
        const unsigned long long ht = tries == 0 ? ht0 : ld_rlx64(&g->hub_tail);
        if (hh >= ht) break;
        const unsigned long long prev = atomicCAS(&g->hub_head, hh, hh + 1ull);
        if (prev == hh) { ticket = hh; break; }
        hh = prev;
      }
    }
    ticket = __shfl_sync(0xFFFFFFFFu, ticket, 0);
    if (ticket != ~0ull) {
      if (lane == 0) {
        const unsigned mask = (1u << ADDS_HUB_RING_LOG2) - 1u;
        unsigned *seq = P.hub_seq + (ticket & mask);
        Waiter w{deadline, 0, ADDS_DEV_TIMEOUT};
        bool ok = true;
        while (ld_acq32(seq) != (unsigned)(ticket + 1ull)) {
          if (!w.spin(g, W_HUB_POP)) { ok = false; break; }
        }
        if (ok) {
          const unsigned *hp = reinterpret_cast<const unsigned *>(P.hub + (ticket & mask));
          const unsigned cq = __ldcg(hp), cu = __ldcg(hp + 1), cdu = __ldcg(hp + 2),
                         ceb = __ldcg(hp + 3), cee = __ldcg(hp + 4);
          __threadfence();
          st_rel32(seq, (unsigned)(ticket + (1ull << ADDS_HUB_RING_LOG2)));
          S.status = ST_HUB;
          S.q = cq;
          S.k = 1;
          S.hub_u = cu;
          S.it_rb[0] = ceb;
          S.it_du[0] = cdu;
          S.it_off[0] = 0;
          S.total_edges = cee - ceb;
          const QueryCtl *ctl = P.qs[cq].ctl;
          const unsigned long long ctrl = ld_rlx64(&ctl->ctrl);
          S.base_b = (unsigned)ctrl & 0x7FFFFFFFu;
          S.base_key = (unsigned)(ctrl >> 32);
          S.shift = ld_rlx32(&ctl->shift);
        } else {
          S.status = ST_EXIT;
        }
      }
      return;
    }
  }
  /* 2. bucket queues, one query at a time starting at the sticky one */
  unsigned q = S.cur_q;
  const unsigned tries = P.nq < 8u ? P.nq : 8u;
  for (unsigned t = 0; t < tries; ++t, q = (q + 1u == P.nq) ? 0u : q + 1u) {
    /* the cached descriptor when it is this query's (shared memory) */
    const QueryDesc &d = (q == S.qd_q) ? S.qd : P.qs[q];
    QueryCtl *ctl = d.ctl;
    const unsigned qdone = ld_rlx32(&ctl->done);
    const unsigned long long ctrl = ld_rlx64(&ctl->ctrl);
    const unsigned qshift = ld_rlx32(&ctl->shift);
    const unsigned qwin = ld_rlx32(&ctl->win);
    if (qdone != 0u) continue;
    const unsigned base_b = (unsigned)ctrl & 0x7FFFFFFFu;
    const bool phase_h = ((unsigned)ctrl & ADDS_PHASE_H) != 0u;
    const unsigned base_key = (unsigned)(ctrl >> 32);
    const unsigned s = (base_b + lane) & (ADDS_NB - 1u);
    SlotCtr *lsc = d.slots + s;
    SlotCtr *hsc = d.slots + ADDS_NB + s;
    const unsigned long long lh = ld_rlx64(&lsc->head), lt = ld_rlx64(&lsc->tail);
    const long long lav = (long long)ld_rlx64((const unsigned long long *)&lsc->avail);
    const unsigned long long hh = ld_rlx64(&hsc->head), ht = ld_rlx64(&hsc->tail);
    const long long hav = (long long)ld_rlx64((const unsigned long long *)&hsc->avail);
    const unsigned lmask = __ballot_sync(0xFFFFFFFFu, lt > lh);
    const unsigned lamask = __ballot_sync(0xFFFFFFFFu, lav > 0);
    const unsigned hmask = __ballot_sync(0xFFFFFFFFu, ht > hh);
    const unsigned hamask = __ballot_sync(0xFFFFFFFFu, hav > 0);
    if ((lmask | hmask) == 0u) {
      if (lane == 0 && ld_rlx32(&ctl->live) == 0u) {
        if (atomicCAS(&ctl->done, 0u, 1u) == 0u) atomicSub(&g->remaining, 1u);
      }
      continue;
    }
    /* the base slot's in-flight counts, read after its head and tail (a
     * claimer raises them before it moves the head); needed only while the
     * base bucket's light queue or heavy list looks empty */
    const bool strict = P.strict_order != 0u;
    unsigned long long li = 0, hi = 0;
    if (strict && ((lmask & hmask & 1u) == 0u)) {
      if (lane == 0) {
        li = ld_rlx64(&lsc->inflight);
        hi = ld_rlx64(&hsc->inflight);
      }
      li = __shfl_sync(0xFFFFFFFFu, li, 0);
      hi = __shfl_sync(0xFFFFFFFFu, hi, 0);
    }
    const bool l_done = !(lmask & 1u) && (!strict || li == 0ull);
    const bool h_done = !(hmask & 1u) && (!strict || hi == 0ull);
    /* base-bucket state machine */
    unsigned eff = 0;      /* base after our transition, relative to base_b */
    bool eff_h = phase_h;
    unsigned long long nc = ctrl;
    if (l_done) {
      if (h_done) {
        /* retire: the next bucket with light entries or a heavy list (a
         * bucket above the base may have finished its light phase inside
         * the window and left only its heavy list), in phase L */
        const unsigned ahead = (lmask | hmask) & ~1u;
        if (ahead) {
          eff = __ffs(ahead) - 1u;
          eff_h = false;
          nc = ((unsigned long long)(base_key + eff) << 32) | ((base_b + eff) & 0x7FFFFFFFu);
        }
      } else if (!phase_h) { /* light phase over: expand the heavy lists */
        eff_h = true;
        nc = ((unsigned long long)base_key << 32) | base_b | ADDS_PHASE_H;
      }
    }
    /* On-device bucket width (adapt, the reference's dynamic delta,
     * wl.h:968-1360): the window of buckets processed at once widens by one
     * when this CTA finds nothing to claim inside it but light entries
     * beyond it (the buckets run thin), and narrows by one, down to the
     * configured window, when the base bucket retires while no CTA is idle.
     * Any window is label-correcting, so the distances do not change. */
    unsigned win = P.window;
    if (P.adapt) {
      win = qwin;
      if (nc != ctrl && eff != 0u && hungry0 == 0u && win > P.window && lane == 0)
        atomicCAS(&ctl->win, win, win - 1u);
    }
    if (nc != ctrl && lane == 0) atomicCAS(&ctl->ctrl, ctrl, nc);
    /* claim: heavy list of a base in phase H (or stale lists outside the
     * window), else the lowest light bucket inside the window */
    const unsigned wmask_l = (eff + win >= 32u) ? (0xFFFFFFFFu << eff)
                                                : (((1u << win) - 1u) << eff);
    /* heavy lists outside the active window belong to settled buckets */
    unsigned hcand = hamask & ~wmask_l;
    if (eff_h && eff == 0u) hcand |= hamask & 1u;  /* the base's heavy lists  */
    const unsigned lcand = lamask & wmask_l;
    bool heavy = hcand != 0u;
    const unsigned j = heavy ? (__ffs(hcand) - 1u) : (lcand ? __ffs(lcand) - 1u : 32u);
    if (j == 32u) {
      if (P.adapt && win < 32u && (lamask & ~wmask_l & ~((1u << eff) - 1u)) != 0u && lane == 0)
        atomicCAS(&ctl->win, win, win + 1u);
      continue;
    }
    unsigned got = 0;
    unsigned long long h0 = 0;
    if (lane == j) got = claim(heavy ? hsc : lsc, heavy ? hav : lav, P, &h0);
    got = __shfl_sync(0xFFFFFFFFu, got, j);
    h0 = __shfl_sync(0xFFFFFFFFu, h0, j);
    if (got == 0u) continue;
    if (lane == 0) {
      const unsigned sid = ((base_b + j) & (ADDS_NB - 1u)) + (heavy ? ADDS_NB : 0u);
      const unsigned long long vp0 = h0 >> ADDS_PAGE_LOG2;
      const unsigned long long vp1 = (h0 + got - 1ull) >> ADDS_PAGE_LOG2;
      if (S.ptc_q != q) { /* cache belongs to another query */
        for (int i = 0; i < NSLOT; ++i) S.ptc_vp[i] = ~0ull;
        S.ptc_q = q;
      }
      const unsigned pi0 = pt_wait(P, d, sid, vp0, deadline, &S.ptc_vp[sid], &S.ptc_pi[sid]);
      const unsigned pi1 = (vp1 == vp0) ? pi0
                           : pt_wait(P, d, sid, vp1, deadline, &S.ptc_vp[sid], &S.ptc_pi[sid]);
      S.status = heavy ? ST_HEAVY : ST_WORK;
      S.q = q;
      S.slot = sid;
      S.h = h0;
      S.k = got;
      S.pi0 = pi0;
      S.pi1 = pi1;
      S.base_b = (base_b + eff) & 0x7FFFFFFFu;
      S.base_key = base_key + eff;
      S.shift = qshift;
      S.win = win;
      S.cur_q = q;
    }
    return;
  }
  if (lane == 0) {
    S.status = ST_IDLE;
    S.cur_q = q;
  }
}

/* ------------------------------------------------------------------------ */
/* Flush staged pushes: counting sort by slot (light buckets and heavy lists)
 * in shared memory.  With `keep`, the entries of the lowest light bucket
 * inside the window (up to local_max) stay in shared memory as this CTA's
 * next batch, so a wavefront advances without a round trip through HBM.
 * Every other slot gets one tail reservation and the entry stores; its
 * avail count is raised after the stores.  Replaces the per-warp match_any
 * + atomicAdd + st.cg + __threadfence + write_done update of push_work
 * (wl.h:1902-1928).
 *
 * The flush that ends a batch also retires the batch: its done_k entries
 * leave the live count and the in-flight count of done_slot (NO_SLOT for a
 * split-row chunk).  The live count takes pushes minus done_k in one atomic
 * before any entry is visible, so it never falls below what is queued or
 * held.  When the CTA keeps entries of the batch's own slot, that slot's
 * in-flight count takes kept minus done_k in one atomic (it stays at least
 * the kept count, so the slot cannot retire under them); otherwise the
 * batch leaves its slot after the new entries are published.  A flush that
 * keeps every push publishes nothing and needs no fence. */
#define NO_SLOT 0xFFFFFFFFu
template <int BLOCK>
__device__ void flush(const EngParams &P, Smem<BLOCK> &S, const QueryDesc &d,
                      unsigned long long deadline, unsigned long long &st_pushes, bool keep,
                      unsigned done_k = 0u, unsigned done_slot = NO_SLOT) {
  const unsigned tid = threadIdx.x;
  const unsigned cnt = S.pcnt;
  if (cnt == 0u) { /* uniform: read after a barrier */
    if (tid == 0u && done_k) {
      if (done_slot != NO_SLOT)
        atomicAdd(&d.slots[done_slot].inflight, (unsigned long long)(0ull - done_k));
      atomicSub(&d.ctl->live, done_k);
    }
    return;
  }
  const unsigned qd = S.q; /* d is this query's descriptor */
  const bool stale_cache = S.ptc_q != qd; /* uniform: read after a barrier */
  /* whether CTAs are idle (keeps fewer entries local), read early */
  const unsigned hungry = (keep && tid < 32u) ? ld_rlx32(&P.g->hungry) : 0u;
  if (tid < NSLOT) {
    S.hist[tid] = 0u;
    if (stale_cache) S.ptc_vp[tid] = ~0ull;
  }
  __syncthreads();
  if (tid == 0u) S.ptc_q = qd;
  for (unsigned i = tid; i < cnt; i += BLOCK)
    S.pb_rank[i] = (unsigned short)atomicAdd(&S.hist[S.pb_s[i]], 1u);
  __syncthreads();
  if (tid < 32u) { /* warp 0: light buckets, local keep, live count */
    const unsigned c = S.hist[tid];
    const unsigned nz = __ballot_sync(0xFFFFFFFFu, c != 0u);
    unsigned ks = 0xFFFFFFFFu, kn = 0u;
    if (keep && nz) {
      const unsigned sh = S.base_b & 31u; /* bit r of rot = slot base_b + r */
      const unsigned rot = sh ? ((nz >> sh) | (nz << (32u - sh))) : nz;
      const unsigned r = __ffs(rot) - 1u;
      if (r < S.win) {
        ks = (S.base_b + r) & (ADDS_NB - 1u);
        const unsigned lmax = hungry ? P.local_max_hungry : P.local_max;
        kn = min(min(__shfl_sync(0xFFFFFFFFu, c, ks), lmax), (unsigned)BLOCK);
      }
    }
    const unsigned cg = c - ((tid == ks) ? kn : 0u);
    const bool merged = kn != 0u && done_slot == ks;
    if (tid == 0u) {
      /* count before any entry is visible: the entries become visible
       * through the avail increments below, each behind two barriers and a
       * (cumulative) fence of the raising thread, which order this update
       * before them as they order the entry stores */
      if (cnt != done_k) atomicAdd(&d.ctl->live, cnt - done_k);
      st_pushes += cnt;
      S.keep_slot = kn ? ks : 0xFFFFFFFFu;
      S.loc_k = kn;
      S.loc_slot = ks;
      S.done_late = (done_k != 0u && done_slot != NO_SLOT && !merged) ? 1u : 0u;
    }
    __syncwarp();
    S.gcnt[tid] = cg;
    if (tid == ks && kn) {
      const unsigned long long add = merged ? (unsigned long long)kn - done_k : kn;
      if (add) atomicAdd(&d.slots[ks].inflight, add);
    }
    if (cg != 0u) {
      unsigned long long b;
      unsigned p0, p1;
      slot_reserve(P, d, tid, cg, deadline, &b, &p0, &p1, &S.ptc_vp[tid], &S.ptc_pi[tid]);
      S.bbase[tid] = b;
      S.bp0[tid] = p0;
      S.bp1[tid] = p1;
    }
  } else if (tid < 64u) { /* warp 1: heavy lists */
    const unsigned sl = tid; /* NB + lane */
    const unsigned c = S.hist[sl];
    S.gcnt[sl] = c;
    if (c != 0u) {
      unsigned long long b;
      unsigned p0, p1;
      slot_reserve(P, d, sl, c, deadline, &b, &p0, &p1, &S.ptc_vp[sl], &S.ptc_pi[sl]);
      S.bbase[sl] = b;
      S.bp0[sl] = p0;
      S.bp1[sl] = p1;
    }
  }
  __syncthreads();
  const unsigned ks = S.keep_slot, kn = S.loc_k;
  for (unsigned i = tid; i < cnt; i += BLOCK) {
    const unsigned s = S.pb_s[i];
    const unsigned r = S.pb_rank[i];
    if (s == ks && r < kn) {
      S.loc_v[r] = S.pb_v[i];
      S.loc_d[r] = S.pb_d[i];
      continue;
    }
    const unsigned long long b = S.bbase[s];
    const unsigned long long idx = b + r - (s == ks ? kn : 0u);
    const unsigned pi = ((idx >> ADDS_PAGE_LOG2) == (b >> ADDS_PAGE_LOG2)) ? S.bp0[s] : S.bp1[s];
    if (pi != PI_BAD) st_rlx64(entry_ptr(P, pi, idx), make_entry(S.pb_v[i], S.pb_d[i], pi));
  }
  /* the entry stores of the whole CTA are ordered before the avail
   * increments by the barrier plus one (cumulative) fence per raising
   * thread; a popper that still sees an old entry waits on its phase bit */
  __syncthreads();
  if (tid < NSLOT && S.gcnt[tid] != 0u) {
    __threadfence();
    atomicAdd((unsigned long long *)&d.slots[tid].avail, (unsigned long long)S.gcnt[tid]);
  }
  if (tid == 0u) {
    S.pcnt = 0u;
    /* the batch leaves its slot after its pushes into that slot are
     * reserved (the tail moved), so the slot is never seen empty between */
    if (S.done_late) atomicAdd(&d.slots[done_slot].inflight, (unsigned long long)(0ull - done_k));
  }
  __syncthreads();
}

/* block-wide exclusive scan of one value per thread */
template <int BLOCK>
__device__ __forceinline__ unsigned block_exscan(Smem<BLOCK> &S, unsigned x, unsigned &total) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= (unsigned)o) incl += y;
  }
  if (lane == 31u) S.wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    unsigned w = lane < BLOCK / 32 ? S.wsum[lane] : 0u;
    unsigned wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= (unsigned)o) wi += y;
    }
    if (lane < BLOCK / 32) S.wsum[lane] = wi - w;
    if (lane == 31u) S.total_edges = wi;
  }
  __syncthreads();
  total = S.total_edges;
  return S.wsum[warp] + incl - x;
}

/* stage one push in shared memory (warp-aggregated slot reservation) */
template <int BLOCK>
__device__ __forceinline__ void stage(Smem<BLOCK> &S, unsigned v, unsigned dd, unsigned slot) {
  cg::coalesced_group grp = cg::coalesced_threads();
  unsigned pos = 0;
  if (grp.thread_rank() == 0) pos = atomicAdd(&S.pcnt, grp.size());
  pos = grp.shfl(pos, 0) + grp.thread_rank();
  S.pb_v[pos] = v;
  S.pb_d[pos] = dd;
  S.pb_s[pos] = (unsigned char)slot;
}

/* ------------------------------------------------------------------------ */
/* the persistent solver                                                      */
template <bool FLT, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) solve_kernel(EngParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<BLOCK> &S = *reinterpret_cast<Smem<BLOCK> *>(smem_raw);
  constexpr int U = Smem<BLOCK>::U;
  constexpr unsigned FLUSH_AT = Smem<BLOCK>::SB - BLOCK * U;
  const unsigned tid = threadIdx.x;
  const unsigned long long deadline = gtimer() + P.timeout_ns;

  unsigned long long st_items = 0, st_stale = 0, st_edges = 0, st_pushes = 0,
                     st_batches = 0, st_hub = 0, st_local = 0, st_hub_stale = 0,
                     st_heavy = 0;
  /* per-phase SM cycle counts (thread 0's view; every phase ends at a
   * barrier, so thread 0 sees the CTA's time) */
  unsigned long long cy_acq = 0, cy_load = 0, cy_edge = 0, cy_flush = 0, cy_idle = 0,
                     cy_mflush = 0, st_mflush = 0;
  const long long cy_start = clock64();
  long long cy_mark = cy_start;
#define CY_LAP(acc)                     \
  do {                                  \
    const long long _n = clock64();     \
    acc += (unsigned long long)(_n - cy_mark); \
    cy_mark = _n;                       \
  } while (0)
  if (tid == 0) {
    /* spread the CTAs evenly over the queries of a batch */
    S.cur_q = (unsigned)(((unsigned long long)blockIdx.x * P.nq) / P.nctas) % P.nq;
    S.pcnt = 0;
    S.idle = 0;
    S.hungry = 0;
    S.hub_chunks = 0;
    S.loc_k = 0;
    S.q = S.cur_q;
    S.ptc_q = 0xFFFFFFFFu;
    S.qd_q = 0xFFFFFFFFu;
    S.win = P.window;
  }
  if (tid < NSLOT) S.ptc_vp[tid] = ~0ull;
  __syncthreads();

  for (;;) {
    /* a local batch reads the window base with its entries' loads and
     * publishes it before the scan's barriers (thread 0) */
    unsigned long long lctrl = 0ull;
    unsigned lshift = 0u, lwin = 0u;
    if (S.loc_k == 0u) { /* uniform: read after a barrier */
      if (tid < 32) acquire<BLOCK>(P, S, deadline);
    } else if (tid == 0) {
      /* next batch = the entries this CTA kept from its own last flush
       * (of the query whose descriptor is cached) */
      S.status = ST_LOCAL;
      S.k = S.loc_k;
      S.slot = S.loc_slot;
      const QueryCtl *ctl = S.qd.ctl;
      lctrl = ld_rlx64(&ctl->ctrl);
      lshift = ld_rlx32(&ctl->shift);
      lwin = ld_rlx32(&ctl->win);
    }
    if (tid == 0 && S.status != ST_IDLE && S.status != ST_EXIT && S.q != S.qd_q) {
      S.qd = P.qs[S.q];
      S.qd_q = S.q;
    }
    __syncthreads();
    const unsigned status = S.status;
    if (status == ST_IDLE || status == ST_EXIT) CY_LAP(cy_idle); else CY_LAP(cy_acq);
    if (status == ST_EXIT) break;
    if (status == ST_IDLE) {
      if (tid == 0) {
        const unsigned n = ++S.idle;
        if (!S.hungry) {
          S.hungry = 1;
          atomicAdd(&P.g->hungry, 1u);
        }
        if (gtimer() > deadline) raise_err(P.g, ADDS_DEV_TIMEOUT, W_IDLE);
        __nanosleep(n < 8 ? 100 : (n < 64 ? 400 : 1000));
      }
      __syncthreads();
      CY_LAP(cy_idle);
      continue;
    }
    if (tid == 0) {
      S.idle = 0;
      if (S.hungry) {
        S.hungry = 0;
        atomicSub(&P.g->hungry, 1u);
      }
    }
    const unsigned q = S.q;
    const QueryDesc &d = S.qd;
    const unsigned *__restrict__ row = d.row;
    const uint2 *__restrict__ edges = d.edges;
    const unsigned *__restrict__ split = d.split;
    unsigned *dist = d.dist;
    const float scale = d.scale;
    unsigned k = 1;
    unsigned cons0 = 0u, cons1 = 0u; /* page counts before this batch (thread 0) */

    if (status != ST_HUB) {
      k = S.k;
      const unsigned long long h = S.h;
      const unsigned myslot = S.slot;
      unsigned deg = 0, rb = 0, dp = 0, chunks = 0;
      if (tid < k) {
        bool ok = true;
        unsigned v = 0;
        if (status == ST_LOCAL) {
          v = S.loc_v[tid];
          dp = S.loc_d[tid];
        } else {
          const unsigned long long idx = h + tid;
          const unsigned pi = ((idx >> ADDS_PAGE_LOG2) == (h >> ADDS_PAGE_LOG2)) ? S.pi0 : S.pi1;
          ok = pi != PI_BAD;
          unsigned long long e = 0;
          if (ok) {
            const unsigned long long *ep = entry_ptr(P, pi, idx);
            Waiter w{deadline, 0, ADDS_DEV_TIMEOUT};
            e = ld_rlx64(ep);
            while (((unsigned)e & 0x80000000u) != (pi & 0x80000000u)) {
              if (!w.spin(P.g, W_ENTRY)) { ok = false; break; }
              e = ld_rlx64(ep);
            }
          }
          v = (unsigned)e & 0x7FFFFFFFu;
          dp = (unsigned)(e >> 32);
        }
        if (ok) {
          /* the row bounds are read with the distance, before the stale
           * check: one memory round trip per batch instead of two (a wave
           * front advances one batch per round trip chain) */
          const unsigned dv = __ldcg(dist + v);
          const unsigned r0 = __ldg(row + v), r1 = __ldg(row + v + 1);
          const unsigned nl = split ? __ldg(split + v) : (r1 - r0);
          ++st_items;
          if (dv < dp) {
            ++st_stale; /* superseded: a later push carries the smaller value */
          } else {
            if (status == ST_HEAVY) { /* settled vertex: its heavy edges */
              rb = r0 + nl;
              deg = r1 - rb;
              ++st_heavy;
            } else {                  /* light edges now, heavy list later */
              rb = r0;
              deg = nl;
              if (nl < r1 - r0) stage<BLOCK>(S, v, dp, ADDS_NB + (myslot & (ADDS_NB - 1u)));
            }
            if (deg > P.hub_threshold) {
              chunks = (deg + P.hub_chunk - 1u) / P.hub_chunk;
              atomicAdd(&S.hub_chunks, chunks);
            } else {
              st_edges += deg; /* split rows are counted chunk by chunk */
            }
          }
        }
        if (chunks) S.loc_v[tid] = v; /* remembered for the chunk records */
      }
      S.it_rb[tid] = rb;
      S.it_du[tid] = dp;
      if (tid == 0 && status == ST_LOCAL) {
        S.base_b = (unsigned)lctrl & 0x7FFFFFFFu;
        S.base_key = (unsigned)(lctrl >> 32);
        S.shift = lshift;
        S.win = P.adapt ? lwin : P.window;
      }
      unsigned tot;
      const unsigned off = block_exscan<BLOCK>(S, chunks ? 0u : deg, tot);
      S.it_off[tid] = off;
      /* retire the claimed range (every entry has been read): the counts are
       * raised now, and pages whose entries are all consumed go back after
       * the expansion, when the counts have long arrived */
      if (tid == 0) {
        if (status != ST_LOCAL) {
          const unsigned c0 = min((unsigned)(ADDS_PAGE - (h & PAGE_MASK)), k);
          cons0 = consume_begin(P, S.pi0, c0);
          if (k > c0) cons1 = consume_begin(P, S.pi1, k - c0);
        } else {
          ++st_local;
        }
        S.loc_k = 0;
        if (S.hub_chunks) {
          atomicAdd(&d.ctl->live, S.hub_chunks);
          __threadfence();
        }
      }
      __syncthreads();
      if (chunks) {
        /* publish this row's chunks for the whole grid (tb_coop_assign,
         * wl.h:1638-1696, widened from one block to all CTAs) */
        const unsigned u = S.loc_v[tid];
        const unsigned mask = (1u << ADDS_HUB_RING_LOG2) - 1u;
        const unsigned long long t0 = atomicAdd(&P.g->hub_tail, (unsigned long long)chunks);
        /* the row's ring cells are free once their sequence words reach
         * their tickets: read eight at a time (one round trip each group),
         * then one fence before all the records and one before all the
         * sequence words, instead of two fences per chunk */
        bool ok = true;
        for (unsigned c0 = 0; c0 < chunks && ok; c0 += 8u) {
          const unsigned nb = min(8u, chunks - c0);
          unsigned sq[8];
#pragma unroll
          for (unsigned j = 0; j < 8u; ++j)
            sq[j] = j < nb ? ld_rlx32(P.hub_seq + ((t0 + c0 + j) & mask)) : 0u;
#pragma unroll
          for (unsigned j = 0; j < 8u; ++j) {
            if (j >= nb || !ok) continue;
            const unsigned long long t = t0 + c0 + j;
            Waiter w{deadline, 0, ADDS_DEV_HUB_OVERFLOW};
            while (sq[j] != (unsigned)t) {
              if (!w.spin(P.g, W_HUB_PUB)) { ok = false; break; }
              sq[j] = ld_rlx32(P.hub_seq + (t & mask));
            }
          }
        }
        if (ok) {
          __threadfence(); /* the cells' last readers are done before they are reused */
          for (unsigned c = 0; c < chunks; ++c) {
            HubChunk hc;
            hc.q = q;
            hc.u = u;
            hc.du = dp;
            hc.eb = rb + c * P.hub_chunk;
            hc.ee = (unsigned)min((unsigned long long)rb + (unsigned long long)(c + 1u) * P.hub_chunk,
                                  (unsigned long long)rb + deg);
            hc.pad[0] = hc.pad[1] = hc.pad[2] = 0u;
            P.hub[(t0 + c) & mask] = hc;
          }
          __threadfence(); /* the records before their sequence words */
          for (unsigned c = 0; c < chunks; ++c)
            st_rlx32(P.hub_seq + ((t0 + c) & mask), (unsigned)(t0 + c + 1ull));
        }
      }
    } else { /* ST_HUB: one chunk of a split row, staged by acquire */
      if (tid == 0) {
        ++st_hub;
        /* the row's vertex improved since the chunk was made: a later
         * expansion covers these edges with the smaller distance */
        if (__ldcg(dist + S.hub_u) < S.it_du[0]) {
          S.total_edges = 0;
          ++st_hub_stale;
        } else {
          st_edges += S.total_edges;
        }
      }
      __syncthreads();
    }
    if (tid == 0) {
      ++st_batches;
      S.hub_chunks = 0;
    }
    /* read after the barriers above (a local batch's base was published
     * before the scan) */
    const unsigned shift = S.shift, base_b = S.base_b, base_key = S.base_key;
    CY_LAP(cy_load);

    /* edge-balanced expansion of the batch: relax + atomicMin + stage push */
    const unsigned E = S.total_edges;
    int lo = 0; /* a thread's edges only increase: each search starts at the last item */
    for (unsigned eb = 0; eb < E; eb += BLOCK * U) {
      unsigned dst[U], nd[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const unsigned e = eb + u * BLOCK + tid;
        nd[u] = 0xFFFFFFFFu;
        dst[u] = 0;
        if (e < E) {
          int hi = (int)k - 1;
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (S.it_off[mid] <= e) lo = mid; else hi = mid - 1;
          }
          const uint2 ed = __ldg(edges + S.it_rb[lo] + (e - S.it_off[lo]));
          const unsigned du = S.it_du[lo];
          dst[u] = ed.x;
          nd[u] = FLT ? __float_as_uint(__fadd_rn(__uint_as_float(du), __uint_as_float(ed.y)))
                      : du + ed.y;
        }
      }
      /* A single solve is a chain of dependent round trips: an improvement on
       * the gathered value is applied with a reduction (no result, so no
       * wait) and pushed at once; where a concurrent smaller value wins, the
       * entry is dropped as stale when it is popped (the reference's int
       * kernel also pushes whatever its atomicMin returned,
       * ads_int/kernel.cu:78-82).  A batch of queries hides that latency
       * behind its other queries and is bound by work instead: it pushes only
       * when its atomicMin won, which spares the duplicate entries (23 % more
       * pops on the batch of 128 grids). */
      unsigned cur[U];
#pragma unroll
      for (int u = 0; u < U; ++u) cur[u] = (nd[u] != 0xFFFFFFFFu) ? __ldcg(dist + dst[u]) : 0u;
      if (P.nq == 1u) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (nd[u] < cur[u]) {
            red_min(dist + dst[u], nd[u]);
            stage<BLOCK>(S, dst[u], nd[u],
                         bucket_slot(dist_key<FLT>(nd[u], scale), shift, base_b, base_key));
          }
        }
      } else {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (nd[u] < cur[u] && atomicMin(dist + dst[u], nd[u]) > nd[u])
            stage<BLOCK>(S, dst[u], nd[u],
                         bucket_slot(dist_key<FLT>(nd[u], scale), shift, base_b, base_key));
        }
      }
      __syncthreads();
      if (S.pcnt > FLUSH_AT) {
        CY_LAP(cy_edge);
        flush<BLOCK>(P, S, d, deadline, st_pushes, false);
        CY_LAP(cy_mflush);
        ++st_mflush;
      }
    }
    if (tid == 0 && (status == ST_WORK || status == ST_HEAVY)) {
      const unsigned c0 = min((unsigned)(ADDS_PAGE - (S.h & PAGE_MASK)), k);
      consume_end(P, S.pi0, c0, cons0);
      if (k > c0) consume_end(P, S.pi1, k - c0, cons1);
    }
    __syncthreads();
    CY_LAP(cy_edge);
    /* batch finished: its k entries (or one chunk) leave the live count and
     * the slot's in-flight count inside the flush */
    flush<BLOCK>(P, S, d, deadline, st_pushes, P.local_max != 0u, k,
                 status != ST_HUB ? S.slot : NO_SLOT);
    CY_LAP(cy_flush);
  }
#undef CY_LAP

  if (tid == 0 && S.hungry) atomicSub(&P.g->hungry, 1u);
  /* statistics */
  {
    GlobalCtl *g = P.g;
#define WSUM(x) \
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xFFFFFFFFu, x, o);
    WSUM(st_items) WSUM(st_stale) WSUM(st_edges) WSUM(st_pushes) WSUM(st_heavy)
#undef WSUM
    if ((tid & 31u) == 0u) {
      if (st_items) atomicAdd(&g->st_items, st_items);
      if (st_stale) atomicAdd(&g->st_stale, st_stale);
      if (st_edges) atomicAdd(&g->st_edges, st_edges);
      if (st_pushes) atomicAdd(&g->st_pushes, st_pushes);
      if (st_heavy) atomicAdd(&g->st_heavy, st_heavy);
      if (tid == 0) {
        atomicAdd(&g->st_cyc[0], cy_acq);
        atomicAdd(&g->st_cyc[1], cy_load);
        atomicAdd(&g->st_cyc[2], cy_edge);
        atomicAdd(&g->st_cyc[3], cy_flush);
        atomicAdd(&g->st_cyc[4], cy_idle);
        atomicAdd(&g->st_cyc[5], (unsigned long long)(clock64() - cy_start));
        atomicAdd(&g->st_pad[0], cy_mflush);
        atomicAdd(&g->st_pad[1], st_mflush);
        if (st_hub) atomicAdd(&g->st_hub, st_hub);
        if (st_local) atomicAdd(&g->st_local, st_local);
        if (st_hub_stale) atomicAdd(&g->st_hub_stale, st_hub_stale);
        atomicAdd(&g->st_batches, st_batches);
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* init: d = INF, d[src] = 0, per-query control reset, source pushed to the
 * lowest bucket (ads_int/kernel.cu:18-27 + assign_manager's source push,
 * wl.h:944-953).  grid = (x, nq). */
__global__ void init_kernel(EngParams P) {
  const unsigned q = blockIdx.y;
  const QueryDesc &d = P.qs[q];
  const unsigned src = (P.single_src != 0xFFFFFFFFu && q == 0u) ? P.single_src : d.src;
  const unsigned inf = P.is_float ? ADDS_INF_F32_BITSV : ADDS_INF_I32_BITS;
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < d.n;
       v += gridDim.x * blockDim.x)
    d.dist[v] = (v == src) ? 0u : inf;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    GlobalCtl *g = P.g;
    if (q == 0) {
      g->remaining = P.nq;
      g->hungry = 0;
      g->st_items = g->st_stale = g->st_edges = g->st_pushes = 0;
      g->st_batches = g->st_hub = g->st_local = g->st_hub_stale = g->st_heavy = 0;
      for (int i = 0; i < 6; ++i) g->st_cyc[i] = 0;
      g->st_pad[0] = g->st_pad[1] = 0;
    }
    QueryCtl *c = d.ctl;
    c->ctrl = 0ull;
    c->done = 0u;
    c->shift = d.shift0;
    c->win = P.window;
    for (int s = 0; s < NSLOT; ++s) d.slots[s].inflight = 0ull;
    c->live = 1u;
    __threadfence();
    const unsigned long long deadline = gtimer() + P.timeout_ns;
    unsigned long long b, cvp = ~0ull;
    unsigned p0, p1, cpi = 0;
    if (slot_reserve(P, d, 0u, 1u, deadline, &b, &p0, &p1, &cvp, &cpi)) {
      st_rlx64(entry_ptr(P, p0, b), make_entry(src, 0u, p0));
      __threadfence();
      atomicAdd((unsigned long long *)&d.slots[0].avail, 1ull);
    }
  }
}

/* reached vertices and their out-edges (m_r, n_r of the GTEPS metric) */
__global__ void reached_kernel(const unsigned *row, const unsigned *dist, unsigned n,
                               unsigned inf, unsigned long long *out) {
  unsigned long long nr = 0, mr = 0;
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    if (dist[v] != inf) {
      ++nr;
      mr += row[v + 1] - row[v];
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    nr += __shfl_down_sync(0xFFFFFFFFu, nr, o);
    mr += __shfl_down_sync(0xFFFFFFFFu, mr, o);
  }
  if ((threadIdx.x & 31u) == 0u) {
    atomicAdd(out, nr);
    atomicAdd(out + 1, mr);
  }
}

/* worklist full reset: free queue holds every page, hub ring sequence = i */
__global__ void wl_reset_kernel(unsigned long long *fq, unsigned fq_cells, unsigned pool_pages,
                                unsigned *hub_seq, unsigned hub_cells) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < fq_cells;
       i += gridDim.x * blockDim.x)
    fq[i] = (i < pool_pages) ? (((unsigned long long)i << 32) | i)
                             : (unsigned long long)(~i); /* tag never equals i */
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < hub_cells;
       i += gridDim.x * blockDim.x)
    hub_seq[i] = i;
}

/* ------------------------------------------------------------------------ */
/* host-side launch helpers (called from api.cu)                              */
template <bool FLT, int BLOCK>
static cudaError_t prep_one(int *max_blocks_per_sm) {
  const size_t smem = sizeof(Smem<BLOCK>);
  cudaError_t e = cudaFuncSetAttribute(solve_kernel<FLT, BLOCK>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(max_blocks_per_sm,
                                                       solve_kernel<FLT, BLOCK>, BLOCK, smem);
}

template <bool FLT, int BLOCK>
static cudaError_t launch_one(const EngParams &P, cudaStream_t st) {
  /* cooperative launch: all CTAs co-resident (they wait on each other's
   * pushes); cudaLaunchKernelEx form so the launch can be graph-captured */
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P.nctas);
  cfg.blockDim = dim3(BLOCK);
  cfg.dynamicSmemBytes = sizeof(Smem<BLOCK>);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, solve_kernel<FLT, BLOCK>, P);
}

}  // namespace adds

/* C++ linkage entry points used by api.cu.  block: 128, 256 or 512 (a
 * 64-thread variant measured 3.6x slower on the 4096^2 grid: its CTAs hold
 * too few of a wave front's vertices per batch). */
cudaError_t adds_engine_prepare(bool flt, int block, int *max_blocks_per_sm) {
  switch (block) {
    case 128: return flt ? adds::prep_one<true, 128>(max_blocks_per_sm) : adds::prep_one<false, 128>(max_blocks_per_sm);
    case 256: return flt ? adds::prep_one<true, 256>(max_blocks_per_sm) : adds::prep_one<false, 256>(max_blocks_per_sm);
    case 512: return flt ? adds::prep_one<true, 512>(max_blocks_per_sm) : adds::prep_one<false, 512>(max_blocks_per_sm);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t adds_engine_launch_init(const EngParams &P, unsigned max_n, cudaStream_t st) {
  unsigned bx = (max_n + 1023u) / 1024u;
  if (bx > 1184u) bx = 1184u; /* 8 x 148 SMs: grid-stride beyond that */
  if (bx == 0u) bx = 1u;
  dim3 grid(bx, P.nq);
  adds::init_kernel<<<grid, 1024, 0, st>>>(P);
  return cudaGetLastError();
}

cudaError_t adds_engine_launch_solve(const EngParams &P, int block, cudaStream_t st) {
  switch (block) {
    case 128: return P.is_float ? adds::launch_one<true, 128>(P, st) : adds::launch_one<false, 128>(P, st);
    case 256: return P.is_float ? adds::launch_one<true, 256>(P, st) : adds::launch_one<false, 256>(P, st);
    case 512: return P.is_float ? adds::launch_one<true, 512>(P, st) : adds::launch_one<false, 512>(P, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t adds_engine_launch_reached(const unsigned *row, const unsigned *dist, unsigned n,
                                       unsigned inf, unsigned long long *out, cudaStream_t st) {
  unsigned bx = (n + 255u) / 256u;
  if (bx > 1184u) bx = 1184u;
  if (bx == 0u) bx = 1u;
  adds::reached_kernel<<<bx, 256, 0, st>>>(row, dist, n, inf, out);
  return cudaGetLastError();
}

cudaError_t adds_engine_launch_reset(unsigned long long *fq, unsigned fq_cells,
                                     unsigned pool_pages, unsigned *hub_seq, unsigned hub_cells,
                                     cudaStream_t st) {
  adds::wl_reset_kernel<<<296, 256, 0, st>>>(fq, fq_cells, pool_pages, hub_seq, hub_cells);
  return cudaGetLastError();
}
