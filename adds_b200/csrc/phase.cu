/*
 * phase.cu — bulk-synchronous bucketed delta-stepping SSSP for sm_100a.
 *
 * Behavioural source: ADDS (ads_int/kernel.cu:30-128 relaxation,
 * ads_int/wl.h:192-1972 bucket worklist).  Kept from the reference:
 *   - circular distance buckets, bucket = key >> shift (wl.h:1958-1972),
 *     the farthest slot collecting everything beyond the ring;
 *   - relax new = d[u] + w, accept if d[v] > new, atomicMin, push
 *     (kernel.cu:112-121); float relaxes fl(d[u] + w) with a 32-bit
 *     atomicMin on the bits of the non-negative float instead of the
 *     reference's 64-bit CAS (ads_float/csr_graph.h:58-70);
 *   - long rows split across workers (tb_coop_assign, wl.h:1638-1696; here
 *     across every CTA of the group);
 *   - the reference's per-thread work counts (wl.h:1835-1839) as statistics.
 * Different: the buckets are settled in phases (Meyer-Sanders light/heavy
 * delta-stepping).  A group of CTAs expands one frontier, meets at a group
 * barrier, and the last CTA to arrive decides the next frontier from the list
 * tails; while frontiers are small that CTA keeps running them alone with
 * block barriers only.  There is no manager block, no CDP launch and no
 * per-push fence; every wait is bounded by a device deadline and reports
 * an error word instead of trapping.
 *
 * Batches: every group takes queries from a shared counter (largest first)
 * and solves each one start to finish, distance initialisation included, so
 * a batch of uneven solves is one launch.
 */
#include <cuda_runtime.h>

#include "phase_internal.h"

namespace adds_phase {

#define PH_M_START 5u /* bootstrap pseudo-phase: nothing ran yet */

/* ------------------------------------------------------------------------ */
/* memory-model helpers (PTX ISA: ld/st .relaxed/.acquire/.release .gpu)     */
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
/* Edge stream load: read-only path, no L1 allocation.  An L2 evict_first
 * hint on these loads measured 2.6 % slower on R-MAT 24 (5.85 vs 5.70 ms):
 * a row's edges are often read again by the next light/heavy phase. */
__device__ __forceinline__ uint2 ld_edge(const uint2 *p) {
  uint2 r;
  asm("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(r.x), "=r"(r.y) : "l"(p));
  return r;
}

enum : unsigned { W_BARRIER = 1, W_PT = 2, W_ALLOC = 3, W_MAPPING = 4, W_HUB = 5, W_COPY = 6 };

__device__ __forceinline__ void raise_err(PhGlobal *g, unsigned code, unsigned where) {
  if (atomicCAS(&g->err, 0u, code) == 0u) st_rlx32(&g->err_where, where);
}

/* Bounded wait: call once per spin iteration; false = give up. */
struct Waiter {
  unsigned long long deadline;
  unsigned it;
  __device__ __forceinline__ bool spin(PhGlobal *g, unsigned where, unsigned sleep_cap) {
    ++it;
    if ((it & 15u) == 0u) {
      if (ld_rlx32(&g->err) != 0u) return false;
      if (gtimer() > deadline) {
        raise_err(g, PH_ERR_TIMEOUT, where);
        return false;
      }
    }
    __nanosleep(it < 32 ? 32 : sleep_cap);
    return true;
  }
};

/* ------------------------------------------------------------------------ */
/* bucket mapping (dist_to_bag_id_int, wl.h:1958-1972)                        */
template <bool FLT>
__device__ __forceinline__ unsigned bucket_of(unsigned d, float scale, unsigned shift) {
  unsigned key = d;
  if (FLT) key = __float2uint_rz(__fmul_rn(__uint_as_float(d), scale));
  return key >> shift;
}
/* A lower bound of every heavy-edge candidate fl(d[u] + w) out of bucket
 * base: a vertex whose distance is at or below it cannot be improved by the
 * bucket's heavy edges.  Integer keys: a heavy edge has w >= 2^shift and d[u]
 * >= base << shift, so the bound is the next bucket's first key (minus one).
 * Float keys: d[u] >= base 2^shift / scale and w >= 2^shift / scale up to the
 * roundings of the key product and of the light threshold, both covered by
 * the 1e-6 margin; the sum is rounded down. */
template <bool FLT>
__device__ __forceinline__ unsigned pull_floor(const PhQuery &Q, unsigned base) {
  if (!FLT) {
    const unsigned long long t = ((unsigned long long)base + 1ull) << Q.shift;
    return t > 0xFFFFFFFFull ? 0xFFFFFFFFu : (unsigned)(t - 1ull);
  }
  const double bw = ldexp(1.0, (int)Q.shift) / (double)Q.scale * (1.0 - 1e-6);
  const float lo = __double2float_rd((double)base * bw);
  const float dw = __double2float_rd(bw);
  return __float_as_uint(__fadd_rd(lo, dw));
}

/* list of a push with bucket b relative to the base bucket being settled;
 * the near-far schedule keeps one far pile instead of the ring */
__device__ __forceinline__ unsigned route(unsigned b, unsigned base, unsigned near_far) {
  if (b <= base) return PH_LNEXT;
  if (near_far) return PH_LFAR;
  const unsigned off = min(b - base, (unsigned)PH_NSLOT - 1u);
  return (base + off) & (PH_NSLOT - 1u);
}

/* ------------------------------------------------------------------------ */
/* shared memory of one CTA                                                   */
#define PH_RES_PAGES 6u /* pages one list reservation may touch (flush size) */
#define PH_EPT 1        /* frontier entries one thread prepares per chunk     */
#define PH_PULL_V 4u    /* vertices one thread selects per pull sub-tile      */
#define PH_PULL_SUB 2u  /* pull sub-tiles per block barrier                  */
/* split-row chunk records one CTA takes at a time */
#define PH_HUB_PER_CLAIM(BLOCK) ((BLOCK) / 16u)

template <int BLOCK, int UU>
struct PSmem {
  static constexpr int U = UU;      /* edges per thread in flight                     */
  static constexpr int SEGI = 2;    /* iterations of U edges between flush checks     */
  static constexpr int EPT = PH_EPT;         /* frontier entries per thread per chunk */
  static constexpr int IC = EPT * BLOCK;     /* items per chunk                        */
  static constexpr int FLUSH_AT = 2 * BLOCK; /* flush once more than this is staged  */
  /* staged pushes: FLUSH_AT, plus one per entry of a chunk, plus one per edge of
   * a segment -- a segment can never overflow the buffer */
  static constexpr int SB = FLUSH_AT + IC + SEGI * U * BLOCK;
  static_assert(SB <= (int)((PH_RES_PAGES - 1u) * PH_PAGE + 1u),
                "a flush must fit in PH_RES_PAGES pages of one list");
  /* the items of the chunk being expanded: row segments [rb, re) */
  unsigned it_rb[IC];
  unsigned it_du[IC];      /* distance the item is expanded with                 */
  unsigned it_off[IC + 1]; /* exclusive scan of the segment lengths              */
  unsigned ck_k, ck_E;        /* items and edges of the chunk                    */
  unsigned pb_v[SB];
  unsigned pb_d[SB];
  unsigned short pb_rank[SB];
  unsigned char pb_l[SB];
  unsigned hist[PH_NLIST];
  unsigned bpg[PH_NLIST][PH_RES_PAGES]; /* pages of each list's reservation  */
  unsigned long long bbase[PH_NLIST];
  unsigned long long ptc_vp[PH_NLIST]; /* per-list page-table cache           */
  unsigned ptc_pi[PH_NLIST];
  unsigned wsum[BLOCK / 32];
  PhDesc D;                            /* the phase being run                 */
  unsigned long long st_items, st_stale, st_heavy, st_repush, st_pushes, st_chunks, st_hubs,
      st_solo;
  unsigned long long claim;
  unsigned long long cy[8]; /* thread 0's cycles: entry prep, record prep (with
                               waits), expand, flush, barrier wait, leader,
                               grid-phase work, total */
  unsigned total, pcnt, leader, gen, pi0, pi1, stop;
  unsigned hub_made; /* this CTA cut a row into records in the current phase */
  unsigned long long tr_e, tr_mi, tr_mp; /* trace: phase edges, counter marks */
  /* -- after the fields above, which keep their offsets -- */
  /* thread 0's claim state and cycle marks (kept here, not in registers) */
  unsigned long long local_claim, pend;
  long long tph, tk, cy0;
  unsigned long long nphase;
  /* pull phase: next tile of the current run, tiles left in it, the tile
   * being expanded, pull_floor of the phase's bucket */
  unsigned pl_t0, pl_k, pl_cur, pl_T;
  unsigned it_d0[IC]; /* pull batch: each vertex's distance before it */
  unsigned it_v[IC];  /* pull batch: the item's vertex                 */
};

/* thread 0's cycle accounting: the cycles since the last mark go to cy[i] */
template <int BLOCK, int UU>
__device__ __forceinline__ void cy_mark(PSmem<BLOCK, UU> &S, int i) {
  if (threadIdx.x == 0) {
    const long long t = clock64();
    S.cy[i] += (unsigned long long)(t - S.tph);
    S.tph = t;
  }
}

/* what a CTA keeps for the kernel's lifetime; the group's arrays are
 * recomputed from the parameters where they are used */
struct Ctx {
  unsigned gi, rank;
  unsigned long long deadline;
  unsigned edges; /* per-thread count; the rest is counted in shared memory */
  unsigned edges_mark; /* trace: c.edges at the end of the last phase         */
};
__device__ __forceinline__ PhGroup *grp_of(const PhParams &P, const Ctx &c) { return P.grp + c.gi; }

__device__ __forceinline__ unsigned long long *pt_cell(const PhParams &P, const Ctx &c, unsigned L,
                                                       unsigned long long vp) {
  return P.pt + ((((unsigned long long)c.gi * PH_NLIST + L) << P.ptn_log2) |
                 (vp & ((1ull << P.ptn_log2) - 1ull)));
}
__device__ __forceinline__ unsigned long long *entry_ptr(const PhParams &P, const Ctx &c,
                                                         unsigned page, unsigned long long idx) {
  return P.pool + ((((unsigned long long)c.gi * P.pages_per_group + page) << PH_PAGE_LOG2) |
                   (idx & (PH_PAGE - 1u)));
}
__device__ __forceinline__ PhHub *hub_of(const PhParams &P, const Ctx &c) {
  return P.hub + (unsigned long long)c.gi * P.hub_cap;
}
__device__ __forceinline__ unsigned *hub_seq_of(const PhParams &P, const Ctx &c) {
  return P.hub_seq + (unsigned long long)c.gi * P.hub_cap;
}

/* Page of virtual page vp of list L; waits for the reservation that owns the
 * page's first entry to map it (a bounded, short wait: that reservation is
 * in flight in the same phase). */
__device__ unsigned pt_wait(const PhParams &P, const Ctx &c, unsigned L, unsigned long long vp,
                            unsigned long long *cvp, unsigned *cpi) {
  if (*cvp == vp) return *cpi;
  unsigned long long *cell = pt_cell(P, c, L, vp);
  Waiter w{c.deadline, 0};
  for (;;) {
    const unsigned long long e = ld_rlx64(cell);
    if ((unsigned)e == (unsigned)vp) {
      *cvp = vp;
      *cpi = (unsigned)(e >> 32);
      return *cpi;
    }
    if (!w.spin(P.g, W_PT, 64)) return 0xFFFFFFFFu;
  }
}

/* Reserves cnt entries at the tail of list L and maps the pages the range
 * touches (at most PH_RES_PAGES) into pgs[].  The reservation holding a
 * page's first entry takes a page from the group's bump counter; it maps the
 * pages it owns before it waits for the first one, so a later reservation
 * never waits behind its wait.  Replaces push_work's reservation and
 * address translation (wl.h:1854-1928). */
__device__ bool list_reserve(const PhParams &P, const Ctx &c, unsigned L, unsigned cnt,
                             unsigned long long *pbase, unsigned *pgs,
                             unsigned long long *cvp, unsigned *cpi) {
  PhGroup *G = grp_of(P, c);
  const unsigned long long base = atomicAdd(&G->tails[L].tail, (unsigned long long)cnt);
  *pbase = base;
  const unsigned long long vp0 = base >> PH_PAGE_LOG2;
  const unsigned long long vp1 = (base + cnt - 1ull) >> PH_PAGE_LOG2;
  for (unsigned j = 0; j < PH_RES_PAGES; ++j) pgs[j] = 0xFFFFFFFFu;
  if (vp1 - vp0 >= PH_RES_PAGES) { /* larger than any flush: engine fault */
    raise_err(P.g, PH_ERR_MAPPING, W_ALLOC);
    return false;
  }
  for (unsigned long long vp = vp1 + 1ull; vp-- > vp0;) {
    if ((vp << PH_PAGE_LOG2) < base) continue;
    const unsigned pg = atomicAdd(&G->page_next, 1u);
    if (pg >= P.pages_per_group) {
      raise_err(P.g, PH_ERR_OVERFLOW, W_ALLOC);
      return false;
    }
    st_rlx64(pt_cell(P, c, L, vp), ((unsigned long long)pg << 32) | (unsigned)vp);
    *cvp = vp;
    *cpi = pg;
    pgs[vp - vp0] = pg;
  }
  if ((vp0 << PH_PAGE_LOG2) < base) { /* first page: mapped by an earlier reservation */
    const unsigned pg = pt_wait(P, c, L, vp0, cvp, cpi);
    if (pg == 0xFFFFFFFFu) return false;
    pgs[0] = pg;
  }
  return true;
}

/* Page of an entry already written in an earlier phase (its mapping is
 * visible after the barrier; a missing one is an engine fault). */
__device__ __forceinline__ unsigned pt_lookup(const PhParams &P, const Ctx &c, unsigned L,
                                              unsigned long long vp) {
  const unsigned long long e = ld_rlx64(pt_cell(P, c, L, vp));
  if ((unsigned)e != (unsigned)vp) {
    raise_err(P.g, PH_ERR_MAPPING, W_MAPPING);
    return 0xFFFFFFFFu;
  }
  return (unsigned)(e >> 32);
}

/* ------------------------------------------------------------------------ */
/* staging and flushing of pushes                                             */

template <int BLOCK, int UU>
__device__ __forceinline__ void stage(PSmem<BLOCK, UU> &S, unsigned v, unsigned d, unsigned L) {
  const unsigned mask = __activemask();
  const unsigned lane = threadIdx.x & 31u;
  const unsigned leader = __ffs(mask) - 1u;
  unsigned pos = 0;
  if (lane == leader) pos = atomicAdd(&S.pcnt, (unsigned)__popc(mask));
  pos = __shfl_sync(mask, pos, leader) + __popc(mask & ((1u << lane) - 1u));
  S.pb_v[pos] = v;
  S.pb_d[pos] = d;
  S.pb_l[pos] = (unsigned char)L;
}

/* Counting sort of the staged pushes by list, one reservation per list, the
 * entry stores.  Nothing else: the phase barrier publishes them.  Replaces the
 * per-warp reservation + st.cg + __threadfence + write_done update of
 * push_work (wl.h:1902-1928).  Call with every thread, after a barrier. */
template <int BLOCK, int UU>
__device__ void flush(const PhParams &P, Ctx &c, PSmem<BLOCK, UU> &S) {
  const unsigned tid = threadIdx.x;
  const unsigned cnt = S.pcnt;
  if (cnt == 0u) return;
  if (tid < PH_NLIST) S.hist[tid] = 0u;
  __syncthreads();
  /* ranks within each list: one shared atomic per distinct list per warp */
  const unsigned lane = tid & 31u;
  for (unsigned i0 = tid - lane; i0 < cnt; i0 += BLOCK) {
    const unsigned i = i0 + lane;
    const bool in = i < cnt;
    const unsigned L = in ? S.pb_l[i] : 0xFFu;
    const unsigned grp = __match_any_sync(0xFFFFFFFFu, L);
    const unsigned first = __ffs(grp) - 1u;
    unsigned b = 0;
    if (in && lane == first) b = atomicAdd(&S.hist[L], (unsigned)__popc(grp));
    b = __shfl_sync(0xFFFFFFFFu, b, first);
    if (in) S.pb_rank[i] = (unsigned short)(b + __popc(grp & ((1u << lane) - 1u)));
  }
  __syncthreads();
  if (tid < PH_NLIST) {
    const unsigned h = S.hist[tid];
    if (h != 0u) {
      /* a dense bucket slot only records that it is non-empty (its bit);
       * the far slot (everything past the ring) never turns dense */
      PhGroup *G = grp_of(P, c);
      const bool far = tid == ((S.D.base + PH_NSLOT - 1u) & (PH_NSLOT - 1u));
      if (P.dense_shift != 0u && far && !((ld_rlx64(&G->fmask) >> tid) & 1ull))
        atomicOr(&G->fmask, 1ull << tid);
      const bool slot = P.dense_shift != 0u && tid < PH_NSLOT && !far &&
                        !((ld_rlx64(&G->fmask) >> tid) & 1ull);
      if (slot && ((ld_rlx64(&G->dmask) >> tid) & 1ull)) {
        S.bbase[tid] = 0ull;
        for (unsigned j = 0; j < PH_RES_PAGES; ++j) S.bpg[tid][j] = 0xFFFFFFFFu; /* no stores */
      } else {
        unsigned long long b;
        unsigned pg[PH_RES_PAGES];
        list_reserve(P, c, tid, h, &b, pg, &S.ptc_vp[tid], &S.ptc_pi[tid]);
        S.bbase[tid] = b;
        for (unsigned j = 0; j < PH_RES_PAGES; ++j) S.bpg[tid][j] = pg[j];
        if (slot) {
          const unsigned n = P.qs[S.D.q].n;
          const unsigned long long thr = max(4096u, n >> P.dense_shift);
          if (b + h - ld_rlx64(&G->head[tid]) > thr) atomicOr(&G->dmask, 1ull << tid);
        }
      }
    }
  }
  __syncthreads();
  for (unsigned i = tid; i < cnt; i += BLOCK) {
    const unsigned L = S.pb_l[i];
    const unsigned long long b = S.bbase[L];
    const unsigned long long idx = b + S.pb_rank[i];
    const unsigned pg = S.bpg[L][(idx >> PH_PAGE_LOG2) - (b >> PH_PAGE_LOG2)];
    if (pg != 0xFFFFFFFFu)
      st_rlx64(entry_ptr(P, c, pg, idx), ((unsigned long long)S.pb_d[i] << 32) | S.pb_v[i]);
  }
  if (tid == 0u) S.st_pushes += cnt;
  __syncthreads();
  if (tid == 0u) S.pcnt = 0u;
  __syncthreads();
}

/* block-wide exclusive scan of one value per thread */
template <int BLOCK, int UU>
__device__ __forceinline__ unsigned block_exscan(PSmem<BLOCK, UU> &S, unsigned x, unsigned &total) {
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
    const unsigned w = lane < BLOCK / 32 ? S.wsum[lane] : 0u;
    unsigned wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= (unsigned)o) wi += y;
    }
    if (lane < BLOCK / 32) S.wsum[lane] = wi - w;
    if (lane == 31u) S.total = wi;
  }
  __syncthreads();
  total = S.total;
  return S.wsum[warp] + incl - x;
}

/* ------------------------------------------------------------------------ */
/* Chunks.  A chunk is up to BLOCK frontier entries (or a few split-row
 * records); each becomes an item, a row segment [rb, re) of the CSR to
 * expand with distance du.  The CTA scans the segment lengths, then every
 * thread walks its share of the chunk's edges with no barrier until the
 * chunk is done.                                                             */

/* Items from one entry (v, d) of a light or heavy phase: the stale check,
 * the far-slot re-push, the light / heavy row segment, the settled push and
 * the split of long rows into records.  Returns the segment in rb/re (empty
 * when nothing is to be expanded) and counts what it did. */
template <bool FLT, int BLOCK, int UU>
__device__ __forceinline__ void entry_item(const PhParams &P, Ctx &c, PSmem<BLOCK, UU> &S,
                                           const PhQuery &Q, unsigned v, unsigned d, unsigned dv,
                                           unsigned &rb, unsigned &re, unsigned &du,
                                           unsigned &nstale, unsigned &nrepush, unsigned &nheavy) {
  PhGroup *G = grp_of(P, c);
  const unsigned mode = S.D.mode, d_base = S.D.base;
  rb = re = du = 0u;
  if (dv != d) {
    ++nstale; /* superseded: a later push carries the smaller value */
    return;
  }
  const unsigned b = bucket_of<FLT>(d, Q.scale, Q.shift);
  if (b > d_base) { /* left in the far slot: move it to its own bucket */
    stage<BLOCK, UU>(S, v, d, route(b, d_base, P.near_far));
    if (P.near_far) {
      /* near-far: the smallest bucket the split sends back to the pile is
       * where the leader may move the threshold next */
      const unsigned am = __activemask();
      const unsigned wm = __reduce_min_sync(am, b);
      if ((threadIdx.x & 31u) == (unsigned)(__ffs(am) - 1)) atomicMin(&G->far_min, wm);
    }
    ++nrepush;
    return;
  }
  const unsigned r0 = __ldg(Q.row + v), r1 = __ldg(Q.row + v + 1);
  const unsigned nl = (Q.split && !S.D.full) ? __ldg(Q.split + v) : (r1 - r0);
  if (mode == PH_M_LIGHT) {
    rb = r0;
    re = r0 + nl;
    if (nl < r1 - r0) stage<BLOCK, UU>(S, v, d, PH_LSETTLED);
  } else {
    rb = r0 + nl;
    re = r1;
    ++nheavy;
  }
  if (re - rb > P.hub_threshold) { /* cut into chunks for the whole group */
    const unsigned deg = re - rb;
    const unsigned nch = (deg + P.hub_chunk - 1u) / P.hub_chunk;
    const unsigned hb = atomicAdd(&G->hub_count, nch);
    S.hub_made = 1u;
    if (hb + nch > P.hub_cap) {
      raise_err(P.g, PH_ERR_HUB_OVERFLOW, W_HUB);
    } else {
      PhHub *hp = hub_of(P, c) + hb;
      unsigned *sq = hub_seq_of(P, c) + hb;
      for (unsigned x = 0; x < nch; ++x)
        __stcg(reinterpret_cast<uint4 *>(hp + x),
               make_uint4(v, d, rb + x * P.hub_chunk, rb + min(deg, (x + 1u) * P.hub_chunk)));
      __threadfence(); /* the records before their sequence words */
      const unsigned ep = S.D.epoch;
      for (unsigned x = 0; x < nch; ++x) st_rlx32(sq + x, ep);
    }
    re = rb;
  }
  du = d;
}

/* Finishes a chunk whose items' lengths are in it_off: statistics, the
 * exclusive scan of the lengths, the chunk totals. */
template <int BLOCK, int UU>
__device__ __forceinline__ void finish_items(PSmem<BLOCK, UU> &S, unsigned k, unsigned nstale,
                                             unsigned nrepush, unsigned nheavy) {
  constexpr int EPT = PSmem<BLOCK, UU>::EPT;
  const unsigned tid = threadIdx.x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nstale += __shfl_down_sync(0xFFFFFFFFu, nstale, o);
    nrepush += __shfl_down_sync(0xFFFFFFFFu, nrepush, o);
    nheavy += __shfl_down_sync(0xFFFFFFFFu, nheavy, o);
  }
  if ((tid & 31u) == 0u) {
    if (nstale) atomicAdd(&S.st_stale, (unsigned long long)nstale);
    if (nrepush) atomicAdd(&S.st_repush, (unsigned long long)nrepush);
    if (nheavy) atomicAdd(&S.st_heavy, (unsigned long long)nheavy);
  }
  __syncthreads();
  /* offsets in item order: thread t owns items [t*EPT, t*EPT + EPT) */
  unsigned lens[EPT], mine = 0;
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    lens[j] = S.it_off[tid * EPT + j];
    mine += lens[j];
  }
  unsigned tot;
  unsigned off = block_exscan<BLOCK, UU>(S, mine, tot);
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    S.it_off[tid * EPT + j] = off;
    off += lens[j];
  }
  if (tid == 0) {
    S.it_off[EPT * BLOCK] = tot;
    S.ck_k = k;
    S.ck_E = tot;
  }
  __syncthreads();
}

/* Claims and prepares the next chunk.  Returns false when the phase has no
 * more chunks.  Every thread calls it; thread 0 keeps the claim state in
 * shared memory (S.local_claim, S.pend), out of every thread's registers. */
template <bool FLT, int BLOCK, int UU>
__device__ bool prepare_chunk(const PhParams &P, Ctx &c, PSmem<BLOCK, UU> &S, bool solo) {
  const unsigned tid = threadIdx.x;
  const unsigned mode = S.D.mode;
  PhGroup *G = grp_of(P, c);
  const PhQuery &Q = P.qs[S.D.q];
  const unsigned long long d_lo = S.D.lo, d_hi = S.D.hi, d_wb = S.D.work_base;
  const unsigned d_base = S.D.base, d_list = S.D.list;
  constexpr unsigned IC = PSmem<BLOCK, UU>::IC;
  const unsigned nx = mode == PH_M_LIGHT ? S.D.nx : 0u; /* ranges past the first */
  unsigned long long count = d_hi - d_lo;
  for (unsigned r = 0; r < nx; ++r) count += S.D.xhi[r] - S.D.xlo[r];
  __syncthreads(); /* everyone has read the previous claim's S.stop */
  if (tid == 0) {
    /* guided self-scheduling: a claim takes about half this CTA's share of
     * what is left (at least 32 entries, at most IC), so a phase starts with
     * large chunks and ends with small ones */
    auto want = [&](unsigned long long seen) {
      const unsigned long long left = count > seen ? count - seen : 0ull;
      const unsigned long long w = (left / (2ull * P.gsize) + 31ull) & ~31ull;
      return (unsigned)min((unsigned long long)IC, max(32ull, w));
    };
    unsigned long long at;
    unsigned n;
    if (solo) {
      at = S.local_claim;
      n = IC;
      S.local_claim = at + IC;
    } else {
      /* the next claim is taken one chunk ahead, so its latency overlaps this
       * chunk's work; claims past the end are simply not used.  pend packs
       * the claim's start (entries since work_base, 40 bits) and size. */
      unsigned long long pend = S.pend;
      if (pend == ~0ull) {
        const unsigned w = want(0ull);
        pend = ((atomicAdd(&G->work, (unsigned long long)w) - d_wb) << 24) | w;
      }
      at = pend >> 24;
      n = (unsigned)(pend & 0xFFFFFFull);
      const unsigned w = want(at + n);
      S.pend = ((atomicAdd(&G->work, (unsigned long long)w) - d_wb) << 24) | w;
    }
    S.claim = at;
    S.stop = at >= count ? 1u : 0u;
    if (!S.stop && nx != 0u) { /* a widened bucket: each thread maps its entry */
      S.ck_k = (unsigned)min((unsigned long long)n, count - at);
      ++S.st_chunks;
      S.st_items += S.ck_k;
    } else if (!S.stop) {
      const unsigned long long s0 = d_lo + at;
      const unsigned long long s1 = min(s0 + n, d_hi) - 1ull;
      S.ck_k = (unsigned)(s1 + 1ull - s0);
      const unsigned long long v0 = s0 >> PH_PAGE_LOG2, v1 = s1 >> PH_PAGE_LOG2;
      S.pi0 = S.ptc_vp[d_list] == v0 ? S.ptc_pi[d_list] : pt_lookup(P, c, d_list, v0);
      S.pi1 = v1 == v0 ? S.pi0 : pt_lookup(P, c, d_list, v1);
      S.ptc_vp[d_list] = v1;
      S.ptc_pi[d_list] = S.pi1;
      ++S.st_chunks;
      S.st_items += s1 + 1ull - s0;
    }
  }
  __syncthreads();
  if (S.stop) return false;
  const unsigned long long s0 = d_lo + S.claim;
  const unsigned k = S.ck_k;
  constexpr int EPT = PSmem<BLOCK, UU>::EPT;
  /* item i = j*BLOCK + tid: neighbouring threads read neighbouring entries;
   * the loads of all EPT entries are issued before their dependants */
  unsigned ev[EPT], ed[EPT], dv[EPT];
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    const unsigned i = j * BLOCK + tid;
    ev[j] = 0xFFFFFFFFu;
    ed[j] = 0u;
    if (i < k && nx != 0u) { /* find the entry's range, then its page */
      unsigned long long pos = S.claim + i, span = d_hi - d_lo, idx = d_lo + pos;
      unsigned L = d_list;
      for (unsigned r = 0; r < nx && pos >= span; ++r) {
        pos -= span;
        L = S.D.xl[r];
        idx = S.D.xlo[r] + pos;
        span = S.D.xhi[r] - S.D.xlo[r];
      }
      const unsigned pg = pt_lookup(P, c, L, idx >> PH_PAGE_LOG2);
      if (pg != 0xFFFFFFFFu) {
        const unsigned long long e = __ldcg(entry_ptr(P, c, pg, idx));
        ev[j] = (unsigned)e;
        ed[j] = (unsigned)(e >> 32);
      }
    } else if (i < k) {
      const unsigned long long idx = s0 + i;
      const unsigned pg = ((idx >> PH_PAGE_LOG2) == (s0 >> PH_PAGE_LOG2)) ? S.pi0 : S.pi1;
      if (pg != 0xFFFFFFFFu) {
        const unsigned long long e = __ldcg(entry_ptr(P, c, pg, idx));
        ev[j] = (unsigned)e;
        ed[j] = (unsigned)(e >> 32);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < EPT; ++j) dv[j] = ev[j] != 0xFFFFFFFFu ? __ldcg(Q.dist + ev[j]) : 0u;
  unsigned nstale = 0, nrepush = 0, nheavy = 0;
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    const unsigned i = j * BLOCK + tid;
    unsigned rb = 0, re = 0, du = 0;
    if (ev[j] != 0xFFFFFFFFu)
      entry_item<FLT, BLOCK, UU>(P, c, S, Q, ev[j], ed[j], dv[j], rb, re, du, nstale, nrepush,
                                 nheavy);
    S.it_rb[i] = rb;
    S.it_du[i] = du;
    S.it_off[i] = re - rb; /* the length, turned into an offset below */
  }
  finish_items<BLOCK, UU>(S, k, nstale, nrepush, nheavy);
  return true;
}

/* Claims the next split-row records of this phase and prepares them as the
 * chunk.  Records are appended by CTAs that are still expanding frontier
 * chunks (the producers); a claim beyond the records appended so far waits
 * (bounded) until they are there or every producer has finished.  Returns
 * false when no record is left.  Every thread calls it. */
template <bool FLT, int BLOCK, int UU>
__device__ bool prepare_records(const PhParams &P, Ctx &c, PSmem<BLOCK, UU> &S) {
  constexpr unsigned K = PH_HUB_PER_CLAIM(BLOCK);
  const unsigned tid = threadIdx.x;
  PhGroup *G = grp_of(P, c);
  const PhQuery &Q = P.qs[S.D.q];
  const unsigned epoch = S.D.epoch;
  __syncthreads(); /* everyone has read the previous claim's S.stop */
  if (tid == 0) {
    const unsigned r = atomicAdd(&G->hub_claim, K);
    unsigned n = 0;
    Waiter w{c.deadline, 0};
    for (;;) {
      const unsigned hc = ld_acq32(&G->hub_count);
      if (hc >= r + K) {
        n = K;
        break;
      }
      if (ld_acq32(&G->producers) == 0u) { /* no record can still appear */
        const unsigned hf = min(ld_acq32(&G->hub_count), P.hub_cap);
        n = hf > r ? min(K, hf - r) : 0u;
        break;
      }
      if (!w.spin(P.g, W_HUB, 128)) break;
    }
    n = r < P.hub_cap ? min(n, P.hub_cap - r) : 0u; /* past the store: overflow */
    S.claim = r;
    S.pi0 = n;
    S.stop = n == 0u ? 1u : 0u;
  }
  __syncthreads();
  if (S.stop) return false;
  const unsigned r = (unsigned)S.claim, k = S.pi0;
  unsigned rb = 0, re = 0, du = 0;
  bool stale = false;
  if (tid < k) {
    /* the record's reservation was counted before it was written */
    const unsigned *sq = hub_seq_of(P, c) + r + tid;
    Waiter w{c.deadline, 0};
    bool ok = true;
    while (ld_acq32(sq) != epoch) {
      if (!w.spin(P.g, W_HUB, 64)) {
        ok = false;
        break;
      }
    }
    if (ok) {
      const uint4 h = __ldcg(reinterpret_cast<const uint4 *>(hub_of(P, c) + r + tid));
      /* h = {v, d, eb, ee}.  The row's vertex improved since the chunk was
       * cut: a later expansion covers these edges with the smaller value */
      if (__ldcg(Q.dist + h.x) == h.y) {
        rb = h.z;
        re = h.w;
        du = h.y;
      } else {
        stale = true;
      }
    }
  }
  S.it_rb[tid] = rb;
  S.it_du[tid] = du;
  const unsigned nstale = __syncthreads_count(stale);
  if (tid == 0) {
    S.st_stale += nstale;
    S.st_hubs += k - nstale;
  }
  unsigned tot;
  const unsigned off = block_exscan<BLOCK, UU>(S, re - rb, tot);
  S.it_off[tid] = off;
  if (tid == 0) {
    S.it_off[BLOCK] = tot;
    S.ck_k = k;
    S.ck_E = tot;
  }
  __syncthreads();
  return true;
}

/* Relaxes the chunk's edges.  In iteration i warp w takes the 32*U edges
 * i*BLOCK*U + w*32*U + [0, 32*U), lane l every 32nd of them, so each load
 * instruction of a warp reads 32 neighbouring edges and a lane's successive
 * edges are 32 apart: its item is found by a short forward (galloping)
 * search from the previous one.  The loads of iteration i+1 are issued
 * before the distance gathers of iteration i.  Every SEGI iterations the CTA
 * meets once to flush staged pushes (the staging buffer is sized so that this
 * is the only barrier needed).  (The pull direction has a loop of its own,
 * pull_tile_warp, in a kernel of its own: a run-time switch inside this loop
 * cost it 37 % of its speed on R-MAT 24.) */
template <bool FLT, int BLOCK, int UU>
__device__ void expand(const PhParams &P, Ctx &c, PSmem<BLOCK, UU> &S, const PhQuery &Q,
                       unsigned base) {
  constexpr int U = PSmem<BLOCK, UU>::U;
  constexpr unsigned R = BLOCK * U;
  const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const unsigned k = S.ck_k, E = S.ck_E;
  const unsigned nit = (E + R - 1u) / R; /* the same for every thread */
  const uint2 *__restrict__ edges = Q.edges;
  unsigned *dist = Q.dist;
  const float scale = Q.scale;
  const unsigned shift = Q.shift;
  const unsigned *off = S.it_off; /* off[k] = E */
  unsigned lo = 0; /* item of the thread's last edge: its edges only move forward */
  uint2 ne[U];
  unsigned nu[U];
  auto find = [&](unsigned e) {
    /* gallop: the last item whose offset is <= e, at or after lo */
    unsigned step = 1u;
    while (lo + step < k && off[lo + step] <= e) {
      lo += step;
      step <<= 1;
    }
    unsigned hi = min(lo + step, k) - 1u; /* off[hi + 1] > e or hi = k - 1 */
    while (lo < hi) {
      const unsigned mid = (lo + hi + 1u) >> 1;
      if (off[mid] <= e) lo = mid; else hi = mid - 1u;
    }
  };
  auto load_round = [&](unsigned eb) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned e = eb + u * 32u;
      nu[u] = 0xFFFFFFFFu;
      ne[u] = make_uint2(0u, 0u);
      if (e < E) {
        find(e);
        ne[u] = ld_edge(edges + S.it_rb[lo] + (e - off[lo]));
        nu[u] = S.it_du[lo];
      }
    }
  };
  const unsigned mine = warp * 32u * U + lane; /* offset of the thread's first edge */
  if (nit) load_round(mine);
  unsigned nedges = 0;
  for (unsigned it = 0; it < nit; ++it) {
    unsigned dst[U], nd[U], cur[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      dst[u] = ne[u].x;
      nd[u] = 0xFFFFFFFFu;
      if (nu[u] != 0xFFFFFFFFu) {
        nd[u] = FLT ? __float_as_uint(__fadd_rn(__uint_as_float(nu[u]), __uint_as_float(ne[u].y)))
                    : nu[u] + ne[u].y;
        ++nedges;
      }
    }
    if (it + 1u < nit) load_round((it + 1u) * R + mine);
#pragma unroll
    for (int u = 0; u < U; ++u) cur[u] = (nd[u] != 0xFFFFFFFFu) ? __ldcg(dist + dst[u]) : 0u;
    /* an improvement on the gathered value is applied with a reduction (no
     * return value, so no wait) and pushed at once; if a concurrent smaller
     * value wins, the pushed entry is dropped as stale when it is popped.
     * The reference's int kernel likewise pushes whether or not its atomicMin
     * won (ads_int/kernel.cu:78-82). */
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (nd[u] < cur[u]) {
        red_min(dist + dst[u], nd[u]);
        stage<BLOCK, UU>(S, dst[u], nd[u],
                         route(bucket_of<FLT>(nd[u], scale, shift), base, P.near_far));
      }
    }
    if ((it % PSmem<BLOCK, UU>::SEGI) == PSmem<BLOCK, UU>::SEGI - 1u || it + 1u == nit) {
      __syncthreads();
      if (S.pcnt > (unsigned)PSmem<BLOCK, UU>::FLUSH_AT) {
        const long long f0 = clock64();
        flush<BLOCK, UU>(P, c, S);
        if (tid == 0) S.cy[3] += (unsigned long long)(clock64() - f0); /* also in expand's */
      }
    }
  }
  c.edges += nedges;
}

/* ------------------------------------------------------------------------ */
/* A heavy phase run as a pull (PH_M_PULL; the leader picks it when the heavy
 * scan counted fewer in-edges into the vertices above pull_floor than heavy
 * edges out of the settled bucket).  Every vertex above pull_floor -- the
 * only ones the bucket's heavy edges can improve -- takes the minimum of
 * fl(d[u] + w) over all its in-edges; one that improves is pushed once, with
 * that value.  The distances equal the push phase's: every candidate is the
 * length of a path, and each heavy edge out of the bucket into such a vertex
 * is one of its in-edges.  Only the thread that owns a vertex writes it in
 * this phase.  The direction choice follows Beamer et al. (SC 2012), applied
 * to delta-stepping's heavy phase as in Chakaravarthy et al. (IPDPS 2014).
 *
 * CTAs claim runs of tiles of PH_PULL_SUB x PH_PULL_V x BLOCK vertices (guided
 * self-scheduling, the next run claimed one run ahead; thread 0 keeps the
 * runs in shared memory) and run each sub-tile through pull_tile_warp.
 * Claims the next tile into S.pl_cur; false when none is left.  Every
 * thread calls it. */
template <bool FLT, int BLOCK, int UU>
__device__ bool prepare_pull(const PhParams &P, Ctx &c, PSmem<BLOCK, UU> &S, const PhQuery &Q) {
  const unsigned tid = threadIdx.x;
  const unsigned long long tv = (unsigned long long)PH_PULL_SUB * PH_PULL_V * BLOCK;
  const unsigned ntile = (unsigned)(((unsigned long long)Q.n + tv - 1ull) / tv);
  __syncthreads(); /* everyone has read the previous tile's S.pl_cur and S.stop */
  if (tid == 0) {
    if (S.pl_k == 0u) { /* the run claimed ahead becomes current; claim the next */
      PhGroup *G = grp_of(P, c);
      const unsigned long long wb = S.D.work_base;
      /* about a quarter of this CTA's share of what is left, 1 to 8 tiles;
       * packed (start << 24) | count */
      auto take = [&](unsigned long long seen) {
        const unsigned long long left = ntile > seen ? ntile - seen : 0ull;
        const unsigned long long w = min(8ull, max(1ull, left / (4ull * P.gsize)));
        return ((atomicAdd(&G->work, w) - wb) << 24) | w;
      };
      unsigned long long pend = S.pend;
      if (pend == ~0ull) pend = take(0ull);
      S.pl_t0 = (unsigned)min(pend >> 24, (unsigned long long)ntile);
      S.pl_k = (unsigned)(pend & 0xFFFFFFull);
      S.pend = take((pend >> 24) + (pend & 0xFFFFFFull));
    }
    S.pl_cur = S.pl_t0;
    S.stop = S.pl_t0 >= ntile ? 1u : 0u;
    ++S.pl_t0;
    --S.pl_k;
  }
  __syncthreads();
  return S.stop == 0u;
}

/* lane-wise inclusive scan over a warp */
__device__ __forceinline__ unsigned warp_incl_scan(unsigned x) {
  const unsigned lane = threadIdx.x & 31u;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= (unsigned)o) x += y;
  }
  return x;
}

/* Sub-tile `sub` of a claimed pull tile (PH_PULL_SUB sub-tiles of PH_PULL_V
 * x BLOCK consecutive vertices, run before one block barrier), each warp on
 * its own 32 x PH_PULL_V of them with no block barrier (the block-wide
 * version spent 40 % of its issue slots waiting at barriers).  A lane
 * selects its vertices above pull_floor that have in-edges; the warp
 * compacts them into its 32-item slice of the chunk arrays, 32 at a time,
 * spreads the slice's in-edges over its lanes (U per lane per round, the
 * next round's edge loads issued before this round's gathers) and lowers
 * each item's best candidate with a shared-memory atomic minimum; a vertex
 * whose best is below its distance stores it (only this lane writes the
 * vertex in the phase) and is staged for its bucket (a tile stages at most
 * one push per vertex, which the staging buffer holds past FLUSH_AT).  Every
 * thread calls it; the caller meets the block at a barrier before the flush
 * check. */
template <bool FLT, int BLOCK, int UU>
__device__ void pull_tile_warp(const PhParams &P, Ctx &c, PSmem<BLOCK, UU> &S,
                               const PhQuery &Q, unsigned sub) {
  constexpr unsigned V = PH_PULL_V, U = PSmem<BLOCK, UU>::U, R = 32u * U;
  constexpr unsigned SB = PSmem<BLOCK, UU>::SB, FLUSH_AT = PSmem<BLOCK, UU>::FLUSH_AT;
  static_assert(PSmem<BLOCK, UU>::IC == BLOCK, "one 32-item slice per warp");
  static_assert(FLUSH_AT + PH_PULL_SUB * V * BLOCK <= SB, "a tile's pushes fit the staging buffer");
  const unsigned tid = threadIdx.x, lane = tid & 31u, sl = tid & ~31u;
  unsigned *const w_rb = S.it_rb + sl, *const w_best = S.it_du + sl, *const w_d0 = S.it_d0 + sl;
  unsigned *const w_v = S.it_v + sl, *const w_off = S.it_off + sl;
  const uint2 *__restrict__ edges = Q.tedges;
  unsigned *const dist = Q.dist;
  const unsigned n = Q.n, T = S.pl_T;
  const unsigned long long v0 =
      (((unsigned long long)S.pl_cur * PH_PULL_SUB + sub) * BLOCK + tid) * V;
  unsigned d[V], rb[V], re[V];
  const bool vec = ((reinterpret_cast<unsigned long long>(Q.dist) |
                     reinterpret_cast<unsigned long long>(Q.trow)) & 15ull) == 0ull;
  if (vec && v0 + V <= n) {
    const uint4 x = __ldcg(reinterpret_cast<const uint4 *>(Q.dist + v0));
    const uint4 r = __ldg(reinterpret_cast<const uint4 *>(Q.trow + v0));
    d[0] = x.x; d[1] = x.y; d[2] = x.z; d[3] = x.w;
    rb[0] = r.x; rb[1] = r.y; rb[2] = r.z; rb[3] = r.w;
    re[0] = r.y; re[1] = r.z; re[2] = r.w; re[3] = __ldg(Q.trow + v0 + 4);
  } else {
#pragma unroll
    for (unsigned j = 0; j < V; ++j) {
      const bool in = v0 + j < n;
      d[j] = in ? __ldcg(Q.dist + v0 + j) : 0u;
      rb[j] = in ? __ldg(Q.trow + v0 + j) : 0u;
      re[j] = in ? __ldg(Q.trow + v0 + j + 1) : 0u;
    }
  }
  unsigned selm = 0;
#pragma unroll
  for (unsigned j = 0; j < V; ++j)
    if (v0 + j < n && d[j] > T && re[j] > rb[j]) selm |= 1u << j;
  const unsigned cnt = __popc(selm), incl = warp_incl_scan(cnt);
  const unsigned total = __shfl_sync(0xFFFFFFFFu, incl, 31), pos0 = incl - cnt;
  if (lane == 0 && total != 0u) atomicAdd(&S.st_items, (unsigned long long)total);
  unsigned nedges = 0;
  for (unsigned r0 = 0; r0 < total; r0 += 32u) {
    __syncwarp(); /* the last batch's items are read */
    unsigned p = pos0;
#pragma unroll
    for (unsigned j = 0; j < V; ++j) {
      if ((selm >> j) & 1u) {
        if (p - r0 < 32u) { /* p in [r0, r0 + 32) */
          const unsigned i = p - r0;
          w_rb[i] = rb[j];
          w_best[i] = d[j]; /* the item's best candidate so far */
          w_d0[i] = d[j];
          w_v[i] = (unsigned)(v0 + j);
          w_off[i] = re[j] - rb[j]; /* the length, turned into an offset below */
        }
        ++p;
      }
    }
    __syncwarp();
    const unsigned k = min(32u, total - r0);
    const unsigned len = lane < k ? w_off[lane] : 0u;
    const unsigned li = warp_incl_scan(len);
    const unsigned E = __shfl_sync(0xFFFFFFFFu, li, 31);
    w_off[lane] = li - len; /* each lane rewrites the slot it read */
    __syncwarp();
    unsigned lo = 0; /* item of the lane's last edge: its edges only move forward */
    uint2 ne[U];
    unsigned nu[U];
    auto find = [&](unsigned e) {
      /* gallop: the last item whose offset is <= e, at or after lo */
      unsigned step = 1u;
      while (lo + step < k && w_off[lo + step] <= e) {
        lo += step;
        step <<= 1;
      }
      unsigned hi = min(lo + step, k) - 1u;
      while (lo < hi) {
        const unsigned mid = (lo + hi + 1u) >> 1;
        if (w_off[mid] <= e) lo = mid; else hi = mid - 1u;
      }
    };
    auto load_round = [&](unsigned eb) {
#pragma unroll
      for (unsigned u = 0; u < U; ++u) {
        const unsigned e = eb + u * 32u + lane;
        nu[u] = 0xFFFFFFFFu;
        ne[u] = make_uint2(0u, 0u);
        if (e < E) {
          find(e);
          ne[u] = ld_edge(edges + w_rb[lo] + (e - w_off[lo]));
          nu[u] = lo;
        }
      }
    };
    const unsigned nit = (E + R - 1u) / R;
    if (nit) load_round(0u);
    for (unsigned it = 0; it < nit; ++it) {
      unsigned src[U], cur[U], wv[U], iv[U], live = 0;
#pragma unroll
      for (unsigned u = 0; u < U; ++u) {
        src[u] = ne[u].x;
        wv[u] = ne[u].y;
        iv[u] = nu[u];
        if (nu[u] != 0xFFFFFFFFu) {
          live |= 1u << u;
          ++nedges;
        }
      }
      if (it + 1u < nit) load_round((it + 1u) * R);
#pragma unroll
      for (unsigned u = 0; u < U; ++u) cur[u] = ((live >> u) & 1u) ? __ldcg(dist + src[u]) : 0u;
#pragma unroll
      for (unsigned u = 0; u < U; ++u) {
        if ((live >> u) & 1u) {
          /* an unreached tail gives INF + w, above every distance */
          const unsigned w = wv[u], i = iv[u];
          const unsigned cand =
              FLT ? __float_as_uint(__fadd_rn(__uint_as_float(cur[u]), __uint_as_float(w)))
                  : cur[u] + w;
          if (cand < w_best[i]) atomicMin(&w_best[i], cand);
        }
      }
    }
    __syncwarp();
    if (lane < k) {
      const unsigned best = w_best[lane];
      if (best < w_d0[lane]) {
        const unsigned v = w_v[lane];
        st_rlx32(dist + v, best);
        stage<BLOCK, UU>(S, v, best, route(bucket_of<FLT>(best, Q.scale, Q.shift), S.D.base,
                                           P.near_far));
      }
    }
  }
  c.edges += nedges;
}


/* ------------------------------------------------------------------------ */
/* One phase (or, solo, the whole of it on this CTA).  PK: the kernel may
 * pick pull phases (sampling scans compiled in). */
template <bool FLT, int BLOCK, int UU, bool PK>
__device__ void run_phase(const PhParams &P, Ctx &c, PSmem<BLOCK, UU> &S, bool solo) {
  constexpr unsigned FLUSH_AT = PSmem<BLOCK, UU>::FLUSH_AT;
  const unsigned tid = threadIdx.x;
  const unsigned mode = S.D.mode;
  /* a pull phase runs in its own kernel (pull_kernel) between two launches */
  if (mode == PH_M_START || mode == PH_M_EXIT || mode == PH_M_PULL) return;
  const PhQuery &Q = P.qs[S.D.q];
  if (mode == PH_M_INIT) {
    const unsigned rank = solo ? 0u : c.rank;
    const unsigned gsize = solo ? 1u : P.gsize;
    const unsigned inf = P.is_float ? 0x7F7FFFFFu : 0x7FFFFFFFu;
    if ((reinterpret_cast<unsigned long long>(Q.dist) & 15ull) == 0ull) {
      uint4 *d4 = reinterpret_cast<uint4 *>(Q.dist);
      const unsigned n4 = Q.n >> 2;
      const uint4 x = make_uint4(inf, inf, inf, inf);
      for (unsigned i = rank * BLOCK + tid; i < n4; i += gsize * BLOCK) __stcg(d4 + i, x);
      if (rank == 0u && tid < (Q.n & 3u)) __stcg(Q.dist + (n4 << 2) + tid, inf);
    } else {
      for (unsigned i = rank * BLOCK + tid; i < Q.n; i += gsize * BLOCK) __stcg(Q.dist + i, inf);
    }
    return;
  }
  if (mode == PH_M_SCAN) {
    /* A scan over the distances.  Light scan (list = the bucket's slot):
     * every vertex whose distance lies in the bucket goes to NEXT, once,
     * with its current distance.  Heavy scan (list = SETTLED): every vertex
     * of the settled bucket that has heavy edges goes to SETTLED, in vertex
     * order, so the heavy phase reads their rows in address order and pops
     * no duplicates.  Nothing relaxes in this phase, so the distances do not
     * move.  A CTA takes tiles of 4 x BLOCK vertices round-robin, SCANG of
     * them per round with all their 16-byte loads issued first; each tile's
     * matches are staged (at most 4 x BLOCK) before the flush check, which
     * the staging buffer's size allows.  A sampling heavy scan (D.sample)
     * stages nothing: over one tile in PH_SAMPLE_STRIDE it sums, for the
     * leader's push-or-pull choice, the heavy out-edges of the bucket and
     * the in-edges of the vertices above pull_floor. */
    constexpr unsigned SCANG = 4;
    const bool heavy = S.D.list == PH_LSETTLED;
    const bool sample = PK && heavy && S.D.sample != 0u;
    const bool count = sample && Q.trow != nullptr;
    const unsigned tstep = sample ? PH_SAMPLE_STRIDE : 1u;
    const unsigned pfl = count ? pull_floor<FLT>(Q, S.D.base) : 0xFFFFFFFFu;
    unsigned long long c_push = 0, c_pull = 0;
    const unsigned target = heavy ? PH_LSETTLED : PH_LNEXT;
    const unsigned base = S.D.base, n = Q.n;
    const unsigned inf = P.is_float ? 0x7F7FFFFFu : 0x7FFFFFFFu;
    const bool vec = (reinterpret_cast<unsigned long long>(Q.dist) & 15ull) == 0ull;
    /* tiles read (every tstep-th tile of 4 x BLOCK vertices) */
    const unsigned ntile = ((n + 4u * BLOCK - 1u) / (4u * BLOCK) + tstep - 1u) / tstep;
    const unsigned r0 = solo ? 0u : c.rank, stride = solo ? 1u : P.gsize;
    for (unsigned t0 = r0; t0 < ntile; t0 += SCANG * stride) {
      unsigned d[SCANG][4];
#pragma unroll
      for (unsigned g = 0; g < SCANG; ++g) {
        const unsigned t = t0 + g * stride;
        const unsigned v0 = t * tstep * 4u * BLOCK + 4u * tid;
        if (t < ntile && vec && v0 + 3u < n) {
          const uint4 x = __ldcg(reinterpret_cast<const uint4 *>(Q.dist + v0));
          d[g][0] = x.x;
          d[g][1] = x.y;
          d[g][2] = x.z;
          d[g][3] = x.w;
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            d[g][j] = (t < ntile && v0 + j < n) ? __ldcg(Q.dist + v0 + j) : inf;
        }
      }
#pragma unroll
      for (unsigned g = 0; g < SCANG; ++g) {
        const unsigned v0 = (t0 + g * stride) * tstep * 4u * BLOCK + 4u * tid;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          bool take = d[g][j] != inf && bucket_of<FLT>(d[g][j], Q.scale, Q.shift) == base;
          if (take && heavy) {
            const unsigned v = v0 + j;
            const unsigned nl = __ldg(Q.split + v), deg = __ldg(Q.row + v + 1) - __ldg(Q.row + v);
            take = nl < deg;
            c_push += deg - nl;
          }
          if (take && !sample) stage<BLOCK, UU>(S, v0 + j, d[g][j], target);
          if (count && d[g][j] > pfl && v0 + j < n)
            c_pull += __ldg(Q.trow + v0 + j + 1) - __ldg(Q.trow + v0 + j);
        }
        __syncthreads();
        if (S.pcnt > FLUSH_AT) flush<BLOCK, UU>(P, c, S);
      }
    }
    flush<BLOCK, UU>(P, c, S);
    if (count) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        c_push += __shfl_down_sync(0xFFFFFFFFu, c_push, o);
        c_pull += __shfl_down_sync(0xFFFFFFFFu, c_pull, o);
      }
      if ((tid & 31u) == 0u) {
        PhGroup *G = grp_of(P, c);
        if (c_push) atomicAdd(&G->pc_push, c_push);
        if (c_pull) atomicAdd(&G->pc_pull, c_pull);
      }
    }
    return;
  }
  const unsigned base = S.D.base;
  /* frontier chunks first, then split-row records (a records-only phase
   * finishes what a solo phase left) */
  bool records = mode == PH_M_HUB;
  if (tid == 0) {
    S.hub_made = 0u; /* read after the claim barriers below */
    S.local_claim = 0ull;
    S.pend = ~0ull;
    S.tph = clock64();
  }
  for (;;) {
    const bool have = records ? prepare_records<FLT, BLOCK, UU>(P, c, S)
                              : prepare_chunk<FLT, BLOCK, UU>(P, c, S, solo);
    cy_mark<BLOCK, UU>(S, records ? 1 : 0);
    if (!have) {
      if (records) break;

      /* no frontier chunk left for this CTA: it appends no more split rows,
       * and helps expand the ones the group has appended */
      records = true;
      /* alone and without records: nothing is left for this phase */
      if (solo && S.hub_made == 0u) break;
      if (tid == 0) {
        __threadfence();
        PhGroup *G = grp_of(P, c);
        atomicSub(&G->producers, 1u);
        /* alone, with many records: leave them to the whole group */
        S.stop = solo && ld_rlx32(&G->hub_count) - ld_rlx32(&G->hub_claim) >
                             2u * PH_HUB_PER_CLAIM(BLOCK);
      }
      __syncthreads();
      if (S.stop) break;
      continue;
    }
    if (S.ck_E != 0u) expand<FLT, BLOCK, UU>(P, c, S, Q, base);
    __syncthreads();
    cy_mark<BLOCK, UU>(S, 2);
    if (S.pcnt > FLUSH_AT) flush<BLOCK, UU>(P, c, S);
    cy_mark<BLOCK, UU>(S, 3);
  }
  flush<BLOCK, UU>(P, c, S);
  cy_mark<BLOCK, UU>(S, 3);
}

/* ------------------------------------------------------------------------ */
/* The leader's decision (warp 0 of the last CTA to reach the barrier): what
 * the group runs next.  Replaces the assign manager's bucket advance and
 * termination logic (wl.h:851-1527) with a read of the list tails.  PK: pull
 * phases may be picked. */
template <bool FLT, int BLOCK, int UU, bool PK>
__device__ void leader_step(const PhParams &P, Ctx &c, PSmem<BLOCK, UU> &S) {
  const unsigned lane = threadIdx.x & 31u;
  PhGroup *G = grp_of(P, c);
  const unsigned prev_mode = S.D.mode, prev_q = S.D.q, prev_list = S.D.list,
                 prev_epoch = S.D.epoch;
  bool hub_only = false;
  unsigned mode = PH_M_EXIT, q = prev_q, list = 0, base = ld_rlx32(&G->base);
  unsigned long long lo = 0, hi = 0;
  unsigned nx = 0, xl[PH_MAXR - 1] = {0u, 0u, 0u}, full = 0u;
  unsigned long long xlo[PH_MAXR - 1] = {0ull, 0ull, 0ull}, xhi[PH_MAXR - 1] = {0ull, 0ull, 0ull};
  bool decide = false, next_query = false;
  unsigned sample = 0u; /* a heavy scan that only counts (pull or push) */
  if (ld_rlx32(&P.g->err) != 0u) {
    mode = PH_M_EXIT;
  } else if (prev_mode == PH_M_START) {
    next_query = true;
  } else if (prev_mode == PH_M_INIT) {
    /* distances are INF: set the source and push it (the first bucket) */
    if (lane == 0) {
      const PhQuery &Q = P.qs[prev_q];
      const unsigned src = (P.single_src != 0xFFFFFFFFu && prev_q == 0u) ? P.single_src : Q.src;
      st_rlx32(Q.dist + src, 0u);
      unsigned long long b, cvp = ~0ull;
      unsigned pg[PH_RES_PAGES], cpi = 0;
      if (list_reserve(P, c, PH_LNEXT, 1u, &b, pg, &cvp, &cpi))
        st_rlx64(entry_ptr(P, c, pg[0], b), (unsigned long long)src);
      st_rlx32(&G->base, 0u);
      st_rlx32(&G->far_min, 0xFFFFFFFFu);
      /* the source's bucket counts as dense: it starts with split rows */
      st_rlx32(&G->lh_dense, 1u);
      st_rlx32(&G->lh_k, 0u);
      st_rlx32(&G->lh_full, 0u);
      st_rlx64(&G->lh_prev, 0ull);
      st_rlx64(&G->dmask, 0ull);
      st_rlx64(&G->fmask, 0ull);
      st_rlx32(&G->hs_block, 0u);
      st_rlx32(&G->pc_state, 0u);
      st_rlx32(&G->wide, 0u);
      __threadfence();
    }
    __syncwarp();
    base = 0u;
    decide = true;
  } else if ((prev_mode == PH_M_LIGHT || prev_mode == PH_M_HEAVY) &&
             ld_rlx32(&G->hub_claim) < ld_rlx32(&G->hub_count)) {
    /* a solo phase left split-row records: the group expands them */
    mode = PH_M_HUB;
    list = prev_list;
    lo = ld_rlx32(&G->hub_claim);
    hi = min(ld_rlx32(&G->hub_count), P.hub_cap);
    hub_only = true;
  } else {
    decide = true;
  }
  if (decide) {
    const unsigned long long tn = ld_rlx64(&G->tails[PH_LNEXT].tail);
    const unsigned long long hn = ld_rlx64(&G->head[PH_LNEXT]);
    const unsigned long long ts = ld_rlx64(&G->tails[PH_LSETTLED].tail);
    const unsigned long long hs = ld_rlx64(&G->head[PH_LSETTLED]);
    if (tn > hn) {
      mode = PH_M_LIGHT;
      list = PH_LNEXT;
      lo = hn;
      hi = tn;
      if (P.lh_adapt) {
        /* another light phase of the same bucket: when it re-improved few of
         * the vertices the last one expanded (under 1 in 20), heavy edges go
         * with the light ones, and a bucket whose second light phase is that
         * small marks the next bucket as sparse.  The first light phase of a
         * bucket collected by a scan (or of the source's bucket) takes the
         * choice made when the bucket opened. */
        const unsigned long long prevc = ld_rlx64(&G->lh_prev);
        const bool few = (tn - hn) * 20ull < prevc;
        const unsigned k = ld_rlx32(&G->lh_k);
        full = k == 0u ? ld_rlx32(&G->lh_full) : (few ? 1u : 0u);
        if (lane == 0) {
          if (full) st_rlx32(&G->hs_block, 1u);
          if (k == 1u && !few) st_rlx32(&G->lh_dense, 1u);
          st_rlx64(&G->lh_prev, tn - hn);
          st_rlx32(&G->lh_k, k + 1u);
        }
      }
    } else if (ts > hs) {
      /* a large settled list (duplicates included) is rebuilt once by a
       * heavy scan: each settled vertex with heavy edges once, in vertex
       * order; the list's entries are dropped.  With an in-edge CSR the scan
       * also counts both directions, and the bucket's heavy edges are then
       * taken as a pull when that reads fewer edges than the push */
      const PhQuery &Qh = P.qs[q];
      const unsigned long long thr = max(4096u, Qh.n >> (P.dense_shift ? P.dense_shift : 31u));
      const bool pull_ok =
          PK && P.pull_ok && Qh.trow != nullptr && Qh.split != nullptr && !P.near_far;
      const unsigned long long pull_thr = max(4096ull, (unsigned long long)(Qh.n >> 6));
      /* 1: the sampling scan just counted for this list; 2: it chose push
       * (no second sample).  Read only where a pull is possible. */
      const unsigned pcs = pull_ok ? ld_rlx32(&G->pc_state) : 0u;
      /* a settled list of one bucket: after a widened light phase it holds
       * vertices of lower buckets too, whose heavy edges can reach vertices
       * at or below pull_floor, which a pull does not visit.  (A light phase
       * that relaxed whole rows is no obstacle: it re-relaxes nothing a pull
       * would miss.) */
      const bool one_bucket = pull_ok && ld_rlx32(&G->wide) == 0u;
      unsigned pc_next = 0u;
      if (one_bucket && pcs == 1u && ld_rlx64(&G->pc_pull) < ld_rlx64(&G->pc_push)) {
        mode = PH_M_PULL;
        list = PH_LSETTLED;
        lo = 0ull;
        hi = Qh.n;
        if (lane == 0) st_rlx64(&G->head[PH_LSETTLED], ts);
      } else if (one_bucket && pcs == 0u && ts - hs > pull_thr) {
        /* count both directions on a sample of the vertices first; the
         * settled list stays for a push */
        mode = PH_M_SCAN;
        list = PH_LSETTLED;
        lo = 0ull;
        hi = Qh.n;
        sample = 1u;
        pc_next = 1u;
        if (lane == 0) {
          st_rlx64(&G->pc_push, 0ull);
          st_rlx64(&G->pc_pull, 0ull);
        }
      } else if (P.dense_shift && Qh.split && ts - hs > thr && ld_rlx32(&G->hs_block) == 0u) {
        mode = PH_M_SCAN;
        list = PH_LSETTLED;
        lo = 0ull;
        hi = Qh.n;
        pc_next = pcs != 0u ? 2u : 0u; /* sampled already: no second sample */
        if (lane == 0) {
          st_rlx64(&G->head[PH_LSETTLED], ts);
          st_rlx32(&G->hs_block, 1u);
        }
      } else {
        mode = PH_M_HEAVY;
        list = PH_LSETTLED;
        lo = hs;
        hi = ts;
      }
      if (lane == 0 && pcs != pc_next) st_rlx32(&G->pc_state, pc_next);
    } else if (P.near_far) {
      /* near-far: the threshold moves up one bucket, or to the smallest
       * bucket pushed to the far pile since it last moved, and the pile is
       * split against it (entries above it are pushed to the pile again) */
      const unsigned long long tf = ld_rlx64(&G->tails[PH_LFAR].tail);
      const unsigned long long hf = ld_rlx64(&G->head[PH_LFAR]);
      if (tf > hf) {
        const unsigned fm = ld_rlx32(&G->far_min);
        mode = PH_M_LIGHT;
        list = PH_LFAR;
        lo = hf;
        hi = tf;
        base = (fm != 0xFFFFFFFFu && fm > base + 1u) ? fm : base + 1u;
        if (lane == 0) {
          st_rlx32(&G->base, base);
          st_rlx32(&G->far_min, 0xFFFFFFFFu);
        }
        if (P.lh_adapt) {
          full = ld_rlx32(&G->lh_dense) != 0u ? 0u : 1u;
          if (lane == 0) {
            st_rlx32(&G->lh_dense, 0u);
            st_rlx64(&G->lh_prev, tf - hf);
            st_rlx32(&G->lh_k, 1u);
          }
        }
      } else {
        next_query = true;
      }
    } else {
      /* advance: the nearest non-empty slot above the base */
      const unsigned offa = lane + 1u, offb = lane + 33u;
      const unsigned sa = (base + offa) & (PH_NSLOT - 1u);
      const unsigned sb = (base + offb) & (PH_NSLOT - 1u);
      const unsigned long long ta = ld_rlx64(&G->tails[sa].tail), ha = ld_rlx64(&G->head[sa]);
      unsigned long long tb = 0, hb = 0;
      if (offb < PH_NSLOT) {
        tb = ld_rlx64(&G->tails[sb].tail);
        hb = ld_rlx64(&G->head[sb]);
      }
      /* a dense slot is non-empty whatever its list holds */
      const unsigned long long dm = P.dense_shift ? ld_rlx64(&G->dmask) : 0ull;
      const unsigned ma = __ballot_sync(0xFFFFFFFFu, ta > ha || ((dm >> sa) & 1ull));
      const unsigned mb =
          __ballot_sync(0xFFFFFFFFu, offb < PH_NSLOT && (tb > hb || ((dm >> sb) & 1ull)));
      const unsigned long long m0 = (unsigned long long)ma | ((unsigned long long)mb << 32);
      const unsigned s0 = m0 ? (base + (unsigned)__ffsll((long long)m0)) & (PH_NSLOT - 1u) : 0u;
      if (m0 != 0ull && ((dm >> s0) & 1ull)) {
        /* the nearest bucket is dense: collect it with one pass over the
         * distances (its list is incomplete and is dropped) */
        mode = PH_M_SCAN;
        list = s0;
        base += (unsigned)__ffsll((long long)m0);
        lo = 0ull;
        hi = P.qs[q].n;
        if (lane == 0) {
          st_rlx32(&G->base, base);
          st_rlx64(&G->head[s0], ld_rlx64(&G->tails[s0].tail));
          atomicAnd(&G->dmask, ~(1ull << s0));
          st_rlx32(&G->lh_full, ld_rlx32(&G->lh_dense) != 0u ? 0u : 1u);
          st_rlx32(&G->lh_dense, 0u);
          st_rlx32(&G->lh_k, 0u);
          st_rlx32(&G->hs_block, 0u);
          st_rlx32(&G->wide, 0u);
        }
      } else if (ma | mb) {
        /* the nearest non-empty slot; with adaptation on, while the entries
         * gathered stay few, the next non-empty slots too (at most PH_MAXR,
         * never the far slot after another): the bucket is widened on the
         * device and the ring re-based at the window's top bucket.  Relaxing
         * a wider bucket is still label-correcting: a distance that a later
         * heavy phase lowers to the window comes back through the NEXT list */
        unsigned long long mask = (unsigned long long)ma | ((unsigned long long)mb << 32);
        const unsigned long long target =
            max(4ull * P.solo_max, 32ull * P.gsize);
        unsigned long long cum = 0;
        unsigned top = 0;
        while (mask != 0ull) {
          const unsigned i = (unsigned)__ffsll((long long)mask) - 1u;
          const unsigned off = i + 1u;
          if (off == PH_NSLOT - 1u && top != 0u) break;
          const unsigned long long t = __shfl_sync(0xFFFFFFFFu, i < 32u ? ta : tb, i & 31u);
          const unsigned long long h = __shfl_sync(0xFFFFFFFFu, i < 32u ? ha : hb, i & 31u);
          const unsigned sl = (base + off) & (PH_NSLOT - 1u);
          if (top != 0u && ((dm >> sl) & 1ull)) break; /* a dense slot opens alone */
          if (top == 0u) {
            list = sl;
            lo = h;
            hi = t;
          } else {
            xl[nx] = sl;
            xlo[nx] = h;
            xhi[nx] = t;
            ++nx;
          }
          top = off;
          cum += t - h;
          mask &= mask - 1ull;
          if (!P.adapt || cum >= target || nx + 1u == PH_MAXR || off == PH_NSLOT - 1u) break;
        }
        mode = PH_M_LIGHT;
        base += top;
        if (lane == 0) st_rlx32(&G->base, base);
        bool hsb = nx != 0u;
        if (P.lh_adapt) {
          /* a new bucket: whole rows unless the last bucket was dense */
          full = ld_rlx32(&G->lh_dense) != 0u ? 0u : 1u;
          if (lane == 0) {
            st_rlx32(&G->lh_dense, 0u);
            st_rlx64(&G->lh_prev, cum);
            st_rlx32(&G->lh_k, 1u);
          }
          hsb = hsb || full != 0u;
        }
        if (lane == 0) {
          st_rlx32(&G->hs_block, hsb ? 1u : 0u);
          st_rlx32(&G->wide, nx != 0u ? 1u : 0u);
        }
      } else {
        next_query = true;
      }
    }
    if ((mode == PH_M_LIGHT || mode == PH_M_HEAVY) && lane == 0) {
      st_rlx64(&G->head[list], hi);
      for (unsigned r = 0; r < nx; ++r) st_rlx64(&G->head[xl[r]], xhi[r]);
      if (P.dense_shift) { /* opened slots: their far entries move on now */
        unsigned long long opened = list < PH_NSLOT ? (1ull << list) : 0ull;
        for (unsigned r = 0; r < nx; ++r) opened |= 1ull << xl[r];
        if (opened) atomicAnd(&G->fmask, ~opened);
      }
      st_rlx32(&G->hub_count, 0u); /* split rows of the coming phase */
      st_rlx32(&G->hub_claim, 0u);
    }
  }
  if (next_query) {
    unsigned qi = 0;
    if (lane == 0) qi = atomicAdd(&P.g->next_q, 1u);
    qi = __shfl_sync(0xFFFFFFFFu, qi, 0);
    if (qi < P.nq) {
      mode = PH_M_INIT;
      q = P.order ? P.order[qi] : qi;
      base = 0u;
      /* a new query: lists start on a page boundary (the pool restarts) */
      for (unsigned L = lane; L < PH_NLIST; L += 32u) {
        const unsigned long long t = ld_rlx64(&G->tails[L].tail);
        const unsigned long long al = (t + PH_PAGE - 1ull) & ~(unsigned long long)(PH_PAGE - 1u);
        st_rlx64(&G->tails[L].tail, al);
        st_rlx64(&G->head[L], al);
      }
      if (lane == 0) {
        st_rlx32(&G->page_next, 0u);
        st_rlx32(&G->hub_count, 0u);
        st_rlx32(&G->q, q);
        st_rlx32(&G->base, 0u);
      }
    } else {
      mode = PH_M_EXIT;
    }
  }
  const unsigned long long wb = ld_rlx64(&G->work);
  unsigned epoch = prev_epoch; /* a records-only phase keeps its producer's */
  if (lane == 0 && !hub_only) {
    epoch = ld_rlx32(&G->epoch) + 1u;
    if (epoch == 0u) epoch = 1u; /* 0 is what a cleared record sequence holds */
    st_rlx32(&G->epoch, epoch);
  }
  __syncwarp();
  unsigned long long total = hi - lo;
  for (unsigned r = 0; r < nx; ++r) total += xhi[r] - xlo[r];
  if (lane == 0 && P.trace && c.gi == 0u) {
    /* the phase that just ended: its work, and its barrier tail */
    const unsigned long long now = gtimer();
    const unsigned long long prev = ld_rlx64(&P.g->st_trace);
    if (prev > 0ull && prev - 1ull < P.trace_cap) {
      PhTrace *t = P.trace + (prev - 1ull);
      const unsigned long long f = ld_rlx64(&G->tr_first);
      t->edges = (unsigned)min(ld_rlx64(&G->tr_edges), 0xFFFFFFFFull);
      t->items = (unsigned)min(ld_rlx64(&G->tr_items), 0xFFFFFFFFull);
      t->pushes = (unsigned)min(ld_rlx64(&G->tr_pushes), 0xFFFFFFFFull);
      t->tail_ns = (f != 0ull && now > f) ? (unsigned)min(now - f, 0xFFFFFFFFull) : 0u;
    }
    st_rlx64(&G->tr_first, 0ull);
    st_rlx64(&G->tr_edges, 0ull);
    st_rlx64(&G->tr_items, 0ull);
    st_rlx64(&G->tr_pushes, 0ull);
    const unsigned long long i = atomicAdd(&P.g->st_trace, 1ull);
    if (i < P.trace_cap) {
      PhTrace tr;
      tr.t_ns = now;
      tr.count = mode == PH_M_INIT ? P.qs[q].n : (unsigned)min(total, 0xFFFFFFFFull);
      tr.mode = (unsigned short)mode;
      tr.base = (unsigned short)base;
      tr.edges = tr.items = tr.pushes = tr.tail_ns = 0u;
      P.trace[i] = tr;
    }
  }
  if (lane == 0) {
    S.D.mode = mode;
    S.D.q = q;
    S.D.list = list;
    S.D.base = base;
    S.D.lo = lo;
    S.D.hi = hi;
    S.D.work_base = wb;
    S.D.epoch = epoch;
    S.D.nx = nx;
    S.D.full = full;
    S.D.sample = sample;
    for (unsigned r = 0; r < PH_MAXR - 1; ++r) {
      S.D.xl[r] = xl[r];
      S.D.xlo[r] = xlo[r];
      S.D.xhi[r] = xhi[r];
    }
    /* entries per claim: BLOCK, or fewer (a multiple of 32) so that a medium
     * frontier reaches every CTA of the group */
    const unsigned long long spread = (total + P.gsize - 1ull) / P.gsize;
    S.D.per = (unsigned)min((unsigned long long)(PH_EPT * BLOCK),
                            max(32ull, (spread + 31ull) & ~31ull));
  }
}

/* Trace of group 0: adds this CTA's work in the phase that just ended to the
 * group's counters (every thread calls it). */
template <int BLOCK, int UU>
__device__ void trace_account(const PhParams &P, Ctx &c, PSmem<BLOCK, UU> &S) {
  unsigned e = c.edges - c.edges_mark;
  c.edges_mark = c.edges;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xFFFFFFFFu, e, o);
  if ((threadIdx.x & 31u) == 0u && e != 0u) atomicAdd(&S.tr_e, (unsigned long long)e);
  __syncthreads();
  if (threadIdx.x == 0) {
    PhGroup *G = grp_of(P, c);
    const unsigned long long it = S.st_items + S.st_hubs, pu = S.st_pushes;
    atomicAdd(&G->tr_edges, S.tr_e);
    atomicAdd(&G->tr_items, it - S.tr_mi);
    atomicAdd(&G->tr_pushes, pu - S.tr_mp);
    S.tr_e = 0ull;
    S.tr_mi = it;
    S.tr_mp = pu;
  }
}

/* A phase descriptor as the leader published it (thread 0; the release of
 * the group's generation orders it). */
__device__ __forceinline__ void read_desc(PhDesc &D, const PhDesc *dp) {
  D.mode = ld_rlx32(&dp->mode);
  D.q = ld_rlx32(&dp->q);
  D.list = ld_rlx32(&dp->list);
  D.base = ld_rlx32(&dp->base);
  D.lo = ld_rlx64(&dp->lo);
  D.hi = ld_rlx64(&dp->hi);
  D.work_base = ld_rlx64(&dp->work_base);
  D.per = ld_rlx32(&dp->per);
  D.epoch = ld_rlx32(&dp->epoch);
  D.nx = ld_rlx32(&dp->nx);
  D.full = ld_rlx32(&dp->full);
  D.sample = ld_rlx32(&dp->sample);
  for (unsigned r = 0; r < PH_MAXR - 1; ++r) {
    D.xl[r] = ld_rlx32(&dp->xl[r]);
    D.xlo[r] = ld_rlx64(&dp->xlo[r]);
    D.xhi[r] = ld_rlx64(&dp->xhi[r]);
  }
}

/* frontiers small enough for the leader alone */
template <int BLOCK, int UU>
__device__ __forceinline__ bool solo_ok(const PhParams &P, const PSmem<BLOCK, UU> &S) {
  const unsigned mode = S.D.mode;
  if (mode == PH_M_LIGHT || mode == PH_M_HEAVY) {
    unsigned long long total = S.D.hi - S.D.lo;
    for (unsigned r = 0; r < S.D.nx; ++r) total += S.D.xhi[r] - S.D.xlo[r];
    return total <= P.solo_max;
  }
  if (mode == PH_M_HUB) return false; /* left by a solo phase because it is large */
  if (mode == PH_M_INIT) return P.qs[S.D.q].n <= 64u * BLOCK;
  return false;
}

/* ------------------------------------------------------------------------ */
/* edges in flight per thread: 8 where a thread may hold 128 registers, 4 at 64 */
#define PH_U(BLOCK, MINB) ((BLOCK) * (MINB) >= 1024 ? 4 : 8)

/* PK: an instantiation that may pick pull phases (P.pull_ok); the one
 * without them is the same code with the sampling scans and the pull choice
 * compiled out -- the extra code alone made the push loop about 7 % slower
 * (R-MAT 24, batches), so launches that cannot pull do not carry it. */
template <bool FLT, int BLOCK, int MINB, bool PK>
__global__ void __launch_bounds__(BLOCK, MINB) phase_kernel(const __grid_constant__ PhParams P) {
  constexpr int UU = PH_U(BLOCK, MINB);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PSmem<BLOCK, UU> &S = *reinterpret_cast<PSmem<BLOCK, UU> *>(smem_raw);
  const unsigned tid = threadIdx.x;
  Ctx c;
  c.gi = blockIdx.x / P.gsize;
  c.rank = blockIdx.x % P.gsize;
  c.deadline = gtimer() + P.timeout_ns;
  c.edges = 0;
  c.edges_mark = 0;
  PhGroup *G = grp_of(P, c);
  if (tid == 0) {
    S.cy0 = clock64();
    S.nphase = 0ull;
    S.gen = ld_acq32(&G->gen);
    S.pcnt = 0u;
    S.D.mode = PH_M_START;
    S.D.q = 0u;
    /* a resumed launch starts from the pull phase the last one ended with
     * (or, when the solve is done, exits at once) */
    if (P.resume) {
      read_desc(S.D, &G->desc[S.gen & 1u]);
      if (S.D.mode != PH_M_PULL) S.D.mode = PH_M_EXIT;
    }
    S.st_items = S.st_stale = S.st_heavy = S.st_repush = S.st_pushes = S.st_chunks = 0;
    S.st_hubs = S.st_solo = 0;
    S.tr_e = S.tr_mi = S.tr_mp = 0ull;
    for (int i = 0; i < 8; ++i) S.cy[i] = 0ull;
  }
  if (tid < PH_NLIST) S.ptc_vp[tid] = ~0ull;
  __syncthreads();
  while (S.D.mode != PH_M_EXIT) { /* left at the end of the body */
    if (tid == 0) S.tk = clock64();
    run_phase<FLT, BLOCK, UU, PK>(P, c, S, false);
    if (tid == 0) { /* run_phase as a whole, grid phases */
      const long long t1 = clock64();
      S.cy[6] += (unsigned long long)(t1 - S.tk);
      S.tk = t1;
    }
    const bool tracing = P.trace != nullptr && c.gi == 0u;
    if (tracing) trace_account<BLOCK, UU>(P, c, S);
    /* group barrier: the last CTA in becomes the leader */
    __syncthreads();
    if (tid == 0) {
      if (tracing) atomicCAS(&G->tr_first, 0ull, gtimer());
      __threadfence();
      const unsigned old = atomicAdd(&G->arrive, 1u);
      S.leader = (old == P.gsize - 1u) ? 1u : 0u;
      if (S.leader) {
        st_rlx32(&G->arrive, 0u);
        __threadfence();
      }
    }
    __syncthreads();
    if (S.leader) {
      for (;;) {
        if (tid < 32) leader_step<FLT, BLOCK, UU, PK>(P, c, S);
        __syncthreads();
        if (tid == 0) ++S.nphase;
        if (!solo_ok<BLOCK, UU>(P, S)) break;
        if (tid == 0) {
          /* this CTA alone expands the phase; no fence: until the group is
           * released (with a fence) nothing outside this CTA reads what the
           * solo phases write, and the CTA's barriers order its own accesses */
          st_rlx32(&G->producers, 1u);
          ++S.st_solo;
          if (P.trace && c.gi == 0u) { /* mark the record just written as solo */
            const unsigned long long i = ld_rlx64(&P.g->st_trace) - 1ull;
            if (i < P.trace_cap) P.trace[i].mode |= 0x100;
          }
        }
        run_phase<FLT, BLOCK, UU, PK>(P, c, S, true);
        if (tracing) trace_account<BLOCK, UU>(P, c, S);
        __syncthreads();
      }
      if (tid == 0) {
        /* a records-only phase has no producers */
        st_rlx32(&G->producers, S.D.mode == PH_M_HUB ? 0u : P.gsize);
        G->desc[(S.gen + 1u) & 1u] = S.D;
        __threadfence();
        st_rel32(&G->gen, S.gen + 1u);
      }
      if (tid == 0) S.cy[5] += (unsigned long long)(clock64() - S.tk);
    } else {
      if (tid == 0) {
        Waiter w{c.deadline, 0};
        bool ok = true;
        while (ld_acq32(&G->gen) == S.gen) {
          if (!w.spin(P.g, W_BARRIER, 128)) {
            ok = false;
            break;
          }
        }
        if (ok) {
          read_desc(S.D, &G->desc[(S.gen + 1u) & 1u]);
        } else {
          S.D.mode = PH_M_EXIT;
        }
      }
      if (tid == 0) S.cy[4] += (unsigned long long)(clock64() - S.tk);
    }
    if (tid == 0) ++S.gen;
    __syncthreads();
    /* a pull phase ends the launch: the pull kernel runs it, and the next
     * launch (resume) continues from its descriptor */
    if (S.D.mode == PH_M_EXIT || S.D.mode == PH_M_PULL) break;
  }
  /* statistics */
  PhGlobal *g = P.g;
  unsigned long long s_edges = c.edges;
  for (int o = 16; o > 0; o >>= 1) s_edges += __shfl_down_sync(0xFFFFFFFFu, s_edges, o);
  if ((tid & 31u) == 0u && s_edges) atomicAdd(&g->st_edges, s_edges);
  if (tid == 0) {
    atomicAdd(&g->st_items, S.st_items);
    atomicAdd(&g->st_stale, S.st_stale);
    atomicAdd(&g->st_heavy, S.st_heavy);
    atomicAdd(&g->st_repush, S.st_repush);
    atomicAdd(&g->st_pushes, S.st_pushes);
    atomicAdd(&g->st_chunks, S.st_chunks);
    atomicAdd(&g->st_hub, S.st_hubs);
    atomicAdd(&g->st_solo, S.st_solo);
    atomicAdd(&g->st_phases, S.nphase);
    S.cy[7] = (unsigned long long)(clock64() - S.cy0);
    for (int i = 0; i < 8; ++i) atomicAdd(&g->st_cyc[i], S.cy[i]);
  }
}

/* The pull phase of a one-query launch chain (PH_M_PULL), in a kernel of its
 * own so that the phase kernel's push loop keeps its registers (the same
 * loop instantiated twice in one kernel, or called out of it, made the push
 * loop up to 40 % slower on R-MAT 24).  Its CTAs are co-resident like the
 * phase kernel's (a list reservation may wait for another CTA's page
 * mapping) and claim vertex tiles until none is left.  A launch with no pull
 * to run -- the solve has ended, or failed -- returns at once. */
template <bool FLT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) pull_kernel(const __grid_constant__ PhParams P) {
  constexpr int UU = PH_U(BLOCK, MINB);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PSmem<BLOCK, UU> &S = *reinterpret_cast<PSmem<BLOCK, UU> *>(smem_raw);
  const unsigned tid = threadIdx.x;
  Ctx c;
  c.gi = 0u; /* one query, one group */
  c.rank = blockIdx.x;
  c.deadline = gtimer() + P.timeout_ns;
  c.edges = 0;
  c.edges_mark = 0;
  PhGroup *G = grp_of(P, c);
  if (tid == 0) {
    read_desc(S.D, &G->desc[ld_acq32(&G->gen) & 1u]);
    if (ld_rlx32(&P.g->err) != 0u) S.D.mode = PH_M_EXIT;
    S.pcnt = 0u;
    S.st_items = S.st_stale = S.st_heavy = S.st_repush = S.st_pushes = S.st_chunks = 0;
    S.st_hubs = S.st_solo = 0;
    S.tr_e = S.tr_mi = S.tr_mp = 0ull;
    S.pend = ~0ull;
    S.pl_k = 0u;
  }
  if (tid < PH_NLIST) S.ptc_vp[tid] = ~0ull;
  __syncthreads();
  if (S.D.mode != PH_M_PULL) return;
  const PhQuery &Q = P.qs[S.D.q];
  if (tid == 0) S.pl_T = pull_floor<FLT>(Q, S.D.base); /* read after prepare's barrier */
  while (prepare_pull<FLT, BLOCK, UU>(P, c, S, Q)) {
    for (unsigned sub = 0; sub < PH_PULL_SUB; ++sub) pull_tile_warp<FLT, BLOCK, UU>(P, c, S, Q, sub);
    __syncthreads();
    if (tid == 0) ++S.st_chunks;
    if (S.pcnt > PSmem<BLOCK, UU>::FLUSH_AT) flush<BLOCK, UU>(P, c, S);
  }
  flush<BLOCK, UU>(P, c, S);
  if (P.trace != nullptr) trace_account<BLOCK, UU>(P, c, S);
  PhGlobal *g = P.g;
  unsigned long long s_edges = c.edges;
  for (int o = 16; o > 0; o >>= 1) s_edges += __shfl_down_sync(0xFFFFFFFFu, s_edges, o);
  if ((tid & 31u) == 0u && s_edges) atomicAdd(&g->st_edges, s_edges);
  if (tid == 0) {
    atomicAdd(&g->st_items, S.st_items);
    atomicAdd(&g->st_pushes, S.st_pushes);
    atomicAdd(&g->st_chunks, S.st_chunks);
  }
}

template <bool FLT, int BLOCK, int MINB>
static cudaError_t prep_one(int *max_blocks_per_sm) {
  const size_t smem = sizeof(PSmem<BLOCK, PH_U(BLOCK, MINB)>);
  cudaError_t e = cudaFuncSetAttribute(phase_kernel<FLT, BLOCK, MINB, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(phase_kernel<FLT, BLOCK, MINB, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(pull_kernel<FLT, BLOCK, MINB>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  /* the grid must be resident for every kernel of a launch chain */
  int a = 0, b = 0, p = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, phase_kernel<FLT, BLOCK, MINB, false>,
                                                    BLOCK, smem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, phase_kernel<FLT, BLOCK, MINB, true>,
                                                      BLOCK, smem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, pull_kernel<FLT, BLOCK, MINB>, BLOCK, smem);
  const int ab = a < b ? a : b;
  *max_blocks_per_sm = ab < p ? ab : p;
  return e;
}

template <bool FLT, int BLOCK, int MINB>
static cudaError_t launch_one(const PhParams &P, cudaStream_t st, bool pull) {
  /* cooperative launch: every CTA of a group waits at the group barrier, so
   * all of them must be resident; the Ex form keeps it graph-capturable.
   * The pull kernel takes the same grid. */
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P.groups * P.gsize);
  cfg.blockDim = dim3(BLOCK);
  cfg.dynamicSmemBytes = sizeof(PSmem<BLOCK, PH_U(BLOCK, MINB)>);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (pull) return cudaLaunchKernelEx(&cfg, pull_kernel<FLT, BLOCK, MINB>, P);
  return P.pull_ok ? cudaLaunchKernelEx(&cfg, phase_kernel<FLT, BLOCK, MINB, true>, P)
                   : cudaLaunchKernelEx(&cfg, phase_kernel<FLT, BLOCK, MINB, false>, P);
}

/* Failure-detection check: thread 0 waits, through the same bounded Waiter
 * as the group barrier, for a flag that nothing sets.  The deadline runs out,
 * the error word records a timeout at the barrier's wait site, and the
 * kernel returns with the context intact.  An iteration cap bounds the loop
 * even if the timer were not to advance. */
__global__ void diag_wait_kernel(const unsigned *flag, PhGlobal *g,
                                 unsigned long long timeout_ns) {
  if (threadIdx.x != 0u || blockIdx.x != 0u) return;
  Waiter w{gtimer() + timeout_ns, 0};
  for (unsigned long long it = 0; ld_acq32(flag) == 0u; ++it) {
    if (it > (1ull << 24)) {
      raise_err(g, PH_ERR_TIMEOUT, W_BARRIER);
      return;
    }
    if (!w.spin(g, W_BARRIER, 1024)) return;
  }
}

}  // namespace adds_phase

int ph_diag_wait(int device, unsigned timeout_ms, unsigned *err, unsigned *where,
                 float *waited_ms) {
  if (cudaSetDevice(device) != cudaSuccess) return -5;
  PhGlobal *g = nullptr;
  unsigned *flag = nullptr;
  cudaEvent_t a = nullptr, z = nullptr;
  int rc = -5;
  if (cudaMalloc(&g, sizeof(PhGlobal)) == cudaSuccess &&
      cudaMalloc(&flag, sizeof(unsigned)) == cudaSuccess &&
      cudaMemset(g, 0, sizeof(PhGlobal)) == cudaSuccess &&
      cudaMemset(flag, 0, sizeof(unsigned)) == cudaSuccess &&
      cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&z) == cudaSuccess) {
    cudaEventRecord(a, 0);
    adds_phase::diag_wait_kernel<<<1, 32>>>(flag, g, (unsigned long long)timeout_ms * 1000000ull);
    cudaEventRecord(z, 0);
    PhGlobal h;
    if (cudaGetLastError() == cudaSuccess && cudaEventSynchronize(z) == cudaSuccess &&
        cudaMemcpy(&h, g, sizeof(PhGlobal), cudaMemcpyDeviceToHost) == cudaSuccess) {
      *err = h.err;
      *where = h.err_where;
      cudaEventElapsedTime(waited_ms, a, z);
      rc = 0;
    }
  }
  if (a) cudaEventDestroy(a);
  if (z) cudaEventDestroy(z);
  if (flag) cudaFree(flag);
  if (g) cudaFree(g);
  return rc;
}

/* Kernel variants: (threads per CTA, CTAs per SM the registers are sized
 * for).  variant 0: 256 x 4, 1: 512 x 2, 2: 1024 x 1, 5: 128 x 8 (64
 * registers per thread), 3: 256 x 2, 4: 512 x 1 (128 registers per thread). */
#define PH_VARIANTS(X) \
  X(0, 256, 4) X(1, 512, 2) X(2, 1024, 1) X(3, 256, 2) X(4, 512, 1) X(5, 128, 8)

int adds_phase_variant_block(int variant) {
#define X(i, b, m) if (variant == i) return b;
  PH_VARIANTS(X)
#undef X
  return 0;
}

cudaError_t adds_phase_prepare(bool flt, int variant, int *max_blocks_per_sm) {
  using namespace adds_phase;
#define X(i, b, m) \
  if (variant == i) return flt ? prep_one<true, b, m>(max_blocks_per_sm) : prep_one<false, b, m>(max_blocks_per_sm);
  PH_VARIANTS(X)
#undef X
  return cudaErrorInvalidValue;
}

cudaError_t adds_phase_launch(const PhParams &P, int variant, cudaStream_t st, bool pull) {
  using namespace adds_phase;
#define X(i, b, m) \
  if (variant == i)  \
    return P.is_float ? launch_one<true, b, m>(P, st, pull) : launch_one<false, b, m>(P, st, pull);
  PH_VARIANTS(X)
#undef X
  return cudaErrorInvalidValue;
}

/* ======================================================================== */
/* host side                                                                  */
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

static unsigned ph_log2_ceil(unsigned long long x) {
  unsigned l = 0;
  while ((1ull << l) < x) ++l;
  return l;
}

void ph_engine_free(PhEngine &E) {
  void *ptrs[] = {E.grp, E.g, E.qs, E.order, E.pool, E.pt, E.hub, E.hub_seq, E.trace};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (E.g_host) cudaFreeHost(E.g_host);
  E = PhEngine();
}

/* Full reset (first use, or after a device error left a barrier or a list
 * half way): group state and page tables back to their initial values. */
int ph_engine_reset(PhEngine &E, cudaStream_t st) {
  if (cudaMemsetAsync(E.grp, 0, (size_t)E.groups * sizeof(PhGroup), st) != cudaSuccess ||
      cudaMemsetAsync(E.pt, 0xFF, ((size_t)E.groups * PH_NLIST << E.ptn_log2) * 8, st) !=
          cudaSuccess ||
      cudaMemsetAsync(E.g, 0, sizeof(PhGlobal), st) != cudaSuccess ||
      cudaMemsetAsync(E.hub_seq, 0, (size_t)E.groups * E.hub_cap * 4, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return -5; /* ADDS_ERR_CUDA */
  return 0;
}

int ph_engine_upload(PhEngine &E, cudaStream_t st) {
  if (cudaMemcpyAsync(E.qs, E.qs_host.data(), E.qs_host.size() * sizeof(PhQuery),
                      cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return -5;
  return 0;
}

static int ph_blocks_per_sm(bool flt, int variant, int *bps) {
  return adds_phase_prepare(flt, variant, bps) == cudaSuccess ? 0 : -5;
}

/* Sizes the per-group pools for the largest query (x grow) and allocates. */
int ph_engine_alloc(PhEngine &E, int device, bool flt, const std::vector<PhQuery> &qv,
                    const PhKnobs &k, unsigned grow, cudaStream_t st) {
  ph_engine_free(E);
  E.device = device;
  E.flt = flt;
  E.nq = (unsigned)qv.size();
  E.variant = (unsigned)k.variant;
  E.block = (unsigned)adds_phase_variant_block(k.variant);
  int bps = 0;
  if (E.block == 0 || ph_blocks_per_sm(flt, k.variant, &bps) || bps < 1)
    return -9; /* ADDS_ERR_UNSUPPORTED */
  if (cudaDeviceGetAttribute(&E.num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return -5;
  const int cps = (k.ctas_per_sm > 0 && k.ctas_per_sm < bps) ? k.ctas_per_sm : bps;
  const unsigned nctas = (unsigned)(cps * E.num_sms);
  E.req_group = k.group_ctas;
  if (E.nq == 1) {
    /* one query: every resident CTA, or fewer when asked (a small graph's
     * phases are short, and a group barrier over fewer CTAs is cheaper) */
    E.gsize = k.group_ctas > 0 ? std::min((unsigned)k.group_ctas, nctas) : nctas;
    E.groups = 1;
  } else {
    /* about 32 groups: enough to run small queries side by side, large
     * enough that a big query still has a few SMs (measured best on the
     * mixed 256-query batch: 18 CTAs per group on 148 SMs) */
    unsigned gs = k.group_ctas > 0 ? (unsigned)k.group_ctas
                                   : std::max(1u, nctas / std::min(E.nq, 32u));
    gs = std::min(gs, nctas);
    E.gsize = gs;
    E.groups = std::min(nctas / gs, E.nq);
  }
  double need = 0;
  unsigned long long mmax = 0;
  for (const PhQuery &q : qv) {
    need = std::max(need, 3.0 * q.n + q.m / 8.0);
    mmax = std::max(mmax, q.m);
    E.max_n = std::max(E.max_n, q.n);
  }
  const unsigned long long pages = (unsigned long long)(need * grow / PH_PAGE) + 2ull * PH_NLIST + 8ull;
  if (pages > 0x3FFFFFFFull) return -4; /* ADDS_ERR_OOM */
  E.pages_per_group = (unsigned)pages;
  E.ptn_log2 = ph_log2_ceil(pages + 2ull);
  /* records per phase: a split row of d edges gives ceil(d / chunk) <= d /
   * chunk + 1 of them and only rows longer than the threshold (>= chunk) are
   * split; a vertex can be expanded twice in one phase */
  E.hub_eff = ph_hub_chunk(k);
  E.hub_cap = (unsigned)std::min<unsigned long long>(
      0x7FFFFFFFull, (4ull * (mmax / E.hub_eff) + 4096ull) * grow);
  E.qs_host = qv;
#define PH_ALLOC(ptr, bytes_)                               \
  do {                                                      \
    size_t _b = (bytes_);                                   \
    if (cudaMalloc((void **)&(ptr), _b) != cudaSuccess) {   \
      cudaGetLastError();                                   \
      ph_engine_free(E);                                    \
      return -4;                                            \
    }                                                       \
    E.bytes += _b;                                          \
  } while (0)
  PH_ALLOC(E.grp, (size_t)E.groups * sizeof(PhGroup));
  PH_ALLOC(E.g, sizeof(PhGlobal));
  PH_ALLOC(E.qs, (size_t)E.nq * sizeof(PhQuery));
  PH_ALLOC(E.order, (size_t)E.nq * 4);
  PH_ALLOC(E.pool, (size_t)E.groups * E.pages_per_group * PH_PAGE * 8);
  PH_ALLOC(E.pt, ((size_t)E.groups * PH_NLIST << E.ptn_log2) * 8);
  PH_ALLOC(E.hub, (size_t)E.groups * E.hub_cap * sizeof(PhHub));
  PH_ALLOC(E.hub_seq, (size_t)E.groups * E.hub_cap * 4);
#undef PH_ALLOC
  if (cudaMallocHost((void **)&E.g_host, sizeof(PhGlobal)) != cudaSuccess) {
    cudaGetLastError();
    ph_engine_free(E);
    return -4;
  }
  memset(E.g_host, 0, sizeof(PhGlobal));
  /* largest queries first: the last group to finish is not stuck with a big one */
  std::vector<unsigned> order(E.nq);
  for (unsigned i = 0; i < E.nq; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](unsigned a, unsigned b) {
    return qv[a].m + qv[a].n > qv[b].m + qv[b].n;
  });
  if (cudaMemcpyAsync(E.order, order.data(), (size_t)E.nq * 4, cudaMemcpyHostToDevice, st) !=
      cudaSuccess)
    return -5;
  int rc = ph_engine_upload(E, st);
  if (rc) return rc;
  return ph_engine_reset(E, st);
}

unsigned ph_hub_chunk(const PhKnobs &k) {
  const unsigned thr = std::max(64u, k.hub_threshold);
  return std::max(64u, std::min(k.hub_chunk, thr));
}

int ph_engine_params(const PhEngine &E, const PhKnobs &k, unsigned single_src, PhParams *P) {
  memset(P, 0, sizeof *P);
  P->qs = E.qs;
  P->order = E.order;
  P->nq = E.nq;
  P->groups = E.groups;
  P->gsize = E.gsize;
  P->grp = E.grp;
  P->g = E.g;
  P->pool = E.pool;
  P->pages_per_group = E.pages_per_group;
  P->pt = E.pt;
  P->ptn_log2 = E.ptn_log2;
  P->hub = E.hub;
  P->hub_seq = E.hub_seq;
  P->hub_cap = E.hub_cap;
  P->hub_threshold = std::max(64u, k.hub_threshold);
  P->hub_chunk = ph_hub_chunk(k);
  if (P->hub_chunk < E.hub_eff) return -9; /* engine sized for longer chunks */
  P->solo_max = k.solo_max;
  P->adapt = k.adapt;
  P->lh_adapt = k.lh_adapt;
  P->near_far = k.near_far ? 1u : 0u;
  P->dense_shift = k.near_far ? 0u : k.dense_shift;
  P->is_float = E.flt ? 1u : 0u;
  /* pull phases: one query on one group, with an in-edge CSR */
  P->pull_ok = (E.nq == 1 && E.groups == 1 && E.qs_host[0].trow != nullptr) ? 1u : 0u;
  P->resume = 0u;
  P->single_src = single_src;
  P->timeout_ns = k.timeout_ns;
  P->trace = E.trace;
  P->trace_cap = E.trace_cap;
  return 0;
}

/* Turns the phase trace of group 0 on (cap > 0, allocates) or off. */
int ph_engine_trace(PhEngine &E, unsigned cap) {
  if (E.trace) cudaFree(E.trace);
  E.trace = nullptr;
  E.trace_cap = 0;
  if (cap == 0) return 0;
  if (cudaMalloc((void **)&E.trace, (size_t)cap * sizeof(PhTrace)) != cudaSuccess) {
    cudaGetLastError();
    return -4;
  }
  E.trace_cap = cap;
  return 0;
}

/* One launch: statistics cleared, the persistent kernel, the control block
 * copied back (it carries the error word).  Graph-capturable. */
int ph_engine_enqueue(PhEngine &E, const PhParams &P, cudaStream_t st, cudaEvent_t k0,
                      cudaEvent_t k1) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return -5;
  const unsigned fl = cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : 0u;
  /* statistics and the batch counter start at zero; the error word is kept,
   * so after a failed solve the ones queued behind it exit at once and the
   * failure reaches the host at the next synchronisation (the host resets
   * the engine once it has reported the error) */
  const size_t keep = offsetof(PhGlobal, next_q);
  if (cudaMemsetAsync(reinterpret_cast<char *>(E.g) + keep, 0, sizeof(PhGlobal) - keep, st) !=
      cudaSuccess)
    return -5;
  if (k0 && cudaEventRecordWithFlags(k0, st, fl) != cudaSuccess) return -5;
  if (adds_phase_launch(P, (int)E.variant, st) != cudaSuccess) return -5;
  if (P.pull_ok) {
    /* a launch that picks a pull phase ends there; each pull kernel runs the
     * phase the launch before it ended with, and the next launch resumes
     * from it.  The last launch picks no pull, so the chain always finishes
     * the solve; launches with nothing left to do return at once. */
    PhParams R = P;
    R.resume = 1u;
    for (unsigned s = 1; s <= PH_PULL_SEGMENTS; ++s) {
      R.pull_ok = s < PH_PULL_SEGMENTS ? 1u : 0u;
      if (adds_phase_launch(R, (int)E.variant, st, true) != cudaSuccess ||
          adds_phase_launch(R, (int)E.variant, st) != cudaSuccess)
        return -5;
    }
  }
  if (k1 && cudaEventRecordWithFlags(k1, st, fl) != cudaSuccess) return -5;
  if (cudaMemcpyAsync(E.g_host, E.g, sizeof(PhGlobal), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return -5;
  return 0;
}

/* device error word -> ABI code (after the stream has been synchronised) */
int ph_engine_status(const PhEngine &E, char *msg, size_t msg_len) {
  const unsigned err = E.g_host->err;
  if (err && msg) snprintf(msg, msg_len, "device error %u at wait site %u", err, E.g_host->err_where);
  switch (err) {
    case 0: return 0;
    case PH_ERR_OVERFLOW: return -7;     /* ADDS_ERR_WL_OVERFLOW    */
    case PH_ERR_HUB_OVERFLOW: return -7;
    case PH_ERR_MAPPING: return -5;      /* engine fault: ADDS_ERR_CUDA */
    default: return -6;                  /* ADDS_ERR_DEVICE_TIMEOUT */
  }
}
