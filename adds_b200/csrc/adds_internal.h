/*
 * adds_internal.h — device data layout of the persistent SSSP engine.
 *
 * The reference worklist (ads_int/wl.h:133-190) keeps 32 circular distance
 * buckets ("bags") as virtual ranges in a paged HBM pool, and three manager
 * warps (alloc / read / assign, wl.h:488-1527) move pages and hand work to
 * worker blocks through global mailboxes.  This engine keeps the bucket ring
 * and the paged pool but removes the manager block: every CTA pops and pushes
 * with atomics on per-bucket counters, pages are allocated on demand by the
 * CTA whose reservation covers a page's first entry, and termination is a
 * per-query live-item count.  Queue entries carry the distance they were
 * pushed with so superseded entries are dropped at pop time.
 */
#ifndef ADDS_INTERNAL_H_
#define ADDS_INTERNAL_H_

#include <stdint.h>

#define ADDS_NB 32                 /* bucket slots per query (wl.h:14 NUM_BAG) */
#define ADDS_PAGE_LOG2 12
#define ADDS_PAGE (1u << ADDS_PAGE_LOG2) /* entries per pool page (8 B each)   */
#define ADDS_HUB_RING_LOG2 16      /* split-row chunk ring capacity            */
#define ADDS_INF_I32_BITS 0x7FFFFFFFu
/* Graph edge arrays are allocated this many entries past m: the phase
 * engine copies row segments rounded out to 16-byte boundaries, so a copy
 * may read one entry past the last row (never relaxed). */
#define ADDS_EDGE_PAD 2u
#define ADDS_INF_F32_BITSV 0x7F7FFFFFu

/* device error codes written to GlobalCtl::err (first one wins) */
#define ADDS_DEV_OK 0u
#define ADDS_DEV_TIMEOUT 1u
#define ADDS_DEV_OVERFLOW 2u
#define ADDS_DEV_HUB_OVERFLOW 3u

/* One bucket slot: monotone 64-bit virtual indices.  Entries [head, tail)
 * are reserved by pushers; `avail` counts reserved, written entries that no
 * popper has claimed yet (pushers add after their stores, poppers claim by
 * fetch-and-subtract, so no popper ever takes an index that was not
 * reserved).  inflight counts claimed-but-unfinished entries (used only to
 * decide when the lowest bucket may be retired).  Each counter has its own
 * 32-byte sector so the fetch-and-adds on them do not share a sector. */
struct __align__(128) SlotCtr {
  unsigned long long head;
  unsigned long long pad0[3];
  unsigned long long tail;
  unsigned long long pad1[3];
  long long avail;
  unsigned long long pad2[3];
  unsigned long long inflight;
  unsigned long long pad3[3];
};

/* Per-query mutable control, one 128-byte line each.  ctrl packs the lowest
 * live bucket: low word = base bucket counter (31 bits) | phase << 31 (0:
 * its light edges are being relaxed, 1: its settled vertices' heavy edges
 * are), high word = the base bucket's key (dist key >> shift). */
#define ADDS_PHASE_H 0x80000000u
struct __align__(128) QueryCtl {
  unsigned long long ctrl;
  unsigned live;           /* entries pushed (queue or hub ring) not finished   */
  unsigned done;           /* 1 once live reached 0                            */
  unsigned shift;          /* bucket shift of the query                        */
  unsigned win;            /* buckets processed at once (on-device adapted)     */
  unsigned pad[26];
};

/* Read-only per-query descriptor. */
struct QueryDesc {
  const unsigned *row;     /* n+1 row offsets (u32)                           */
  const uint2 *edges;      /* m x {dst, weight bits}, rows sorted by weight   */
  const unsigned *split;   /* per vertex: count of light edges (w < delta) at
                              the start of its row; NULL = every edge light  */
  unsigned *dist;          /* n distance words                                */
  unsigned n;
  unsigned src;
  float scale;             /* float graphs: key = floor(d*scale)              */
  unsigned ptn_log2;       /* page-table ring size per slot (log2)            */
  unsigned long long *pt;  /* [2*ADDS_NB << ptn_log2] page-table entries      */
  SlotCtr *slots;          /* [2*ADDS_NB]: light buckets, then heavy lists    */
  QueryCtl *ctl;
  unsigned shift0;         /* initial bucket shift                            */
  unsigned graph_id;       /* index of the distinct graph (backward pass)     */
};

struct __align__(32) HubChunk { /* a slice of one long row                    */
  unsigned q;
  unsigned u;                   /* the row's vertex: stale chunks are skipped */
  unsigned du;
  unsigned eb;
  unsigned ee;
  unsigned pad[3];
};

/* Engine-wide control block. */
struct __align__(128) GlobalCtl {
  unsigned remaining;       /* queries not yet finished                       */
  unsigned err;             /* ADDS_DEV_* (first error wins)                  */
  unsigned err_where;       /* diagnostic: which wait gave up                 */
  unsigned pad0[29];
  unsigned long long fq_head; unsigned long long pad1[15]; /* page free queue */
  unsigned long long fq_tail; unsigned long long pad2[15];
  unsigned long long hub_head; unsigned long long pad3[15]; /* chunk ring     */
  unsigned long long hub_tail; unsigned long long pad4[15];
  unsigned hungry;          /* CTAs currently without work                   */
  unsigned pad5[31];
  /* statistics */
  unsigned long long st_items;
  unsigned long long st_stale;
  unsigned long long st_edges;
  unsigned long long st_pushes;
  unsigned long long st_batches;
  unsigned long long st_hub;
  unsigned long long st_local;   /* batches taken from the CTA's own pushes     */
  unsigned long long st_hub_stale;
  unsigned long long st_heavy;    /* heavy-edge lists expanded                   */
  unsigned long long st_cyc[6];   /* SM cycles: acquire, load, edges, flush,
                                     idle, total (summed over CTAs)            */
  unsigned long long st_pad[2];   /* diagnostics: mid-batch flush cycles, count */
};

/* Kernel parameters (passed by value). */
struct EngParams {
  const QueryDesc *qs;
  unsigned nq;
  unsigned nctas;
  GlobalCtl *g;
  unsigned long long *pool;     /* pool_pages * ADDS_PAGE entries            */
  unsigned *pgen;               /* per page allocation generation            */
  unsigned *pcons;              /* per page consumed-entry count             */
  unsigned long long *fq;       /* free-page queue cells {tag:32 | page:32}  */
  unsigned fq_mask;
  unsigned pool_pages;
  HubChunk *hub;                /* [1 << ADDS_HUB_RING_LOG2]                 */
  unsigned *hub_seq;            /* Vyukov sequence numbers                   */
  unsigned long long timeout_ns;
  unsigned long long alloc_wait_ns;
  unsigned window;              /* buckets popped concurrently               */
  unsigned batch_max;           /* items per CTA batch (<= block size)       */
  unsigned hub_threshold;       /* split rows with more edges than this      */
  unsigned hub_chunk;           /* edges per split chunk                     */
  unsigned strict_order;
  unsigned adapt;
  unsigned is_float;
  unsigned single_src;          /* init: override source of query 0 if != ~0 */
  unsigned local_max;           /* own pushes kept as the next batch         */
  unsigned local_max_hungry;    /* ... while other CTAs are waiting for work */
  unsigned block;               /* threads per CTA (selects the kernel)      */
  unsigned greed;               /* claim share = avail / (nctas >> greed)    */
};

#endif /* ADDS_INTERNAL_H_ */
