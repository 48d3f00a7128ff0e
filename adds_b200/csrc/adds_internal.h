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
#define ADDS_INF_F32_BITSV 0x7F7FFFFFu

/* device error codes written to GlobalCtl::err (first one wins) */
#define ADDS_DEV_OK 0u
#define ADDS_DEV_TIMEOUT 1u
#define ADDS_DEV_OVERFLOW 2u
#define ADDS_DEV_HUB_OVERFLOW 3u

/* One bucket slot: monotone 64-bit virtual indices.  Entries [head, tail)
 * are pushed but not popped.  inflight counts popped-but-unfinished entries
 * (used only to decide when the lowest bucket may be retired). */
struct __align__(32) SlotCtr {
  unsigned long long head;
  unsigned long long tail;
  unsigned long long inflight;
  unsigned long long pad;
};

/* Per-query mutable control, one 128-byte line each. */
struct __align__(128) QueryCtl {
  unsigned long long ctrl; /* (base_key << 32) | base_bucket                  */
  unsigned live;           /* entries pushed (queue or hub ring) not finished   */
  unsigned done;           /* 1 once live reached 0                            */
  unsigned shift;          /* current bucket shift (device-adapted)            */
  unsigned adapt_state;
  unsigned long long pushes_at_base; /* controller bookkeeping                 */
  unsigned pad[24];
};

/* Read-only per-query descriptor. */
struct QueryDesc {
  const unsigned *row;     /* n+1 row offsets (u32)                           */
  const uint2 *edges;      /* m x {dst, weight bits}                          */
  unsigned *dist;          /* n distance words                                */
  unsigned n;
  unsigned src;
  float scale;             /* float graphs: key = floor(d*scale)              */
  unsigned ptn_log2;       /* page-table ring size per slot (log2)            */
  unsigned long long *pt;  /* [ADDS_NB << ptn_log2] page-table entries        */
  SlotCtr *slots;          /* [ADDS_NB]                                       */
  QueryCtl *ctl;
  unsigned shift0;         /* initial bucket shift                            */
  unsigned graph_id;       /* index of the distinct graph (backward pass)     */
};

struct HubChunk {          /* a slice of one long row                         */
  unsigned q;
  unsigned du;
  unsigned eb;
  unsigned ee;
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
  /* statistics */
  unsigned long long st_items;
  unsigned long long st_stale;
  unsigned long long st_edges;
  unsigned long long st_pushes;
  unsigned long long st_batches;
  unsigned long long st_hub;
  unsigned long long st_pad[10];
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
};

#endif /* ADDS_INTERNAL_H_ */
