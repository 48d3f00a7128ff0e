/*
 * phase_internal.h — device data layout of the bulk-synchronous bucket
 * engine (phase.cu).
 *
 * The reference worklist (ads_int/wl.h:133-190) keeps 32 circular distance
 * buckets as virtual ranges of a paged HBM pool and lets workers pop and push
 * asynchronously under three manager warps (wl.h:488-1527).  This engine keeps
 * the bucket ring and the paged pool but runs the buckets in phases: a group
 * of CTAs expands one frontier (a range of one list), meets at a group
 * barrier, and the last CTA to arrive (the leader) decides the next frontier.
 * Inside a phase nothing waits for anything but a page mapping, so the edge
 * stream runs at full width; between phases the leader's decision is one read
 * of a few list tails.
 *
 * Lists are append-only for the life of the engine: a list is a monotone
 * 64-bit index space [head, tail) whose 4096-entry virtual pages map to pool
 * pages through a per-list ring of page-table cells tagged with the virtual
 * page number.  Pool pages are handed out by a per-group bump counter that is
 * reset when the group starts a query (the lists of the previous query are
 * empty by then), so nothing is ever freed or recycled inside a solve.
 */
#ifndef ADDS_PHASE_INTERNAL_H_
#define ADDS_PHASE_INTERNAL_H_

#include <stdint.h>

#define PH_NSLOT 64                /* bucket ring (the reference has 32 bags)   */
#define PH_LNEXT PH_NSLOT          /* list: current bucket's next frontier     */
#define PH_LSETTLED (PH_NSLOT + 1) /* list: settled vertices with heavy edges  */
#define PH_NLIST (PH_NSLOT + 2)
#define PH_LFAR (PH_NSLOT - 1)     /* near-far schedule: the far pile          */
#define PH_PAGE_LOG2 12
#define PH_PAGE (1u << PH_PAGE_LOG2) /* entries per pool page (8 B each)      */

/* phase modes */
#define PH_M_INIT 0u   /* fill the query's distances with INF                 */
#define PH_M_LIGHT 1u  /* expand light edges of a list range                  */
#define PH_M_HEAVY 2u  /* expand heavy edges of settled vertices              */
#define PH_M_HUB 3u    /* (reserved: split rows are expanded inside their phase) */
#define PH_M_EXIT 4u   /* no more queries for this group                      */
#define PH_M_SCAN 6u   /* collect a dense bucket from the distances into NEXT  */
#define PH_M_PULL 7u   /* heavy phase as a pull: every vertex above the bucket
                          takes the minimum over its in-edges                */

/* device error codes (first one wins) */
#define PH_ERR_TIMEOUT 1u
#define PH_ERR_OVERFLOW 2u
#define PH_ERR_HUB_OVERFLOW 3u
#define PH_ERR_MAPPING 4u
#define PH_ERR_INPUT 5u    /* caller's arrays failed validation (no-alloc path);
                              err_where holds the failed checks            */

/* Read-only per-query descriptor. */
struct PhQuery {
  const unsigned *row;   /* n+1 row offsets                                   */
  const uint2 *edges;    /* m x {dst, weight bits}; rows weight-sorted when
                            split != NULL                                     */
  const unsigned *split; /* light edges (w < delta) at the start of each row  */
  unsigned *dist;        /* n distance words                                  */
  unsigned n;
  unsigned src;
  float scale;           /* float graphs: key = floor(d * scale)              */
  unsigned shift;        /* bucket = key >> shift                             */
  unsigned long long m;
  /* in-edge CSR (the transposed graph: {tail vertex, weight bits} per edge)
   * for heavy phases run as a pull; NULL = push only */
  const unsigned *trow;
  const uint2 *tedges;
};

/* One split-row chunk: edges [eb, ee) of vertex v expanded with distance d. */
struct __align__(16) PhHub {
  unsigned v, d, eb, ee;
};

/* What every CTA of a group needs for one phase (written by the leader before
 * it releases the barrier; double-buffered by barrier generation). */
#define PH_MAXR 4 /* list ranges one light phase may read (widened bucket) */
/* launches of the phase kernel one solve may be split into by pull phases
 * (each pull runs in a kernel between two of them) */
#define PH_PULL_SEGMENTS 2u
#define PH_SAMPLE_STRIDE 16u /* a sampling heavy scan reads every 16th tile */
struct __align__(64) PhDesc {
  unsigned mode;
  unsigned q;                  /* query index                                */
  unsigned list;               /* list the frontier is read from             */
  unsigned base;               /* absolute bucket being settled              */
  unsigned long long lo, hi;   /* entry range of the list (hub: record range) */
  unsigned long long work_base; /* claim counter value at phase start        */
  unsigned per;                /* entries per claim                           */
  unsigned epoch;              /* phase number: marks its split-row records    */
  /* a light phase whose bucket the leader widened over thin slots reads
   * nx further ranges after (list, lo, hi) */
  unsigned nx;
  unsigned xl[PH_MAXR - 1];
  unsigned long long xlo[PH_MAXR - 1], xhi[PH_MAXR - 1];
  unsigned full;               /* light phase relaxes whole rows, no SETTLED */
  unsigned sample;             /* heavy scan that only counts push and pull
                                  work, over one tile in PH_SAMPLE_STRIDE  */
  unsigned pad[2];
};

/* Per-group state.  `arrive` and `gen` sit in lines of their own; the list
 * tails are hit by reservations from every CTA of the group, each in its own
 * 128-byte line. */
struct __align__(128) PhTail {
  unsigned long long tail;
  unsigned long long pad[15];
};

struct __align__(128) PhGroup {
  unsigned arrive;
  unsigned pad0[31];
  unsigned gen;
  unsigned pad1[31];
  unsigned long long work;     /* chunk claim counter (monotone)             */
  unsigned long long pad2[15];
  unsigned hub_count;          /* split-row records appended this phase      */
  unsigned pad3[31];
  unsigned hub_claim;          /* split-row records claimed this phase       */
  unsigned pad3b[31];
  unsigned producers;          /* CTAs that may still append records         */
  unsigned pad3c[31];
  unsigned page_next;          /* bump allocator: next free page (relative)  */
  unsigned pad4[31];
  PhDesc desc[2];
  /* leader-only control state */
  unsigned q;                  /* current query                              */
  unsigned base;               /* absolute base bucket                       */
  unsigned mode;               /* mode of the phase that just ran            */
  unsigned epoch;              /* phases decided so far                      */
  /* trace of group 0 only: the running phase's work and its first arrival */
  unsigned long long tr_first, tr_edges, tr_items, tr_pushes;
  /* adaptive light/heavy: entries of the bucket's last light phase, light
   * phases run in it, whether it re-improved many of its own vertices */
  unsigned long long lh_prev;
  unsigned lh_k, lh_dense;
  /* near-far schedule: smallest bucket pushed to the far list since the
   * threshold last moved */
  unsigned far_min;
  /* first light phase of a bucket opened by a scan: whole rows or not */
  unsigned lh_full;
  /* the settled list of the current bucket may not be rebuilt by a heavy
   * scan: it was already, or a light phase relaxed whole rows, or the
   * bucket was widened over several slots */
  unsigned hs_block;
  unsigned pad5[13];
  /* dense bucket slots (bit per slot): a slot whose pushes passed the dense
   * threshold stops storing entries; its bucket is collected by a scan of
   * the distances when it opens (PH_M_SCAN) */
  unsigned long long dmask;
  /* slots holding far-slot entries (buckets beyond the ring when they were
   * pushed): such a slot never turns dense, since a scan collects one bucket
   * only; the bit clears when the slot opens and its entries move on */
  unsigned long long fmask;
  unsigned long long pad6[14];
  unsigned long long head[PH_NLIST];
  PhTail tails[PH_NLIST];
  /* pull or push for a settled bucket's heavy edges (kept after the other
   * fields, which keep their offsets): a sampling heavy scan sums the heavy
   * out-edges of the bucket (pc_push) and the in-edges of every vertex a
   * heavy edge could still improve (pc_pull) over the same sample; pc_state
   * is 1 while those sums belong to the decision about to be made, 2 right
   * after it chose push (no second sample).  wide: the current bucket was
   * widened over several slots, so its settled list holds vertices of lower
   * buckets too (no pull). */
  unsigned pc_state;
  unsigned wide;
  unsigned pad7[30];
  unsigned long long pc_push, pc_pull;
  unsigned long long pad8[14];
};

/* Engine-wide control and statistics. */
struct __align__(128) PhGlobal {
  unsigned err;
  unsigned err_where;
  unsigned pad0[30];
  unsigned next_q;             /* batch: next query to hand to a group       */
  unsigned pad1[31];
  unsigned long long st_items, st_stale, st_edges, st_pushes, st_chunks, st_hub,
      st_phases, st_solo, st_heavy, st_repush, st_pages;
  unsigned long long st_cyc[8]; /* SM cycles summed over CTAs: entry chunk
                                   preparation, record preparation (with its
                                   waits), expansion, flushes, barrier wait,
                                   leader (solo phases included), grid-phase
                                   work, total                                */
  unsigned long long st_trace;  /* trace records written (may exceed the cap) */
};

/* One record of the phase trace (group 0 only): when the leader decided a
 * phase, what it was and how big. */
struct PhTrace {
  unsigned long long t_ns;  /* %globaltimer at the decision                  */
  unsigned count;           /* entries (hub: chunk records; init: vertices)   */
  unsigned short mode;      /* PH_M_* | 0x100 if run by the leader alone      */
  unsigned short base;      /* low 16 bits of the base bucket                 */
  unsigned edges;           /* edges the phase relaxed                        */
  unsigned items;           /* entries and records it prepared                */
  unsigned pushes;          /* entries it appended                           */
  unsigned tail_ns;         /* first CTA at the barrier to the decision       */
};

/* Kernel parameters (by value). */
struct PhParams {
  const PhQuery *qs;
  const unsigned *order;       /* query order (largest first); NULL = 0..nq-1 */
  unsigned nq;
  unsigned groups;             /* CTA groups; gridDim.x = groups * gsize      */
  unsigned gsize;              /* CTAs per group                             */
  PhGroup *grp;                /* [groups]                                   */
  PhGlobal *g;
  unsigned long long *pool;    /* groups * pages_per_group * PH_PAGE entries  */
  unsigned pages_per_group;
  unsigned long long *pt;      /* groups * PH_NLIST << ptn_log2 cells         */
  unsigned ptn_log2;
  PhHub *hub;                  /* groups * hub_cap records                    */
  unsigned *hub_seq;           /* groups * hub_cap: epoch of each written record */
  unsigned hub_cap;
  unsigned hub_threshold;      /* rows with more expanded edges are split     */
  unsigned hub_chunk;          /* edges per split chunk                       */
  unsigned solo_max;           /* frontiers up to this size run on the leader */
  unsigned adapt;              /* merge thin bucket slots into one phase      */
  unsigned lh_adapt;           /* whole rows in light phases of sparse buckets */
  unsigned near_far;           /* two lists instead of the bucket ring         */
  unsigned dense_shift;        /* a bucket slot that receives more than
                                  max(n >> dense_shift, 4096) pushes turns
                                  dense (collected by a scan); 0 = never      */
  unsigned is_float;
  /* pull phases (one query per launch): the leader may pick PH_M_PULL,
   * which ends this launch; the pull kernel runs the phase and a launch
   * with resume = 1 continues from its descriptor */
  unsigned pull_ok;
  unsigned resume;
  unsigned single_src;         /* overrides query 0's source when != ~0       */
  unsigned long long timeout_ns;
  PhTrace *trace;              /* optional phase trace of group 0              */
  unsigned trace_cap;
};

#ifdef __cplusplus
#include <cuda_runtime.h>
#include <vector>

/* Host-side handle of one engine instance (phase.cu). */
struct PhEngine {
  int device = -1;
  bool flt = false;
  unsigned nq = 0, groups = 0, gsize = 0, block = 0, variant = 0;
  int req_group = 0; /* group_ctas knob the engine was sized with */
  unsigned pages_per_group = 0, ptn_log2 = 0, hub_cap = 0, max_n = 0;
  unsigned hub_eff = 0; /* split-row chunk length the record store is sized for */
  PhGroup *grp = nullptr;
  PhGlobal *g = nullptr;
  PhQuery *qs = nullptr;
  unsigned *order = nullptr;
  unsigned long long *pool = nullptr, *pt = nullptr;
  PhHub *hub = nullptr;
  unsigned *hub_seq = nullptr;
  PhGlobal *g_host = nullptr; /* pinned copy of the statistics and error word */
  PhTrace *trace = nullptr;    /* phase trace buffer (allocated on request)  */
  unsigned trace_cap = 0;
  std::vector<PhQuery> qs_host;
  size_t bytes = 0;
  int num_sms = 0;
};

/* knobs of one launch */
struct PhKnobs {
  int variant;        /* kernel variant (threads x CTAs per SM), phase.cu      */
  int ctas_per_sm;    /* <= 0: as many as fit                                 */
  int group_ctas;     /* CTAs per group (batches); <= 0: automatic            */
  unsigned hub_threshold, hub_chunk, solo_max, adapt, lh_adapt;
  unsigned near_far;  /* near-far schedule instead of the bucket ring          */
  unsigned dense_shift; /* dense bucket slots (PhParams::dense_shift), 0 = off  */
  unsigned long long timeout_ns;
};


/* phase.cu host API (C++ linkage) */
int adds_phase_variant_block(int variant);
cudaError_t adds_phase_prepare(bool flt, int variant, int *max_blocks_per_sm);
/* pull = true launches the pull kernel of a launch chain (ph_engine_enqueue) */
cudaError_t adds_phase_launch(const PhParams &P, int variant, cudaStream_t st, bool pull = false);
int ph_engine_alloc(PhEngine &E, int device, bool flt, const std::vector<PhQuery> &qv,
                    const PhKnobs &k, unsigned grow, cudaStream_t st);
void ph_engine_free(PhEngine &E);
int ph_engine_reset(PhEngine &E, cudaStream_t st);
/* bounded wait on a flag nothing sets (failure-detection check): the error
 * word and wait site it left, and how long the kernel ran */
int ph_diag_wait(int device, unsigned timeout_ms, unsigned *err, unsigned *where,
                 float *waited_ms);
int ph_engine_upload(PhEngine &E, cudaStream_t st);
int ph_engine_params(const PhEngine &E, const PhKnobs &k, unsigned single_src, PhParams *P);
int ph_engine_enqueue(PhEngine &E, const PhParams &P, cudaStream_t st, cudaEvent_t k0,
                      cudaEvent_t k1);
int ph_engine_status(const PhEngine &E, char *msg, size_t msg_len);
int ph_engine_trace(PhEngine &E, unsigned cap);
unsigned ph_hub_chunk(const PhKnobs &k); /* effective split-row chunk length */
#endif

#endif /* ADDS_PHASE_INTERNAL_H_ */
