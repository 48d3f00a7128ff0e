/*
 * adds.h — C ABI of the B200-native asynchronous delta-stepping SSSP engine.
 *
 * The reference (UCLA-VAST/adds) has no library API: its only boundary is the
 * `sssp` process (ads_int/support.cu:11-76, ads_int/kernel.cu:290-305) plus the
 * CSR graph object handed to gg_main (ads_int/kernel.cu:185) and the host half
 * of the worklist (ads_int/wl.h:160-165).  Every entry point below names the
 * reference interface it replaces.  All functions return 0 (ADDS_OK) or a
 * negative ADDS_ERR_* code; none of them calls exit() or traps on the device.
 *
 * Conventions
 *   - Vertex ids are uint32 (reference index_type is `unsigned`,
 *     ads_int/csr_graph.h:20); edge counts must be < 2^32 for the same reason.
 *   - Distances are 32-bit words: int32 for ADDS_I32 graphs (INF = INT32_MAX,
 *     ads_int/csr_graph.h:23) and float32 for ADDS_F32 graphs
 *     (INF = FLT_MAX, ads_float/csr_graph.h:49).
 *   - Weights must be non-negative (int32 in [0, INT32_MAX], float32 >= 0 and
 *     not NaN).  -0.0f is stored as +0.0f (same sums).
 *   - A pointer argument documented as "host or device" is classified with
 *     cudaPointerGetAttributes; device pointers must live on the graph's GPU.
 *   - Handles are not thread-safe: concurrent calls on one handle race;
 *     distinct handles may be used from distinct threads.
 */
#ifndef ADDS_H_
#define ADDS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ADDS_ABI_VERSION 2

typedef enum { ADDS_I32 = 0, ADDS_F32 = 1 } adds_wtype;

enum {
  ADDS_OK = 0,
  ADDS_ERR_INVALID = -1,        /* bad argument                                  */
  ADDS_ERR_IO = -2,             /* file could not be opened/read/written         */
  ADDS_ERR_FORMAT = -3,         /* malformed .gr file                             */
  ADDS_ERR_OOM = -4,            /* device or host allocation failed               */
  ADDS_ERR_CUDA = -5,           /* a CUDA runtime call failed                     */
  ADDS_ERR_DEVICE_TIMEOUT = -6, /* a bounded device wait ran out                  */
  ADDS_ERR_WL_OVERFLOW = -7,    /* worklist pool exhausted after all regrowths    */
  ADDS_ERR_NO_DEVICE = -8,      /* no usable sm_100 device                        */
  ADDS_ERR_UNSUPPORTED = -9     /* request outside what this build supports       */
};

#define ADDS_INF_I32 0x7FFFFFFF
#define ADDS_INF_F32_BITS 0x7F7FFFFFu /* FLT_MAX */

typedef struct adds_graph adds_graph; /* device-resident CSR, library-owned */
typedef struct adds_batch adds_batch; /* many solves in one persistent launch */

/* Solver knobs.  Zero / negative means "choose automatically".
 * Replaces the compile-time tuning of ads_int/wl.h:14-25,777-849 and the
 * runtime delta choice of worklist::set_param (ads_int/wl.h:395-449). */
typedef struct adds_opts {
  void *stream;          /* cudaStream_t to run on; NULL = per-graph stream      */
  int32_t delta_shift;   /* bucket width 2^shift key units; <0 = auto            */
  float delta_scale;     /* float graphs: key = floor(dist*scale); <=0 = auto   */
  int32_t window;        /* buckets popped concurrently (1..32); 0 = auto        */
  int32_t ctas_per_sm;   /* persistent CTAs per SM; 0 = auto                     */
  int32_t batch_max;     /* max vertices one CTA pops per batch; 0 = auto        */
  int32_t hub_threshold; /* out-degree above which a row is split across CTAs   */
  int32_t timeout_ms;    /* bound on every device wait; 0 = 20000 ms             */
  int32_t adapt;         /* on-device bucket widening.  Phase engine: the leader
                            merges up to 4 thin consecutive bucket slots into
                            one light phase.  Async engine: the window of
                            buckets processed at once grows by one while CTAs
                            find nothing inside it but entries beyond it, and
                            shrinks back towards `window` as the base bucket
                            retires with no CTA idle.  -1 auto (the tuned
                            value, else on in the async engine and off in
                            the phase engine), 0 off, 1 on                  */
  int32_t strict_order;  /* 1: advance a bucket only when its work is done       */
  int32_t local_max;     /* own pushes a CTA keeps as its next batch; <0 = auto,
                            0 = always go through the HBM queues              */
  int32_t light_heavy;   /* 1: relax heavy edges (w >= delta) once per settled
                            vertex from a weight-sorted row copy; 0: off;
                            2 (phase engine): per bucket — split rows while a
                            bucket keeps re-improving its own vertices, whole
                            rows in one light phase once buckets turn sparse
                            (the asynchronous engine treats 2 as 1);
                            <0 = auto (2 phase engine, 1 async)              */
  int32_t block_threads; /* threads per persistent CTA: async engine 128, 256 or
                            512; phase engine 256, 512 or 1024; 0 = auto       */
  int32_t greed;         /* async engine: a claim takes avail / (CTAs >> greed)
                            entries; <0 = auto                                 */
  int32_t engine;        /* ADDS_ENGINE_*: 0 = auto (phase)                      */
  int32_t group_ctas;    /* phase engine: CTAs that solve one query together
                            (batches: the group size; plain solves: the CTAs
                            launched, fewer making each phase's barrier
                            cheaper on small graphs); 0 = auto              */
  int32_t solo_max;      /* phase engine: frontiers of at most this many entries
                            run on one CTA without a group barrier; <0 = auto  */
  int32_t near_far;      /* phase engine, 1: near-far schedule (the Galois GPU
                            nf comparator, nf_int.patch): one far pile instead
                            of the bucket ring, split against a threshold that
                            moves one bucket at a time (or to the smallest
                            bucket in the pile); 0 = bucket ring             */
  int32_t dense_scan;    /* phase engine: a bucket slot that receives more than
                            max(n >> dense_scan, 4096) pushes stops storing
                            them, and its bucket is collected by one pass over
                            the distances when it opens (no duplicate or stale
                            entries); 0 = auto (off unless tuned), < 0 = off,
                            6 = n/64                                        */
  int32_t pull;          /* phase engine, light/heavy split on: the heavy edges
                            of a large settled bucket may be relaxed as a pull
                            -- every vertex they could still improve takes the
                            minimum over its in-edges -- when a count over the
                            distances finds that this reads fewer edges than
                            the push.  Keeps a transposed copy of the graph
                            (8 B per edge, built on first use).  0 = auto
                            (on), < 0 = off, 1 = on                         */
  int32_t reserved[2];
} adds_opts;

/* Engines.  PHASE settles the buckets in bulk-synchronous phases (light
 * edges to convergence, then heavy edges once) with the frontier spread
 * over every CTA; ASYNC pops and pushes bucket entries asynchronously with
 * per-bucket counters, as the reference's worklist does. */
enum { ADDS_ENGINE_AUTO = 0, ADDS_ENGINE_ASYNC = 1, ADDS_ENGINE_PHASE = 2 };

/* Per-solve statistics (reference: work_count + fd-3 record,
 * ads_int/kernel.cu:264-282). */
typedef struct adds_stats {
  double ms;                /* device time of the solve(s), CUDA events        */
  double kernel_ms;         /* of which the persistent solver kernel(s)        */
  uint64_t items_popped;    /* queue entries popped (reference int work count) */
  uint64_t items_stale;     /* popped entries skipped as superseded            */
  uint64_t edges_scanned;   /* edges of expanded vertices (float work count)   */
  uint64_t pushes;          /* queue entries pushed                            */
  uint64_t batches;         /* CTA-level pops (phase engine: frontier chunks)  */
  uint64_t hub_chunks;      /* split row chunks processed                      */
  uint64_t hub_stale;       /* of which skipped (row's vertex had improved)    */
  uint64_t local_batches;   /* batches a CTA took from its own pushes          */
  uint64_t heavy_lists;     /* settled vertices whose heavy edges were relaxed */
  uint64_t phase_cycles[6]; /* SM cycles summed over CTAs.  Async engine:
                               acquire, load, edges, flush, idle, total.
                               Phase engine: chunk preparation, split-row
                               record preparation (waits included), edge
                               expansion, flushes, group-barrier wait, leader
                               (solo phases included)                         */
  uint64_t mid_flush_cycles; /* async: edge-phase flushes of a full buffer;
                                phase: cycles in grid phases                  */
  uint64_t mid_flushes;     /* async: their count; phase: total cycles        */
  uint64_t reached;         /* vertices with finite distance (filled on request) */
  uint64_t reached_edges;   /* out-edges of reached vertices (filled on request) */
  int32_t delta_shift;      /* bucket shift at the end of the solve            */
  int32_t retries;          /* worklist regrowths needed                       */
  int32_t ctas;             /* persistent CTAs launched                        */
  int32_t engine;           /* ADDS_ENGINE_ASYNC or ADDS_ENGINE_PHASE          */
  int32_t launches;         /* kernel launches per solve: async 2 (init, solver);
                               phase 1, or 5 with pull phases possible (phase,
                               pull, phase, pull, phase; unused ones return at
                               once)                                         */
  int32_t reserved[3];
  uint64_t phases;          /* phase engine: phases decided (solo included)    */
  uint64_t solo_phases;     /* phase engine: phases run by one CTA             */
  uint64_t repushes;        /* phase engine: far-slot entries moved on         */
} adds_stats;

typedef struct adds_graph_info_t {
  uint32_t n;
  uint64_t m;
  adds_wtype wtype;
  int device;
  uint32_t max_degree;
  double avg_degree;
  double avg_weight;      /* sampled mean weight (as ads_int/kernel.cu:153-183) */
  uint64_t device_bytes;  /* bytes held on the GPU by the graph                  */
} adds_graph_info_t;

/* ---- library ------------------------------------------------------------ */
int adds_abi_version(void);
const char *adds_strerror(int code);
void adds_opts_init(adds_opts *o);
/* Last CUDA error text seen by this thread (diagnostics only). */
const char *adds_last_cuda_error(void);

/* ---- graphs ------------------------------------------------------------- */
/* Replaces CSRGraph::read/readFromGR + copy_to_gpu
 * (ads_int/csr_graph.cu:203-296,309-328; float: ads_float/csr_graph.cu).
 * Galois .gr v1 layout: u64 version=1, u64 sizeEdgeTy, u64 n, u64 m,
 * u64 out_end[n], u32 dst[m], (u32 pad if m odd), u32|f32 w[m].
 * sizeEdgeTy==0 gives all-zero weights, as the reference does. */
int adds_graph_load_gr(const char *path, adds_wtype wt, int device,
                       adds_graph **out);
/* Builds a device graph from host CSR arrays (copied; caller keeps them).
 * row_start has n+1 entries, row_start[0]==0, row_start[n]==m. */
int adds_graph_from_csr(uint32_t n, uint64_t m, const uint64_t *row_start,
                        const uint32_t *dst, const void *w, adds_wtype wt,
                        int device, adds_graph **out);
int adds_graph_info(const adds_graph *g, adds_graph_info_t *info);
/* Copies the CSR back to host buffers (any may be NULL).  Replaces
 * CSRGraph::copy_to_cpu (ads_int/csr_graph.cu:330-350) minus the distances. */
int adds_graph_download(const adds_graph *g, uint64_t *row_start, uint32_t *dst,
                        void *w);
/* Overwrites the m edge weights (host or device pointer, CSR order). */
int adds_graph_set_weights(adds_graph *g, const void *w);
/* Writes the graph as a Galois .gr v1 file (input side of run_all.sh). */
int adds_graph_save_gr(const adds_graph *g, const char *path);
void adds_graph_free(adds_graph *g);

/* Seeded synthetic generators, run on the GPU; identical to the numpy
 * generators in adds_b200/graphs.py.  kind: 0 = R-MAT, 1 = 2-D grid with
 * local shortcuts, 2 = Erdos-Renyi, 3 = plain 2-D grid. */
typedef struct adds_gen_spec {
  int32_t kind;
  int32_t scale;        /* R-MAT: n = 2^scale                                 */
  int32_t edge_factor;  /* R-MAT / ER: directed draws = edge_factor * n       */
  uint32_t n;           /* ER: vertex count                                   */
  uint32_t side_x, side_y; /* grids                                           */
  double a, b, c;       /* R-MAT quadrant probabilities (d = 1-a-b-c)         */
  double shortcut_frac; /* grid: shortcut pairs = frac * grid edges           */
  int32_t shortcut_radius;
  adds_wtype wtype;
  double w_lo, w_hi;    /* int: uniform [lo,hi]; float: uniform [lo,hi)       */
  uint64_t seed;
} adds_gen_spec;
int adds_graph_generate(const adds_gen_spec *spec, int device, adds_graph **out);

/* ---- plain solve -------------------------------------------------------- */
/* One SSSP from src.  Replaces gg_main's solve (ads_int/kernel.cu:185-288):
 * init kernel, profiler_kernel + set_param delta choice, and the
 * driver_kernel/wl_kernel/sssp_kernel pair, as one init + one persistent
 * cooperative launch.  dist_out (n words, host or device) may be NULL to keep
 * the result on the device (read it with adds_graph_last_dist). */
int adds_sssp(adds_graph *g, uint32_t src, void *dist_out, const adds_opts *opts,
              adds_stats *stats);
/* Enqueues a solve on the graph's stream and returns at once (no host
 * synchronisation); adds_graph_sync waits for all enqueued solves and
 * reports the first device error.  A solve that ran out of worklist space
 * (ADDS_ERR_WL_OVERFLOW) is not an error there: the pool grows and the
 * enqueued solves run again one at a time, as adds_sssp does.  The
 * distances of the last solve stay in the graph. */
int adds_sssp_async(adds_graph *g, uint32_t src, const adds_opts *opts);
int adds_graph_sync(adds_graph *g, adds_stats *stats);
/* Copies the distances of the last solve on g (host or device pointer). */
int adds_graph_last_dist(adds_graph *g, void *dist_out);
/* Several sources on one graph, one solve each, result i in dist_out[i]
 * (n words each, host or device; an entry may repeat a buffer, later results
 * overwrite earlier ones).  Replaces the reference's one-process-per-source
 * loop (run_all.sh:4-18 calls `sssp -s <src>` per source; gg_main,
 * ads_int/kernel.cu:185-288, copies the result back after the solve): here
 * the copy of result i to host memory runs on a second stream while solve
 * i+1 runs.  stats sums the solve times; the other counters are the last
 * solve's. */
int adds_sssp_sources(adds_graph *g, const uint32_t *srcs, uint32_t ns, void *const *dist_out,
                      const adds_opts *opts, adds_stats *stats);
/* Fills stats->reached and stats->reached_edges for the last solve on g. */
int adds_graph_reached(adds_graph *g, uint64_t *reached, uint64_t *reached_edges);

/* ---- batched solves ----------------------------------------------------- */
/* nq solves (graph graphs[i], source srcs[i]) run in ONE persistent launch
 * with per-query bucket queues sharing one page pool; the launch is captured
 * in a CUDA graph on first run and replayed afterwards.  No reference
 * counterpart (the reference runs one source per process).  Each query
 * takes its graph's tuned bucket width (else the heuristic).  The
 * launch-wide knobs are opts' or the defaults, not a graph's tuned ones
 * (those are for a plain solve that has the whole GPU).  With opts->engine
 * 0 the engine follows the largest query's graph: asynchronous for an
 * average degree under 6 (grids, road networks), phase otherwise. */
int adds_batch_create(adds_graph *const *graphs, const uint32_t *srcs,
                      uint32_t nq, const adds_opts *opts, adds_batch **out);
int adds_batch_run(adds_batch *b, adds_stats *stats);
/* Enqueues a run on the batch's stream without waiting; adds_batch_sync
 * waits and reports device errors. */
int adds_batch_launch(adds_batch *b);
int adds_batch_sync(adds_batch *b, adds_stats *stats);
int adds_batch_dist(adds_batch *b, uint32_t q, void *dist_out);
/* All queries' distances in one copy: query q occupies out[offsets[q] ..
 * offsets[q] + n_q) (words; offsets are padded to 32-word multiples) and
 * *total words are written.  out (host or device) may be NULL to only fill
 * offsets (nq entries) and *total. */
int adds_batch_dist_all(adds_batch *b, void *out, uint64_t *offsets, uint64_t *total);
/* Device pointer to query q's distance array (valid until adds_batch_free). */
int adds_batch_dist_ptr(adds_batch *b, uint32_t q, void **dptr);
int adds_batch_set_sources(adds_batch *b, const uint32_t *srcs);
void adds_batch_free(adds_batch *b);

/* ---- adjoint (backward) ------------------------------------------------- */
/* Float graphs only.  For every query q of the batch, takes dL/d dist_q
 * (n_q floats, device pointer) and ACCUMULATES dL/dw into grad_w[g] (m_g
 * floats, device pointer) for each distinct graph, summing over queries in
 * query order.  The predecessor of v is the tight in-edge (u->v) with
 * fl(d[u]+w)==d[v] and d[u]<d[v] of smallest CSR index; zero-gap ties are
 * resolved breadth-first, again by smallest index.  No reference counterpart. */
int adds_batch_backward(adds_batch *b, const float *const *grad_dist,
                        float *const *grad_w);
/* Single-graph convenience: ns solves from srcs, dist/grad_dist are [ns][n]
 * device arrays laid out row-major, grad_w (m floats, device) is overwritten. */
int adds_sssp_backward(adds_graph *g, uint32_t ns, const uint32_t *srcs,
                       const float *dist, const float *grad_dist, float *grad_w,
                       const adds_opts *opts);

/* ---- solve without allocating -------------------------------------------- */
/* No counterpart in the reference.  For callers that may not let a library
 * allocate device memory: a framework that owns all device memory through
 * its own allocator or a fixed arena (a foreign cudaMalloc takes memory
 * outside its budget; cudaFree synchronises the device), or a service loop
 * that cannot afford those implicit synchronisations.  Nothing is allocated:
 * the caller passes device arrays it owns, and the engine's working memory
 * is one fixed device array of ADDS_NOALLOC_SCRATCH_BYTES inside this
 * library, held on every GPU that loads the library until the process
 * exits.
 *   row_start: n+1 u32 row offsets; edges: 2*m u32 words, {dst, weight bits}
 *   per edge in CSR order; dist: n words, overwritten (same INF values as
 *   adds_sssp); all three on the current device.  stream: cudaStream_t or
 *   NULL.  The call waits once for that stream, at its end, and returns
 *   after the solve has finished.
 * The arrays are checked on the device before the solver reads them (row
 * offsets start at 0, never decrease and end at m; dst < n; weights not
 * negative and, for floats, not NaN; -0.0f is accepted and sums like
 * +0.0f); a failed check returns ADDS_ERR_FORMAT with dist untouched.
 * Graphs above ADDS_NOALLOC_MAX_N vertices or ADDS_NOALLOC_MAX_M edges are
 * rejected (ADDS_ERR_UNSUPPORTED); a graph within the limits whose queues
 * outgrow the fixed pool reports ADDS_ERR_WL_OVERFLOW.  The first call on a
 * device looks up the array's device address and prepares the kernels for
 * that device.  All calls share the array (each clears what it needs
 * first): calls that overlap on the GPU race, so issue them one after
 * another. */
#define ADDS_NOALLOC_SCRATCH_BYTES (64u << 20)
#define ADDS_NOALLOC_MAX_N (1u << 20)
#define ADDS_NOALLOC_MAX_M (1u << 24)
int adds_sssp_noalloc(uint32_t n, uint64_t m, const uint32_t *row_start,
                      const uint32_t *edges, adds_wtype wt, uint32_t src,
                      uint32_t *dist, void *stream);

/* ---- phase trace (diagnostics) ------------------------------------------ */
/* One record per phase the phase engine decided, in order (the leader's
 * %globaltimer at the decision; a phase lasts until the next record).
 * Extends the reference's per-run work record (ads_int/kernel.cu:264-282)
 * down to the phase; the reference has no tracing of its own. */
typedef struct adds_phase_trace {
  uint64_t t_ns;  /* device clock at the decision, ns                       */
  uint32_t count; /* frontier entries (split rows: chunks; init: vertices)   */
  uint16_t mode;  /* 0 init, 1 light, 2 heavy, 3 split rows, 4 exit,
                     6 scan (a dense bucket collected from the distances);
                     | 0x100 when one CTA ran it alone                      */
  uint16_t base;  /* low 16 bits of the bucket being settled                */
  uint32_t edges;   /* edges the phase relaxed                              */
  uint32_t items;   /* frontier entries and split-row records it prepared   */
  uint32_t pushes;  /* entries it appended to the bucket lists               */
  uint32_t tail_ns; /* from the first CTA reaching the phase's barrier to the
                       next decision: the phase's load imbalance (0 solo)   */
} adds_phase_trace;
/* Records up to cap phases of each later plain solve on g (0 = off). */
int adds_graph_trace(adds_graph *g, uint32_t cap);
/* Copies the last solve's records (at most cap) to host memory; *written
 * receives how many the solve produced (it may exceed the capacity). */
int adds_graph_trace_read(adds_graph *g, adds_phase_trace *out, uint32_t cap,
                          uint64_t *written);

/* ---- relaxation ceiling (diagnostics) ----------------------------------- */
/* No counterpart in the reference.  Solves from src, then times one pass over
 * every edge of g with those final distances resident, four ways: ms_out[0]
 * streaming each edge and its source's distance (12 B per edge), [1] the same
 * plus the random gather of dist[dst] and the comparison, [2] plus a
 * min-reduction where the comparison succeeds, [3] a min-reduction on every
 * edge without the gather.  [1] bounds any push-based relaxation schedule on
 * this GPU.  Allocates (the pass needs 4 B per edge and two distance arrays). */
int adds_diag_relax_pass(adds_graph *g, uint32_t src, double ms_out[4]);
/* Failure-detection check, no counterpart in the reference (whose worklist
 * traps with a device assert, ads_int/wl.h:614-619): one thread waits, through
 * the engine's bounded barrier wait, for a flag that nothing sets.  After
 * timeout_ms (1..10000) the wait gives up and the call returns
 * ADDS_ERR_DEVICE_TIMEOUT with the GPU context intact; waited_ms (may be
 * NULL) receives the kernel's duration. */
int adds_diag_wait_timeout(int device, int timeout_ms, double *waited_ms);

/* ---- autotuner ---------------------------------------------------------- */
/* Times candidate settings on the sample sources and stores the fastest in
 * the graph (used whenever a later call passes "auto" knobs): delta, then for
 * the phase engine the kernel variant (threads x CTAs per SM), the solo
 * threshold, the split-row threshold and the light/heavy split; for the async
 * engine window, batch, hub threshold, block, greed, CTAs/SM, order and local
 * chaining.  best may be NULL; if not, best->engine selects the engine to
 * tune on input (0 = auto) and *best receives the winner. */
int adds_tune(adds_graph *g, const uint32_t *srcs, uint32_t ns,
              adds_opts *best, double *best_ms);

/* ---- text output -------------------------------------------------------- */
/* Writes n lines "<v> <dist>" / "<v> INF" exactly as support.cu:78-97 (int,
 * "%d %d") and the Galois float writer (cpu_sssp_float.patch:241-247,
 * "%d %f").  dist is a host array of 32-bit words. */
int adds_write_dist_text(const char *path, uint32_t n, const void *dist,
                         adds_wtype wt);

#ifdef __cplusplus
}
#endif
#endif /* ADDS_H_ */
