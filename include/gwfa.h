/*
 * gwfa.h — drop-in C ABI of the B200 GWFA sequence-to-graph edit-distance path.
 *
 * The graph types keep the exact layout of the reference's gwfa.h:6-18, so a caller that
 * already builds a gwf_graph_t (for example through gwf_gfa2gwf, main.cu:294-345) passes it
 * unchanged. Every entry point is plain C: pointers and sizes, no CUDA or C++ types.
 *
 * Error model: functions returning int return 0 on success or a negative GWF_E_* code.
 * gwf_ed returns the distance (>= 0), -1 when no alignment exists (reference behaviour,
 * gwf-ed.cu:1336), or a GWF_E_* code (<= -2). gwf_last_error() gives a message for the
 * last failure in the calling thread.
 */
#ifndef GWFA_B200_H
#define GWFA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- graph types: same layout as the reference (gwfa.h:6-18) ---- */
typedef struct {
	uint64_t a; /* source vertex << 32 | target vertex */
	int32_t o;  /* overlap on the target: the walk enters the target at offset o */
} gwf_arc_t;

typedef struct {
	uint32_t n_vtx, n_arc;
	uint32_t *len;   /* vertex lengths */
	uint32_t *src;   /* original oriented GFA vertex (segment << 1 | strand) */
	char **seq;      /* NUL-terminated vertex sequences */
	gwf_arc_t *arc;  /* arcs; sorted by a after gwf_ed_index */
	uint64_t *aux;   /* CSR: first_arc << 32 | n_arcs per vertex, filled by gwf_ed_index */
} gwf_graph_t;

/* ---- status / error codes ---- */
#define GWF_OK               0
#define GWF_NO_ALIGNMENT    (-1) /* distance value: wavefront emptied (gwf-ed.cu:1336) */
#define GWF_E_BAD_INPUT     (-2) /* ql <= 0, v0/v1 out of range, null pointer */
#define GWF_E_UNSUPPORTED   (-3) /* gwf_ed with traceback != 0: the reference has none (paths come
                                   * from gwf_ed_batch_path); max_lag is accepted and ignored, as the
                                   * reference ignores it, unless GWF_F_MAX_LAG is set */
#define GWF_E_CAPACITY      (-4) /* read did not fit the largest wavefront arena class */
#define GWF_E_CUDA          (-5) /* CUDA runtime failure or no usable B200 device */
#define GWF_E_NOT_INDEXED   (-6) /* gwf_ed_index was not called for this graph */
#define GWF_E_BAD_GRAPH     (-7) /* zero-length vertex, arc overlap >= target length, bad CSR */
#define GWF_E_TIMEOUT       (-8) /* a bounded device/host wait gave up (serving loop) */
#define GWF_E_NOMEM         (-9) /* device or host allocation failed */
#define GWF_E_BUSY          (-10) /* serving: the server is shutting down */

/* batch flags */
#define GWF_F_EXACT_START   0x1 /* exact edit distance at the start of the read. By default the
                                   library reproduces two reference rules about the start state
                                   k = -1: gwf_extend1 does not extend it when v0 or the query is
                                   shorter than 32 bases (signed k against an unsigned max_k,
                                   gwf-ed.cu:809,833), and gwf_ed_extend_batch drops insertion
                                   candidates with k = -1 (uint32_t vl, gwf-ed.cu:895,993), so an
                                   alignment cannot begin with an insertion. Both add cost to
                                   some reads. Default off = reference-identical distances. */
#define GWF_F_MAX_LAG       0x2 /* apply the batch call's max_lag (no reference counterpart: the
                                   reference's prune call is commented out, gwf-ed.cu:1286-1287).
                                   After each score step, the states whose query position d + k
                                   is more than max_lag behind the furthest state's are dropped.
                                   A heuristic: distances can only grow, or become -1 when no
                                   state is left. Off = max_lag ignored, as in the reference. */

#define GWF_F_BOTH_STRANDS  0x4 /* align each read and its reverse complement (IUPAC complement,
                                   made on the device) from the same v0 in one launch; the read's
                                   distance is the smaller one (-1 when neither aligns).
                                   gwf_ed_batch_strand also returns which strand gave it. No
                                   reference counterpart: the reference aligns the read as given,
                                   from v0's orientation only (main.cu:370, TODO at main.cu:404).
                                   Honoured by the batch, resident-batch and serving calls. */

/* execution forms */
#define GWF_MODE_AUTO        0 /* persistent cost-ordered queue */
#define GWF_MODE_PLAIN       1 /* one launch per batch, one warp per read */
#define GWF_MODE_PERSISTENT  2 /* persistent kernel fed by a cost-ordered device queue */

typedef struct {
	int32_t mode;        /* GWF_MODE_* */
	int32_t flags;       /* GWF_F_* */
	int32_t device;      /* CUDA device ordinal (-1 = current) */
	int32_t warps_per_read; /* persistent form: warps that align one read together (1, 2, 4 or 8).
	                           0 = per read: the gwf_tune value of its length bucket for
	                           GWF_MODE_AUTO, else by its share of the batch's work (cost ql^2
	                           against the persistent grid's warp slots) and by its arena size:
	                           reads costing more than one slot's even share, or (in batches of
	                           fewer than 3 reads per warp slot) whose arenas over every slot
	                           would pass 16 GiB, get 2, 4 or 8 warps, the others one.
	                           The plain form uses one warp per read. */
	int32_t ctas_per_sm;   /* persistent grid; 0 = the autotuned value for GWF_MODE_AUTO (see
	                          gwf_tune), else the occupancy limit */
	int32_t use_graph;     /* 1 = replay the persistent form's launch sequence as a CUDA graph */
	int32_t reserved[10];
} gwf_batch_opts_t;

/* ---- index / cleanup (reference gwfa.h:87-88, main.cu:246-277) ---- */

/* Replaces gwf_ed_index (main.cu:265-270): sorts g->arc by a, fills g->aux (calloc'd, as the
 * reference does) and uploads a device-resident CSR with 2-bit packed vertex sequences to the
 * current CUDA device. The device copy is kept in a side table keyed by g. On a device failure
 * the host CSR is still built; gwf_last_error() reports the device error. */
void gwf_ed_index(gwf_graph_t *g);

/* Replaces gwf_cleanup (main.cu:273-277): frees g->aux and the device copy of g. */
void gwf_cleanup(gwf_graph_t *g);

/* Host-callable single alignment. Replaces the device-only
 * gwf_ed(g, ql, q, v0, v1, max_lag, buf, diag_shared) of gwfa.h:95 with the upstream GWFA
 * signature. km is accepted and ignored (kalloc.c is empty in the reference). Synchronous.
 * max_lag is ignored as in the reference; traceback != 0 returns GWF_E_UNSUPPORTED (this signature
 * has no path output: gwf_ed_batch_path returns paths). Returns the edit distance, -1 if no
 * alignment, or a GWF_E_* code. */
int32_t gwf_ed(void *km, const gwf_graph_t *g, int32_t ql, const char *q, int32_t v0, int32_t v1,
               uint32_t max_lag, int32_t traceback);

/* Batch alignment of n reads given as separate strings. Replaces the caller-side stream loop of
 * main.cu:620-735 plus gwf_ed_kernel (main.cu:151-236). v0 is per read (the reference kernel
 * hard-codes 0, main.cu:217). dist[i] receives the distance or -1; status[i] GWF_OK or a
 * per-read GWF_E_* code. Returns 0, or a negative code when the whole call failed. */
int gwf_ed_batch(const gwf_graph_t *g, int32_t n, const char *const *q, const int32_t *ql,
                 const int32_t *v0, int32_t v1, uint32_t max_lag, int32_t *dist, int32_t *status,
                 const gwf_batch_opts_t *opt);

/* Same as gwf_ed_batch with the reads concatenated in one host buffer (the layout of
 * all_sequences_host in main.cu:481-531): read i is seqs[offs[i] .. offs[i]+ql[i]). */
int gwf_ed_batch_concat(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs,
                        const int32_t *ql, const int32_t *v0, int32_t v1, uint32_t max_lag,
                        int32_t *dist, int32_t *status, const gwf_batch_opts_t *opt);

/* gwf_ed_batch_concat with GWF_F_BOTH_STRANDS (implied), plus strand[i]: 0 when read i aligns
 * best as given (ties included), 1 when its reverse complement does, -1 when neither aligns or
 * the read has a non-OK status. A strand that ends with a per-read error (GWF_E_CAPACITY after
 * the retries) makes status[i] that error and dist[i] = -1. */
int gwf_ed_batch_strand(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs,
                        const int32_t *ql, const int32_t *v0, int32_t v1, uint32_t max_lag,
                        int32_t *dist, int32_t *status, int32_t *strand, const gwf_batch_opts_t *opt);

/* ---- traceback: the alignment path ----
 * The reference computes distances only: gwf_ed's traceback argument is unused there
 * (README.md:117-118; no path output in gwfa.h:95), so this entry point has no counterpart; it
 * stands where upstream GWFA returns its path. Reads as in gwf_ed_batch_concat, flags as in
 * gwf_batch_opts_t.flags; the distances equal gwf_ed_batch_concat's. For read i (rows are max_nv
 * wide, row i starts at i * max_nv):
 *   path_n[i]           vertices on the path; only the first min(path_n[i], max_nv) are written
 *   path_v[row + j]     j-th vertex, path_v[row] = v0[i]
 *   path_arc[row + j]   index in g->arc (as sorted by gwf_ed_index) of the arc from vertex j-1
 *                       to vertex j; the alignment enters vertex j at that arc's overlap
 *                       offset o; -1 for j = 0
 *   end_off[i]          offset in the last vertex of the last base the alignment consumes
 * The path spells seq[v0][0 ..] then seq[w][o ..] for each later vertex, through end_off of the
 * last; aligning the read end to end against that text costs at most dist[i] (exactly dist[i]
 * with GWF_F_EXACT_START and v1 = -1). path_n[i] = 0 and end_off[i] = -1 when the read has no
 * alignment or a non-OK status. Synchronous; returns 0 or a negative GWF_E_* code. */
int gwf_ed_batch_path(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs,
                      const int32_t *ql, const int32_t *v0, int32_t v1, int32_t flags, int32_t max_nv,
                      int32_t *dist, int32_t *status, int32_t *end_off, int32_t *path_n,
                      int32_t *path_v, int32_t *path_arc);

/* gwf_ed_batch_path plus the base-level alignment of each read against the text its path spells,
 * as a CIGAR (no counterpart in the reference either). Row i of cigar (max_ops wide) holds
 * cigar_n[i] runs len << 4 | op with the BAM codes 7 '=' (equal bases), 8 'X' (substitution),
 * 1 'I' (a read base the path text lacks), 2 'D' (a path base the read lacks); only the first
 * min(cigar_n[i], max_ops) are written. The CIGAR consumes the whole read and the whole text and
 * is an optimal end-to-end alignment of the two: its cost (X + I + D) is at most dist[i], equal
 * with GWF_F_EXACT_START and v1 = -1. cigar_n[i] = -1 when read i has no CIGAR: no alignment, a
 * per-read error, a path longer than max_nv, or a wavefront table ((dist + 1)^2 int32) larger
 * than 2 GiB or the memory budget. max_ops = 0 is gwf_ed_batch_path. */
int gwf_ed_batch_align(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs,
                       const int32_t *ql, const int32_t *v0, int32_t v1, int32_t flags, int32_t max_nv,
                       int32_t max_ops, int32_t *dist, int32_t *status, int32_t *end_off, int32_t *path_n,
                       int32_t *path_v, int32_t *path_arc, int32_t *cigar_n, uint32_t *cigar);

/* ---- device-resident batches (inputs uploaded once; used to time the kernel alone) ---- */
typedef struct gwf_batch_s gwf_batch_t;
gwf_batch_t *gwf_batch_create(const gwf_graph_t *g, int32_t n, const char *seqs,
                              const int64_t *offs, const int32_t *ql, const int32_t *v0,
                              int32_t v1, const gwf_batch_opts_t *opt);
/* Runs the whole batch on the device (including overflow retries). Returns 0 or GWF_E_*.
 * *kernel_ms receives the device time of the run measured with CUDA events. */
int gwf_batch_run(gwf_batch_t *b, const gwf_batch_opts_t *opt, float *kernel_ms);
int gwf_batch_results(gwf_batch_t *b, int32_t *dist, int32_t *status);
/* Number of kernel launches issued by the last gwf_batch_run. */
int32_t gwf_batch_launches(const gwf_batch_t *b);
/* Score steps each read took in the last run (diagnostics and cost models). */
int gwf_batch_steps(gwf_batch_t *b, int32_t *steps);
void gwf_batch_destroy(gwf_batch_t *b);

/* ---- batch alignment that allocates nothing ----
 * No counterpart in the reference. For callers that must not allocate device memory while they
 * align, such as a framework whose caching allocator owns the device heap, or a latency-bound
 * serving loop that cannot afford cudaMalloc's implicit device synchronisation. The caller passes
 * device buffers; the call allocates nothing. Its warp arenas live in one fixed device array of
 * GWF_NOALLOC_SCRATCH_BYTES (64 MiB) that every GPU loading the library holds until exit.
 * Limits: at most GWF_NOALLOC_MAX_READS reads per call and GWF_NOALLOC_MAX_QL bases per read
 * (max_ql = the longest read; larger calls return GWF_E_CAPACITY), and a read whose wavefront
 * outgrows its arena gets per-read status GWF_E_CAPACITY (there is no larger arena to retry in).
 * Layout: read i is d_seqs[d_offs[i] .. d_offs[i]+d_ql[i]); d_seqs must be 8-byte aligned with
 * 16 readable bytes after the last read. The graph must have been indexed on the current device
 * (gwf_ed_index). flags: only GWF_F_EXACT_START is honoured; any other bit returns
 * GWF_E_BAD_INPUT (this call has no lag pruning). Asynchronous on `stream` (a cudaStream_t, NULL =
 * legacy default stream): d_dist / d_status are valid once the stream has completed. The first
 * call on a device does a one-time set-up (symbol lookup, a small init kernel, and a wait for it
 * on `stream`); make that first call before any stream capture. All calls share the one array,
 * so calls that overlap on the GPU (e.g. on two streams) race; serialise them. Returns 0 or a
 * GWF_E_* code. */
#define GWF_NOALLOC_MAX_READS     262144
#define GWF_NOALLOC_MAX_QL        2048
#define GWF_NOALLOC_SCRATCH_BYTES (64LL << 20)
int gwf_ed_batch_noalloc(const gwf_graph_t *g, int32_t n, int32_t max_ql, const char *d_seqs,
                         const int64_t *d_offs, const int32_t *d_ql, const int32_t *d_v0,
                         int32_t v1, int32_t *d_dist, int32_t *d_status, int32_t flags,
                         void *stream);

/* ---- autotuner (no reference counterpart) ----
 * Times the persistent form with 1, 2, 4 and 8 warps per read at 1..(occupancy limit) CTAs per
 * SM, and the plain form, on the given reads, separately for each read-length bucket (ql < 1500,
 * < 3000, < 6000, < 12000, longer; at most max_reads_per_bucket evenly spread reads each, 0 =
 * 8192), and keeps the fastest shape per bucket for the graph's device. Batch calls with mode
 * GWF_MODE_AUTO then align each read with the warps per read of its own bucket (warps_per_read =
 * 0), and take the form and CTAs per SM (ctas_per_sm = 0) of the bucket holding most of the
 * batch's work (sum of ql^2). json_path != NULL also writes the table as JSON; gwf_tune_load
 * reads it back (device -1 = current). */
#define GWF_TUNE_NBUCKETS 5
int gwf_tune(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs, const int32_t *ql,
             const int32_t *v0, int32_t v1, int32_t max_reads_per_bucket, const char *json_path);
int gwf_tune_load(const char *json_path, int32_t device);
/* 1 = the bucket has an entry (form = GWF_MODE_*, ctas_per_sm, measured reads/s), 0 = none. */
int gwf_tune_get(int32_t device, int32_t bucket, int32_t *form, int32_t *ctas_per_sm, float *reads_per_s);
/* gwf_tune_get plus the bucket's warps per read. */
int gwf_tune_get_shape(int32_t device, int32_t bucket, int32_t *form, int32_t *ctas_per_sm,
                       int32_t *warps_per_read, float *reads_per_s);
void gwf_tune_clear(int32_t device);

/* Page-locked host memory for read buffers, so that batch copies run at full PCIe speed. */
void *gwf_pinned_alloc(int64_t bytes);
void gwf_pinned_free(void *p);

/* ---- serving: continuous batching on a resident graph ----
 * No reference counterpart. One resident kernel aligns reads pulled from a device queue, one
 * warp per read. Reads of queued requests are admitted in FIFO order while a slot is free and
 * the arena budget holds the read's wavefront arena (sized for its own length); a read that
 * overflows its arena is queued again in a 4x larger one, up to three times, ahead of new
 * reads. Results equal those of gwf_ed_batch for the same reads, whatever else is in flight. */
typedef struct gwf_srv_s gwf_srv_t;
typedef struct {
	int64_t arena_budget_bytes; /* device bytes for in-flight wavefront arenas; 0 = 1/4 of free */
	int32_t max_inflight_reads; /* reads admitted at once (queued or running); 0 = 16384 */
	int32_t flags;              /* GWF_F_* */
	int32_t device;
	int32_t max_lag;            /* with GWF_F_MAX_LAG in flags: the lag of the pruning */
	int32_t warps_per_read;     /* warps that align one read together: 1, 2, 4 or 8; 0 = 8. More
	                               warps per read lower the latency of each read; one warp per read
	                               gives more throughput on short reads of sparse graphs */
	int32_t reserved[5];
} gwf_srv_opts_t;
gwf_srv_t *gwf_srv_create(const gwf_graph_t *g, const gwf_srv_opts_t *opt);
/* Queues one request of n reads; returns a request id >= 0 or a GWF_E_* code. Copies the
 * reads, so the caller's buffers can be reused on return. */
int64_t gwf_srv_submit(gwf_srv_t *s, int32_t n, const char *seqs, const int64_t *offs,
                       const int32_t *ql, const int32_t *v0, int32_t v1);
/* 1 = done (dist/status filled), 0 = pending, < 0 = error. */
int gwf_srv_poll(gwf_srv_t *s, int64_t req, int32_t *dist, int32_t *status);
/* Waits at most timeout_s seconds. Returns 1 done, GWF_E_TIMEOUT, or another error. */
int gwf_srv_wait(gwf_srv_t *s, int64_t req, int32_t *dist, int32_t *status, double timeout_s);
/* With GWF_F_BOTH_STRANDS in the server's flags, every read of a request is aligned on both
 * strands (its reverse complement is queued as a read of its own) and poll / wait return the
 * better distance; this gives the strand of each read of a finished request (as
 * gwf_ed_batch_strand). Returns 0 or a GWF_E_* code. */
int gwf_srv_strand(gwf_srv_t *s, int64_t req, int32_t *strand);
/* Submit, first-admission and completion times (seconds, steady clock) of a finished request. */
int gwf_srv_times(gwf_srv_t *s, int64_t req, double *t_submit, double *t_admit, double *t_done);
/* Counters of the server, in this order: kernel launches, reads re-queued in a larger arena,
 * arena bytes in use, queue positions published, completion records consumed, reads admitted
 * and not finished, requests not fully admitted, kernel running (0/1). Fills min(n_out,
 * GWF_SRV_NSTATS) values and returns GWF_SRV_NSTATS. */
#define GWF_SRV_NSTATS 8
int gwf_srv_stats(gwf_srv_t *s, int64_t *out, int32_t n_out);
void gwf_srv_destroy(gwf_srv_t *s);

/* ---- GFA input side (reference gfa-io.c, gfa-base.c, gfa-sub.c, main.cu:294-359) ---- */

/* gfa_read + gfa_finalize + gwf_gfa2gwf in one call. start_seg = segment name of v0 on the
 * forward strand (main.cu:399-407), or the name followed by '+' or '-' to choose the strand
 * (the reference leaves that as a TODO, main.cu:404); NULL = first segment, forward. Vertex 0
 * of the result is the start segment on that strand. Returns NULL on failure. path may be
 * gzip-compressed, or "-" for standard input. The text is parsed on one thread per core (at
 * least 1 MiB each; the environment variable GWF_GFA_THREADS sets the count) and applied in file
 * order, so the result does not depend on the thread count. */
gwf_graph_t *gwf_gfa_load(const char *path, const char *start_seg);
/* Same from an in-memory GFA text. */
gwf_graph_t *gwf_gfa_load_mem(const char *text, int64_t len, const char *start_seg);
/* Frees a graph from gwf_gfa_load* (gwf_free, main.cu:347-352); also calls gwf_cleanup. */
void gwf_graph_free(gwf_graph_t *g);
/* Writes the gwf_graph_print dump (main.cu:354-359) to buf. Returns the full length; writes at
 * most cap bytes (NUL-terminated when it fits). */
int64_t gwf_graph_dump(const gwf_graph_t *g, char *buf, int64_t cap);

/* ---- read sets (replaces the reference's two-pass FASTA reading, main.cu:459-534) ----
 * FASTA or FASTQ (four-line records), plain or gzip, "-" = standard input. The sequences are
 * concatenated in file order into seqs (16 zero bytes after the last), read i being
 * seqs[offs[i] .. offs[i] + lens[i]), ready for gwf_ed_batch_concat. FASTA is parsed on one
 * thread per core (at least 4 MiB each; GWF_READS_THREADS sets the count). Returns NULL on
 * failure; free with gwf_reads_free. */
typedef struct {
	int32_t n;
	int64_t n_bases;
	char *seqs;
	int64_t *offs;
	int32_t *lens;
} gwf_reads_t;
gwf_reads_t *gwf_reads_load(const char *path);
void gwf_reads_free(gwf_reads_t *r);

/* ---- diagnostics ---- */
const char *gwf_last_error(void);
const char *gwf_version(void);

#ifdef __cplusplus
}
#endif

#endif
