/*
 * gwf_oracle.h — TEST INFRASTRUCTURE ONLY. CPU restatement of the reference GWFA
 * edit-distance path (gwf-ed.cu:80-1337 with single-lane semantics) plus an independent
 * sequence-to-graph dynamic program. Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it; the product never does.
 */
#ifndef GWF_ORACLE_H
#define GWF_ORACLE_H

#include <stdint.h>
#include "../include/gwfa.h"

#ifdef __cplusplus
extern "C" {
#endif

/* flags: reference capacity limits that this read would hit (main.cu:498-505 sizing).
 * SAFE ones only reduce pruning; UNSAFE ones corrupt memory or drop states in the reference. */
#define GWFO_F_TMP_DROP     0x001 /* safe:   tmp interval dropped (gwf-ed.cu:1008,1177) */
#define GWFO_F_SWAP_DROP    0x002 /* safe:   intv not copied, n_swap=0 (gwf-ed.cu:754-758) */
#define GWFO_F_HASH_FULL    0x010 /* unsafe: hash set full, absent=0 (gwf-ed.cu:1054-1061) */
#define GWFO_F_A_WRAP       0x020 /* unsafe: ring A overran its capacity (gwf-ed.cu:848-852) */
#define GWFO_F_B_OVER       0x040 /* unsafe: B wrote past max_B (gwf-ed.cu:879-888) */
#define GWFO_F_A_COPY_OVER  0x080 /* unsafe: n_B > max_a on the B->a copy (gwf-ed.cu:1263-1270) */
#define GWFO_F_INTV_OVER    0x100 /* unsafe: merged intervals > max_intv (gwf-ed.cu:300-348) */
#define GWFO_F_OOO_OVER     0x200 /* unsafe: n_a > max_ooo in gwf_diag_sort (gwf-ed.cu:546) */
#define GWFO_F_NONTERM      0x400 /* reference never terminates: first query-end state has k=-1
                                     (gwf-ed.cu:1233 with 1327) or ql=0 */
#define GWFO_F_UNSAFE_MASK  0x7f0

/* options */
#define GWFO_O_EXACT_START  0x1 /* disable the two k=-1 unsigned-compare rules of the start
                                     state (see gwf_oracle.c): exact edit distance */
#define GWFO_O_ENTRY_KEY    0x2 /* the library's arrival key: (entry id, query position), the
                                     entry id telling apart arcs into one vertex with different
                                     overlaps. The reference keys on (vertex, query position)
                                     (gwf-ed.cu:1196), so where the arcs into a vertex carry
                                     different overlaps its result depends on its FIFO order; with
                                     one overlap per vertex both keys are the same. */

typedef struct {
	int32_t steps;        /* score steps executed (s + 1 when an end is found) */
	int32_t flags;        /* GWFO_F_* */
	int64_t W;            /* sum over steps of wavefront size entering the step */
	int64_t E;            /* character pairs compared by extension */
	int64_t n_keys;       /* distinct arrival keys inserted into the hash set */
	int32_t max_na, max_nB, max_nA, max_ntmp, max_nintv;
	int32_t pad;
} gwfo_stats_t;

/* Builds g->aux like gwf_ed_index (main.cu:246-270): arcs sorted by a, CSR off<<32|n. */
void gwfo_index(gwf_graph_t *g);
void gwfo_index_free(gwf_graph_t *g);

/* One read. Returns the reference distance (or -1). st may be NULL. */
int32_t gwfo_ed(const gwf_graph_t *g, int32_t ql, const char *q, int32_t v0, int32_t v1,
                int32_t opts, gwfo_stats_t *st);

/* gwfo_ed with the product's lag pruning after each step (max_lag > 0; 0 = gwfo_ed). */
int32_t gwfo_ed_lag(const gwf_graph_t *g, int32_t ql, const char *q, int32_t v0, int32_t v1,
                    int32_t opts, int32_t max_lag, gwfo_stats_t *st);

/* Many reads over a thread pool (n_threads <= 0: all online cores). st may be NULL.
 * Returns the number of threads used. */
int32_t gwfo_ed_batch(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs,
                      const int32_t *ql, const int32_t *v0, int32_t v1, int32_t opts,
                      int32_t *dist, gwfo_stats_t *st, int32_t n_threads);

/* Independent ground truth: minimum edit distance of q against any walk that starts before
 * offset 0 of v0, follows arcs (entering w at offset o), and ends anywhere (v1 < 0) or at the
 * last base of v1. 0-1 BFS over (graph position, query prefix). Small inputs only. */
int32_t gwfo_dp(const gwf_graph_t *g, int32_t ql, const char *q, int32_t v0, int32_t v1);

#ifdef __cplusplus
}
#endif
#endif
