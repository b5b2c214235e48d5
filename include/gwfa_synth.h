/*
 * gwfa_synth.h — seeded synthetic inputs for the GWFA path: a variation graph written as GFA
 * (S lines plus "L a + b + 0M" links, like exposed_testing/generated/grafo_test.gfa) and reads
 * sampled along random walks with substitution:insertion:deletion errors at 6:2:2.
 * The reference ships no generator and no benchmark data; these stand in for its missing read
 * sets (exposed_testing/generated/ref*.fa). No counterpart in the reference's C ABI.
 */
#ifndef GWFA_SYNTH_H
#define GWFA_SYNTH_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Graph: uniform ACGT backbone of backbone_len bases. Every site_every bases a variant site:
 * a SNP with probability p_snp (1-bp ref and alt segments), otherwise an indel of U{1..indel_max}
 * bases, insertion or deletion 50/50, as an extra segment plus a bypass arc. Every sv_every bases
 * (0 = none) a structural variant of U{sv_min..sv_max} bases, insertion or deletion 50/50.
 * Segments are named s1, s2, ... in creation order (= GFA segment id order). */
void *gwf_synth_graph_new(int64_t backbone_len, int32_t site_every, double p_snp,
                          int32_t indel_max, int32_t sv_every, int32_t sv_min, int32_t sv_max,
                          uint64_t seed);
void gwf_synth_graph_free(void *g);
/* GFA text; returns the full length, copies at most cap bytes. */
int64_t gwf_synth_graph_gfa(void *g, char *buf, int64_t cap);
int32_t gwf_synth_graph_nseg(void *g);

/* Reads. len_kind: 0 = fixed len_a; 1 = lognormal(median len_a, sigma len_b); 2 = uniform
 * [len_a, len_b]. Lengths are the true (graph) lengths, clipped to [len_min, len_max]; errors are
 * then applied per base with a rate drawn uniformly from [err_min, err_max]. Each read starts at
 * offset 0 of a backbone segment (its origin, reported as a 0-based segment id) and follows a
 * random walk choosing branches uniformly. */
void *gwf_synth_reads_new(void *g, int32_t n, int32_t len_kind, double len_a, double len_b,
                          int32_t len_min, int32_t len_max, double err_min, double err_max,
                          uint64_t seed);
int64_t gwf_synth_reads_bytes(void *r);
/* seqs: reads_bytes bytes; offs/lens/origin/err: n entries each (err may be NULL). */
void gwf_synth_reads_copy(void *r, char *seqs, int64_t *offs, int32_t *lens, int32_t *origin,
                          float *err);
void gwf_synth_reads_free(void *r);

#ifdef __cplusplus
}
#endif
#endif
