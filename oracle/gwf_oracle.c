/*
 * gwf_oracle.c — TEST INFRASTRUCTURE ONLY (the checker, never the product path).
 *
 * A single-threaded C restatement of the reference GWFA edit-distance routine, gwf-ed.cu of
 * MarafonGiacomo/GWFA-CUDA-VERSION, with converged-warp ("single-lane") semantics: every
 * warp-parallel step of the reference (ballot compactions, merge-path merges, parallel sorts)
 * becomes the serial loop it computes. Each function cites the reference lines it restates.
 *
 * It reproduces the reference's observable behaviour, including four quirks found by reading:
 *  1. gwf_extend1 (gwf-ed.cu:806-839) compares a signed k against an unsigned max_k. With
 *     k = -1 the serial tail loop never runs, so the start state does not extend when
 *     min(ql - d, vl) < 32. GWFO_O_EXACT_START disables this for the ground-truth comparison.
 *  2. gwf_diag_is_sorted / gwf_intv_is_sorted (gwf-ed.cu:219-263, 372-417) skip element 32 and,
 *     when n <= 33, the last element. ref_is_sorted() emulates the 32 lanes literally.
 *  3. gwf_ed_extend_batch (gwf-ed.cu:895, 993) holds the vertex length in a uint32_t, so its
 *     successor filter `p->k < vl` drops every candidate with k = -1: an alignment cannot begin
 *     with an insertion before the first base of v0. GWFO_O_EXACT_START disables this too.
 *  4. The reference never terminates when the first query-end state it pops has k = -1
 *     (gwf-ed.cu:1233 sets end_off = -1, gwf-ed.cu:1327 then keeps looping). The oracle stops,
 *     returns s and sets GWFO_F_NONTERM.
 * Capacity limits of the reference arena (main.cu:498-505) are emulated where they are safe
 * (tmp / swap truncation only reduces pruning) and flagged where they corrupt memory.
 *
 * The independent ground truth gwfo_dp() is at the end of the file.
 */
#define _GNU_SOURCE
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <pthread.h>
#include <unistd.h>
#include "gwf_oracle.h"

#define SHIFT 0x40000000 /* gwf-ed.cu:11 */

typedef struct { uint64_t vd; int32_t k; uint32_t xo; } od_t; /* gwf_diag_t, gwfa.h:27-31 */

static inline uint64_t gen_vd(uint32_t v, int32_t d) /* gwf-ed.cu:80-83 */
{
	return (uint64_t)v << 32 | (uint32_t)(SHIFT + d);
}

/* ------------------------------------------------------------------ growable storage */
#define GROW(ptr, cap, need) do { \
		if ((int64_t)(need) > (cap)) { \
			int64_t nc_ = (cap) ? (cap) : 64; \
			while (nc_ < (int64_t)(need)) nc_ <<= 1; \
			(ptr) = realloc((ptr), (size_t)nc_ * sizeof(*(ptr))); \
			(cap) = nc_; \
		} \
	} while (0)

typedef struct {
	const gwf_graph_t *g;
	int32_t ql, v1, opts, max_lag;
	const char *q;
	/* reference arena caps (main.cu:498-505) */
	int64_t max_a, max_B, max_A, max_intv, max_tmp, max_swap, max_ooo;
	uint64_t ha_cap;
	/* wavefront a: SoA (gwfa.h:20-25) */
	uint64_t *a_vd; int32_t *a_k; uint32_t *a_xo; int64_t a_cap, a_cap2, a_cap3;
	od_t *B; int64_t B_cap;
	od_t *A; int64_t A_cap, A_head;
	uint64_t *intv0, *intv1, *tmp0, *tmp1, *swap0, *swap1;
	int64_t intv_cap0, intv_cap1, tmp_cap0, tmp_cap1, swap_cap0, swap_cap1;
	od_t *ooo, *scr; int64_t ooo_cap, scr_cap;
	/* arrival set (static_set64_put semantics, unbounded) */
	uint64_t *hk; uint64_t h_mask, h_n;
	/* counters (gwfa.h:44-52) */
	int32_t n_intv, n_tmp, n_swap, n_A, n_B, n_a;
	gwfo_stats_t st;
} ows_t;

/* ------------------------------------------------------------------ arrival set */
static inline uint64_t mix64(uint64_t x)
{
	x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
	return x;
}

static void hset_init(ows_t *w)
{
	w->h_mask = 1023; w->h_n = 0;
	w->hk = calloc(w->h_mask + 1, 8);
}

static void hset_grow(ows_t *w)
{
	uint64_t om = w->h_mask, i, *ok = w->hk;
	w->h_mask = (om + 1) * 2 - 1;
	w->hk = calloc(w->h_mask + 1, 8);
	for (i = 0; i <= om; ++i)
		if (ok[i]) {
			uint64_t j = mix64(ok[i]) & w->h_mask;
			while (w->hk[j]) j = (j + 1) & w->h_mask;
			w->hk[j] = ok[i];
		}
	free(ok);
}

/* static_set64_put (gwf-ed.cu:1020-1062): absent = 1 iff key is new. key == 0 is never
 * absent. A full reference table (h_n == cap) would answer 0: flagged, then treated as absent. */
static int hset_put(ows_t *w, uint64_t key)
{
	uint64_t j;
	if (key == 0) return 0;
	j = mix64(key) & w->h_mask;
	while (w->hk[j]) {
		if (w->hk[j] == key) return 0;
		j = (j + 1) & w->h_mask;
	}
	if (w->h_n >= w->ha_cap) w->st.flags |= GWFO_F_HASH_FULL;
	w->hk[j] = key, ++w->h_n;
	if (w->h_n * 2 > w->h_mask) hset_grow(w);
	return 1;
}

/* ------------------------------------------------------------------ extension */
/* gwf_extend1 (gwf-ed.cu:806-839). max_k is uint32 in the reference: with k = -1 the tail loop
 * condition (k < max_k) is false, and the 32-wide loop only runs when max_k >= 31. */
static int32_t o_extend1(ows_t *w, int32_t d, int32_t k, int32_t vl, const char *ts)
{
	int64_t m = (int64_t)(w->ql - d < vl ? w->ql - d : vl) - 1;
	const char *qs = w->q;
	if (k < 0 && m < 31 && !(w->opts & GWFO_O_EXACT_START)) return k;
	while (k < m && ts[k + 1] == qs[d + k + 1]) ++k, ++w->st.E;
	if (k < m) ++w->st.E;
	return k;
}

/* ------------------------------------------------------------------ sortedness (quirk 2) */
/* gwf_diag_is_sorted / gwf_intv_is_sorted (gwf-ed.cu:372-417, 219-263), emulating the 32 lanes
 * and the diag_shared[64] double buffer literally. */
static int ref_is_sorted(const uint64_t *x, int32_t n)
{
	uint64_t sh[64], curr[32], first;
	int32_t idx, cb = 0, nb = 32, l, t;
	memset(sh, 0, sizeof(sh));
	for (l = 0; l < 32; ++l) if (l < n) sh[l] = x[l];
	first = sh[0];
	idx = 33;
	while (idx - 32 < n) {
		for (l = 0; l < 32; ++l) if (idx + l < n) sh[nb + l] = x[idx + l];
		for (l = 0; l < 32; ++l) curr[l] = (idx - 32) + l < n ? sh[cb + l] : 0;
		for (l = 0; l < 32; ++l) {
			uint64_t prev = l == 0 ? first : curr[l - 1];
			if ((idx - 32) + l < n && prev > curr[l]) return 0;
		}
		first = curr[31];
		idx += 32;
		t = cb, cb = nb, nb = t;
	}
	return 1;
}

/* ------------------------------------------------------------------ stable sorts */
/* fast_parallel_sort (gwf-ed.cu:85-216) and sort_gwf_diags (gwf-ed.cu:419-524) are both stable
 * (odd-even transposition swaps only on >, merge takes left on <=), so any stable sort gives
 * the same permutation. */
typedef struct { uint64_t k, v; } okv_t;

static void stable_sort_kv(okv_t *a, int64_t n, okv_t *tmp)
{
	int64_t width, i;
	if (n < 2) return;
	for (width = 1; width < n; width <<= 1) {
		for (i = 0; i < n; i += 2 * width) {
			int64_t l = i, m = i + width < n ? i + width : n, r = i + 2 * width < n ? i + 2 * width : n;
			int64_t p = l, q = m, o = l;
			while (p < m && q < r) tmp[o++] = a[p].k <= a[q].k ? a[p++] : a[q++];
			while (p < m) tmp[o++] = a[p++];
			while (q < r) tmp[o++] = a[q++];
		}
		memcpy(a, tmp, (size_t)n * sizeof(okv_t));
	}
}

static void stable_sort_diag(od_t *a, int64_t n, od_t *tmp)
{
	int64_t width, i;
	if (n < 2) return;
	for (width = 1; width < n; width <<= 1) {
		for (i = 0; i < n; i += 2 * width) {
			int64_t l = i, m = i + width < n ? i + width : n, r = i + 2 * width < n ? i + 2 * width : n;
			int64_t p = l, q = m, o = l;
			while (p < m && q < r) tmp[o++] = a[p].vd <= a[q].vd ? a[p++] : a[q++];
			while (p < m) tmp[o++] = a[p++];
			while (q < r) tmp[o++] = a[q++];
		}
		memcpy(a, tmp, (size_t)n * sizeof(od_t));
	}
}

/* ------------------------------------------------------------------ intervals */
/* gwf_intv_merge_adj (gwf-ed.cu:266-296) */
static int32_t o_intv_merge_adj(int32_t n, uint64_t *a0, uint64_t *a1)
{
	int32_t i, k;
	uint64_t st, en;
	if (n == 0) return 0;
	st = a0[0], en = a1[0];
	for (i = 1, k = 0; i < n; ++i) {
		if (a0[i] > en) a0[k] = st, a1[k++] = en, st = a0[i], en = a1[i];
		else en = en > a1[i] ? en : a1[i];
	}
	a0[k] = st, a1[k++] = en;
	return k;
}

/* gwf_intv_merge2 (gwf-ed.cu:300-348): merge path evaluated per output index exactly as the
 * lanes do, so an unsorted input gives the same (lossy) result as the reference. */
static int32_t o_intv_merge2(uint64_t *a0, uint64_t *a1, int32_t n_b, const uint64_t *b0,
                             const uint64_t *b1, int32_t n_c, const uint64_t *c0, const uint64_t *c1)
{
	int32_t total = n_b + n_c, k;
	if (total == 0) return 0;
	for (k = 0; k < total; ++k) {
		int32_t low = k - n_c > 0 ? k - n_c : 0, high = k < n_b ? k : n_b, i, j, tb;
		while (low < high) {
			int32_t mid = (low + high) >> 1;
			int cond = b0[mid] <= c0[k - 1 - mid];
			low = cond ? mid + 1 : low;
			high = cond ? high : mid;
		}
		i = low, j = k - i;
		tb = i < n_b && (j >= n_c || b0[i] <= c0[j]);
		a0[k] = tb ? b0[i] : c0[j];
		a1[k] = tb ? b1[i] : c1[j];
	}
	return o_intv_merge_adj(total, a0, a1);
}

/* ------------------------------------------------------------------ diagonal dedup */
/* gwf_diag_sort (gwf-ed.cu:527-651): split by the ooo bit into b (clear) and c (set), sort c,
 * clear its bits, merge path b and c back into a. */
static void o_diag_sort(ows_t *w, int32_t n_a)
{
	int32_t n_b = 0, n_c = 0, j, total, k;
	od_t *b, *c;
	if (n_a > w->max_ooo) w->st.flags |= GWFO_F_OOO_OVER;
	GROW(w->ooo, w->ooo_cap, n_a);
	GROW(w->scr, w->scr_cap, n_a);
	for (j = 0; j < n_a; ++j) if (w->a_xo[j] & 1) ++n_c;
	n_b = n_a - n_c;
	b = w->ooo, c = w->ooo + n_b;
	{
		int32_t tb = 0, tc = 0;
		for (j = 0; j < n_a; ++j) {
			od_t x = { w->a_vd[j], w->a_k[j], w->a_xo[j] };
			if (x.xo & 1) c[tc++] = x; else b[tb++] = x;
		}
	}
	stable_sort_diag(c, n_c, w->scr);
	for (j = 0; j < n_c; ++j) c[j].xo &= 0xfffffffeU;
	total = n_b + n_c;
	for (k = 0; k < total; ++k) {
		int32_t low = k - n_c > 0 ? k - n_c : 0, high = k < n_b ? k : n_b, i, jj;
		od_t best;
		while (low < high) {
			int32_t mid = (low + high) >> 1;
			int cond = b[mid].vd <= c[k - 1 - mid].vd;
			low = cond ? mid + 1 : low;
			high = cond ? high : mid;
		}
		i = low, jj = k - i;
		best = (i < n_b && (jj >= n_c || b[i].vd <= c[jj].vd)) ? b[i] : c[jj];
		w->a_vd[k] = best.vd, w->a_k[k] = best.k, w->a_xo[k] = best.xo;
	}
}

/* gwf_diag_dedup (gwf-ed.cu:653-687) */
static int32_t o_diag_dedup(ows_t *w, int32_t n_a)
{
	int32_t i, n, st;
	if (!ref_is_sorted(w->a_vd, n_a)) o_diag_sort(w, n_a);
	for (i = 1, st = 0, n = 0; i <= n_a; ++i) {
		if (i == n_a || w->a_vd[i] != w->a_vd[st]) {
			int32_t j, max_j = st;
			for (j = st + 1; j < i; ++j)
				if (w->a_k[max_j] < w->a_k[j]) max_j = j;
			w->a_vd[n] = w->a_vd[max_j], w->a_k[n] = w->a_k[max_j], w->a_xo[n] = w->a_xo[max_j];
			++n, st = i;
		}
	}
	return n;
}

/* gwf_mixed_dedup (gwf-ed.cu:691-747): drop diagonals inside a forbidden interval, found by
 * the reference's binary search (exact even when the interval list is not sorted). */
static int32_t o_mixed_dedup(ows_t *w, int32_t n_a)
{
	int32_t j, kw = 0;
	for (j = 0; j < n_a; ++j) {
		uint64_t vd = w->a_vd[j];
		int keep = 1, low = 0, high = w->n_intv - 1;
		while (low <= high) {
			int32_t mid = (low + high) / 2;
			if (vd >= w->intv0[mid] && vd < w->intv1[mid]) { keep = 0; break; }
			if (vd < w->intv0[mid]) high = mid - 1; else low = mid + 1;
		}
		if (keep) w->a_vd[kw] = vd, w->a_k[kw] = w->a_k[j], w->a_xo[kw] = w->a_xo[j], ++kw;
	}
	return kw;
}

/* gwf_dedup (gwf-ed.cu:780-804) with static_intv_copy (gwf-ed.cu:751-778) */
static int32_t o_dedup(ows_t *w, int32_t n_a)
{
	if (w->n_intv + w->n_tmp > 0) {
		int32_t total;
		if (!ref_is_sorted(w->tmp0, w->n_tmp)) {
			okv_t *kv = malloc(sizeof(okv_t) * (size_t)(w->n_tmp + 1) * 2);
			int32_t j;
			for (j = 0; j < w->n_tmp; ++j) kv[j].k = w->tmp0[j], kv[j].v = w->tmp1[j];
			stable_sort_kv(kv, w->n_tmp, kv + w->n_tmp);
			for (j = 0; j < w->n_tmp; ++j) w->tmp0[j] = kv[j].k, w->tmp1[j] = kv[j].v;
			free(kv);
		}
		if (w->n_intv > w->max_swap) {
			w->n_swap = 0;
			w->st.flags |= GWFO_F_SWAP_DROP;
		} else {
			GROW(w->swap0, w->swap_cap0, w->n_intv + 1);
			GROW(w->swap1, w->swap_cap1, w->n_intv + 1);
			memcpy(w->swap0, w->intv0, sizeof(uint64_t) * (size_t)w->n_intv);
			memcpy(w->swap1, w->intv1, sizeof(uint64_t) * (size_t)w->n_intv);
			w->n_swap = w->n_intv;
		}
		total = w->n_swap + w->n_tmp;
		if (total > w->max_intv) w->st.flags |= GWFO_F_INTV_OVER;
		GROW(w->intv0, w->intv_cap0, total + 1);
		GROW(w->intv1, w->intv_cap1, total + 1);
		w->n_intv = o_intv_merge2(w->intv0, w->intv1, w->n_swap, w->swap0, w->swap1,
		                          w->n_tmp, w->tmp0, w->tmp1);
		if (w->n_intv > w->st.max_nintv) w->st.max_nintv = w->n_intv;
	}
	n_a = o_diag_dedup(w, n_a);
	if (w->n_intv > 0) n_a = o_mixed_dedup(w, n_a);
	return n_a;
}

/* Lag pruning (no reference body: the call at gwf-ed.cu:1286-1287 is commented out and gwfa.h
 * declares no gwf_prune). The product's rule: keep the states whose query position d + k is
 * within max_lag of the furthest state's, in order. */
static int32_t o_prune(ows_t *w, int32_t n_a)
{
	int32_t i, far = INT32_MIN, kw = 0;
	for (i = 0; i < n_a; ++i) {
		int32_t x = (int32_t)w->a_vd[i] - SHIFT + w->a_k[i];
		if (x > far) far = x;
	}
	for (i = 0; i < n_a; ++i)
		if ((int32_t)w->a_vd[i] - SHIFT + w->a_k[i] >= far - w->max_lag)
			w->a_vd[kw] = w->a_vd[i], w->a_k[kw] = w->a_k[i], w->a_xo[kw] = w->a_xo[i], ++kw;
	return kw;
}

/* ------------------------------------------------------------------ queues */
static void A_push(ows_t *w, uint64_t vd, int32_t k, uint32_t xo) /* static_A_pushp :841-857 */
{
	int64_t tail = w->A_head + w->n_A;
	if (w->n_A >= w->max_A) w->st.flags |= GWFO_F_A_WRAP;
	GROW(w->A, w->A_cap, tail + 1);
	w->A[tail].vd = vd, w->A[tail].k = k, w->A[tail].xo = xo;
	++w->n_A;
	if (w->n_A > w->st.max_nA) w->st.max_nA = w->n_A;
}

static void B_push(ows_t *w, uint32_t v, int32_t d, int32_t k, uint32_t xo, uint32_t ooo) /* :879-888 */
{
	if (w->n_B >= w->max_B) w->st.flags |= GWFO_F_B_OVER;
	GROW(w->B, w->B_cap, w->n_B + 1);
	w->B[w->n_B].vd = gen_vd(v, d), w->B[w->n_B].k = k, w->B[w->n_B].xo = xo << 1 | ooo;
	++w->n_B;
}

static int diag_update(od_t *p, uint32_t v, int32_t d, int32_t k, uint32_t x, uint32_t ooo) /* :355-370 */
{
	uint64_t vd = gen_vd(v, d);
	if (p->vd == vd) {
		p->xo = p->k > k ? p->xo : x << 1 | ooo;
		p->k = p->k > k ? p->k : k;
		return 0;
	}
	return 1;
}

static void tmp_push(ows_t *w, uint64_t val) /* :1008-1014, :1177-1183 */
{
	if (w->n_tmp < w->max_tmp) {
		GROW(w->tmp0, w->tmp_cap0, w->n_tmp + 1);
		GROW(w->tmp1, w->tmp_cap1, w->n_tmp + 1);
		w->tmp0[w->n_tmp] = val, w->tmp1[w->n_tmp] = val + 1;
		++w->n_tmp;
		if (w->n_tmp > w->st.max_ntmp) w->st.max_ntmp = w->n_tmp;
	} else w->st.flags |= GWFO_F_TMP_DROP;
}

/* ------------------------------------------------------------------ one score step */
/* gwf_ed_extend_batch (gwf-ed.cu:891-1018): n consecutive diagonals of one vertex at off. */
static void o_extend_batch(ows_t *w, int32_t n, int32_t off)
{
	const gwf_graph_t *g = w->g;
	uint32_t v = (uint32_t)(w->a_vd[off] >> 32);
	int32_t vl = (int32_t)g->len[v], j, m, ql = w->ql;
	const char *ts = g->seq[v];
	uint64_t *vd = w->a_vd + off;
	int32_t *ak = w->a_k + off;
	uint32_t *xo = w->a_xo + off;
	od_t *b;

	for (j = 0; j < n; ++j) {
		int32_t k = o_extend1(w, (int32_t)vd[j] - SHIFT, ak[j], vl, ts);
		xo[j] += (uint32_t)(k - ak[j]) << 2;
		ak[j] = k;
	}
	if (w->n_B + n + 2 > w->max_B) w->st.flags |= GWFO_F_B_OVER;
	GROW(w->B, w->B_cap, w->n_B + n + 2);
	b = &w->B[w->n_B];
	b[0].vd = vd[0] - 1, b[0].xo = xo[0] + 2, b[0].k = ak[0] + 1;
	{
		int c = n == 1 || ak[0] > ak[1];
		b[1].vd = vd[0];
		b[1].xo = c ? xo[0] + 4 : xo[1] + 2;
		b[1].k = (c ? ak[0] : ak[1]) + 1;
	}
	for (j = 1; j < n - 1; ++j) {
		uint32_t x = xo[j - 1] + 2;
		int32_t k = ak[j - 1];
		x = k > ak[j] + 1 ? x : xo[j] + 4;
		k = k > ak[j] + 1 ? k : ak[j] + 1;
		x = k > ak[j + 1] + 1 ? x : xo[j + 1] + 2;
		k = k > ak[j + 1] + 1 ? k : ak[j + 1] + 1;
		b[j + 1].vd = vd[j], b[j + 1].k = k, b[j + 1].xo = x;
	}
	if (n >= 2) {
		int c = ak[n - 2] > ak[n - 1] + 1;
		b[n].vd = vd[n - 1];
		b[n].xo = c ? xo[n - 2] + 2 : xo[n - 1] + 4;
		b[n].k = c ? ak[n - 2] : ak[n - 1] + 1;
	}
	b[n + 1].vd = vd[n - 1] + 1, b[n + 1].xo = xo[n - 1] + 2, b[n + 1].k = ak[n - 1];

	for (j = 0; j < n; ++j) {
		int32_t d = (int32_t)vd[j] - SHIFT;
		if (ak[j] == vl - 1 || d + ak[j] == ql - 1) {
			xo[j] |= 1;
			A_push(w, vd[j], ak[j], xo[j]);
		}
	}
	/* vl is uint32_t in the reference (gwf-ed.cu:895), so `p->k < vl` is an unsigned compare:
	 * a candidate with k = -1 (an insertion before the first base of the vertex) is dropped */
	for (j = 0, m = 0; j < n + 2; ++j) {
		od_t *p = &b[j];
		int32_t d = (int32_t)p->vd - SHIFT;
		int k_ok = (w->opts & GWFO_O_EXACT_START) ? p->k < vl : (uint32_t)p->k < (uint32_t)vl;
		if (d + p->k < ql && k_ok) b[m++] = *p;
		else if (p->k == vl) tmp_push(w, gen_vd(v, d));
	}
	w->n_B += m;
	if (w->n_B > w->st.max_nB) w->st.max_nB = w->n_B;
}

/* gwf_ed_extend (gwf-ed.cu:1064-1290). Returns 1 when the query end was reached. */
static int o_extend(ows_t *w, int32_t *end_v, int32_t *end_off)
{
	const gwf_graph_t *g = w->g;
	int32_t i, x, n = w->n_a, do_dedup = 1, ql = w->ql, v1 = w->v1;
	const char *q = w->q;

	w->n_A = 0, w->A_head = 0, w->n_B = 0;
	*end_v = *end_off = -1;
	w->n_tmp = 0;
	w->st.W += n;
	if (n > w->st.max_na) w->st.max_na = n;

	for (x = 0, i = 1; i <= n; ++i)
		if (i == n || w->a_vd[i] != w->a_vd[i - 1] + 1) {
			o_extend_batch(w, i - x, x);
			x = i;
		}
	if (w->n_A == 0) do_dedup = 0;

	while (w->n_A > 0) {
		od_t t = w->A[w->A_head];
		uint32_t x0, ooo;
		int32_t v, d, k, ii, vl;
		++w->A_head, --w->n_A; /* static_A_shift :859-877 */
		ooo = t.xo & 1;
		v = (int32_t)(t.vd >> 32);
		d = (int32_t)t.vd - SHIFT;
		vl = (int32_t)g->len[v];
		k = o_extend1(w, d, t.k, vl, g->seq[v]);
		ii = k + d;
		x0 = (t.xo >> 1) + ((uint32_t)(k - t.k) << 1);
		if (k + 1 < vl && ii + 1 < ql) {
			int push1 = 1, push2 = 1;
			if (w->n_B >= 2) push1 = diag_update(&w->B[w->n_B - 2], v, d - 1, k + 1, x0 + 1, ooo);
			if (w->n_B >= 1) push2 = diag_update(&w->B[w->n_B - 1], v, d, k + 1, x0 + 2, ooo);
			if (push1) B_push(w, v, d - 1, k + 1, x0 + 1, 1);
			if (push2 || push1) B_push(w, v, d, k + 1, x0 + 2, 1);
			B_push(w, v, d + 1, k, x0 + 1, ooo);
		} else if (ii + 1 < ql) {
			int32_t ov = (int32_t)(g->aux[v] >> 32), nv = (int32_t)g->aux[v], n_ext = 0, j;
			tmp_push(w, gen_vd(v, d));
			for (j = 0; j < nv; ++j) {
				uint32_t wv = (uint32_t)g->arc[ov + j].a;
				int32_t ol = g->arc[ov + j].o;
				/* GWFO_O_ENTRY_KEY: the library's arrival key, whose vertex part is the arc's entry
				 * id (gwfo_index), so that arrivals at one query position through arcs of different
				 * overlaps into one vertex stay distinct */
				uint32_t kv = (w->opts & GWFO_O_ENTRY_KEY) ? (uint32_t)g->aux[g->n_vtx + ov + j] : wv;
				int absent = hset_put(w, (uint64_t)kv << 32 | (uint32_t)(ii + 1));
				if (q[ii + 1] == g->seq[wv][ol]) {
					++n_ext;
					if (absent) A_push(w, gen_vd(wv, ii + 1 - ol), ol, (x0 + 2) << 1 | 1);
				} else if (absent) {
					B_push(w, wv, ii - ol, ol, x0 + 1, 1);
					B_push(w, wv, ii + 1 - ol, ol, x0 + 2, 1);
				}
			}
			if (nv == 0 || n_ext != nv) B_push(w, v, d + 1, k, x0 + 1, 1);
		} else if (v1 < 0 || (v == v1 && k + 1 == vl)) {
			*end_v = v, *end_off = k;
			w->n_A = 0;
			return 1;
		} else if (k + 1 < vl) {
			B_push(w, v, d - 1, k + 1, x0 + 1, ooo);
		} else if (v != v1) {
			int32_t ov = (int32_t)(g->aux[v] >> 32), nv = (int32_t)g->aux[v], j;
			for (j = 0; j < nv; ++j)
				B_push(w, (uint32_t)g->arc[ov + j].a, ii - g->arc[ov + j].o, g->arc[ov + j].o, x0 + 1, 1);
		}
	}
	if (w->n_B > w->st.max_nB) w->st.max_nB = w->n_B;

	/* B -> a (gwf-ed.cu:1261-1276) */
	if (w->n_B > w->max_a) w->st.flags |= GWFO_F_A_COPY_OVER;
	GROW(w->a_vd, w->a_cap, w->n_B + 1);
	GROW(w->a_k, w->a_cap2, w->n_B + 1);
	GROW(w->a_xo, w->a_cap3, w->n_B + 1);
	for (i = 0; i < w->n_B; ++i)
		w->a_vd[i] = w->B[i].vd, w->a_k[i] = w->B[i].k, w->a_xo[i] = w->B[i].xo;
	w->n_a = w->n_B, w->n_B = 0;
	if (do_dedup) w->n_a = o_dedup(w, w->n_a);
	if (w->max_lag > 0 && w->n_a > 0) w->n_a = o_prune(w, w->n_a);
	return 0;
}

static uint32_t next_pow2_u32(uint32_t x) /* main.cu:279-292 */
{
	if (x == 0) return 0;
	--x;
	x |= x >> 1, x |= x >> 2, x |= x >> 4, x |= x >> 8, x |= x >> 16;
	return x + 1;
}

/* gwf_ed (gwf-ed.cu:1292-1337); max_lag > 0 adds o_prune after each step */
int32_t gwfo_ed_lag(const gwf_graph_t *g, int32_t ql, const char *q, int32_t v0, int32_t v1,
                    int32_t opts, int32_t max_lag, gwfo_stats_t *st)
{
	ows_t w;
	int32_t s = 0, end_v = -1, end_off = -1, ret;
	memset(&w, 0, sizeof(w));
	w.g = g, w.ql = ql, w.q = q, w.v1 = v1, w.opts = opts, w.max_lag = max_lag;
	/* main.cu:498-505 */
	w.max_a = (uint32_t)(((4 * (size_t)(ql > 0 ? ql : 0) * 0.1) + 1) * 4);
	w.max_B = 3 * w.max_a + 1;
	w.max_A = w.max_intv = w.max_swap = w.max_a;
	w.max_tmp = w.max_ooo = w.max_B;
	w.ha_cap = (uint64_t)next_pow2_u32((uint32_t)(ql > 0 ? ql : 0) * 32);
	hset_init(&w);
	GROW(w.a_vd, w.a_cap, 16);
	GROW(w.a_k, w.a_cap2, 16);
	GROW(w.a_xo, w.a_cap3, 16);
	w.a_vd[0] = gen_vd((uint32_t)v0, 0), w.a_k[0] = -1, w.a_xo[0] = 0;
	w.n_a = 1;
	if (ql <= 0) w.st.flags |= GWFO_F_NONTERM;
	while (w.n_a > 0) {
		int found = o_extend(&w, &end_v, &end_off);
		++w.st.steps;
		if (found && end_off < 0) { w.st.flags |= GWFO_F_NONTERM; break; }
		if (end_off >= 0 || w.n_a == 0) break;
		++s;
	}
	ret = end_v >= 0 ? s : -1;
	w.st.n_keys = (int64_t)w.h_n;
	if (st) *st = w.st;
	free(w.a_vd), free(w.a_k), free(w.a_xo), free(w.B), free(w.A);
	free(w.intv0), free(w.intv1), free(w.tmp0), free(w.tmp1), free(w.swap0), free(w.swap1);
	free(w.ooo), free(w.scr), free(w.hk);
	return ret;
}

int32_t gwfo_ed(const gwf_graph_t *g, int32_t ql, const char *q, int32_t v0, int32_t v1,
                int32_t opts, gwfo_stats_t *st)
{
	return gwfo_ed_lag(g, ql, q, v0, v1, opts, 0, st);
}

/* ------------------------------------------------------------------ index (main.cu:242-270) */
static int arc_cmp(const void *x, const void *y)
{
	const gwf_arc_t *a = (const gwf_arc_t *)x, *b = (const gwf_arc_t *)y;
	return a->a < b->a ? -1 : a->a > b->a ? 1 : 0;
}

/* entry ids of the arcs, for GWFO_O_ENTRY_KEY (the library's rule, gwf_runtime.cu upload_graph):
 * the target vertex w when every arc into w has the same overlap, else an id >= n_vtx that is
 * the same for the arcs into w with the same overlap and differs otherwise */
typedef struct { uint64_t key; uint32_t e; } oentry_t;
static int entry_cmp(const void *x, const void *y)
{
	const oentry_t *a = (const oentry_t *)x, *b = (const oentry_t *)y;
	return a->key < b->key ? -1 : a->key > b->key ? 1 : (a->e > b->e) - (a->e < b->e);
}

static void entry_ids(gwf_graph_t *g, uint64_t *eid)
{
	int32_t *first = (int32_t *)malloc(sizeof(int32_t) * (g->n_vtx ? g->n_vtx : 1));
	uint8_t *mixed = (uint8_t *)calloc(g->n_vtx ? g->n_vtx : 1, 1);
	oentry_t *t = (oentry_t *)malloc(sizeof(oentry_t) * (g->n_arc ? g->n_arc : 1));
	uint32_t e, n = 0, v, next = g->n_vtx;
	for (v = 0; v < g->n_vtx; ++v) first[v] = -1;
	for (e = 0; e < g->n_arc; ++e) {
		uint32_t w = (uint32_t)g->arc[e].a;
		if (first[w] < 0) first[w] = g->arc[e].o;
		else if (first[w] != g->arc[e].o) mixed[w] = 1;
	}
	for (e = 0; e < g->n_arc; ++e) {
		uint32_t w = (uint32_t)g->arc[e].a;
		eid[e] = w;
		if (mixed[w]) t[n].key = (uint64_t)w << 32 | (uint32_t)g->arc[e].o, t[n++].e = e;
	}
	qsort(t, n, sizeof(oentry_t), entry_cmp);
	for (e = 0; e < n; ++e) {
		if (e > 0 && t[e].key != t[e - 1].key) ++next;
		eid[t[e].e] = next;
	}
	free(first), free(mixed), free(t);
}

void gwfo_index(gwf_graph_t *g)
{
	uint32_t i, st;
	qsort(g->arc, g->n_arc, sizeof(gwf_arc_t), arc_cmp);
	/* aux[0 .. n_vtx) is the reference's CSR; aux[n_vtx + e] holds arc e's entry id */
	g->aux = (uint64_t *)calloc((size_t)g->n_vtx + g->n_arc + 1, sizeof(uint64_t));
	for (st = 0, i = 1; i <= g->n_arc; ++i)
		if (i == g->n_arc || g->arc[i].a >> 32 != g->arc[st].a >> 32) {
			uint32_t v = (uint32_t)(g->arc[st].a >> 32);
			if (v < g->n_vtx) g->aux[v] = (uint64_t)st << 32 | (i - st);
			st = i;
		}
	entry_ids(g, g->aux + g->n_vtx);
}

void gwfo_index_free(gwf_graph_t *g)
{
	free(g->aux);
	g->aux = 0;
}

/* ------------------------------------------------------------------ thread pool */
typedef struct {
	const gwf_graph_t *g;
	int32_t n, v1, opts;
	const char *seqs;
	const int64_t *offs;
	const int32_t *ql, *v0;
	int32_t *dist;
	gwfo_stats_t *st;
	int64_t next;
} pool_t;

static void *pool_worker(void *arg)
{
	pool_t *p = (pool_t *)arg;
	for (;;) {
		int64_t i = __atomic_fetch_add(&p->next, 1, __ATOMIC_RELAXED);
		if (i >= p->n) break;
		p->dist[i] = gwfo_ed(p->g, p->ql[i], p->seqs + p->offs[i], p->v0[i], p->v1, p->opts,
		                     p->st ? &p->st[i] : 0);
	}
	return 0;
}

int32_t gwfo_ed_batch(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs,
                      const int32_t *ql, const int32_t *v0, int32_t v1, int32_t opts,
                      int32_t *dist, gwfo_stats_t *st, int32_t n_threads)
{
	pool_t p;
	pthread_t *th;
	int32_t t;
	if (n_threads <= 0) n_threads = (int32_t)sysconf(_SC_NPROCESSORS_ONLN);
	if (n_threads < 1) n_threads = 1;
	if (n_threads > n && n > 0) n_threads = n;
	p.g = g, p.n = n, p.v1 = v1, p.opts = opts, p.seqs = seqs, p.offs = offs, p.ql = ql;
	p.v0 = v0, p.dist = dist, p.st = st, p.next = 0;
	th = malloc(sizeof(pthread_t) * (size_t)n_threads);
	for (t = 0; t < n_threads; ++t) pthread_create(&th[t], 0, pool_worker, &p);
	for (t = 0; t < n_threads; ++t) pthread_join(th[t], 0);
	free(th);
	return n_threads;
}

/* ------------------------------------------------------------------ ground truth */
/* Shortest path over states (position u, i query bases consumed). u = P is the virtual start
 * before offset 0 of v0; u < P is a base of the graph. Weights are 0/1, so two frontier lists
 * suffice (Dijkstra with buckets). */
int32_t gwfo_dp(const gwf_graph_t *g, int32_t ql, const char *q, int32_t v0, int32_t v1)
{
	int64_t P = 0, *base, nst, i;
	int32_t *dist, *vof, res = -1, d;
	int64_t *cur = 0, *nxt = 0, n_cur = 0, n_nxt = 0, c_cur = 0, c_nxt = 0;
	uint32_t v;
	if (ql < 0 || v0 < 0 || (uint32_t)v0 >= g->n_vtx) return -2;
	base = malloc(sizeof(int64_t) * (g->n_vtx + 1));
	for (v = 0; v < g->n_vtx; ++v) base[v] = P, P += g->len[v];
	base[g->n_vtx] = P;
	vof = malloc(sizeof(int32_t) * (size_t)(P + 1));
	for (v = 0; v < g->n_vtx; ++v) for (i = base[v]; i < base[v + 1]; ++i) vof[i] = (int32_t)v;
	nst = (P + 1) * (ql + 1);
	dist = malloc(sizeof(int32_t) * (size_t)nst);
	for (i = 0; i < nst; ++i) dist[i] = 0x7fffffff;
#define ST(u, ii) ((int64_t)(u) * (ql + 1) + (ii))
#define PUSH(arr, n, c, x) do { GROW(arr, c, (n) + 1); (arr)[(n)++] = (x); } while (0)
	dist[ST(P, 0)] = 0;
	PUSH(cur, n_cur, c_cur, ST(P, 0));
	for (d = 0; n_cur > 0; ++d) {
		int64_t h;
		for (h = 0; h < n_cur; ++h) {
			int64_t s = cur[h], u = s / (ql + 1), succ[64];
			int32_t ii = (int32_t)(s % (ql + 1)), ns = 0, t;
			if (dist[s] != d) continue;
			if (ii == ql) {
				if (v1 < 0) { res = d; goto done; }
				if (u < P && vof[u] == v1 && u == base[v1 + 1] - 1) { res = d; goto done; }
			}
			if (u == P) succ[ns++] = base[v0];
			else {
				int32_t vv = vof[u];
				if (u + 1 < base[vv + 1]) succ[ns++] = u + 1;
				else if (g->aux) {
					int32_t ov = (int32_t)(g->aux[vv] >> 32), nv = (int32_t)g->aux[vv], j;
					for (j = 0; j < nv && ns < 64; ++j) {
						uint32_t w = (uint32_t)g->arc[ov + j].a;
						int32_t o = g->arc[ov + j].o;
						if (o >= 0 && (uint32_t)o < g->len[w]) succ[ns++] = base[w] + o;
					}
				}
			}
			for (t = 0; t < ns; ++t) {
				int64_t un = succ[t], s2;
				if (ii < ql) {
					int wgt = q[ii] != g->seq[vof[un]][un - base[vof[un]]];
					s2 = ST(un, ii + 1);
					if (dist[s2] > d + wgt) {
						dist[s2] = d + wgt;
						if (wgt) PUSH(nxt, n_nxt, c_nxt, s2); else PUSH(cur, n_cur, c_cur, s2);
					}
				}
				s2 = ST(un, ii);
				if (dist[s2] > d + 1) { dist[s2] = d + 1; PUSH(nxt, n_nxt, c_nxt, s2); }
			}
			if (ii < ql) {
				int64_t s2 = ST(u, ii + 1);
				if (dist[s2] > d + 1) { dist[s2] = d + 1; PUSH(nxt, n_nxt, c_nxt, s2); }
			}
		}
		{ int64_t *t = cur; cur = nxt; nxt = t; }
		{ int64_t t = c_cur; c_cur = c_nxt; c_nxt = t; }
		n_cur = n_nxt, n_nxt = 0;
	}
done:
#undef ST
#undef PUSH
	free(cur), free(nxt), free(dist), free(vof), free(base);
	return res;
}
