// gwf_cigar.cuh — base-level alignment (CIGAR) of each read against the text its traced path
// spells. No reference counterpart: the reference computes distances only (README.md:117-118).
//
// One warp per read. The text is the path's bases: seq[v0][0..], then seq[w][o..] for each later
// vertex w entered over an arc of overlap o, through the end offset in the last vertex. The warp
// copies it into the read's arena, then runs an edit-distance wavefront over (query, text): at
// score s, diagonal k = j - i holds the furthest text position j reached with s edits, from
//   mismatch  W[s-1][k] + 1,  deletion (text base only)  W[s-1][k-1] + 1,
//   insertion (query base only)  W[s-1][k+1],
// then extended over equal bytes. Every wavefront is kept ((D + 1)^2 entries for the traced
// distance D, which bounds the optimum on the path), so lane 0 can walk back from the end
// (diagonal m - ql at offset m) recomputing each step's candidates, and emit the operations in
// runs: '=' 7, 'X' 8, 'I' 1 (query base), 'D' 2 (text base), as BAM codes len << 4 | op.
#pragma once
#include "gwf_device.cuh"

namespace gwfb {

struct CigarParams {
	DevGraph g;
	DevReads r;
	const int32_t *order;     // reads of this launch
	int32_t n_order;
	int32_t max_nv, max_ops;  // widths of the path and CIGAR rows
	uint8_t *ws;              // arenas
	const int64_t *slot_off;  // arena byte offset per launch position
	const int32_t *dist, *status, *end_off, *path_n, *path_v, *path_arc;
	int32_t *cigar_n;         // runs, -1 when there is no CIGAR for the read
	uint32_t *cigar;          // n x max_ops runs
};

constexpr uint32_t CIG_I = 1, CIG_D = 2, CIG_EQ = 7, CIG_X = 8;
constexpr int32_t WF_NONE = INT32_MIN / 4;

// Arena of one read with query length ql and distance bound d: the text (at most ql + d bases
// plus padding), the wavefronts, the reversed runs.
__host__ __device__ inline int64_t cigar_text_cap(int32_t ql, int32_t d) { return (int64_t)ql + d + 16; }
__host__ __device__ inline int64_t cigar_arena_bytes(int32_t ql, int32_t d)
{
	return al16(cigar_text_cap(ql, d)) + al16(4LL * (d + 1) * (d + 1)) + al16(4LL * (2LL * d + 2));
}

#ifdef __CUDACC__
// Candidate offset on diagonal k from diagonal kk of the previous wavefront (band s1), moved by
// add text positions; WF_NONE when kk is outside the band, unreached, or the move leaves the
// (query, text) rectangle.
__device__ __forceinline__ int32_t wf_cand(const int32_t *Wp, int32_t s1, int32_t kk, int32_t add, int32_t k,
                                           int32_t m, int32_t ql)
{
	if (kk < -s1 || kk > s1) return WF_NONE;
	const int32_t v = Wp[kk + s1];
	if (v < 0) return WF_NONE;
	const int32_t j = v + add, i = j - k;
	return j <= m && i >= 0 && i <= ql ? j : WF_NONE;
}

__global__ void __launch_bounds__(256) k_cigar(const __grid_constant__ CigarParams p)
{
	const int lane = threadIdx.x & 31;
	const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
	if (gw >= p.n_order) return;
	const int32_t r = p.order[gw];
	const int32_t d = p.dist[r], pn = p.path_n[r], ql = p.r.ql[r];
	if (p.status[r] != 0 || d < 0 || pn < 1 || pn > p.max_nv || ql <= 0) {
		if (lane == 0) p.cigar_n[r] = -1;
		return;
	}
	uint8_t *const wsb = p.ws + p.slot_off[gw];
	const int64_t t_cap = cigar_text_cap(ql, d);
	uint8_t *const t = wsb;
	int32_t *const W = (int32_t *)(wsb + al16(t_cap));
	uint32_t *const runs = (uint32_t *)(wsb + al16(t_cap) + al16(4LL * (d + 1) * (d + 1)));
	const uint8_t *const q = p.r.raw + p.r.raw_off[r];
	const int64_t row = (int64_t)r * p.max_nv;

	// 1. the text of the path (warp-uniform loop over the path, lanes copy the bases)
	int64_t m = 0;
	bool bad = false;
	for (int32_t j = 0; j < pn; ++j) {
		const int32_t v = p.path_v[row + j], a = p.path_arc[row + j];
		if (v < 0 || (uint32_t)v >= p.g.n_vtx || (j > 0 && a < 0)) {
			bad = true;
			break;
		}
		const int32_t vl = (int32_t)__ldg(p.g.len + v);
		const int32_t o = j == 0 ? 0 : (int32_t)__ldg(p.g.arc + a).y;
		const int32_t e = j == pn - 1 ? p.end_off[r] + 1 : vl;
		if (o < 0 || e < o || e > vl || m + (e - o) > t_cap - 16) {
			bad = true;
			break;
		}
		const uint8_t *src = p.g.raw + __ldg(p.g.base + v) + o;
		for (int32_t x = lane; x < e - o; x += 32) t[m + x] = src[x];
		m += e - o;
	}
	__syncwarp();
	const int32_t mm = (int32_t)m, kend = mm - ql;

	// 2. the wavefronts, s = 0 .. d at most
	int32_t s_fin = -1;
	for (int32_t s = 0; s <= d && !bad; ++s) {
		int32_t *const Ws = W + (int64_t)s * s;
		const int32_t *const Wp = s > 0 ? W + (int64_t)(s - 1) * (s - 1) : W;
		bool done = false;
		for (int32_t kb = -s; kb <= s; kb += 32) {
			const int32_t k = kb + lane;
			if (k > s) continue;
			int32_t j = WF_NONE;
			if (s == 0) {
				j = 0;
			} else {
				const int32_t cm = wf_cand(Wp, s - 1, k, 1, k, mm, ql);
				const int32_t cd = wf_cand(Wp, s - 1, k - 1, 1, k, mm, ql);
				const int32_t ci = wf_cand(Wp, s - 1, k + 1, 0, k, mm, ql);
				j = max(cm, max(cd, ci));
			}
			if (j >= 0) {
				while (j < mm && j - k < ql && t[j] == q[j - k]) ++j;
				if (k == kend && j == mm) done = true;
			} else
				j = -1;
			Ws[k + s] = j;
		}
		__syncwarp();
		if (__any_sync(FULL, done)) {
			s_fin = s;
			break;
		}
	}

	// 3. walk back from the end, recomputing each step's candidates; runs are collected in reverse
	if (lane == 0) {
		bool ok = !bad && s_fin >= 0;
		int32_t n_runs = 0;
		uint32_t cur_op = 0, cur_len = 0;
		auto emit = [&](uint32_t op, int32_t len) {
			if (len <= 0) return;
			if (cur_len && op == cur_op) {
				cur_len += (uint32_t)len;
				return;
			}
			if (cur_len) runs[n_runs++] = cur_len << 4 | cur_op;
			cur_op = op, cur_len = (uint32_t)len;
		};
		int32_t s = s_fin, k = kend, j = mm;
		while (ok && s > 0) {
			const int32_t *const Wp = W + (int64_t)(s - 1) * (s - 1);
			const int32_t cm = wf_cand(Wp, s - 1, k, 1, k, mm, ql);
			const int32_t cd = wf_cand(Wp, s - 1, k - 1, 1, k, mm, ql);
			const int32_t ci = wf_cand(Wp, s - 1, k + 1, 0, k, mm, ql);
			const int32_t j0 = max(cm, max(cd, ci));
			if (j0 < 0 || j0 > j || n_runs + 2 > 2 * d + 2) {
				ok = false;
				break;
			}
			emit(CIG_EQ, j - j0);
			if (cm == j0) emit(CIG_X, 1), j = j0 - 1;
			else if (cd == j0) emit(CIG_D, 1), j = j0 - 1, --k;
			else emit(CIG_I, 1), j = j0, ++k;
			--s;
		}
		if (ok && k != 0) ok = false;
		if (ok) {
			emit(CIG_EQ, j);
			if (cur_len) runs[n_runs++] = cur_len << 4 | cur_op;
			const int64_t crow = (int64_t)r * p.max_ops;
			for (int32_t x = 0; x < n_runs && x < p.max_ops; ++x) p.cigar[crow + x] = runs[n_runs - 1 - x];
		}
		p.cigar_n[r] = ok ? n_runs : -1;
	}
}
#endif

} // namespace gwfb
