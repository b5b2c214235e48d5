// gwf_group.cuh — one read aligned by a group of NW warps (NW = 2, 4 or 8) of one CTA, and the
// class-ordered persistent kernel that runs long reads on groups and short reads on single warps.
//
// The score loop is the one of align_read_t (gwf_kernels.cuh), phase for phase (extension,
// in-vertex successors, arc waves, ended intervals and the next wavefront; the reference lines
// are cited there). Every list pass runs over the group's 32 * NW threads instead of one warp's
// 32 lanes. Lists whose order matters (in-vertex candidates, ended points, intervals, the
// merged wavefront) are compacted with a group prefix sum: one named barrier per 32 * NW
// entries. Lists whose order does not matter (vertex-end and entered states, arc-side
// candidates, ended points of arcs: they are sorted or deduplicated later) take their positions
// from per-group counters in shared memory with one atomic add per warp, and need no barrier.
// Every overflow check and every exit test goes through a barrier reduction, so that the group
// takes each branch as a whole. Long candidate lists are radix-sorted with one histogram per
// warp (stable in the warp order), the same dense-key mapping as warp_radix_sort.
#pragma once
#include "gwf_kernels.cuh"

namespace gwfb {

struct GrpShm {              // per group, in shared memory
	uint64_t part[2][8];     // per-warp partials of scans and reductions, double-buffered
	uint32_t red[2][8][4];   // per-warp min/max quadruples of the radix sort, double-buffered
	uint32_t ctr[8];         // append counters (monotonic; positions are relative to a base)
	int32_t claim;           // queue position claimed for the group
	int32_t pad[5];
	long long claim64;       // serving: queue position claimed for the group (-1 = leave)
};
enum { C_E = 0, C_N, C_F, C_BA, C_TA, C_KEYS };

template <int NW>
struct Grp {
	static constexpr int GS = 32 * NW;
	int rank, wid, lane, bar, ph;
	GrpShm *sh;

	__device__ __forceinline__ void init(GrpShm *s, int gi)
	{
		sh = s;
		lane = threadIdx.x & 31;
		wid = (threadIdx.x >> 5) % NW;
		rank = wid * 32 + lane;
		bar = 1 + gi; // named barrier per group; 0 is __syncthreads
		ph = 0;
	}
	__device__ __forceinline__ void sync() const
	{
		asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(GS) : "memory");
	}
	__device__ __forceinline__ uint32_t ctr(int k) const { return *(volatile const uint32_t *)&sh->ctr[k]; }
	// OR of x over the group (a barrier)
	__device__ __forceinline__ uint32_t or_bits(uint32_t x)
	{
		x = __reduce_or_sync(FULL, x);
		uint64_t *b = sh->part[ph];
		ph ^= 1;
		if (lane == 0) b[wid] = x;
		sync();
		uint32_t r = 0;
#pragma unroll
		for (int w = 0; w < NW; ++w) r |= (uint32_t)b[w];
		return r;
	}
	// exclusive prefix of c over the group in rank order; *tot = the group's sum (a barrier)
	__device__ __forceinline__ uint32_t scan(uint32_t c, uint32_t *tot)
	{
		uint32_t x = c;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t y = __shfl_up_sync(FULL, x, o);
			if (lane >= o) x += y;
		}
		uint64_t *b = sh->part[ph];
		ph ^= 1;
		if (lane == 31) b[wid] = x;
		sync();
		uint32_t pre = 0, t = 0;
#pragma unroll
		for (int w = 0; w < NW; ++w) {
			const uint32_t v = (uint32_t)b[w];
			pre += w < wid ? v : 0;
			t += v;
		}
		*tot = t;
		return pre + x - c;
	}
	__device__ __forceinline__ uint32_t scan1(bool f, uint32_t *tot)
	{
		const uint32_t m = __ballot_sync(FULL, f);
		uint64_t *b = sh->part[ph];
		ph ^= 1;
		if (lane == 0) b[wid] = __popc(m);
		sync();
		uint32_t pre = 0, t = 0;
#pragma unroll
		for (int w = 0; w < NW; ++w) {
			const uint32_t v = (uint32_t)b[w];
			pre += w < wid ? v : 0;
			t += v;
		}
		*tot = t;
		return pre + __popc(m & lanemask_lt());
	}
	// group max of a signed int (a barrier)
	__device__ __forceinline__ int32_t max_i32(int32_t x)
	{
		x = __reduce_max_sync(FULL, x);
		uint64_t *b = sh->part[ph];
		ph ^= 1;
		if (lane == 0) b[wid] = (uint64_t)(uint32_t)x;
		sync();
		int32_t r = INT32_MIN;
#pragma unroll
		for (int w = 0; w < NW; ++w) {
			const int32_t v = (int32_t)(uint32_t)b[w];
			r = v > r ? v : r;
		}
		return r;
	}
	// inclusive prefix max of a u64 over the group in rank order: *below = max of the warps
	// before this one, *all = the group's max (a barrier)
	__device__ __forceinline__ uint64_t incl_max(uint64_t x, uint64_t *below, uint64_t *all)
	{
		x = warp_incl_max(x);
		uint64_t *b = sh->part[ph];
		ph ^= 1;
		if (lane == 31) b[wid] = x;
		sync();
		uint64_t lo = 0, a = 0;
#pragma unroll
		for (int w = 0; w < NW; ++w) {
			const uint64_t v = b[w];
			if (w < wid) lo = v > lo ? v : lo;
			a = v > a ? v : a;
		}
		*below = lo, *all = a;
		return x > lo ? x : lo;
	}
	// c items appended to the list behind counter k, in no particular order between warps:
	// returns the counter value before this thread's items (no barrier)
	__device__ __forceinline__ uint32_t append(uint32_t c, int k)
	{
		uint32_t x = c;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t y = __shfl_up_sync(FULL, x, o);
			if (lane >= o) x += y;
		}
		uint32_t base = 0;
		if (lane == 31 && x) base = atomicAdd(&sh->ctr[k], x);
		base = __shfl_sync(FULL, base, 31);
		return base + x - c;
	}
	__device__ __forceinline__ uint32_t append1(bool f, int k)
	{
		const uint32_t m = __ballot_sync(FULL, f);
		uint32_t base = 0;
		if (lane == 0 && m) base = atomicAdd(&sh->ctr[k], (uint32_t)__popc(m));
		base = __shfl_sync(FULL, base, 0);
		return base + __popc(m & lanemask_lt());
	}
};

// Stable LSD radix sort of n diagonals by the group (the dense keys and passes of
// warp_radix_sort). Warp w sorts the contiguous range w*per .. into its own 256-bin histogram in
// hist[w * 256 ..]; the bins are scanned digit-major across the warps, so that equal digits keep
// their input order. Returns false (nothing done) when the dense keys need more than 48 bits.
template <int NW>
static __device__ __noinline__ bool grp_radix_sort(Grp<NW> &G, uint64_t *keys, int32_t *vals, int32_t n,
                                                   uint64_t *tmp_keys, int32_t *tmp_vals, uint32_t *hist)
{
	constexpr int GS = 32 * NW, D = 256 / GS; // digits per thread in the bin scan
	const int lane = G.lane, wid = G.wid, rank = G.rank;
	uint32_t vmin = 0xffffffffu, vmax = 0, dmin = 0xffffffffu, dmax = 0;
	for (int32_t i = rank; i < n; i += GS) {
		const uint64_t k = keys[i];
		const uint32_t v = (uint32_t)(k >> 32), d = (uint32_t)k;
		vmin = v < vmin ? v : vmin, vmax = v > vmax ? v : vmax;
		dmin = d < dmin ? d : dmin, dmax = d > dmax ? d : dmax;
	}
	vmin = __reduce_min_sync(FULL, vmin), vmax = __reduce_max_sync(FULL, vmax);
	dmin = __reduce_min_sync(FULL, dmin), dmax = __reduce_max_sync(FULL, dmax);
	{
		uint32_t(*r)[4] = G.sh->red[G.ph];
		G.ph ^= 1;
		if (lane == 0) r[wid][0] = vmin, r[wid][1] = vmax, r[wid][2] = dmin, r[wid][3] = dmax;
		G.sync();
#pragma unroll
		for (int w = 0; w < NW; ++w) {
			vmin = r[w][0] < vmin ? r[w][0] : vmin, vmax = r[w][1] > vmax ? r[w][1] : vmax;
			dmin = r[w][2] < dmin ? r[w][2] : dmin, dmax = r[w][3] > dmax ? r[w][3] : dmax;
		}
	}
	const uint64_t span_d = (uint64_t)(dmax - dmin) + 1;
	const uint32_t span_v = vmax - vmin;
	if ((span_v ? 32 - __clz(span_v) : 0) + (64 - __clzll((long long)span_d)) > 48) return false;
	const uint64_t top = (uint64_t)span_v * span_d + (dmax - dmin);
	const int32_t bits = 64 - __clzll((long long)top);
	const int32_t passes = bits > 0 ? (bits + 7) / 8 : 1;
	const int32_t per = (n + NW - 1) / NW, lo = wid * per < n ? wid * per : n, hi = lo + per < n ? lo + per : n;
	uint32_t *const h = hist + wid * 256;
	uint64_t *src_k = keys, *dst_k = tmp_keys;
	int32_t *src_v = vals, *dst_v = tmp_vals;
	for (int32_t pass = 0; pass < passes; ++pass) {
		const int32_t shift = 8 * pass;
		for (int32_t b = lane; b < 256; b += 32) h[b] = 0;
		__syncwarp();
		for (int32_t base = lo; base < hi; base += 32) {
			const int32_t i = base + lane;
			const bool act = i < hi;
			uint32_t digit = 256 + lane;
			if (act) {
				const uint64_t k = src_k[i];
				const uint64_t dk = (uint64_t)((uint32_t)(k >> 32) - vmin) * span_d + ((uint32_t)k - dmin);
				digit = (uint32_t)(dk >> shift) & 255u;
			}
			const uint32_t same = __match_any_sync(FULL, digit);
			if (act && (same & lanemask_lt()) == 0) h[digit] += __popc(same);
			__syncwarp();
		}
		G.sync();
		// bins in digit-major order: start of (digit d, warp w) = all of digits < d + warps < w of d
		uint32_t dt[D], tsum = 0;
#pragma unroll
		for (int t = 0; t < D; ++t) {
			const int d = rank * D + t;
			uint32_t run = 0;
#pragma unroll
			for (int w = 0; w < NW; ++w) {
				const uint32_t c = hist[w * 256 + d];
				hist[w * 256 + d] = run;
				run += c;
			}
			dt[t] = run, tsum += run;
		}
		uint32_t tot;
		uint32_t pre = G.scan(tsum, &tot);
#pragma unroll
		for (int t = 0; t < D; ++t) {
			const int d = rank * D + t;
#pragma unroll
			for (int w = 0; w < NW; ++w) hist[w * 256 + d] += pre;
			pre += dt[t];
		}
		G.sync();
		for (int32_t base = lo; base < hi; base += 32) {
			const int32_t i = base + lane;
			const bool act = i < hi;
			uint32_t digit = 256 + lane;
			uint64_t k = 0;
			int32_t v = 0;
			if (act) {
				k = src_k[i];
				if (src_v) v = src_v[i];
				const uint64_t dk = (uint64_t)((uint32_t)(k >> 32) - vmin) * span_d + ((uint32_t)k - dmin);
				digit = (uint32_t)(dk >> shift) & 255u;
			}
			const uint32_t same = __match_any_sync(FULL, digit);
			const uint32_t pos = act ? h[digit] + __popc(same & lanemask_lt()) : 0;
			__syncwarp();
			if (act) {
				dst_k[pos] = k;
				if (src_v) dst_v[pos] = v;
				if ((same & lanemask_lt()) == 0) h[digit] += __popc(same);
			}
			__syncwarp();
		}
		G.sync();
		uint64_t *tk = src_k;
		src_k = dst_k, dst_k = tk;
		int32_t *tv = src_v;
		src_v = src_v ? dst_v : nullptr, dst_v = tv;
	}
	if (src_k != keys) {
		for (int32_t i = rank; i < n; i += GS) {
			keys[i] = src_k[i];
			if (vals) vals[i] = src_v[i];
		}
		G.sync();
	}
	return true;
}

// Sorts n diagonals (optional int32 values) for the group: short lists on the first warp (rank
// sort or bitonic network), long ones by the group's radix sort (the first warp's bitonic
// network when the dense keys are too wide, or the histograms do not fit the scratch).
template <int NW>
__device__ __forceinline__ void grp_sort(Grp<NW> &G, uint64_t *keys, int32_t *vals, int32_t n, uint64_t *tmp_keys,
                                         int32_t *tmp_vals, uint32_t *hist, bool hist_fits)
{
	if (n > kRadixMin && hist_fits && grp_radix_sort<NW>(G, keys, vals, n, tmp_keys, tmp_vals, hist)) return;
	if (G.wid == 0) warp_bitonic_sort(keys, vals, n);
	G.sync();
}

// align_read_t<false, LAG> for a group of NW warps: same arena layout (caps_for(min(ql, ql_cap),
// level)), same results. All threads of the group call it with the same arguments.
template <int NW, bool LAG>
__device__ __noinline__ void align_read_grp(const KParams &p, int32_t r, uint8_t *wsb, int32_t ql_cap, int32_t level,
                                            GrpShm *gsh, int gi)
{
	constexpr int GS = 32 * NW;
	Grp<NW> G;
	G.init(gsh, gi);
	const int rank = G.rank, lane = G.lane;
	const Caps c = caps_for(p.r.ql[r] < ql_cap ? p.r.ql[r] : ql_cap, level, p.dens_milli);
	const DevGraph &g = p.g;
	const WsOff o = ws_layout(c);
	uint64_t *const h = (uint64_t *)(wsb + o.h);
	uint32_t off_a_vd = (uint32_t)o.a_vd, off_x_vd = (uint32_t)o.x_vd;
	const uint32_t off_ba_vd = (uint32_t)o.ba_vd;
	uint32_t off_e_vd = (uint32_t)o.w0_vd, off_f_vd = (uint32_t)o.w1_vd;
	const uint32_t off_n_vd = (uint32_t)o.n_vd, off_tb = (uint32_t)o.tb, off_ta = (uint32_t)o.ta;
	const uint32_t off_ilo = (uint32_t)o.i0_lo, off_ihi = (uint32_t)o.i0_hi;
	const uint32_t off_clo = (uint32_t)o.i1_lo, off_chi = (uint32_t)o.i1_hi;
	uint32_t off_a_k = (uint32_t)o.a_k, off_x_k = (uint32_t)o.x_k;
	const uint32_t off_ba_k = (uint32_t)o.ba_k;
	uint32_t off_e_k = (uint32_t)o.w0_k, off_f_k = (uint32_t)o.w1_k;
	const uint32_t off_n_k = (uint32_t)o.n_k;
#define A_VD ((uint64_t *)(wsb + off_a_vd))
#define X_VD ((uint64_t *)(wsb + off_x_vd))
#define BA_VD ((uint64_t *)(wsb + off_ba_vd))
#define E_VD ((uint64_t *)(wsb + off_e_vd))
#define F_VD ((uint64_t *)(wsb + off_f_vd))
#define N_VD ((uint64_t *)(wsb + off_n_vd))
#define TB ((uint64_t *)(wsb + off_tb))
#define TA ((uint64_t *)(wsb + off_ta))
#define ILO ((uint64_t *)(wsb + off_ilo))
#define IHI ((uint64_t *)(wsb + off_ihi))
#define CLO ((uint64_t *)(wsb + off_clo))
#define CHI ((uint64_t *)(wsb + off_chi))
#define A_K ((int32_t *)(wsb + off_a_k))
#define X_K ((int32_t *)(wsb + off_x_k))
#define BA_K ((int32_t *)(wsb + off_ba_k))
#define E_K ((int32_t *)(wsb + off_e_k))
#define F_K ((int32_t *)(wsb + off_f_k))
#define N_K ((int32_t *)(wsb + off_n_k))
	// radix histograms, one per warp: the interval scratch, free whenever a sort runs
	uint32_t *const radix_hist = (uint32_t *)(wsb + off_clo);
	const bool hist_fits = 8LL * (c.iv + c.tb + c.ta) >= 1024LL * NW;

	ReadCtx rc;
	rc.ql = p.r.ql[r];
	rc.v1 = p.r.v1;
	rc.qpk = p.r.pk + p.r.pk_off[r];
	rc.qraw = p.r.raw + p.r.raw_off[r];
	rc.packed = g.pure && p.r.pure[r];
	rc.quirk = !(p.flags & 1);
	const int32_t ql = rc.ql, v1 = rc.v1;
	const int32_t v0 = p.r.v0[r];

	int32_t dist = -1, st = ST_OK, steps = 0;
	int64_t W = 0;
	if (ql <= 0 || v0 < 0 || (uint32_t)v0 >= g.n_vtx || (v1 >= 0 && (uint32_t)v1 >= g.n_vtx)) {
		if (rank == 0) p.dist[r] = -1, p.status[r] = ST_BAD_INPUT;
		return;
	}
	if (o.total > 0xffffffffLL) {
		if (rank == 0) p.dist[r] = -1, p.status[r] = ST_CAPACITY;
		return;
	}
	{
		uint4 *h4 = (uint4 *)h;
		const uint4 z = make_uint4(0, 0, 0, 0);
		for (int32_t i = rank; i < c.h / 2; i += GS) h4[i] = z;
	}
	if (rank == 0) A_VD[0] = gen_vd((uint32_t)v0, 0), A_K[0] = -1; // gwf-ed.cu:1303-1308
	G.sync();
	// counter bases: every append of the previous read is behind the barrier above
	uint32_t uE = G.ctr(C_E), uN = G.ctr(C_N), uF = G.ctr(C_F), uBA = G.ctr(C_BA), uTA = G.ctr(C_TA);
	const uint32_t uKEYS = G.ctr(C_KEYS);
	const uint32_t hmask = (uint32_t)c.h - 1;
	const int32_t hlimit = c.h - c.h / 4;
	int32_t n_a = 1, n_i = 0;
	uint64_t i_min = 0, i_max = 0;

	for (int32_t s = 0;; ++s) {
		if (s >= c.max_steps) {
			st = ST_CAPACITY;
			break;
		}
		++steps;
		W += n_a;
		bool found = false, ovf = false;

		// ---- phase 1: extension; vertex-end / query-end states to the first wave (unordered)
		int32_t n_e;
		{
			bool f_l = false, o_l = false;
			for (int32_t base = 0; base < n_a; base += GS) {
				const int32_t j = base + rank;
				bool toE = false;
				uint64_t vd = 0;
				int32_t k = 0;
				if (j < n_a) {
					vd = A_VD[j];
					k = A_K[j];
					const uint32_t v = vd_v(vd);
					const int32_t d = vd_d(vd), vl = (int32_t)__ldg(g.len + v);
					k = ext(g, rc, v, d, k, vl);
					A_K[j] = k;
					const bool vend = k == vl - 1, qend = d + k == ql - 1;
					if (qend) {
						if (v1 < 0 || ((int32_t)v == v1 && vend)) f_l = true;
						else toE = true;
					} else if (vend)
						toE = true;
				}
				const uint32_t pos = G.append1(toE, C_E) - uE;
				if (toE) {
					if (pos < (uint32_t)c.w) E_VD[pos] = vd, E_K[pos] = k;
					else o_l = true;
				}
			}
			const uint32_t fl = G.or_bits((uint32_t)f_l | (uint32_t)o_l << 1);
			if (fl & 1) {
				dist = s;
				break;
			}
			const uint32_t ce = G.ctr(C_E);
			n_e = (int32_t)(ce - uE);
			uE = ce;
			if (fl & 2) ovf = true;
		}

		// ---- phase 2: in-vertex successors, in diagonal order (group prefix sums)
		int32_t n_x = 0, n_tb = 0;
		for (int32_t base = 0; base < n_a; base += GS) {
			const int32_t j = base + rank;
			uint64_t cv[3];
			int32_t ck[3];
			bool keep[3] = {false, false, false}, tmp[3] = {false, false, false};
			if (j < n_a) {
				const uint64_t vd = A_VD[j];
				const int32_t k = A_K[j];
				const int32_t vl = (int32_t)__ldg(g.len + vd_v(vd));
				const uint64_t pv = j > 0 ? A_VD[j - 1] : 0;
				const int32_t pk = j > 0 ? A_K[j - 1] : 0;
				const uint64_t nv = j + 1 < n_a ? A_VD[j + 1] : 0;
				const int32_t nk = j + 1 < n_a ? A_K[j + 1] : 0;
				const bool left_in = j > 0 && pv == vd - 1, left2 = j > 0 && pv == vd - 2;
				const bool right_in = j + 1 < n_a && nv == vd + 1, right2 = j + 1 < n_a && nv == vd + 2;
				bool has[3];
				has[0] = !left_in;
				cv[0] = vd - 1;
				ck[0] = k + 1;
				if (left2 && pk > ck[0]) ck[0] = pk;
				has[1] = true;
				cv[1] = vd;
				ck[1] = k + 1;
				if (left_in && pk > ck[1]) ck[1] = pk;
				if (right_in && nk + 1 > ck[1]) ck[1] = nk + 1;
				has[2] = !right_in && !right2;
				cv[2] = vd + 1;
				ck[2] = k;
#pragma unroll
				for (int t = 0; t < 3; ++t)
					if (has[t]) {
						const int32_t dd = vd_d(cv[t]);
						const bool kin = rc.quirk ? (uint32_t)ck[t] < (uint32_t)vl : ck[t] < vl;
						if (dd + ck[t] < ql && kin) keep[t] = true;
						else if (ck[t] == vl) tmp[t] = true;
					}
				// as in align_read_t: the first wave records this diagonal's end already
				if (tmp[1] && k == vl - 1 && vd_d(vd) + k != ql - 1) tmp[1] = false;
			}
			const uint32_t kc = (uint32_t)keep[0] + keep[1] + keep[2], tc = (uint32_t)tmp[0] + tmp[1] + tmp[2];
			uint32_t tot;
			const uint32_t pre = G.scan(kc | tc << 16, &tot);
			int32_t off = n_x + (int32_t)(pre & 0xffff), offt = n_tb + (int32_t)(pre >> 16);
#pragma unroll
			for (int t = 0; t < 3; ++t)
				if (keep[t]) {
					if (off < c.x) X_VD[off] = cv[t], X_K[off] = ck[t];
					++off;
				}
#pragma unroll
			for (int t = 0; t < 3; ++t)
				if (tmp[t]) {
					if (offt < c.tb) TB[offt] = cv[t];
					++offt;
				}
			n_x += (int32_t)(tot & 0xffff), n_tb += (int32_t)(tot >> 16);
		}
		if (n_x > c.x || n_tb > c.tb) ovf = true;

		// ---- phase 3: arc waves (unordered appends; barrier reductions decide every branch)
		int32_t n_ba = 0, n_ta = 0;
		for (int32_t wave = 0; n_e > 0 && !ovf; ++wave) {
			if (wave > ql + 2) {
				ovf = true;
				break;
			}
			bool o_l = false;
			uint32_t nk = 0; // arrival keys this thread inserted in this wave
			for (int32_t base = 0; base < n_e; base += GS) {
				const int32_t j = base + rank;
				bool act = j < n_e, isq = false, isv = false;
				uint64_t vd = 0;
				int32_t k = 0, d = 0, vl = 0, i = 0, nv = 0;
				uint32_t v = 0, aoff = 0;
				if (act) {
					vd = E_VD[j], k = E_K[j];
					v = vd_v(vd), d = vd_d(vd), vl = (int32_t)__ldg(g.len + v), i = d + k;
					isq = i == ql - 1;
					isv = !isq;
					aoff = __ldg(g.arc_off + v);
					const int32_t deg = (int32_t)(__ldg(g.arc_off + v + 1) - aoff);
					if (isv || (k + 1 == vl && (int32_t)v != v1)) nv = deg;
				}
				{
					const uint32_t pos = G.append1(isv, C_TA) - uTA;
					if (isv) {
						if (pos < (uint32_t)c.ta) TA[pos] = vd;
						else o_l = true;
					}
				}
				const int32_t max_nv = __reduce_max_sync(FULL, (uint32_t)nv);
				int32_t n_ext = 0;
				for (int32_t t = 0; t < max_nv; ++t) {
					bool enter = false, two = false, one = false;
					uint32_t w = 0;
					int32_t ol = 0;
					if (t < nv) {
						const uint2 e = __ldg(g.arc + aoff + t);
						w = e.x, ol = (int32_t)e.y;
						if (isv) {
							const uint32_t kv = g.arc_key ? __ldg(g.arc_key + aoff + t) : w;
							const int ins = hset_insert(h, hmask, (uint64_t)kv << 32 | (uint32_t)(i + 1));
							if (ins < 0) o_l = true;
							const bool absent = ins == 1;
							if (base_eq(g, rc, w, ol, i + 1)) {
								++n_ext;
								enter = absent;
							} else
								two = absent;
							nk += absent;
						} else
							one = true;
					}
					const uint32_t pe = G.append1(enter, C_N) - uN;
					if (enter) {
						if (pe < (uint32_t)c.w) N_VD[pe] = gen_vd(w, i + 1 - ol), N_K[pe] = ol;
						else o_l = true;
					}
					const uint32_t pb = G.append(two ? 2u : (one ? 1u : 0u), C_BA) - uBA;
					if (two) {
						if (pb + 1 < (uint32_t)c.ba) {
							BA_VD[pb] = gen_vd(w, i - ol), BA_K[pb] = ol;
							BA_VD[pb + 1] = gen_vd(w, i + 1 - ol), BA_K[pb + 1] = ol;
						} else
							o_l = true;
					} else if (one) {
						if (pb < (uint32_t)c.ba) BA_VD[pb] = gen_vd(w, i - ol), BA_K[pb] = ol;
						else o_l = true;
					}
				}
				// (first wave: phase 2 covers diagonal d + 1 already, as in align_read_t)
				const bool ins = isv && wave > 0 && (nv == 0 || n_ext != nv);
				const bool qdel = isq && k + 1 < vl;
				const uint32_t pi = G.append1(ins || qdel, C_BA) - uBA;
				if (ins || qdel) {
					if (pi < (uint32_t)c.ba) {
						BA_VD[pi] = ins ? gen_vd(v, d + 1) : gen_vd(v, d - 1);
						BA_K[pi] = ins ? k : k + 1;
					} else
						o_l = true;
				}
			}
			{ // the read's arrival keys so far: the warp that adds the last ones sees the total
				const uint32_t kp = G.append(nk, C_KEYS) - uKEYS;
				if (nk && kp + nk > (uint32_t)hlimit) o_l = true;
			}
			if (G.or_bits(o_l)) {
				ovf = true;
				break;
			}
			const uint32_t cn = G.ctr(C_N);
			const int32_t n_n = (int32_t)(cn - uN);
			uN = cn;
			// extend the entered states (gwf-ed.cu:1132-1160)
			bool f_l = false;
			o_l = false;
			for (int32_t base = 0; base < n_n; base += GS) {
				const int32_t j = base + rank;
				bool toF = false, three = false;
				uint64_t vd = 0;
				int32_t k = 0, d = 0;
				uint32_t v = 0;
				if (j < n_n) {
					vd = N_VD[j], k = N_K[j];
					v = vd_v(vd), d = vd_d(vd);
					const int32_t vl = (int32_t)__ldg(g.len + v);
					k = ext(g, rc, v, d, k, vl);
					const int32_t i = d + k;
					if (i == ql - 1) {
						if (v1 < 0 || ((int32_t)v == v1 && k == vl - 1)) f_l = true;
						else toF = true;
					} else if (k + 1 < vl)
						three = true;
					else
						toF = true;
				}
				const uint32_t pf = G.append1(toF, C_F) - uF;
				if (toF) {
					if (pf < (uint32_t)c.w) F_VD[pf] = vd, F_K[pf] = k;
					else o_l = true;
				}
				const uint32_t p3 = G.append(three ? 3u : 0u, C_BA) - uBA;
				if (three) {
					if (p3 + 2 < (uint32_t)c.ba) {
						BA_VD[p3] = gen_vd(v, d - 1), BA_K[p3] = k + 1;
						BA_VD[p3 + 1] = gen_vd(v, d), BA_K[p3 + 1] = k + 1;
						BA_VD[p3 + 2] = gen_vd(v, d + 1), BA_K[p3 + 2] = k;
					} else
						o_l = true;
				}
			}
			const uint32_t fl = G.or_bits((uint32_t)f_l | (uint32_t)o_l << 1);
			if (fl & 1) {
				found = true;
				break;
			}
			if (fl & 2) {
				ovf = true;
				break;
			}
			const uint32_t cf = G.ctr(C_F);
			n_e = (int32_t)(cf - uF);
			uF = cf;
			const uint32_t tv = off_e_vd, tk = off_e_k;
			off_e_vd = off_f_vd, off_e_k = off_f_k, off_f_vd = tv, off_f_k = tk;
		}
		if (found) {
			dist = s;
			break;
		}
		if (ovf) {
			st = ST_CAPACITY;
			break;
		}
		{ // every append of this step's waves is behind the wave loop's last barrier
			const uint32_t cb = G.ctr(C_BA), ct = G.ctr(C_TA);
			n_ba = (int32_t)(cb - uBA), n_ta = (int32_t)(ct - uTA);
			uBA = cb, uTA = ct;
		}
		G.sync();

		// ---- phase 4: ended-diagonal intervals, then the next wavefront
		if (n_tb + n_ta > 0) {
			const int32_t n_c = n_i + n_tb + n_ta;
			if (n_c > c.iv + c.tb + c.ta) {
				st = ST_CAPACITY;
				break;
			}
			if (n_c <= 32) {
				if (G.wid == 0) {
					uint64_t lo = PAD_KEY, hi = 0;
					if (lane < n_i) lo = ILO[lane], hi = IHI[lane];
					else if (lane < n_i + n_tb) lo = TB[lane - n_i], hi = lo + 1;
					else if (lane < n_c) lo = TA[lane - n_i - n_tb], hi = lo + 1;
					int32_t rk = 0;
					for (int32_t t = 0; t < n_c; ++t) {
						const uint64_t o2 = __shfl_sync(FULL, lo, t);
						rk += o2 < lo || (o2 == lo && t < lane);
					}
					__syncwarp();
					if (lane < n_c) CLO[rk] = lo, CHI[rk] = hi;
				}
			} else {
				grp_sort<NW>(G, TA, nullptr, n_ta, A_VD, A_K, radix_hist, hist_fits);
				for (int32_t j = rank; j < n_i; j += GS) {
					const uint64_t x = ILO[j];
					const int32_t pos = j + lower_bound_u64(TB, n_tb, x) + lower_bound_u64(TA, n_ta, x);
					CLO[pos] = x, CHI[pos] = IHI[j];
				}
				for (int32_t j = rank; j < n_tb; j += GS) {
					const uint64_t x = TB[j];
					const int32_t pos = j + upper_bound_u64(ILO, n_i, x) + lower_bound_u64(TA, n_ta, x);
					CLO[pos] = x, CHI[pos] = x + 1;
				}
				for (int32_t j = rank; j < n_ta; j += GS) {
					const uint64_t x = TA[j];
					const int32_t pos = j + upper_bound_u64(ILO, n_i, x) + upper_bound_u64(TB, n_tb, x);
					CLO[pos] = x, CHI[pos] = x + 1;
				}
			}
			G.sync();
			// coalesce (gwf_intv_merge_adj, gwf-ed.cu:266-296): a group prefix max with carry
			int32_t n_new = 0;
			uint64_t carry = 0;
			for (int32_t base = 0; base < n_c; base += GS) {
				const int32_t j = base + rank;
				const bool act = j < n_c;
				const uint64_t lo = act ? CLO[j] : 0, hi = act ? CHI[j] : 0;
				uint64_t below, all;
				uint64_t pm = G.incl_max(hi, &below, &all);
				if (carry > pm) pm = carry;
				uint64_t prev = __shfl_up_sync(FULL, pm, 1);
				if (lane == 0) prev = below > carry ? below : carry;
				const bool start = act && (j == 0 || lo > prev);
				const bool end = act && (j + 1 == n_c || CLO[j + 1] > pm);
				uint32_t tot;
				const uint32_t pre = G.scan1(start, &tot);
				if (start) {
					const int32_t rk = n_new + (int32_t)pre;
					if (rk < c.iv) ILO[rk] = lo;
				}
				if (end) {
					const int32_t rk = n_new + (int32_t)pre + (start ? 1 : 0) - 1;
					if (rk < c.iv) IHI[rk] = pm;
				}
				n_new += (int32_t)tot;
				carry = all > carry ? all : carry;
			}
			n_i = n_new;
			if (n_i > c.iv) {
				st = ST_CAPACITY;
				break;
			}
			G.sync();
			i_min = ILO[0], i_max = IHI[n_i - 1];
		}
		int32_t n_new = 0;
		if (n_ba == 0) {
			for (int32_t base = 0; base < n_x; base += GS) {
				const int32_t j = base + rank;
				uint64_t vd = 0;
				int32_t k = 0;
				bool keep = false;
				if (j < n_x) {
					vd = X_VD[j], k = X_K[j];
					keep = !in_ranges(ILO, IHI, n_i, vd, i_min, i_max);
				}
				uint32_t tot;
				const uint32_t pre = G.scan1(keep, &tot);
				if (keep) {
					const int32_t pos = n_new + (int32_t)pre;
					X_VD[pos] = vd, X_K[pos] = k;
				}
				n_new += (int32_t)tot;
			}
			const uint32_t tv = off_a_vd, tk = off_a_k;
			off_a_vd = off_x_vd, off_a_k = off_x_k, off_x_vd = tv, off_x_k = tk;
			G.sync();
		} else {
			// 0. before the sort, drop the arc-side candidates inside an ended interval and fold
			// those on an in-vertex diagonal into that entry, as align_read_t does; copies of one
			// diagonal can sit in different warps of the group, so the fold is an atomic max, which
			// the group barriers order before step 2 reads the in-vertex candidates
			int32_t n_s = 0;
			for (int32_t base = 0; base < n_ba; base += GS) {
				const int32_t j = base + rank;
				bool keep = false;
				uint64_t vd = 0;
				int32_t k = 0;
				if (j < n_ba) {
					vd = BA_VD[j], k = BA_K[j];
					if (!in_ranges(ILO, IHI, n_i, vd, i_min, i_max)) {
						const int32_t px = upper_bound_u64(X_VD, n_x, vd);
						if (px > 0 && X_VD[px - 1] == vd) atomicMax(&X_K[px - 1], k);
						else keep = true;
					}
				}
				uint32_t tot;
				const uint32_t pre = G.scan1(keep, &tot); // a barrier: the chunk's loads come first
				if (keep) {
					const int32_t pos = n_s + (int32_t)pre;
					BA_VD[pos] = vd, BA_K[pos] = k;
				}
				n_s += (int32_t)tot;
			}
			G.sync();
			grp_sort<NW>(G, BA_VD, BA_K, n_s, A_VD, A_K, radix_hist, hist_fits);
			// 1. the surviving arc-side candidates: furthest k per diagonal
			int32_t n_b = 0;
			for (int32_t base = 0; base < n_s; base += GS) {
				const int32_t j = base + rank;
				bool keep = false;
				uint64_t vd = 0;
				int32_t k = 0;
				if (j < n_s) {
					vd = BA_VD[j], k = BA_K[j];
					if (j == 0 || BA_VD[j - 1] != vd) {
						for (int32_t t = j + 1; t < n_s && BA_VD[t] == vd; ++t) {
							const int32_t kt = BA_K[t];
							k = kt > k ? kt : k;
						}
						keep = true;
					}
				}
				uint32_t tot;
				const uint32_t pre = G.scan1(keep, &tot);
				if (keep) {
					const int32_t pos = n_b + (int32_t)pre;
					BA_VD[pos] = vd, BA_K[pos] = k;
				}
				n_b += (int32_t)tot;
			}
			G.sync();
			// 2. in-vertex candidates outside the intervals to their merged rank; per 32 entries,
			// the kept count before them and their keep mask
			uint64_t *const chunk = TB;
			int32_t n_kx = 0;
			for (int32_t base = 0; base < n_x; base += GS) {
				const int32_t j = base + rank;
				bool keep = false;
				uint64_t vd = 0;
				int32_t k = 0;
				if (j < n_x) {
					vd = X_VD[j], k = X_K[j];
					keep = !in_ranges(ILO, IHI, n_i, vd, i_min, i_max);
				}
				uint32_t tot;
				const uint32_t pre = G.scan1(keep, &tot);
				const uint32_t m = __ballot_sync(FULL, keep);
				const uint32_t wpre = __shfl_sync(FULL, pre, 0);
				if (lane == 0 && base + G.wid * 32 < n_x) chunk[j >> 5] = (uint64_t)(uint32_t)(n_kx + (int32_t)wpre) << 32 | m;
				if (keep) {
					const int32_t pos = n_kx + (int32_t)pre + lower_bound_u64(BA_VD, n_b, vd);
					A_VD[pos] = vd, A_K[pos] = k;
				}
				n_kx += (int32_t)tot;
			}
			G.sync();
			// 3. arc-side candidates after the kept in-vertex candidates below them
			const int32_t n_chunks = (n_x + 31) >> 5;
			for (int32_t j = rank; j < n_b; j += GS) {
				const uint64_t vd = BA_VD[j];
				const int32_t px = upper_bound_u64(X_VD, n_x, vd), cx = px >> 5;
				int32_t below = n_kx;
				if (cx < n_chunks) {
					const uint64_t info = chunk[cx];
					below = (int32_t)(info >> 32) + __popc((uint32_t)info & ((1u << (px & 31)) - 1));
				}
				A_VD[j + below] = vd, A_K[j + below] = BA_K[j];
			}
			n_new = n_kx + n_b;
			G.sync();
		}
		n_a = n_new;
		if (LAG && n_a > 0) {
			int32_t far = INT32_MIN;
			for (int32_t j = rank; j < n_a; j += GS) {
				const int32_t i = vd_d(A_VD[j]) + A_K[j];
				far = i > far ? i : far;
			}
			far = G.max_i32(far);
			const int32_t lo = far - p.max_lag;
			int32_t n_keep = 0;
			for (int32_t base = 0; base < n_a; base += GS) {
				const int32_t j = base + rank;
				uint64_t vd = 0;
				int32_t k = 0;
				bool keep = false;
				if (j < n_a) {
					vd = A_VD[j], k = A_K[j];
					keep = vd_d(vd) + k >= lo;
				}
				uint32_t tot;
				const uint32_t pre = G.scan1(keep, &tot);
				if (keep) {
					const int32_t pos = n_keep + (int32_t)pre;
					A_VD[pos] = vd, A_K[pos] = k;
				}
				n_keep += (int32_t)tot;
			}
			n_a = n_keep;
			G.sync();
		}
		if (n_a == 0) break;
		if (n_a > c.a) {
			st = ST_CAPACITY;
			break;
		}
	}
	if (rank == 0) {
		p.dist[r] = st == ST_OK ? dist : -1;
		p.status[r] = st;
		if (st == ST_CAPACITY && p.retry_list) {
			const int32_t q = atomicAdd(p.retry_n, 1);
			p.retry_list[q] = r;
		}
		if (p.steps_out) p.steps_out[r] = steps;
		if (p.w_out) p.w_out[r] = W;
	}
#undef A_VD
#undef X_VD
#undef BA_VD
#undef E_VD
#undef F_VD
#undef N_VD
#undef TB
#undef TA
#undef ILO
#undef IHI
#undef CLO
#undef CHI
#undef A_K
#undef X_K
#undef BA_K
#undef E_K
#undef F_K
#undef N_K
}

// Read classes of one launch of k_align_classes, in the order they run: class k's reads are
// order[k][0 .. n[k]) (longest first), aligned by groups of nw[k] warps, each group in its own
// arena of slot[k] bytes sized for ql_cap[k]. Every CTA holds cta_bytes of arena.
struct ClassParams {
	const int32_t *order[4];
	int32_t *head;         // 4 queue heads
	int64_t slot[4];
	int32_t n[4], nw[4], ql_cap[4];
	int32_t n_cls;
	int64_t cta_bytes;
};

template <int NW>
__device__ __forceinline__ void run_class(const KParams &p, const ClassParams &cp, int k, uint8_t *cta_ws,
                                          GrpShm *gsh)
{
	const int gi = (threadIdx.x >> 5) / NW;
	uint8_t *wsb = cta_ws + gi * cp.slot[k];
	const int32_t n = cp.n[k];
	const int32_t *order = cp.order[k];
	if (NW == 1) {
		const int lane = threadIdx.x & 31;
		for (int32_t guard = 0; guard < n + 1; ++guard) {
			int32_t qi = 0;
			if (lane == 0) qi = atomicAdd(cp.head + k, 1);
			qi = __shfl_sync(FULL, qi, 0);
			if (qi >= n) break;
			align_read(p, order[qi], wsb, cp.ql_cap[k], p.level);
		}
	} else {
		Grp<NW> G;
		G.init(gsh + gi, gi);
		for (int32_t guard = 0; guard < n + 1; ++guard) {
			if (G.rank == 0) gsh[gi].claim = atomicAdd(cp.head + k, 1);
			G.sync();
			const int32_t qi = *(volatile int32_t *)&gsh[gi].claim;
			G.sync(); // every thread has the claim before the next one is written
			if (qi >= n) break;
			if (p.max_lag > 0) align_read_grp<NW, true>(p, order[qi], wsb, cp.ql_cap[k], p.level, gsh + gi, gi);
			else align_read_grp<NW, false>(p, order[qi], wsb, cp.ql_cap[k], p.level, gsh + gi, gi);
		}
	}
}

#ifndef GWF_KERNELS_DECL_ONLY
// Serving form with groups of NW warps: k_serve's claim, pack, align and completion steps, with
// one read per group. The group's first thread claims (the same bounded, backed-off polling and
// closing rule as k_serve, the leader group closing the kernel), the group packs the read and
// aligns it with align_read_grp, and the first thread writes the completion record.
template <int NW>
__global__ void __launch_bounds__(256, 3) k_serve_grp(const __grid_constant__ SrvParams p)
{
	__shared__ GrpShm gsh[4];
	if (threadIdx.x < 4 * 8) ((uint32_t *)gsh[threadIdx.x >> 3].ctr)[threadIdx.x & 7] = 0;
	__syncthreads();
	const int gi = (threadIdx.x >> 5) / NW;
	Grp<NW> G;
	G.init(gsh + gi, gi);
	constexpr int GS = 32 * NW;
	const bool leader = blockIdx.x == 0 && gi == 0;
	for (int64_t guard = 0; guard < (1LL << 40); ++guard) {
		if (G.rank == 0) {
			long long h = -1;
			const uint64_t t0 = globaltimer_ns();
			uint32_t ns = 128;
			for (int64_t spin = 0; spin < (1LL << 32); ++spin) {
				if (ld_acquire_s32(p.stop)) break;
				const unsigned long long head = *(volatile const unsigned long long *)p.q_head;
				if (head & SRV_CLOSED) break;
				const unsigned long long tail = ld_acquire_u64(p.q_tail);
				if (head < tail) {
					atomicAdd(p.busy, 1);
					if (atomicCAS(p.q_head, head, head + 1) == head) {
						h = (long long)head;
						break;
					}
					atomicSub(p.busy, 1);
					continue;
				}
				const int64_t idle = (int64_t)(globaltimer_ns() - t0);
				if (idle > p.max_idle_ns ||
				    (leader && idle > p.idle_ns && *(volatile const int32_t *)p.busy == 0)) {
					atomicCAS(p.q_head, head, head | SRV_CLOSED);
					continue;
				}
				__nanosleep(ns);
				if (ns < 32768) ns *= 2;
			}
			gsh[gi].claim64 = h;
		}
		G.sync();
		const long long h = *(volatile long long *)&gsh[gi].claim64;
		G.sync(); // every thread has the claim before the next one is written
		if (h < 0) break;
		asm volatile("fence.acq_rel.gpu;" ::: "memory");
		const SrvEntry *ep = p.q + (h & p.qmask);
		const uint32_t seq = __ldcg((const unsigned int *)&ep->seq);
		if (seq != (uint32_t)(h + 1)) {
			if (G.rank == 0) {
				atomicOr(p.err, SRV_ERR_SEQ);
				atomicOr(p.q_head, SRV_CLOSED);
				atomicSub(p.busy, 1);
			}
			break;
		}
		const int32_t tag = __ldcg(&ep->tag), ql = __ldcg(&ep->ql), v0 = __ldcg(&ep->v0);
		const int32_t v1 = __ldcg(&ep->v1), level = __ldcg(&ep->level);
		const long long aoff = __ldcg((const long long *)&ep->arena_off);
		const long long abytes = __ldcg((const long long *)&ep->arena_bytes);
		uint8_t *ab = p.arena + aoff;
		SrvHdr *hdr = (SrvHdr *)ab;
		uint64_t *pk = (uint64_t *)(ab + 256);
		const uint8_t *raw = ab + 256 + srv_pk_bytes(ql);
		const int32_t L = ql > 0 ? ql : 0;
		const int32_t nwords = (L + 31) / 32 + 2;
		bool ok = true;
		for (int32_t w = G.rank; w < nwords; w += GS) {
			uint64_t word = 0;
			for (int32_t t = 0; t < 32; ++t) {
				const int32_t i = w * 32 + t;
				if (i < L) {
					const uint8_t ch = (uint8_t)__ldcg((const unsigned char *)raw + i);
					ok &= (ch == 'A' || ch == 'C' || ch == 'G' || ch == 'T');
					word |= (uint64_t)((ch >> 1) & 3) << (2 * t);
				}
			}
			pk[w] = word;
		}
		const bool pure = G.or_bits(ok ? 0u : 1u) == 0;
		if (G.rank == 0) {
			hdr->zero = 0, hdr->ql = ql, hdr->v0 = v0, hdr->pure = pure ? 1 : 0;
			hdr->dist = -1, hdr->status = ST_CAPACITY;
		}
		G.sync();
		int32_t dist = -1, st = ST_CAPACITY;
		const int64_t qb = srv_qbytes(ql);
		const Caps c = caps_for(ql, level, p.dens_milli);
		if (qb + ws_layout(c).total <= abytes) {
			KParams lp;
			memset(&lp, 0, sizeof lp);
			lp.g = p.g;
			lp.r.pk = pk;
			lp.r.pk_off = &hdr->zero;
			lp.r.raw = raw;
			lp.r.raw_off = &hdr->zero;
			lp.r.ql = &hdr->ql;
			lp.r.v0 = &hdr->v0;
			lp.r.pure = &hdr->pure;
			lp.r.v1 = v1;
			lp.r.n = 1;
			lp.dens_milli = p.dens_milli;
			lp.flags = p.flags;
			lp.max_lag = p.max_lag;
			lp.dist = &hdr->dist;
			lp.status = &hdr->status;
			if (p.max_lag > 0) align_read_grp<NW, true>(lp, 0, ab + qb, ql, level, gsh + gi, gi);
			else align_read_grp<NW, false>(lp, 0, ab + qb, ql, level, gsh + gi, gi);
			G.sync();
			dist = *(volatile int32_t *)&hdr->dist;
			st = *(volatile int32_t *)&hdr->status;
		}
		if (G.rank == 0) {
			const unsigned long long pos = atomicAdd(p.cq_tail, 1ULL);
			volatile SrvDone *d = p.cq + (pos & p.cmask);
			d->tag = tag, d->dist = dist, d->status = st;
			__threadfence_system();
			d->gen = (int32_t)((pos >> p.cq_shift) + 1);
			atomicSub(p.busy, 1);
		}
		G.sync();
	}
}

// Persistent form with read classes: the CTA's 8 warps run class 0's reads as groups of nw[0]
// warps, then (after a CTA barrier) class 1's as groups of nw[1], and so on. The classes come
// longest reads first, so the long reads start early and the short ones fill the tail.
__global__ void __launch_bounds__(256, 3) k_align_classes(const __grid_constant__ KParams p,
                                                          const __grid_constant__ ClassParams cp)
{
	__shared__ GrpShm gsh[4];
	if (threadIdx.x < 4 * 8) ((uint32_t *)gsh[threadIdx.x >> 3].ctr)[threadIdx.x & 7] = 0;
	__syncthreads();
	uint8_t *cta_ws = p.ws + (int64_t)blockIdx.x * cp.cta_bytes;
	for (int k = 0; k < cp.n_cls; ++k) {
		switch (cp.nw[k]) {
		case 2: run_class<2>(p, cp, k, cta_ws, gsh); break;
		case 4: run_class<4>(p, cp, k, cta_ws, gsh); break;
		case 8: run_class<8>(p, cp, k, cta_ws, gsh); break;
		default: run_class<1>(p, cp, k, cta_ws, gsh); break;
		}
		__syncthreads();
	}
}
#endif

} // namespace gwfb
