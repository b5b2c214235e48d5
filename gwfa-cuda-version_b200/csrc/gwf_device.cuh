// gwf_device.cuh — device side of the B200 GWFA path.
//
// One warp aligns one read. The wavefront of a score step is a sorted list of diagonals
// (vd = vertex << 32 | d + 2^30, k = offset of the last matched base in the vertex), processed
// lane-parallel: every lane extends its own diagonal with 32-base XOR compares on 2-bit packed
// sequences, then emits the next step's candidates in sorted order. The steps of one score s are
// those of the reference's gwf_ed_extend (gwf-ed.cu:1064-1290):
//   1. extension of every diagonal                         (gwf-ed.cu:902-910, 806-839)
//   2. successors inside the vertex: deletion d-1 / mismatch d / insertion d+1, max k per
//      diagonal; successors past the vertex end become "ended diagonal" points
//                                                           (gwf-ed.cu:912-1016)
//   3. vertex-end states expand over arcs in waves: a free match enters the next vertex at the
//      same score and is extended again; otherwise deletion+mismatch enter at score s+1; the
//      arrival set (vertex w, query position) is kept for the whole read (gwf-ed.cu:1106-1255,
//      static_set64_put :1020)
//   4. new wavefront = merge(step 2, step 3) with the max k per diagonal, minus diagonals that
//      already passed their vertex end (gwf_dedup / gwf_mixed_dedup, gwf-ed.cu:780-804, 691-747)
// The result is the first s at which a state consumes the whole query.
// Every buffer has a capacity; an overflow aborts the read with GWF_E_CAPACITY (the host re-runs
// it with a larger arena), so nothing is dropped silently. Every loop is bounded.
#pragma once
#include <cstdint>

namespace gwfb {

constexpr uint32_t FULL = 0xffffffffu;
constexpr int32_t SHIFT = 0x40000000; // gwf-ed.cu:11
constexpr uint64_t EMPTY_KEY = 0;
constexpr uint64_t PAD_KEY = ~0ULL;

// status codes (mirror gwfa.h)
constexpr int32_t ST_OK = 0;
constexpr int32_t ST_BAD_INPUT = -2;
constexpr int32_t ST_CAPACITY = -4;

struct DevGraph {
	const uint32_t *len;     // [n_vtx]
	const uint64_t *base;    // [n_vtx] first base of the vertex in the concatenated sequence
	const uint64_t *pk;      // 2-bit packed sequence, 32 bases per word, +2 padding words
	const uint8_t *raw;      // raw bytes (buffer 8-byte aligned, +16 padding bytes)
	const uint32_t *arc_off; // [n_vtx + 1] CSR offsets
	const uint2 *arc;        // (target, overlap)
	const uint32_t *arc_key; // vertex part of the arrival key per arc (entry id), or null when
	                         // every vertex's in-arcs share one overlap (the key is the target)
	uint32_t n_vtx;
	int32_t pure;            // 1 when every graph byte is A/C/G/T
};

struct DevReads {
	const uint64_t *pk;     // packed reads
	const int64_t *pk_off;  // word offset of read r in pk
	const uint8_t *raw;     // raw reads, concatenated as given by the caller (+16 padding bytes)
	const int64_t *raw_off; // byte offset of read r in raw
	const int32_t *ql;
	const int32_t *v0;
	const uint8_t *pure;    // 1 when the read is A/C/G/T only
	int32_t v1;
	int32_t n;
};

// Per-warp arena capacities (entries).
struct Caps {
	int32_t a;  // wavefront (allocated a + ba, the merge target)
	int32_t x;  // in-vertex candidates of one step
	int32_t ba; // arc-side candidates of one step (power of two: bitonic sort)
	int32_t w;  // one wave of vertex-end / newly entered states
	int32_t tb; // ended-diagonal points from step 2
	int32_t ta; // ended-diagonal points from step 3 (power of two)
	int32_t iv; // merged ended-diagonal intervals
	int32_t h;  // arrival-set slots (power of two)
	int32_t max_steps;
	int32_t pad;
};

__host__ __device__ inline int32_t pow2ceil_i(int32_t x)
{
	int32_t p = 1;
	while (p < x) p <<= 1;
	return p;
}

// Arena sizing from the read length, the retry level and the graph density
// (dens_milli = 1000 * vertices per base). Shared by host (allocation) and device (carving).
__host__ __device__ inline Caps caps_for(int32_t ql, int32_t level, int32_t dens_milli)
{
	Caps c;
	int64_t q = ql < 64 ? 64 : ql;
	int64_t a = (q * 3) / 4 + 256;
	int64_t mult = (int64_t)1 << (2 * level);
	a *= mult;
	if (a > (1 << 24)) a = 1 << 24;
	c.a = (int32_t)((a + 31) & ~31LL);
	c.x = 2 * c.a;
	c.ba = pow2ceil_i(c.a);
	c.w = c.a;
	c.tb = c.a;
	c.ta = pow2ceil_i(c.a / 2 > 64 ? c.a / 2 : 64);
	c.iv = c.a / 2 + 64;
	// expected arrival keys ~ density * 0.1 * ql^2 (the reference caps its set at 32 * ql keys;
	// reads of 20 kbp on a graph with a variant every 50 bp reach ~90 * ql, so cap at 64 * ql and
	// let the retry classes take the rest)
	int64_t est = (int64_t)dens_milli * q * q / 10000;
	if (est < 256) est = 256;
	if (est > 64 * q) est = 64 * q;
	est = est * 2 * mult;
	if (est > (1 << 26)) est = 1 << 26;
	c.h = pow2ceil_i((int32_t)est);
	c.max_steps = (int32_t)(4 * q + 1024);
	c.pad = 0;
	return c;
}

struct WsOff { // byte offsets in one warp arena
	int64_t a_vd, a_k, x_vd, x_k, ba_vd, ba_k, w0_vd, w0_k, w1_vd, w1_k, n_vd, n_k, tb, ta, i0_lo,
	    i0_hi, i1_lo, i1_hi, h, total;
};
// The wavefront ping-pongs between the a and x buffers (each x + ba entries): step 2 writes the
// in-vertex candidates into the buffer not holding the wavefront.

__host__ __device__ inline int64_t al16(int64_t x) { return (x + 15) & ~15LL; }

__host__ __device__ inline WsOff ws_layout(const Caps &c)
{
	WsOff o;
	int64_t p = 0;
	int64_t na = (int64_t)c.x + c.ba; // merge target of step 4
	o.h = p, p = al16(p + 8LL * c.h); // first: 16-byte aligned for vector clears
	o.a_vd = p, p = al16(p + 8 * na);
	o.x_vd = p, p = al16(p + 8 * na);
	o.ba_vd = p, p = al16(p + 8LL * c.ba);
	o.w0_vd = p, p = al16(p + 8LL * c.w);
	o.w1_vd = p, p = al16(p + 8LL * c.w);
	o.n_vd = p, p = al16(p + 8LL * c.w);
	o.tb = p, p = al16(p + 8LL * c.tb);
	o.ta = p, p = al16(p + 8LL * c.ta);
	o.i0_lo = p, p = al16(p + 8LL * c.iv);
	o.i0_hi = p, p = al16(p + 8LL * c.iv);
	o.i1_lo = p, p = al16(p + 8LL * (c.iv + c.tb + c.ta));
	o.i1_hi = p, p = al16(p + 8LL * (c.iv + c.tb + c.ta));
	o.a_k = p, p = al16(p + 4 * na);
	o.x_k = p, p = al16(p + 4 * na);
	o.ba_k = p, p = al16(p + 4LL * c.ba);
	o.w0_k = p, p = al16(p + 4LL * c.w);
	o.w1_k = p, p = al16(p + 4LL * c.w);
	o.n_k = p, p = al16(p + 4LL * c.w);
	o.total = al16(p);
	return o;
}

// Traceback form only: the trace id (int32) beside every k array, the (k, trace) pairs of the
// arc-side candidates while they are sorted by index, and the trace log. A log record is
// (arc index, parent record): one per arc transition (a free-match entry, or the deletion and
// mismatch pair into a vertex), record 0 is the start state. Parents precede their children.
struct TrOff {
	int64_t a_t, x_t, ba_t, bk, w0_t, w1_t, n_t, log, total;
	int32_t log_cap;
};

__host__ __device__ inline TrOff tr_layout(const Caps &c, int64_t base)
{
	TrOff o;
	int64_t p = base;
	const int64_t na = (int64_t)c.x + c.ba;
	o.log_cap = c.h + 4 * c.a; // absent arrivals stay below c.h; the rest are query-end deletions
	o.log = p, p = al16(p + 8LL * o.log_cap);
	o.bk = p, p = al16(p + 8LL * c.ba);
	o.a_t = p, p = al16(p + 4 * na);
	o.x_t = p, p = al16(p + 4 * na);
	o.ba_t = p, p = al16(p + 4LL * c.ba);
	o.w0_t = p, p = al16(p + 4LL * c.w);
	o.w1_t = p, p = al16(p + 4LL * c.w);
	o.n_t = p, p = al16(p + 4LL * c.w);
	o.total = al16(p);
	return o;
}

#ifdef __CUDACC__

__device__ __forceinline__ uint64_t gen_vd(uint32_t v, int32_t d)
{
	return (uint64_t)v << 32 | (uint32_t)(SHIFT + d);
}
__device__ __forceinline__ int32_t vd_d(uint64_t vd) { return (int32_t)(uint32_t)vd - SHIFT; }
__device__ __forceinline__ uint32_t vd_v(uint64_t vd) { return (uint32_t)(vd >> 32); }

__device__ __forceinline__ uint32_t lanemask_lt()
{
	uint32_t m;
	asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
	return m;
}

// exclusive prefix sum of c over the warp; *total receives the warp sum
__device__ __forceinline__ int32_t warp_excl_scan(int32_t c, int32_t *total)
{
	const int lane = threadIdx.x & 31;
	int32_t x = c;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		int32_t y = __shfl_up_sync(FULL, x, o);
		if (lane >= o) x += y;
	}
	*total = __shfl_sync(FULL, x, 31);
	return x - c;
}

// inclusive prefix max of a u64 over the warp
__device__ __forceinline__ uint64_t warp_incl_max(uint64_t x)
{
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		uint64_t y = __shfl_up_sync(FULL, x, o);
		if (lane >= o) x = x > y ? x : y;
	}
	return x;
}

// 8 consecutive bytes starting at p + pos, read as two aligned words (the buffer behind p starts
// 8-byte aligned and carries 16 bytes of padding).
// RO: the bytes are read-only for the kernel's lifetime (graph), so the non-coherent path is
// allowed; query bytes may be written earlier in the same kernel (serving) and use plain loads.
template <bool RO>
__device__ __forceinline__ uint64_t window8(const uint8_t *p, int64_t pos)
{
	const uintptr_t a = (uintptr_t)(p + pos);
	const uint64_t *w = (const uint64_t *)(a & ~(uintptr_t)7);
	const int sh = (int)(a & 7) * 8;
	const uint64_t lo = RO ? __ldg(w) : w[0], hi = RO ? __ldg(w + 1) : w[1];
	return sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
}

struct ReadCtx {
	const uint64_t *qpk;  // packed query words
	const uint8_t *qraw;  // raw query bytes
	int32_t ql, v1;
	bool packed;          // graph and read are A/C/G/T only
	bool quirk;           // reference start-state rules (ext, and the k=-1 filter of step 2)
};

// 32 bases starting at base position pos of a 2-bit packed sequence, as (lo, hi) 16-base
// halves: three aligned 32-bit loads and two funnel shifts (the arrays carry padding words).
template <bool RO>
__device__ __forceinline__ void window32(const uint32_t *pk, int64_t pos, uint32_t &lo, uint32_t &hi)
{
	const uint32_t *w = pk + (pos >> 4);
	const uint32_t sh = (uint32_t)(pos & 15) * 2;
	const uint32_t w0 = RO ? __ldg(w) : w[0], w1 = RO ? __ldg(w + 1) : w[1], w2 = RO ? __ldg(w + 2) : w[2];
	lo = __funnelshift_r(w0, w1, sh);
	hi = __funnelshift_r(w1, w2, sh);
}

// gwf_extend1 (gwf-ed.cu:806-839): last matching offset on diagonal d from offset k. With
// rc.quirk the start state (k = -1) does not extend when min(ql - d, vl) < 32, as in the
// reference, whose unsigned max_k disables its serial loop for k = -1.
__device__ __forceinline__ int32_t ext(const DevGraph &g, const ReadCtx &rc, uint32_t v, int32_t d,
                                       int32_t k, int32_t vl)
{
	const int32_t m = (rc.ql - d < vl ? rc.ql - d : vl) - 1;
	if (k < 0 && m < 31 && rc.quirk) return k;
	const int64_t gb = (int64_t)__ldg(g.base + v);
	if (rc.packed) {
		const uint32_t *gp = (const uint32_t *)g.pk, *qp = (const uint32_t *)rc.qpk;
		for (int guard = 0; k < m && guard < (1 << 26); ++guard) {
			uint32_t glo, ghi, qlo, qhi;
			window32<true>(gp, gb + k + 1, glo, ghi);
			window32<false>(qp, (int64_t)d + k + 1, qlo, qhi);
			uint32_t xlo = glo ^ qlo, xhi = ghi ^ qhi;
			const int32_t rem = m - k; // bases left to compare, >= 1
			if (rem < 16) xlo |= ~0u << (2 * rem), xhi = ~0u;
			else if (rem < 32) xhi |= (rem == 16 ? ~0u : ~0u << (2 * (rem - 16)));
			if ((xlo | xhi) == 0) {
				k += 32;
				continue;
			}
			k += xlo ? (__ffs(xlo) - 1) >> 1 : 16 + ((__ffs(xhi) - 1) >> 1);
			break;
		}
	} else {
		for (int guard = 0; k < m && guard < (1 << 28); ++guard) {
			const int32_t rem = m - k;
			uint64_t x = window8<true>(g.raw, gb + k + 1) ^ window8<false>(rc.qraw, (int64_t)d + k + 1);
			if (rem < 8) x |= ~0ULL << (8 * rem);
			if (x == 0) {
				k += 8;
				continue;
			}
			k += __ffsll((long long)x) - 1 >> 3;
			break;
		}
	}
	return k < m ? k : m;
}

// q[i] == seq(w)[o] (gwf-ed.cu:1199)
__device__ __forceinline__ bool base_eq(const DevGraph &g, const ReadCtx &rc, uint32_t w, int32_t o,
                                        int32_t i)
{
	const int64_t gp = (int64_t)__ldg(g.base + w) + o;
	if (rc.packed) {
		uint64_t a = __ldg(g.pk + (gp >> 5)) >> ((gp & 31) * 2);
		uint64_t b = rc.qpk[i >> 5] >> ((i & 31) * 2);
		return ((a ^ b) & 3) == 0;
	}
	return __ldg(g.raw + gp) == rc.qraw[i];
}

// Arrival set (static_set64_put, gwf-ed.cu:1020-1062): open addressing, linear probing,
// atomicCAS insert. Returns 1 if the key is new, 0 if present, -1 if the probe limit was reached.
// Key 0 is never new, as in the reference (gwf-ed.cu:1022-1026).
__device__ __forceinline__ int hset_insert(uint64_t *h, uint32_t mask, uint64_t key)
{
	if (key == 0) return 0;
	uint64_t x = key * 0x9E3779B97F4A7C15ULL;
	uint32_t i = (uint32_t)(x >> 32) & mask;
	for (uint32_t p = 0; p <= mask; ++p) {
		unsigned long long old = atomicCAS((unsigned long long *)&h[i], 0ULL, (unsigned long long)key);
		if (old == 0ULL) return 1;
		if (old == key) return 0;
		i = (i + 1) & mask;
	}
	return -1;
}

// first index in sorted keys[0..n) with keys[i] >= x (lower) or > x (upper)
__device__ __forceinline__ int32_t lower_bound_u64(const uint64_t *keys, int32_t n, uint64_t x)
{
	int32_t lo = 0, hi = n;
	while (lo < hi) {
		int32_t mid = (lo + hi) >> 1;
		if (keys[mid] < x) lo = mid + 1; else hi = mid;
	}
	return lo;
}
__device__ __forceinline__ int32_t upper_bound_u64(const uint64_t *keys, int32_t n, uint64_t x)
{
	int32_t lo = 0, hi = n;
	while (lo < hi) {
		int32_t mid = (lo + hi) >> 1;
		if (keys[mid] <= x) lo = mid + 1; else hi = mid;
	}
	return lo;
}

// vd inside one of the sorted disjoint ranges [lo, hi)? lo_min / hi_max bound all ranges.
__device__ __forceinline__ bool in_ranges(const uint64_t *lo, const uint64_t *hi, int32_t n, uint64_t vd,
                                          uint64_t lo_min, uint64_t hi_max)
{
	if (n == 0 || vd < lo_min || vd >= hi_max) return false;
	int32_t j = upper_bound_u64(lo, n, vd) - 1;
	return j >= 0 && vd < hi[j];
}

// Stable LSD radix sort of n diagonals (vd keys, optional int32 values) by one warp, for long
// lists. The keys are first mapped to a dense mixed-radix integer, (v - v_min) * span_d +
// (d - d_min), which keeps their order and usually needs 20-30 bits, then sorted 8 bits per pass
// with a 256-bin histogram (hist: 256 words of scratch owned by this warp). Equal digits
// keep their input order: lanes with the same digit are ranked with __match_any_sync. tmp_keys /
// tmp_vals hold n entries; the result is left in keys / vals. Returns false (nothing done) when
// the dense keys would need more than 48 bits.
static __device__ __noinline__ bool warp_radix_sort(uint64_t *keys, int32_t *vals, int32_t n,
                                                    uint64_t *tmp_keys, int32_t *tmp_vals, uint32_t *hist)
{
	const int lane = threadIdx.x & 31;
	uint32_t vmin = 0xffffffffu, vmax = 0;
	uint32_t dmin = 0xffffffffu, dmax = 0; // the low word, d + 2^30, is unsigned
	for (int32_t i = lane; i < n; i += 32) {
		const uint64_t k = keys[i];
		const uint32_t v = (uint32_t)(k >> 32), d = (uint32_t)k;
		vmin = v < vmin ? v : vmin, vmax = v > vmax ? v : vmax;
		dmin = d < dmin ? d : dmin, dmax = d > dmax ? d : dmax;
	}
	vmin = __reduce_min_sync(FULL, vmin), vmax = __reduce_max_sync(FULL, vmax);
	dmin = __reduce_min_sync(FULL, dmin), dmax = __reduce_max_sync(FULL, dmax);
	const uint64_t span_d = (uint64_t)(dmax - dmin) + 1;
	const uint32_t span_v = vmax - vmin;
	if ((span_v ? 32 - __clz(span_v) : 0) + (64 - __clzll((long long)span_d)) > 48) return false;
	const uint64_t top = (uint64_t)span_v * span_d + (dmax - dmin); // largest dense key, < 2^48
	const int32_t bits = 64 - __clzll((long long)top);
	const int32_t passes = bits > 0 ? (bits + 7) / 8 : 1;
	uint64_t *src_k = keys, *dst_k = tmp_keys;
	int32_t *src_v = vals, *dst_v = tmp_vals;
	for (int32_t pass = 0; pass < passes; ++pass) {
		const int32_t shift = 8 * pass;
		for (int32_t b = lane; b < 256; b += 32) hist[b] = 0;
		__syncwarp();
		for (int32_t base = 0; base < n; base += 32) {
			const int32_t i = base + lane;
			const bool act = i < n;
			uint32_t digit = 256 + lane; // distinct and out of range for idle lanes
			if (act) {
				const uint64_t k = src_k[i];
				const uint64_t dk = (uint64_t)((uint32_t)(k >> 32) - vmin) * span_d + ((uint32_t)k - dmin);
				digit = (uint32_t)(dk >> shift) & 255u;
			}
			const uint32_t same = __match_any_sync(FULL, digit);
			if (act && (same & lanemask_lt()) == 0) hist[digit] += __popc(same);
			__syncwarp();
		}
		// exclusive scan of the 256 bins: 8 per lane, then across the warp
		uint32_t c[8], sum = 0;
#pragma unroll
		for (int t = 0; t < 8; ++t) c[t] = hist[lane * 8 + t], sum += c[t];
		int32_t tot;
		uint32_t run = (uint32_t)warp_excl_scan((int32_t)sum, &tot);
#pragma unroll
		for (int t = 0; t < 8; ++t) hist[lane * 8 + t] = run, run += c[t];
		__syncwarp();
		for (int32_t base = 0; base < n; base += 32) {
			const int32_t i = base + lane;
			const bool act = i < n;
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
			const uint32_t pos = act ? hist[digit] + __popc(same & lanemask_lt()) : 0;
			__syncwarp();
			if (act) {
				dst_k[pos] = k;
				if (src_v) dst_v[pos] = v;
				if ((same & lanemask_lt()) == 0) hist[digit] += __popc(same);
			}
			__syncwarp();
		}
		uint64_t *tk = src_k;
		src_k = dst_k, dst_k = tk;
		int32_t *tv = src_v;
		src_v = src_v ? dst_v : nullptr, dst_v = tv;
	}
	if (src_k != keys) { // an odd number of passes: copy back
		for (int32_t i = lane; i < n; i += 32) {
			keys[i] = src_k[i];
			if (vals) vals[i] = src_v[i];
		}
	}
	__syncwarp();
	return true;
}

// Warp bitonic sort of keys[0..n) with int payload in global memory; buffers hold pow2ceil(n)
// entries. For lists longer than 32 (kept out of line).
static __device__ __noinline__ void warp_bitonic_sort_global(uint64_t *keys, int32_t *vals, int32_t n)
{
	const int lane = threadIdx.x & 31;
	int32_t N = pow2ceil_i(n);
	for (int32_t i = n + lane; i < N; i += 32) keys[i] = PAD_KEY;
	__syncwarp();
	for (int32_t k = 2; k <= N; k <<= 1)
		for (int32_t j = k >> 1; j > 0; j >>= 1) {
			for (int32_t i = lane; i < N; i += 32) {
				int32_t l = i ^ j;
				if (l > i) {
					uint64_t a = keys[i], b = keys[l];
					bool up = (i & k) == 0;
					if ((a > b) == up) {
						keys[i] = b, keys[l] = a;
						if (vals) {
							int32_t t = vals[i];
							vals[i] = vals[l], vals[l] = t;
						}
					}
				}
			}
			__syncwarp();
		}
}

__device__ __forceinline__ void warp_bitonic_sort(uint64_t *keys, int32_t *vals, int32_t n)
{
	const int lane = threadIdx.x & 31;
	if (n <= 1) return;
	if (n <= 32) {
		// one element per lane; its rank is the number of smaller keys (equal keys by lane)
		__syncwarp();
		const uint64_t key = lane < n ? keys[lane] : PAD_KEY;
		const int32_t val = (vals && lane < n) ? vals[lane] : 0;
		int32_t rank = 0;
		for (int32_t t = 0; t < n; ++t) {
			const uint64_t o = __shfl_sync(FULL, key, t);
			rank += o < key || (o == key && t < lane);
		}
		__syncwarp();
		if (lane < n) {
			keys[rank] = key;
			if (vals) vals[rank] = val;
		}
		__syncwarp();
		return;
	}
	warp_bitonic_sort_global(keys, vals, n);
}

#endif // __CUDACC__

} // namespace gwfb
