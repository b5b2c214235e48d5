// gwf_kernels.cuh — the alignment kernel (plain and persistent forms) and the read packer.
// See gwf_device.cuh for the algorithm outline and the reference lines each phase restates.
#pragma once
#include "gwf_device.cuh"

namespace gwfb {

struct KParams {
	DevGraph g;
	DevReads r;
	const int32_t *order;   // read index per queue position (cost-ordered for persistent)
	int32_t n_order;
	int32_t *head;          // persistent: next queue position
	uint8_t *ws;            // warp arenas
	int64_t slot_bytes;     // persistent: bytes per warp arena
	const int64_t *slot_off;// plain: arena byte offset per queue position
	int32_t level;          // arena size class (retry level)
	int32_t dens_milli;     // graph density for arena sizing
	int32_t ql_cap;         // persistent: arenas sized for this read length
	int32_t flags;          // bit 0: exact start (no reference start-state quirk)
	int32_t max_lag;        // > 0: after each step drop the states whose query position lags the
	                        // furthest state's by more than max_lag (0 = keep all)
	int32_t *dist;
	int32_t *status;
	int32_t *retry_list;    // reads that overflowed their arena
	int32_t *retry_n;
	int32_t *steps_out;     // optional per-read score steps
	int64_t *w_out;         // optional per-read sum of wavefront sizes
	// traceback form only (per read r; the path rows are max_nv wide)
	int32_t *end_off;       // offset in the last vertex of the last base consumed, -1 if none
	int32_t *path_n;        // vertices on the path (only the first max_nv are written)
	int32_t *path_v;        // path vertices from v0
	int32_t *path_arc;      // arc index into path_v[j] (-1 for j = 0)
	int32_t max_nv;
};

// ---- serving: one resident kernel, warps pull single reads from a device queue
//
// Each queued read owns an arena (allocated by the host from a fixed budget) laid out as
//   [0, 256)              SrvHdr
//   [256, 256 + pkb)      2-bit packed read, written by the warp
//   [.., + rawb)          raw read bytes (+16 padding), copied in by the host before publication
//   [srv_qbytes(ql), ..)  wavefront workspace for caps_for(ql, level)
struct SrvEntry {         // queue entry, 48 bytes
	uint32_t seq;         // queue position + 1 (checks that the entry is the one claimed)
	int32_t tag;          // host slot of the read
	int64_t arena_off;    // byte offset of the read's arena in the pool
	int64_t arena_bytes;
	int32_t ql, v0, v1, level;
	int32_t pad[2];
};
struct SrvDone {          // completion record in host-mapped memory
	int32_t tag, dist, status, gen; // gen = pass over the ring + 1, written last
};
struct SrvHdr {
	int64_t zero;
	int32_t ql, v0, dist, status;
	uint8_t pure, pad[7];
};
struct SrvParams {
	DevGraph g;
	const SrvEntry *q;                 // device ring, qmask + 1 entries
	const unsigned long long *q_tail;  // published by the host (device memory)
	unsigned long long *q_head;        // next position to claim
	const int32_t *stop;               // host sets 1 to end the kernel
	int32_t *busy;                     // warps holding a read
	unsigned long long *cq_tail;       // next completion position
	SrvDone *cq;                       // host-mapped ring, cmask + 1 records
	int32_t *err;                      // host-mapped error bits (SRV_ERR_*)
	uint8_t *arena;                    // arena pool
	uint32_t qmask, cmask;
	int32_t cq_shift;                  // log2(cmask + 1)
	int32_t dens_milli, flags;
	int32_t max_lag;                   // > 0: lag pruning of each read (GWF_F_MAX_LAG)
	int32_t pad_;
	int64_t idle_ns;                   // the leader warp closes the kernel after this idle
	                                   // time when no warp is busy
	int64_t max_idle_ns;               // any warp closes it after this idle time
};
constexpr int32_t SRV_ERR_SEQ = 1;     // a claimed entry did not carry its position
// Set in q_head when the kernel closes. Claims and the closing mark both change q_head with
// atomicCAS, so a read is either claimed before the mark or stays queued for the next launch.
constexpr unsigned long long SRV_CLOSED = 1ULL << 62;

__host__ __device__ inline int64_t srv_al256(int64_t x) { return (x + 255) & ~255LL; }
__host__ __device__ inline int64_t srv_pk_bytes(int32_t ql) { return srv_al256(8LL * ((ql + 31) / 32 + 2)); }
__host__ __device__ inline int64_t srv_qbytes(int32_t ql)
{
	return 256 + srv_pk_bytes(ql) + srv_al256((int64_t)ql + 16);
}

#ifndef GWF_KERNELS_DECL_ONLY
// Aligns read r with one warp. All control flow is warp-uniform.
// Candidate lists longer than this are radix-sorted; shorter ones by rank or a bitonic network.
constexpr int32_t kRadixMin = 128;

// The arena capacities are those of caps_for(min(ql, ql_cap), level): the arena at wsb must hold
// them (callers size it for ql_cap, or for the read itself). With TR, the arena also holds
// tr_layout's arrays after ws_layout's, every state carries the id of the trace record of the
// last arc it crossed, and the read's path is written to p.path_*. With LAG, each step ends with
// the lag pruning of p.max_lag (a separate instantiation, so that the distance kernel's code is
// untouched by it).
template <bool TR, bool LAG>
__device__ __forceinline__ void align_read_body(const KParams &p, int32_t r, uint8_t *wsb, int32_t ql_cap,
                                                int32_t level)
{
	const int lane = threadIdx.x & 31;
	const Caps c = caps_for(p.r.ql[r] < ql_cap ? p.r.ql[r] : ql_cap, level, p.dens_milli);

	const DevGraph &g = p.g;
	const WsOff o = ws_layout(c);
	uint64_t *const h = (uint64_t *)(wsb + o.h);
	// The arena's arrays, as 32-bit byte offsets from wsb (32-bit offsets hold fewer registers
	// than 64-bit pointers); the upper-case names are the arrays.
	uint32_t off_a_vd = (uint32_t)o.a_vd;
	uint32_t off_x_vd = (uint32_t)o.x_vd;
	const uint32_t off_ba_vd = (uint32_t)o.ba_vd;
	uint32_t off_e_vd = (uint32_t)o.w0_vd;
	uint32_t off_f_vd = (uint32_t)o.w1_vd;
	const uint32_t off_n_vd = (uint32_t)o.n_vd;
	const uint32_t off_tb = (uint32_t)o.tb;
	const uint32_t off_ta = (uint32_t)o.ta;
	const uint32_t off_ilo = (uint32_t)o.i0_lo;
	const uint32_t off_ihi = (uint32_t)o.i0_hi;
	const uint32_t off_clo = (uint32_t)o.i1_lo;
	const uint32_t off_chi = (uint32_t)o.i1_hi;
	uint32_t off_a_k = (uint32_t)o.a_k;
	uint32_t off_x_k = (uint32_t)o.x_k;
	const uint32_t off_ba_k = (uint32_t)o.ba_k;
	uint32_t off_e_k = (uint32_t)o.w0_k;
	uint32_t off_f_k = (uint32_t)o.w1_k;
	const uint32_t off_n_k = (uint32_t)o.n_k;
	// traceback arrays (dead code without TR)
	const TrOff to = tr_layout(c, o.total);
	uint32_t off_a_t = (uint32_t)to.a_t;
	uint32_t off_x_t = (uint32_t)to.x_t;
	const uint32_t off_ba_t = (uint32_t)to.ba_t;
	uint32_t off_e_t = (uint32_t)to.w0_t;
	uint32_t off_f_t = (uint32_t)to.w1_t;
	const uint32_t off_n_t = (uint32_t)to.n_t;
	const uint32_t off_bk = (uint32_t)to.bk;
	const uint32_t off_log = (uint32_t)to.log;
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
#define A_T ((int32_t *)(wsb + off_a_t))
#define X_T ((int32_t *)(wsb + off_x_t))
#define BA_T ((int32_t *)(wsb + off_ba_t))
#define E_T ((int32_t *)(wsb + off_e_t))
#define F_T ((int32_t *)(wsb + off_f_t))
#define N_T ((int32_t *)(wsb + off_n_t))
#define BK ((int2 *)(wsb + off_bk))
#define TLOG ((uint2 *)(wsb + off_log))
	// radix-sort histogram (256 bins): the interval scratch, free whenever a sort runs
	uint32_t *const radix_hist = (uint32_t *)(wsb + off_clo);


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
		if (lane == 0) {
			p.dist[r] = -1, p.status[r] = ST_BAD_INPUT;
			if constexpr (TR) p.path_n[r] = 0, p.end_off[r] = -1;
		}
		return;
	}
	if (o.total > 0xffffffffLL || (TR && to.total > 0xffffffffLL)) { // the 32-bit offsets above
		if (lane == 0) {
			p.dist[r] = -1, p.status[r] = ST_CAPACITY;
			if constexpr (TR) p.path_n[r] = 0, p.end_off[r] = -1;
		}
		return;
	}

	// clear the arrival set (16-byte stores; h is 16-byte aligned, c.h is a power of two >= 256)
	{
		uint4 *h4 = (uint4 *)h;
		const uint4 z = make_uint4(0, 0, 0, 0);
		for (int32_t i = lane; i < c.h / 2; i += 32) h4[i] = z;
	}
	if (lane == 0) A_VD[0] = gen_vd((uint32_t)v0, 0), A_K[0] = -1; // gwf-ed.cu:1303-1308
	int32_t n_log = 1;                  // trace records in use
	int32_t tr_t = -1, tr_k = -1;       // trace record and offset of the state that ends the read
	if constexpr (TR) {
		if (lane == 0) A_T[0] = 0, TLOG[0] = make_uint2(0xffffffffu, 0xffffffffu);
	}
	__syncwarp();
	const uint32_t hmask = (uint32_t)c.h - 1;
	const int32_t hlimit = c.h - c.h / 4;
	int32_t n_a = 1, n_i = 0, n_keys = 0;
	uint64_t i_min = 0, i_max = 0; // bounds of the ended-diagonal intervals

	for (int32_t s = 0;; ++s) {
		if (s >= c.max_steps) {
			st = ST_CAPACITY;
			break;
		}
		++steps;
		W += n_a;
		bool found = false, ovf = false;
		int32_t f_j = 0x7fffffff, f_t = -1, f_k = -1; // TR: this lane's first end state

		// ---- phases 1 and 2, in one pass over the wavefront. Phase 1 extends every diagonal and
		// collects the vertex-end (and, for v1 >= 0, query-end) states into the first wave
		// (gwf-ed.cu:902-910, 965-984). Phase 2 forms the in-vertex successors, sorted and unique by
		// construction (gwf_ed_extend_batch, gwf-ed.cu:912-1016). Phase 2 runs one diagonal behind
		// phase 1, so that both neighbours of a diagonal are extended when its successors are
		// formed: in the chunk at `base`, lane l extends diagonal base+l and forms the successors of
		// diagonal base+l-1. The diagonal and its left neighbour come by rotating shuffles; lanes 30
		// and 31 hand over their diagonals of the previous chunk (o_*), which are the left
		// neighbours of the chunk's first two.
		int32_t n_e = 0, n_x = 0, n_tb = 0;
		uint64_t o_vd = 0;
		int32_t o_k = 0, o_t = 0, o_vl = 0;
		const int src1 = (lane + 31) & 31, src2 = (lane + 30) & 31;
		for (int32_t base = 0; base <= n_a; base += 32) {
			const int32_t j = base + lane;
			bool toE = false;
			uint64_t vd = 0;
			int32_t k = 0, t = 0, vl = 0;
			if (j < n_a) {
				vd = A_VD[j];
				k = A_K[j];
				if constexpr (TR) t = A_T[j];
				const uint32_t v = vd_v(vd);
				const int32_t d = vd_d(vd);
				vl = (int32_t)__ldg(g.len + v);
				k = ext(g, rc, v, d, k, vl);
				const bool vend = k == vl - 1, qend = d + k == ql - 1;
				if (qend) {
					if (v1 < 0 || ((int32_t)v == v1 && vend)) {
						found = true;
						if (TR && j < f_j) f_j = j, f_t = t, f_k = k;
					} else
						toE = true;
				} else if (vend)
					toE = true;
			}
			{
				const uint32_t m = __ballot_sync(FULL, toE);
				const int32_t pos = n_e + __popc(m & lanemask_lt());
				if (toE && pos < c.w) {
					E_VD[pos] = vd, E_K[pos] = k;
					if constexpr (TR) E_T[pos] = t;
				}
				n_e += __popc(m);
			}

			// diagonal e = j - 1 (mine) and e - 1 (left); e + 1 (right) is this lane's own
			const bool h1 = lane == 31, h2 = lane >= 30;
			const uint64_t my_vd = __shfl_sync(FULL, h1 ? o_vd : vd, src1);
			const int32_t my_k = __shfl_sync(FULL, h1 ? o_k : k, src1);
			const int32_t my_vl = __shfl_sync(FULL, h1 ? o_vl : vl, src1);
			const uint64_t pv = __shfl_sync(FULL, h2 ? o_vd : vd, src2);
			const int32_t pk = __shfl_sync(FULL, h2 ? o_k : k, src2);
			int32_t tt = 0, pt = 0;
			if constexpr (TR) {
				tt = __shfl_sync(FULL, h1 ? o_t : t, src1);
				pt = __shfl_sync(FULL, h2 ? o_t : t, src2);
			}
			o_vd = vd, o_k = k, o_vl = vl, o_t = t;
			const int32_t e = j - 1;
			uint64_t cv[3];
			int32_t ck[3], ct[3] = {0, 0, 0};
			bool keep[3] = {false, false, false}, tmp[3] = {false, false, false};
			if (e >= 0 && e < n_a) {
				const bool has_l = e > 0, has_r = j < n_a;
				const bool left_in = has_l && pv == my_vd - 1, left2 = has_l && pv == my_vd - 2;
				const bool right_in = has_r && vd == my_vd + 1, right2 = has_r && vd == my_vd + 2;
				bool has[3];
				// L: diagonal d-1 when absent from a: deletion from d, insertion from d-2
				has[0] = !left_in;
				cv[0] = my_vd - 1;
				ck[0] = my_k + 1, ct[0] = tt;
				if (left2 && pk > ck[0]) ck[0] = pk, ct[0] = pt;
				// S: diagonal d: mismatch, insertion from d-1, deletion from d+1
				has[1] = true;
				cv[1] = my_vd;
				ck[1] = my_k + 1, ct[1] = tt;
				if (left_in && pk > ck[1]) ck[1] = pk, ct[1] = pt;
				if (right_in && k + 1 > ck[1]) ck[1] = k + 1, ct[1] = t;
				// R: diagonal d+1 when neither d+1 nor d+2 is in a: insertion from d
				has[2] = !right_in && !right2;
				cv[2] = my_vd + 1;
				ck[2] = my_k, ct[2] = tt;
				// the reference keeps vl in a uint32_t here (gwf-ed.cu:895, 993): a candidate
				// with k = -1 (insertion before the first base of v0) fails `k < vl` and is dropped
#pragma unroll
				for (int q = 0; q < 3; ++q)
					if (has[q]) {
						const int32_t dd = vd_d(cv[q]);
						const bool kin = rc.quirk ? (uint32_t)ck[q] < (uint32_t)my_vl : ck[q] < my_vl;
						if (dd + ck[q] < ql && kin) keep[q] = true;
						else if (ck[q] == my_vl) tmp[q] = true;
					}
				// a diagonal that ended its vertex short of the query end is a vertex-end state
				// of the first wave, which records it as an ended point already: its own
				// successor at k == vl would repeat that point
				if (tmp[1] && my_k == my_vl - 1 && vd_d(my_vd) + my_k != ql - 1) tmp[1] = false;
			}
			{
				const uint32_t lt = lanemask_lt();
				const uint32_t k0 = __ballot_sync(FULL, keep[0]), k1 = __ballot_sync(FULL, keep[1]),
				               k2 = __ballot_sync(FULL, keep[2]);
				int32_t off = n_x + __popc(k0 & lt) + __popc(k1 & lt) + __popc(k2 & lt);
#pragma unroll
				for (int q = 0; q < 3; ++q)
					if (keep[q]) {
						if (off < c.x) {
							X_VD[off] = cv[q], X_K[off] = ck[q];
							if constexpr (TR) X_T[off] = ct[q];
						}
						++off;
					}
				n_x += __popc(k0) + __popc(k1) + __popc(k2);
				const uint32_t t0 = __ballot_sync(FULL, tmp[0]), t1 = __ballot_sync(FULL, tmp[1]),
				               t2 = __ballot_sync(FULL, tmp[2]);
				if (t0 | t1 | t2) {
					int32_t offt = n_tb + __popc(t0 & lt) + __popc(t1 & lt) + __popc(t2 & lt);
#pragma unroll
					for (int q = 0; q < 3; ++q)
						if (tmp[q]) {
							if (offt < c.tb) TB[offt] = cv[q];
							++offt;
						}
					n_tb += __popc(t0) + __popc(t1) + __popc(t2);
				}
			}
		}
		if (__any_sync(FULL, found)) {
			dist = s;
			if constexpr (TR) {
				const int32_t mj = (int32_t)__reduce_min_sync(FULL, (uint32_t)f_j);
				const int src = __ffs(__ballot_sync(FULL, f_j == mj)) - 1;
				tr_t = __shfl_sync(FULL, f_t, src), tr_k = __shfl_sync(FULL, f_k, src);
			}
			break;
		}
		if (n_e > c.w) ovf = true;
		if (n_x > c.x || n_tb > c.tb) ovf = true;
		__syncwarp();

		// ---- phase 3: vertex-end states over arcs, in waves until no state is entered with a
		// free match (gwf-ed.cu:1106-1255)
		int32_t n_ba = 0, n_ta = 0;
		for (int32_t wave = 0; n_e > 0 && !ovf; ++wave) {
			if (wave > ql + 2) {
				ovf = true;
				break;
			}
			int32_t n_n = 0;
			for (int32_t base = 0; base < n_e; base += 32) {
				const int32_t j = base + lane;
				bool act = j < n_e, isq = false, isv = false;
				uint64_t vd = 0;
				int32_t k = 0, d = 0, vl = 0, i = 0, nv = 0, et = 0;
				uint32_t v = 0, aoff = 0;
				if (act) {
					vd = E_VD[j], k = E_K[j];
					if constexpr (TR) et = E_T[j];
					v = vd_v(vd), d = vd_d(vd), vl = (int32_t)__ldg(g.len + v), i = d + k;
					isq = i == ql - 1;
					isv = !isq;
					aoff = __ldg(g.arc_off + v);
					const int32_t deg = (int32_t)(__ldg(g.arc_off + v + 1) - aoff);
					if (isv || (k + 1 == vl && (int32_t)v != v1)) nv = deg;
				}
				// ended-diagonal point of a vertex-end state (gwf-ed.cu:1177-1183)
				{
					const uint32_t m = __ballot_sync(FULL, isv);
					const int32_t pos = n_ta + __popc(m & lanemask_lt());
					if (isv && pos < c.ta) TA[pos] = vd;
					n_ta += __popc(m);
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
							// arrival key (w, i + 1) as in the reference (gwf-ed.cu:1196), or the
							// arc's entry id in place of w where w's in-arcs differ in overlap
							const uint32_t kv = g.arc_key ? __ldg(g.arc_key + aoff + t) : w;
							const int ins = hset_insert(h, hmask, (uint64_t)kv << 32 | (uint32_t)(i + 1));
							if (ins < 0) ovf = true;
							const bool absent = ins == 1;
							if (base_eq(g, rc, w, ol, i + 1)) {
								++n_ext;
								enter = absent;
							} else
								two = absent;
							if (absent) ++n_keys; // per-lane; reduced below
						} else
							one = true; // v1 >= 0: query end at a vertex end, delete into w
					}
					int32_t rec = 0; // TR: the record of this arc transition
					if constexpr (TR) {
						const bool mk = enter || two || one;
						const uint32_t mr = __ballot_sync(FULL, mk);
						rec = n_log + __popc(mr & lanemask_lt());
						if (mk && rec < to.log_cap) TLOG[rec] = make_uint2(aoff + (uint32_t)t, (uint32_t)et);
						n_log += __popc(mr);
					}
					const uint32_t me = __ballot_sync(FULL, enter);
					const int32_t pe = n_n + __popc(me & lanemask_lt());
					if (enter && pe < c.w) {
						N_VD[pe] = gen_vd(w, i + 1 - ol), N_K[pe] = ol;
						if constexpr (TR) N_T[pe] = rec;
					}
					n_n += __popc(me);
					// positions in lane order: two entries per `two` lane, one per `one` lane
					const uint32_t m2 = __ballot_sync(FULL, two), m1 = __ballot_sync(FULL, one);
					const uint32_t lt = lanemask_lt();
					const int32_t pb = n_ba + 2 * __popc(m2 & lt) + __popc(m1 & lt);
					const int32_t tot = 2 * __popc(m2) + __popc(m1);
					if (two) {
						if (pb + 1 < c.ba) {
							BA_VD[pb] = gen_vd(w, i - ol), BA_K[pb] = ol;         // deletion
							BA_VD[pb + 1] = gen_vd(w, i + 1 - ol), BA_K[pb + 1] = ol; // mismatch
							if constexpr (TR) BA_T[pb] = rec, BA_T[pb + 1] = rec;
						}
					} else if (one) {
						if (pb < c.ba) {
							BA_VD[pb] = gen_vd(w, i - ol), BA_K[pb] = ol;
							if constexpr (TR) BA_T[pb] = rec;
						}
					}
					n_ba += tot;
				}
				// insertion at the vertex end (gwf-ed.cu:1225-1226); v1 >= 0 query-end deletion
				// inside the vertex (gwf-ed.cu:1237-1241). In the first wave the state is a
				// wavefront diagonal d, and phase 2 has already given diagonal d + 1 an in-vertex
				// candidate with k >= vl - 1 or an ended point, which the insertion (d + 1,
				// vl - 1) could only repeat; only entered states (later waves) need it.
				const bool ins = isv && wave > 0 && (nv == 0 || n_ext != nv);
				const bool qdel = isq && k + 1 < vl;
				const uint32_t mi = __ballot_sync(FULL, ins || qdel);
				const int32_t pi = n_ba + __popc(mi & lanemask_lt());
				if ((ins || qdel) && pi < c.ba) {
					BA_VD[pi] = ins ? gen_vd(v, d + 1) : gen_vd(v, d - 1);
					BA_K[pi] = ins ? k : k + 1;
					if constexpr (TR) BA_T[pi] = et;
				}
				n_ba += __popc(mi);
			}
			if ((int32_t)__reduce_add_sync(FULL, (uint32_t)n_keys) > hlimit) ovf = true;
			if (n_n > c.w || n_ba > c.ba || n_ta > c.ta) ovf = true;
			if (TR && n_log > to.log_cap) ovf = true;
			if (__any_sync(FULL, ovf)) {
				ovf = true;
				break;
			}
			__syncwarp();
			// extend the entered states (gwf-ed.cu:1132-1160)
			int32_t n_f = 0;
			for (int32_t base = 0; base < n_n; base += 32) {
				const int32_t j = base + lane;
				bool toF = false, three = false;
				uint64_t vd = 0;
				int32_t k = 0, d = 0, nt = 0;
				uint32_t v = 0;
				if (j < n_n) {
					vd = N_VD[j], k = N_K[j];
					if constexpr (TR) nt = N_T[j];
					v = vd_v(vd), d = vd_d(vd);
					const int32_t vl = (int32_t)__ldg(g.len + v);
					k = ext(g, rc, v, d, k, vl);
					const int32_t i = d + k;
					if (i == ql - 1) {
						if (v1 < 0 || ((int32_t)v == v1 && k == vl - 1)) {
							found = true;
							if (TR && j < f_j) f_j = j, f_t = nt, f_k = k;
						} else
							toF = true;
					} else if (k + 1 < vl)
						three = true;
					else
						toF = true;
				}
				const uint32_t mf = __ballot_sync(FULL, toF);
				const int32_t pf = n_f + __popc(mf & lanemask_lt());
				if (toF && pf < c.w) {
					F_VD[pf] = vd, F_K[pf] = k;
					if constexpr (TR) F_T[pf] = nt;
				}
				n_f += __popc(mf);
				const uint32_t m3 = __ballot_sync(FULL, three);
				const int32_t p3 = n_ba + 3 * __popc(m3 & lanemask_lt());
				if (three && p3 + 2 < c.ba) {
					BA_VD[p3] = gen_vd(v, d - 1), BA_K[p3] = k + 1;     // deletion
					BA_VD[p3 + 1] = gen_vd(v, d), BA_K[p3 + 1] = k + 1; // mismatch
					BA_VD[p3 + 2] = gen_vd(v, d + 1), BA_K[p3 + 2] = k; // insertion
					if constexpr (TR) BA_T[p3] = nt, BA_T[p3 + 1] = nt, BA_T[p3 + 2] = nt;
				}
				n_ba += 3 * __popc(m3);
			}
			if (__any_sync(FULL, found)) break;
			if (n_f > c.w || n_ba > c.ba) {
				ovf = true;
				break;
			}
			__syncwarp();
			const uint32_t tv = off_e_vd, tk = off_e_k, tt = off_e_t;
			off_e_vd = off_f_vd, off_e_k = off_f_k, off_f_vd = tv, off_f_k = tk;
			off_e_t = off_f_t, off_f_t = tt;
			n_e = n_f;
		}
		if (__any_sync(FULL, found)) {
			dist = s;
			if constexpr (TR) {
				const int32_t mj = (int32_t)__reduce_min_sync(FULL, (uint32_t)f_j);
				const int src = __ffs(__ballot_sync(FULL, f_j == mj)) - 1;
				tr_t = __shfl_sync(FULL, f_t, src), tr_k = __shfl_sync(FULL, f_k, src);
			}
			break;
		}
		if (__any_sync(FULL, ovf)) {
			st = ST_CAPACITY;
			break;
		}
		__syncwarp();

		// ---- phase 4: ended-diagonal intervals, then the next wavefront
		// (gwf_dedup / gwf_intv_merge2 / gwf_diag_dedup / gwf_mixed_dedup, gwf-ed.cu:780-804)
		if (n_tb + n_ta > 0) {
			const int32_t n_c = n_i + n_tb + n_ta;
			if (n_c > c.iv + c.tb + c.ta) {
				st = ST_CAPACITY;
				break;
			}
			if (n_c <= 32) {
				// few ranges: one per lane, ordered by rank of the lower end (the union that the
				// coalescing below computes does not depend on the order of equal ends)
				uint64_t lo = PAD_KEY, hi = 0;
				if (lane < n_i) lo = ILO[lane], hi = IHI[lane];
				else if (lane < n_i + n_tb) lo = TB[lane - n_i], hi = lo + 1;
				else if (lane < n_c) lo = TA[lane - n_i - n_tb], hi = lo + 1;
				int32_t rank = 0;
				for (int32_t t = 0; t < n_c; ++t) {
					const uint64_t o2 = __shfl_sync(FULL, lo, t);
					rank += o2 < lo || (o2 == lo && t < lane);
				}
				__syncwarp();
				if (lane < n_c) CLO[rank] = lo, CHI[rank] = hi;
			} else {
			if (n_ta <= kRadixMin || !warp_radix_sort(TA, nullptr, n_ta, A_VD, A_K, radix_hist))
				warp_bitonic_sort(TA, nullptr, n_ta);
			// rank-merge the old ranges with both point lists, ties ordered I < TB < TA
			for (int32_t j = lane; j < n_i; j += 32) {
				const uint64_t x = ILO[j];
				const int32_t pos = j + lower_bound_u64(TB, n_tb, x) + lower_bound_u64(TA, n_ta, x);
				CLO[pos] = x, CHI[pos] = IHI[j];
			}
			for (int32_t j = lane; j < n_tb; j += 32) {
				const uint64_t x = TB[j];
				const int32_t pos = j + upper_bound_u64(ILO, n_i, x) + lower_bound_u64(TA, n_ta, x);
				CLO[pos] = x, CHI[pos] = x + 1;
			}
			for (int32_t j = lane; j < n_ta; j += 32) {
				const uint64_t x = TA[j];
				const int32_t pos = j + upper_bound_u64(ILO, n_i, x) + upper_bound_u64(TB, n_tb, x);
				CLO[pos] = x, CHI[pos] = x + 1;
			}
			}
			__syncwarp();
			// coalesce overlapping or touching ranges (gwf_intv_merge_adj, gwf-ed.cu:266-296)
			int32_t n_new = 0;
			uint64_t carry = 0;
			for (int32_t base = 0; base < n_c; base += 32) {
				const int32_t j = base + lane;
				const bool act = j < n_c;
				const uint64_t lo = act ? CLO[j] : 0, hi = act ? CHI[j] : 0;
				uint64_t pm = warp_incl_max(hi);
				if (base > 0 && carry > pm) pm = carry;
				uint64_t prev = __shfl_up_sync(FULL, pm, 1);
				if (lane == 0) prev = carry;
				const bool start = act && (j == 0 || lo > prev);
				const bool end = act && (j + 1 == n_c || CLO[j + 1] > pm);
				const uint32_t ms = __ballot_sync(FULL, start);
				if (start) {
					const int32_t rk = n_new + __popc(ms & lanemask_lt());
					if (rk < c.iv) ILO[rk] = lo;
				}
				if (end) {
					const int32_t rk = n_new + __popc(ms & (lanemask_lt() | (1u << lane))) - 1;
					if (rk < c.iv) IHI[rk] = pm;
				}
				n_new += __popc(ms);
				carry = __shfl_sync(FULL, pm, 31);
			}
			n_i = n_new;
			if (n_i > c.iv) {
				st = ST_CAPACITY;
				break;
			}
			__syncwarp();
			i_min = ILO[0], i_max = IHI[n_i - 1];
		}
		int32_t n_new = 0;
		if (n_ba == 0) {
			// only in-vertex candidates: already sorted and unique; drop ended diagonals in place
			// and make the candidate buffer the wavefront
			for (int32_t base = 0; base < n_x; base += 32) {
				const int32_t j = base + lane;
				uint64_t vd = 0;
				int32_t k = 0, t = 0;
				bool keep = false;
				if (j < n_x) {
					vd = X_VD[j], k = X_K[j];
					if constexpr (TR) t = X_T[j];
					keep = !in_ranges(ILO, IHI, n_i, vd, i_min, i_max);
				}
				const uint32_t m = __ballot_sync(FULL, keep);
				if (keep) {
					const int32_t pos = n_new + __popc(m & lanemask_lt());
					X_VD[pos] = vd, X_K[pos] = k;
					if constexpr (TR) X_T[pos] = t;
				}
				n_new += __popc(m);
			}
			const uint32_t tv = off_a_vd, tk = off_a_k, tt = off_a_t;
			off_a_vd = off_x_vd, off_a_k = off_x_k, off_x_vd = tv, off_x_k = tk;
			off_a_t = off_x_t, off_x_t = tt;
			__syncwarp();
		} else {
			// TR: the candidates' (k, trace) pairs move aside and the sort carries their indices
			if constexpr (TR) {
				for (int32_t j = lane; j < n_ba; j += 32) BK[j] = make_int2(BA_K[j], BA_T[j]), BA_K[j] = j;
				__syncwarp();
			}
			int32_t n_sort = n_ba; // candidates left to sort
			if constexpr (!TR) {
				// 0. before the sort, drop the arc-side candidates inside an ended interval and fold
				// those whose diagonal is among the in-vertex candidates into that entry (of a
				// chunk's copies of one diagonal, the one with the largest k writes; chunks go in
				// order). Most candidates end here (config 3: ~27 per step, ~4.4 left), so only the
				// rest are sorted. The result is that of step 1 below on the whole list: the
				// interval test depends on the diagonal alone, and the fold keeps the largest k.
				int32_t n_s = 0;
				for (int32_t base = 0; base < n_ba; base += 32) {
					const int32_t j = base + lane;
					uint64_t vd = 0;
					int32_t k = 0, px = 0;
					bool fold = false, keep = false;
					if (j < n_ba) {
						vd = BA_VD[j], k = BA_K[j];
						if (!in_ranges(ILO, IHI, n_i, vd, i_min, i_max)) {
							px = upper_bound_u64(X_VD, n_x, vd);
							fold = px > 0 && X_VD[px - 1] == vd;
							keep = !fold;
						}
					}
					// ~lane is no diagonal (its vertex part would be 2^32 - 1)
					const uint32_t same = __match_any_sync(FULL, fold ? vd : ~(uint64_t)lane);
					uint32_t rest = fold ? same & ~(1u << lane) : 0u;
					bool lead = fold;
					while (__any_sync(FULL, rest != 0)) { // at most 31 rounds, one per copy
						const int q = rest ? __ffs(rest) - 1 : lane;
						const int32_t kq = __shfl_sync(FULL, k, q);
						if (rest) {
							if (kq > k || (kq == k && q < lane)) lead = false;
							rest &= rest - 1;
						}
					}
					if (lead && k > X_K[px - 1]) X_K[px - 1] = k;
					const uint32_t m = __ballot_sync(FULL, keep);
					__syncwarp(); // the chunk's loads before the in-place writes
					if (keep) {
						const int32_t pos = n_s + __popc(m & lanemask_lt());
						BA_VD[pos] = vd, BA_K[pos] = k;
					}
					n_s += __popc(m);
					__syncwarp();
				}
				n_sort = n_s;
			}
			// the wavefront buffer a is free until this step's merge writes it: sort scratch
			if (n_sort <= kRadixMin || !warp_radix_sort(BA_VD, BA_K, n_sort, A_VD, A_K, radix_hist))
				warp_bitonic_sort(BA_VD, BA_K, n_sort);
			// 1. arc-side candidates: one per diagonal with the furthest k, minus those inside an
			// ended interval; a diagonal also present among the in-vertex candidates folds its k
			// into that entry (each in-vertex entry receives at most one, as the list is unique).
			// Without TR, step 0 did the interval test and the fold already.
			int32_t n_b = 0;
			for (int32_t base = 0; base < n_sort; base += 32) {
				const int32_t j = base + lane;
				bool keep = false;
				uint64_t vd = 0;
				int32_t k = 0, tk = 0;
				if (j < n_sort) {
					vd = BA_VD[j], k = BA_K[j];
					if constexpr (TR) {
						const int2 e = BK[k];
						k = e.x, tk = e.y;
					}
					if (j == 0 || BA_VD[j - 1] != vd) {
						for (int32_t t = j + 1; t < n_sort && BA_VD[t] == vd; ++t) {
							if constexpr (TR) {
								const int2 e = BK[BA_K[t]];
								if (e.x > k) k = e.x, tk = e.y;
							} else {
								const int32_t kt = BA_K[t];
								k = kt > k ? kt : k;
							}
						}
						if constexpr (TR) {
							keep = !in_ranges(ILO, IHI, n_i, vd, i_min, i_max);
							if (keep) {
								const int32_t px = upper_bound_u64(X_VD, n_x, vd);
								if (px > 0 && X_VD[px - 1] == vd) {
									if (k > X_K[px - 1]) X_K[px - 1] = k, X_T[px - 1] = tk;
									keep = false;
								}
							}
						} else
							keep = true;
					}
				}
				__syncwarp();
				const uint32_t m = __ballot_sync(FULL, keep);
				if (keep) {
					const int32_t pos = n_b + __popc(m & lanemask_lt());
					BA_VD[pos] = vd, BA_K[pos] = k;
					if constexpr (TR) BA_T[pos] = tk;
				}
				n_b += __popc(m);
				__syncwarp();
			}
			// 2. in-vertex candidates outside the ended intervals go to their merged rank; TB
			// keeps, per chunk of 32, the kept count before the chunk and the chunk's keep mask
			uint64_t *const chunk = TB;
			int32_t n_kx = 0;
			for (int32_t base = 0; base < n_x; base += 32) {
				const int32_t j = base + lane;
				bool keep = false;
				uint64_t vd = 0;
				int32_t k = 0, t = 0;
				if (j < n_x) {
					vd = X_VD[j], k = X_K[j];
					if constexpr (TR) t = X_T[j];
					keep = !in_ranges(ILO, IHI, n_i, vd, i_min, i_max);
				}
				const uint32_t m = __ballot_sync(FULL, keep);
				if (lane == 0) chunk[base >> 5] = (uint64_t)(uint32_t)n_kx << 32 | m;
				if (keep) {
					const int32_t pos = n_kx + __popc(m & lanemask_lt()) + lower_bound_u64(BA_VD, n_b, vd);
					A_VD[pos] = vd, A_K[pos] = k;
					if constexpr (TR) A_T[pos] = t;
				}
				n_kx += __popc(m);
			}
			__syncwarp();
			// 3. arc-side candidates after the kept in-vertex candidates below them
			const int32_t n_chunks = (n_x + 31) >> 5;
			for (int32_t j = lane; j < n_b; j += 32) {
				const uint64_t vd = BA_VD[j];
				const int32_t px = upper_bound_u64(X_VD, n_x, vd), cx = px >> 5;
				int32_t below = n_kx;
				if (cx < n_chunks) {
					const uint64_t info = chunk[cx];
					below = (int32_t)(info >> 32) + __popc((uint32_t)info & ((1u << (px & 31)) - 1));
				}
				A_VD[j + below] = vd, A_K[j + below] = BA_K[j];
				if constexpr (TR) A_T[j + below] = BA_T[j];
			}
			n_new = n_kx + n_b;
			__syncwarp();
		}
		n_a = n_new;
		if (LAG && n_a > 0) {
			// lag pruning, where the reference's commented-out call sits (gwf-ed.cu:1286-1287):
			// keep the states whose query position d + k is within max_lag of the furthest
			int32_t far = INT32_MIN;
			for (int32_t j = lane; j < n_a; j += 32) {
				const int32_t i = vd_d(A_VD[j]) + A_K[j];
				far = i > far ? i : far;
			}
			far = __reduce_max_sync(FULL, far);
			const int32_t lo = far - p.max_lag;
			int32_t n_keep = 0;
			for (int32_t base = 0; base < n_a; base += 32) {
				const int32_t j = base + lane;
				uint64_t vd = 0;
				int32_t k = 0, t = 0;
				bool keep = false;
				if (j < n_a) {
					vd = A_VD[j], k = A_K[j];
					if constexpr (TR) t = A_T[j];
					keep = vd_d(vd) + k >= lo;
				}
				const uint32_t m = __ballot_sync(FULL, keep);
				if (keep) {
					const int32_t pos = n_keep + __popc(m & lanemask_lt());
					A_VD[pos] = vd, A_K[pos] = k;
					if constexpr (TR) A_T[pos] = t;
				}
				n_keep += __popc(m);
			}
			n_a = n_keep;
			__syncwarp();
		}
		if (n_a == 0) break; // wavefront emptied: no alignment (gwf-ed.cu:1313, 1336)
		if (n_a > c.a) {
			st = ST_CAPACITY;
			break;
		}
	}
	if (lane == 0) {
		p.dist[r] = st == ST_OK ? dist : -1;
		p.status[r] = st;
		if (st == ST_CAPACITY && p.retry_list) {
			const int32_t q = atomicAdd(p.retry_n, 1);
			p.retry_list[q] = r;
		}
		if (p.steps_out) p.steps_out[r] = steps;
		if (p.w_out) p.w_out[r] = W;
	}
	if constexpr (TR) {
		// walk the trace records from the end state back to the start (parents precede their
		// children, so every step lowers the index), then write the first max_nv vertices
		if (lane == 0) {
			int32_t nvp = 0;
			const bool ok = st == ST_OK && dist >= 0 && tr_t >= 0 && tr_t < n_log;
			if (ok) {
				for (int32_t t = tr_t; t >= 0; ++nvp) {
					const int32_t par = (int32_t)TLOG[t].y;
					t = par < t ? par : -1;
				}
				int32_t pos = nvp - 1;
				const int64_t row = (int64_t)r * p.max_nv;
				for (int32_t t = tr_t; t >= 0 && pos >= 0; --pos) {
					const uint2 e = TLOG[t];
					if (pos < p.max_nv) {
						const bool root = e.x == 0xffffffffu;
						p.path_v[row + pos] = root ? v0 : (int32_t)__ldg(g.arc + e.x).x;
						p.path_arc[row + pos] = root ? -1 : (int32_t)e.x;
					}
					t = (int32_t)e.y < t ? (int32_t)e.y : -1;
				}
			}
			p.path_n[r] = nvp;
			p.end_off[r] = ok ? tr_k : -1;
		}
	}
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
#undef A_T
#undef X_T
#undef BA_T
#undef E_T
#undef F_T
#undef N_T
#undef BK
#undef TLOG

// Out-of-line copy of the read loop, for the kernels that hold it beside other work (serving,
// read classes, traceback). The two batch kernels below inline the body, one instantiation per
// kernel, and run four CTAs of 8 warps per SM at 64 registers. Inlined, the body spills less at a
// given register count (-Xptxas -v at 80 registers: 200 B stack against 264 B out of line); at 64
// registers it spills about as much as the out-of-line body did at 80, and the 32 warps per SM
// hide more load latency than 24 (config 3: 438 -> 416 ms; config 2: 33.6 -> 32.2 ms; config 4
// unchanged).
template <bool TR, bool LAG>
__device__ __noinline__ void align_read_t(const KParams &p, int32_t r, uint8_t *wsb, int32_t ql_cap, int32_t level)
{
	align_read_body<TR, LAG>(p, r, wsb, ql_cap, level);
}

__device__ __forceinline__ void align_read(const KParams &p, int32_t r, uint8_t *wsb, int32_t ql_cap, int32_t level)
{
	if (p.max_lag > 0) align_read_t<false, true>(p, r, wsb, ql_cap, level);
	else align_read_t<false, false>(p, r, wsb, ql_cap, level);
}

// Plain form: one warp per queue position, arena offsets per read (main.cu:151-236 layout).
// LAG = (p.max_lag > 0), chosen by the host.
template <bool LAG>
__global__ void __launch_bounds__(256, 4) k_align_plain(const __grid_constant__ KParams p)
{
	const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
	if (gw >= p.n_order) return;
	const int32_t r = p.order[gw];
	align_read_body<false, LAG>(p, r, p.ws + p.slot_off[gw], p.r.ql[r], p.level);
}

// Traceback form: the plain form's launch shape, arenas with the trace arrays, paths written out.
__global__ void __launch_bounds__(256, 2) k_align_trace(const __grid_constant__ KParams p)
{
	const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
	if (gw >= p.n_order) return;
	const int32_t r = p.order[gw];
	align_read_t<true, false>(p, r, p.ws + p.slot_off[gw], p.r.ql[r], p.level);
}

// Persistent form: each warp owns one arena (sized for ql_cap) and pulls reads from the
// cost-ordered queue; each read uses the capacities of its own length, so a short read clears
// and touches only the arena it needs. LAG = (p.max_lag > 0), chosen by the host.
template <bool LAG>
__global__ void __launch_bounds__(256, 4) k_align_persistent(const __grid_constant__ KParams p)
{
	const int lane = threadIdx.x & 31;
	const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
	uint8_t *wsb = p.ws + gw * p.slot_bytes;
	for (int32_t guard = 0; guard < p.n_order + 1; ++guard) {
		int32_t qi = 0;
		if (lane == 0) qi = atomicAdd(p.head, 1);
		qi = __shfl_sync(FULL, qi, 0);
		if (qi >= p.n_order) break;
		const int32_t r = p.order[qi];
		align_read_body<false, LAG>(p, r, wsb, p.ql_cap, p.level);
	}
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p)
{
	unsigned long long v;
	asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ int32_t ld_acquire_s32(const int32_t *p)
{
	int32_t v;
	asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}

// Serving form. A warp claims the next published queue position (bounded, backed-off polling of
// device memory), packs the read that the host copied into its arena, aligns it at the entry's
// capacity class, and writes a completion record into host-mapped memory (an arena overflow
// comes back as GWF_E_CAPACITY; the host re-queues the read in a larger arena).
// The kernel ends as a whole: one leader warp marks q_head closed after idle_ns with nothing
// queued and no warp busy (any warp does after max_idle_ns), and every warp leaves when it sees
// the mark. A warp counts itself busy before it tries to claim, so the leader never closes
// under a claim in progress. The host relaunches the kernel when positions are queued and it
// has ended.
__global__ void __launch_bounds__(256, 3) k_serve(const __grid_constant__ SrvParams p)
{
	const int lane = threadIdx.x & 31;
	const bool leader = blockIdx.x == 0 && (threadIdx.x >> 5) == 0;
	for (int64_t guard = 0; guard < (1LL << 40); ++guard) {
		long long h = -1;
		if (lane == 0) {
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
					atomicCAS(p.q_head, head, head | SRV_CLOSED); // fails if a read was claimed
					continue;
				}
				__nanosleep(ns);
				if (ns < 32768) ns *= 2;
			}
		}
		h = __shfl_sync(FULL, h, 0);
		if (h < 0) break;
		__syncwarp();
		asm volatile("fence.acq_rel.gpu;" ::: "memory");
		const SrvEntry *ep = p.q + (h & p.qmask);
		const uint32_t seq = __ldcg((const unsigned int *)&ep->seq);
		if (seq != (uint32_t)(h + 1)) { // cannot happen while the host keeps its ring bounds
			if (lane == 0) {
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
		// pack as k_pack_reads does; the raw bytes came by DMA, so they are read from L2
		const int32_t L = ql > 0 ? ql : 0;
		const int32_t nw = (L + 31) / 32 + 2;
		bool ok = true;
		for (int32_t w = lane; w < nw; w += 32) {
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
		ok = __all_sync(FULL, ok);
		if (lane == 0) {
			hdr->zero = 0, hdr->ql = ql, hdr->v0 = v0, hdr->pure = ok ? 1 : 0;
			hdr->dist = -1, hdr->status = ST_CAPACITY;
		}
		__syncwarp();
		int32_t dist = -1, st = ST_CAPACITY;
		const int64_t qb = srv_qbytes(ql);
		const Caps c = caps_for(ql, level, p.dens_milli);
		if (qb + ws_layout(c).total <= abytes) { // the host sized it so; else report capacity
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
			align_read(lp, 0, ab + qb, ql, level);
			__syncwarp();
			dist = *(volatile int32_t *)&hdr->dist;
			st = *(volatile int32_t *)&hdr->status;
		}
		if (lane == 0) {
			const unsigned long long pos = atomicAdd(p.cq_tail, 1ULL);
			volatile SrvDone *d = p.cq + (pos & p.cmask);
			d->tag = tag, d->dist = dist, d->status = st;
			__threadfence_system();
			d->gen = (int32_t)((pos >> p.cq_shift) + 1);
			atomicSub(p.busy, 1);
		}
		__syncwarp();
	}
}

// IUPAC complement (upper and lower case; other bytes map to themselves), as the GFA loader
// complements reverse-strand segments.
__device__ __forceinline__ uint8_t comp_byte(uint8_t c)
{
	switch (c) {
	case 'A': return 'T';
	case 'T': return 'A';
	case 'C': return 'G';
	case 'G': return 'C';
	case 'a': return 't';
	case 't': return 'a';
	case 'c': return 'g';
	case 'g': return 'c';
	case 'R': return 'Y';
	case 'Y': return 'R';
	case 'K': return 'M';
	case 'M': return 'K';
	case 'B': return 'V';
	case 'V': return 'B';
	case 'D': return 'H';
	case 'H': return 'D';
	case 'r': return 'y';
	case 'y': return 'r';
	case 'k': return 'm';
	case 'm': return 'k';
	case 'b': return 'v';
	case 'v': return 'b';
	case 'd': return 'h';
	case 'h': return 'd';
	case 'U': return 'A';
	case 'u': return 'a';
	default: return c;
	}
}

// Both strands: read n + r (at raw_off[n + r]) becomes the reverse complement of read r. One
// warp per read.
__global__ void __launch_bounds__(256) k_revcomp_reads(uint8_t *__restrict__ raw, const int64_t *__restrict__ raw_off,
                                                       const int32_t *__restrict__ ql, int32_t n)
{
	const int lane = threadIdx.x & 31;
	const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
	if (r >= n) return;
	const uint8_t *src = raw + raw_off[r];
	uint8_t *dst = raw + raw_off[n + r];
	const int32_t L = ql[r] > 0 ? ql[r] : 0;
	for (int32_t i = lane; i < L; i += 32) dst[L - 1 - i] = comp_byte(src[i]);
}

// Packs reads to 2 bits per base (A=0 C=1 T=2 G=3 from bits 1-2 of the ASCII code) and flags
// reads that contain anything but A/C/G/T. One warp per read; lane l builds words l, l+32, ...
__global__ void __launch_bounds__(256) k_pack_reads(const uint8_t *__restrict__ raw,
                                                    const int64_t *__restrict__ raw_off,
                                                    const int32_t *__restrict__ ql,
                                                    const int64_t *__restrict__ pk_off,
                                                    uint64_t *__restrict__ pk, uint8_t *__restrict__ pure,
                                                    int32_t n)
{
	const int lane = threadIdx.x & 31;
	const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
	if (r >= n) return;
	const uint8_t *q = raw + raw_off[r];
	const int32_t L = ql[r] > 0 ? ql[r] : 0;
	const int32_t nw = (L + 31) / 32 + 2;
	uint64_t *out = pk + pk_off[r];
	bool ok = true;
	for (int32_t w = lane; w < nw; w += 32) {
		uint64_t word = 0;
		const int32_t b0 = w * 32;
		for (int32_t t = 0; t < 32; ++t) {
			const int32_t i = b0 + t;
			if (i < L) {
				const uint8_t ch = q[i];
				ok &= (ch == 'A' || ch == 'C' || ch == 'G' || ch == 'T');
				word |= (uint64_t)((ch >> 1) & 3) << (2 * t);
			}
		}
		out[w] = word;
	}
	ok = __all_sync(FULL, ok);
	if (lane == 0) pure[r] = ok ? 1 : 0;
}
#endif // GWF_KERNELS_DECL_ONLY

} // namespace gwfb
