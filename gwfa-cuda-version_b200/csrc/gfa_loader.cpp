// gfa_loader.cpp — GFA input side of the GWFA path: parse S/L lines (and FASTA-as-graph),
// finalize the bidirected graph, extract the topologically ordered subgraph reachable from the
// start vertex, and convert it to a gwf_graph_t.
//
// Behaviour follows the reference loader so that vertex numbering, sequences and arcs match
// `gwf-test -p` byte for byte:
//   parsing            gfa-io.c:115-220 (S), gfa-io.c:222-324 (L), gfa-io.c:326-427 (FASTA, read)
//   finalize           gfa-base.c:455-466 (no_seg, arc sort/index, semi arcs, symmetric arcs,
//                      arc lengths, cleanup), gfa-base.c:235-371
//   subgraph order     gfa-sub.c:41-272 (Kahn's algorithm with an ordered queue keyed by
//                      (in-degree left, distance, vertex) and the orphan / forced rules)
//   conversion         main.cu:294-345 (gwf_gfa2gwf), dump main.cu:354-359
// The containers are this file's own (std::vector, std::set, byte pools for names and sequences,
// and an open-addressing table of segment names).
#include <zlib.h>
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <string_view>
#include <thread>
#include <vector>

#include "../../include/gwfa.h"
#include "gwfa_internal.h"

namespace {

// Names and sequences live in two byte pools; a redefined segment (a second S line with the same
// name) points at its new bytes and leaves the old ones unused.
struct Seg {
	uint64_t seq_off = 0;
	uint32_t seq_len = 0;
	int32_t len = 0;
	bool has_seq = false;
	bool del = false;
};

struct Arc {
	uint64_t v_lv = 0; // vertex << 32 | lv
	uint64_t link_id = 0;
	uint32_t w = 0;
	int32_t ov = 0, ow = 0;
	bool del = false, comp = false;
	uint32_t head() const { return (uint32_t)(v_lv >> 32); }
};

// Segment names -> ids: open addressing, load <= 1/2. Each name is one pool entry (its id, its
// length, its bytes); a slot holds the high 24 bits of the name's hash above the entry's offset
// (0 = empty; the pool starts with a pad), so a probe reads one slot and, when the tags agree,
// one pool entry.
struct NameTable {
	std::vector<uint64_t> slot;
	std::vector<char> pool = std::vector<char>(8, 0);
	size_t n = 0;
	static constexpr uint64_t kOffMask = (1ULL << 40) - 1;
	static uint64_t hash(std::string_view k)
	{
		uint64_t h = 1469598103934665603ULL;
		for (unsigned char c : k) h = (h ^ c) * 1099511628211ULL;
		return h ^ h >> 29;
	}
	static uint64_t tag(uint64_t h) { return h >> 40 << 40; }
	uint32_t entry_id(uint64_t off) const
	{
		uint32_t id;
		memcpy(&id, pool.data() + off, 4);
		return id;
	}
	std::string_view entry_name(uint64_t off) const
	{
		uint32_t len;
		memcpy(&len, pool.data() + off + 4, 4);
		return std::string_view(pool.data() + off + 8, len);
	}
	int64_t find(std::string_view k, uint64_t h) const
	{
		if (slot.empty()) return -1;
		const size_t mask = slot.size() - 1;
		const uint64_t t = tag(h);
		for (size_t i = (size_t)h & mask;; i = (i + 1) & mask) {
			const uint64_t e = slot[i];
			if (!e) return -1;
			if ((e & ~kOffMask) == t && entry_name(e & kOffMask) == k) return entry_id(e & kOffMask);
		}
	}
	void place(uint64_t h, uint64_t off)
	{
		const size_t mask = slot.size() - 1;
		size_t i = (size_t)h & mask;
		while (slot[i]) i = (i + 1) & mask;
		slot[i] = tag(h) | off;
	}
	// sizes an empty table for n names (no growth below that)
	void reserve(size_t n_names, size_t name_bytes)
	{
		if (n) return;
		size_t cap = 1024;
		while (cap < 2 * (n_names + 1)) cap <<= 1;
		slot.assign(cap, 0);
		pool.reserve(pool.size() + name_bytes + 8 * n_names);
	}
	void prefetch(uint64_t h) const
	{
		if (!slot.empty()) __builtin_prefetch(slot.data() + (h & (slot.size() - 1)));
	}
	// second stage: the pool entry of the first slot whose tag agrees (its slot was prefetched)
	void prefetch_entry(uint64_t h) const
	{
		if (slot.empty()) return;
		const size_t mask = slot.size() - 1;
		const uint64_t t = tag(h);
		for (size_t i = (size_t)h & mask, probes = 0; probes < 4; i = (i + 1) & mask, ++probes) {
			const uint64_t e = slot[i];
			if (!e) return;
			if ((e & ~kOffMask) == t) {
				__builtin_prefetch(pool.data() + (e & kOffMask));
				return;
			}
		}
	}
	// appends the name with the given id; the caller has checked that it is absent
	void add(std::string_view k, uint64_t h, uint32_t id)
	{
		const uint64_t off = pool.size();
		const uint32_t len = (uint32_t)k.size();
		pool.resize(off + 8 + len);
		memcpy(pool.data() + off, &id, 4);
		memcpy(pool.data() + off + 4, &len, 4);
		memcpy(pool.data() + off + 8, k.data(), len);
		if (2 * (n + 1) > slot.size()) {
			std::vector<uint64_t> old;
			old.swap(slot);
			slot.assign(old.empty() ? 1024 : old.size() * 2, 0);
			for (uint64_t e : old)
				if (e) place(hash(entry_name(e & kOffMask)), e & kOffMask);
		}
		place(h, off), ++n;
	}
};

struct Gfa {
	std::vector<Seg> seg;
	NameTable names;
	std::vector<char> seq_pool;
	std::vector<Arc> arc;
	std::vector<uint64_t> idx; // per vertex: first << 32 | n
	int threads = 1;           // for the parallel steps of finalize (the parse's thread count)

	int64_t find_seg(std::string_view name) const { return names.find(name, NameTable::hash(name)); }
	uint32_t add_seg(std::string_view name) { return add_seg(name, NameTable::hash(name)); }
	uint32_t add_seg(std::string_view name, uint64_t h)
	{
		const int64_t f = names.find(name, h);
		if (f >= 0) return (uint32_t)f;
		const uint32_t id = (uint32_t)seg.size();
		seg.emplace_back();
		names.add(name, h, id);
		return id;
	}
	void set_seq(Seg &s, std::string_view sq)
	{
		s.seq_off = seq_pool.size(), s.seq_len = (uint32_t)sq.size();
		seq_pool.insert(seq_pool.end(), sq.begin(), sq.end());
	}
	const char *seq(const Seg &s) const { return seq_pool.data() + s.seq_off; }
	uint32_t n_vtx() const { return (uint32_t)seg.size() << 1; }
	uint32_t arc_n(uint32_t v) const { return v < idx.size() ? (uint32_t)idx[v] : 0; }
	uint32_t arc_off(uint32_t v) const { return v < idx.size() ? (uint32_t)(idx[v] >> 32) : 0; }
	void add_arc(uint32_t v, uint32_t w, int32_t ov, int32_t ow, int64_t link_id, bool comp)
	{
		Arc a;
		a.v_lv = (uint64_t)v << 32;
		a.w = w, a.ov = ov, a.ow = ow;
		a.link_id = link_id >= 0 ? (uint64_t)link_id : (uint64_t)arc.size();
		a.comp = comp;
		arc.push_back(a);
	}
	void arc_sort()
	{
		// arcs without lengths yet (low word 0) sort by their head vertex alone: a stable counting
		// sort over 2 * segments buckets; otherwise a stable comparison sort on the full key
		bool heads_only = true;
		uint32_t max_head = 0;
		for (const Arc &a : arc) {
			if ((uint32_t)a.v_lv) {
				heads_only = false;
				break;
			}
			max_head = std::max(max_head, a.head());
		}
		if (!heads_only || arc.size() < 64) {
			std::stable_sort(arc.begin(), arc.end(),
			                 [](const Arc &x, const Arc &y) { return x.v_lv < y.v_lv; });
			return;
		}
		std::vector<uint32_t> start((size_t)max_head + 2, 0);
		for (const Arc &a : arc) ++start[(size_t)a.head() + 1];
		for (size_t i = 1; i < start.size(); ++i) start[i] += start[i - 1];
		std::vector<Arc> out(arc.size());
		for (const Arc &a : arc) out[start[a.head()]++] = a;
		arc.swap(out);
	}
	void arc_index() // gfa-base.c:214-229
	{
		idx.assign((size_t)seg.size() * 2, 0);
		size_t n = arc.size(), last = 0;
		for (size_t i = 1; i <= n; ++i)
			if (i == n || arc[i - 1].head() != arc[i].head()) {
				uint32_t h = arc[i - 1].head();
				if (h < idx.size()) idx[h] = (uint64_t)last << 32 | (i - last);
				last = i;
			}
	}
};

// ---------------------------------------------------------------- tag helpers
using Fields = std::vector<std::string_view>;

// Finds "XY:T:value" among tab-separated optional fields; returns a pointer to value or null.
// The value runs to the next tab or the end of the line, so strtol stops where it should.
const char *find_tag(const Fields &f, size_t first, const char *key, char type)
{
	for (size_t i = first; i < f.size(); ++i) {
		const std::string_view t = f[i];
		if (t.size() >= 5 && t[2] == ':' && t[4] == ':' &&
		    (t[3] == 'A' || t[3] == 'i' || t[3] == 'f' || t[3] == 'Z' || t[3] == 'B') && t[0] == key[0] &&
		    t[1] == key[1] && t[3] == type)
			return t.data() + 5;
	}
	return nullptr;
}

void split_tabs(std::string_view line, Fields &out)
{
	out.clear();
	size_t st = 0;
	for (size_t i = 0; i <= line.size(); ++i)
		if (i == line.size() || line[i] == '\t') {
			out.emplace_back(line.data() + st, i - st);
			st = i + 1;
		}
}

// One S or L line, parsed without touching the graph (the views point into the line), so that
// lines can be parsed on several threads and applied in file order.
struct SRec {
	std::string_view name, seq;
	uint64_t h;
	int32_t len;
	bool has_seq;
};
struct LRec {
	std::string_view v, w;
	uint64_t hv, hw;
	int32_t ov, ow, l1, l2;
	uint8_t oriv, oriw;
	bool has_l1, has_l2;
};

// gfa-io.c:115-220; false for a line the reference skips
bool scan_S(std::string_view line, Fields &f, SRec &r)
{
	split_tabs(line, f); // f[0] == "S"
	if (f.size() < 3) return false;
	const std::string_view name = f[1], sq = f[2];
	int32_t LN = -1;
	if (const char *p = find_tag(f, 3, "LN", 'i')) LN = (int32_t)strtol(p, nullptr, 10);
	const bool has_seq = !(sq.size() > 0 && sq[0] == '*');
	int32_t len = 0;
	if (!has_seq) {
		if (LN >= 0) len = LN;
	} else
		len = (int32_t)sq.size();
	r.name = name, r.seq = sq, r.h = NameTable::hash(name), r.len = len, r.has_seq = has_seq;
	return true;
}

void apply_S(Gfa &g, const SRec &r)
{
	const uint32_t sid = g.add_seg(r.name, r.h);
	Seg &s = g.seg[sid];
	s.len = r.len;
	s.has_seq = r.has_seq;
	if (r.has_seq) g.set_seq(s, r.seq);
	else s.seq_len = 0;
}

// gfa-io.c:222-324; false for a line the reference skips
bool scan_L(std::string_view line, Fields &f, LRec &r)
{
	split_tabs(line, f);
	if (f.size() < 5) return false;
	const std::string_view segv = f[1], segw = f[3];
	if (f[2].empty() || (f[2][0] != '+' && f[2][0] != '-')) return false;
	if (f[4].empty() || (f[4][0] != '+' && f[4][0] != '-')) return false;
	int oriv = f[2][0] != '+', oriw = f[4][0] != '+';
	int32_t ov = 0, ow = 0;
	size_t tags_from = f.size();
	if (f.size() >= 6) {
		// the field ends at a tab or at the end of the line: strtol and isdigit stop there
		const char *q = f[5].data();
		const char *qe = q + f[5].size();
		bool ok = false;
		if (q < qe && *q == '*') {
			ov = ow = 0, ok = true;
		} else if (q < qe && *q == ':') {
			ov = INT32_MAX;
			ow = q + 1 < qe && isdigit((unsigned char)q[1]) ? (int32_t)strtol(q + 1, nullptr, 10) : INT32_MAX;
			ok = true;
		} else if (q < qe && isdigit((unsigned char)*q)) {
			char *rr;
			long first = strtol(q, &rr, 10);
			if (rr < qe && isupper((unsigned char)*rr)) { // CIGAR
				ov = ow = 0;
				const char *p = q;
				do {
					char *e;
					long l = strtol(p, &e, 10);
					p = e;
					if (*p == 'M' || *p == 'D' || *p == 'N') ov += (int32_t)l;
					if (*p == 'M' || *p == 'I' || *p == 'S') ow += (int32_t)l;
					++p;
				} while (p < qe && isdigit((unsigned char)*p));
				ok = true;
			} else if (rr < qe && *rr == ':') {
				ov = (int32_t)first;
				ow = rr + 1 < qe && isdigit((unsigned char)rr[1]) ? (int32_t)strtol(rr + 1, nullptr, 10) : INT32_MAX;
				ok = true;
			}
		}
		if (!ok) ov = ow = 0; // unparsable overlap: treated like a missing field (gfa-io.c:277)
		tags_from = 6;
	}
	r.v = segv, r.w = segw, r.hv = NameTable::hash(segv), r.hw = NameTable::hash(segw);
	r.ov = ov, r.ow = ow, r.oriv = (uint8_t)oriv, r.oriw = (uint8_t)oriw;
	const char *p1 = find_tag(f, tags_from, "L1", 'i'), *p2 = find_tag(f, tags_from, "L2", 'i');
	r.has_l1 = p1 != nullptr, r.has_l2 = p2 != nullptr;
	r.l1 = p1 ? (int32_t)strtol(p1, nullptr, 10) : 0;
	r.l2 = p2 ? (int32_t)strtol(p2, nullptr, 10) : 0;
	return true;
}

void apply_L(Gfa &g, const LRec &r)
{
	const uint32_t v = g.add_seg(r.v, r.hv) << 1 | r.oriv;
	const uint32_t w = g.add_seg(r.w, r.hw) << 1 | r.oriw;
	g.add_arc(v, w, r.ov, r.ow, -1, false);
	if (r.has_l1 && r.ov != INT32_MAX) {
		Seg &s = g.seg[v >> 1];
		if (r.ov + r.l1 > s.len) s.len = r.ov + r.l1;
	}
	if (r.has_l2 && r.ow != INT32_MAX) {
		Seg &s = g.seg[w >> 1];
		if (r.ow + r.l2 > s.len) s.len = r.ow + r.l2;
	}
}

int parse_S(Gfa &g, std::string_view line, Fields &f)
{
	SRec r;
	if (!scan_S(line, f, r)) return -1;
	apply_S(g, r);
	return 0;
}

int parse_L(Gfa &g, std::string_view line, Fields &f)
{
	LRec r;
	if (!scan_L(line, f, r)) return -1;
	apply_L(g, r);
	return 0;
}

// ---------------------------------------------------------------- finalize (gfa-base.c)
void fix_no_seg(Gfa &g)
{
	for (auto &s : g.seg)
		if (s.len == 0) s.del = true;
}

void fix_semi_arc(Gfa &g) // gfa-base.c:269-301
{
	uint32_t nvt = g.n_vtx();
	for (uint32_t v = 0; v < nvt; ++v) {
		uint32_t nv = g.arc_n(v), ofs = g.arc_off(v);
		for (uint32_t i = 0; i < nv; ++i) {
			Arc &avi = g.arc[ofs + i];
			if (avi.del || (avi.ow != INT32_MAX && avi.ov != INT32_MAX)) continue;
			uint32_t w = avi.w ^ 1;
			uint32_t nw = g.arc_n(w), ow_ = g.arc_off(w);
			int c = 0, jv = -1;
			bool multi = false;
			for (uint32_t j = 0; j < nw; ++j)
				if (!g.arc[ow_ + j].del && g.arc[ow_ + j].w == (v ^ 1)) ++c, jv = (int)j;
			if (c == 1) {
				const Arc &awj = g.arc[ow_ + jv];
				if (avi.ov != INT32_MAX && awj.ow != INT32_MAX && avi.ov != awj.ow) multi = true;
				if (avi.ow != INT32_MAX && awj.ov != INT32_MAX && avi.ow != awj.ov) multi = true;
			}
			if (c == 1 && !multi) {
				const Arc &awj = g.arc[ow_ + jv];
				if (awj.ov != INT32_MAX) avi.ow = awj.ov;
				if (awj.ow != INT32_MAX) avi.ov = awj.ow;
			} else
				avi.del = true;
		}
	}
}

// For each arc e = v -> w, the first arc of w^1's list that could be its complement (not
// deleted, w^1 -> v^1 with the overlaps swapped), whether or not an earlier arc claims it; -1 if
// none. Read-only over the arcs, so it runs on threads for large graphs.
std::vector<int64_t> complement_candidates(const Gfa &g, size_t n0)
{
	std::vector<int64_t> cand(n0, -1);
	auto scan = [&](size_t lo, size_t hi) {
		for (size_t e = lo; e < hi; ++e) {
			const Arc &avi = g.arc[e];
			if (avi.del) continue;
			const uint32_t v = avi.head(), nw = g.arc_n(avi.w ^ 1), ow_ = g.arc_off(avi.w ^ 1);
			for (uint32_t j = 0; j < nw; ++j) {
				const Arc &awj = g.arc[ow_ + j];
				if (!awj.del && awj.w == (v ^ 1) && awj.ov == avi.ow && awj.ow == avi.ov) {
					cand[e] = (int64_t)ow_ + j;
					break;
				}
			}
		}
	};
	const size_t nt = std::max<size_t>(1, (size_t)g.threads);
	std::vector<std::thread> th;
	for (size_t t = 1; t < nt; ++t) th.emplace_back(scan, n0 * t / nt, n0 * (t + 1) / nt);
	scan(0, n0 / nt);
	for (auto &x : th) x.join();
	return cand;
}

void fix_symm_add(Gfa &g) // gfa-base.c:303-338
{
	// arcs in order (the lists are sorted by head, so list order is array order); each claims
	// the first unclaimed complement of its target's list, or gets a new complement arc. The
	// candidates come precomputed; a claimed candidate sends the arc back to the plain scan.
	const size_t n0 = g.arc.size();
	const std::vector<int64_t> cand = complement_candidates(g, n0);
	g.arc.reserve(2 * n0); // at most one complement per arc
	for (size_t e = 0; e < n0; ++e) {
		const Arc avi = g.arc[e];
		if (avi.del || avi.comp) continue;
		int64_t j = cand[e];
		if (j >= 0 && g.arc[(size_t)j].comp) {
			const uint32_t v = avi.head(), nw = g.arc_n(avi.w ^ 1), ow_ = g.arc_off(avi.w ^ 1);
			j = -1;
			for (uint32_t t = 0; t < nw; ++t) {
				const Arc &awj = g.arc[ow_ + t];
				if (awj.del || awj.comp) continue;
				if (awj.w == (v ^ 1) && awj.ov == avi.ow && awj.ow == avi.ov) {
					j = (int64_t)ow_ + t;
					break;
				}
			}
		}
		if (j >= 0) {
			g.arc[(size_t)j].comp = true;
			g.arc[(size_t)j].link_id = avi.link_id;
		} else
			g.add_arc(avi.w ^ 1, avi.head() ^ 1, avi.ow, avi.ov, (int64_t)avi.link_id, true);
	}
	if (g.arc.size() > n0) {
		g.arc_sort();
		g.arc_index();
	}
}

void fix_arc_len(Gfa &g) // gfa-base.c:249-267
{
	for (auto &a : g.arc) {
		uint32_t v = a.head(), w = a.w;
		Seg &sv = g.seg[v >> 1];
		if (!sv.del && sv.len < a.ov) a.ov = sv.len;
		if (sv.del || g.seg[w >> 1].del)
			a.del = true;
		else
			a.v_lv |= (uint32_t)(sv.len - a.ov);
	}
}

void cleanup(Gfa &g) // gfa-base.c:340-371
{
	// deleted segments as a bitmap (small enough to stay in cache, unlike the segment records)
	std::vector<uint64_t> gone((g.seg.size() + 63) / 64, 0);
	for (size_t i = 0; i < g.seg.size(); ++i)
		if (g.seg[i].del) gone[i >> 6] |= 1ULL << (i & 63);
	auto is_gone = [&](uint32_t sid) { return (gone[sid >> 6] >> (sid & 63)) & 1; };
	size_t n = 0;
	for (size_t e = 0; e < g.arc.size(); ++e) {
		const Arc &a = g.arc[e];
		if (!a.del && !is_gone(a.head() >> 1) && !is_gone(a.w >> 1)) g.arc[n++] = a;
	}
	g.arc.resize(n);
	bool sorted = true;
	for (size_t e = 1; e < g.arc.size(); ++e)
		if (g.arc[e - 1].v_lv > g.arc[e].v_lv) {
			sorted = false;
			break;
		}
	if (!sorted) g.arc_sort();
	g.arc_index();
}

void finalize(Gfa &g) // gfa-base.c:455-466
{
	fix_no_seg(g);
	g.arc_sort();
	g.arc_index();
	fix_semi_arc(g);
	fix_symm_add(g);
	fix_arc_len(g);
	cleanup(g);
}

// ---------------------------------------------------------------- reader (gfa-io.c:354-427)
struct LineSource { // lines of an in-memory text, without their '\n' and one trailing '\r'
	const char *mem = nullptr;
	int64_t mem_len = 0, mem_pos = 0;

	bool getline(std::string_view &s)
	{
		if (mem_pos >= mem_len) return false;
		const char *p = mem + mem_pos, *e = mem + mem_len;
		const char *nl = (const char *)memchr(p, '\n', (size_t)(e - p));
		const char *stop = nl ? nl : e;
		s = std::string_view(p, (size_t)(stop - p));
		mem_pos += (int64_t)(stop - p) + (nl ? 1 : 0);
		if (!s.empty() && s.back() == '\r') s.remove_suffix(1);
		return true;
	}
};

bool read_gfa(LineSource &src, Gfa &g)
{
	std::string_view s;
	std::string fa_seq;
	Fields fields;
	bool is_fa = false;
	int64_t fa_seg = -1;
	auto flush_fa = [&]() {
		if (fa_seg >= 0) {
			Seg &sg = g.seg[(size_t)fa_seg];
			g.set_seq(sg, fa_seq);
			sg.has_seq = true, sg.len = (int32_t)fa_seq.size();
		}
	};
	while (src.getline(s)) {
		if (!s.empty() && s[0] == '>') {
			is_fa = true;
			flush_fa();
			char nb[32];
			snprintf(nb, sizeof nb, "s%u", (unsigned)g.seg.size() + 1);
			fa_seg = g.add_seg(nb);
			fa_seq.clear();
		} else if (is_fa) {
			if (s.size() >= 3 && s[1] == '\t') {
				flush_fa();
				fa_seg = -1, is_fa = false;
			} else
				fa_seq += s;
		}
		if (is_fa) continue;
		if (s.size() < 3 || s[1] != '\t') continue;
		int ret = 0;
		if (s[0] == 'S') ret = parse_S(g, s, fields);
		else if (s[0] == 'L') ret = parse_L(g, s, fields);
		(void)ret; // the reference reports and skips invalid lines
	}
	if (is_fa) flush_fa();
	finalize(g);
	return true;
}

// ---------------------------------------------------------------- parallel parse
// The text is cut at line ends into one chunk per thread. Each thread scans its chunk into S and
// L records (fields, numbers, name hashes); the records are then applied on one thread in file
// order, so segment ids (first appearance) and arc order are those of the sequential parse.
// Name lookups are prefetched a few records ahead. Inputs with FASTA-style records ('>' lines)
// go to the sequential parser.
struct Chunk {
	std::vector<uint8_t> kind; // 'S' or 'L', in line order
	std::vector<SRec> s;
	std::vector<LRec> l;
	bool fasta = false;
};

void scan_chunk(const char *b, const char *e, Chunk &c)
{
	Fields f;
	while (b < e) {
		const char *nl = (const char *)memchr(b, '\n', (size_t)(e - b));
		const char *le = nl ? nl : e;
		std::string_view line(b, (size_t)(le - b));
		b = nl ? nl + 1 : e;
		if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
		if (!line.empty() && line[0] == '>') {
			c.fasta = true;
			return;
		}
		if (line.size() < 3 || line[1] != '\t') continue;
		if (line[0] == 'S') {
			SRec r;
			if (scan_S(line, f, r)) c.s.push_back(r), c.kind.push_back('S');
		} else if (line[0] == 'L') {
			LRec r;
			if (scan_L(line, f, r)) c.l.push_back(r), c.kind.push_back('L');
		}
	}
}

// Threads for a text of len bytes: GWF_GFA_THREADS if set, else one per core with at least
// 1 MiB each, at most 16.
int parse_threads(size_t len)
{
	if (const char *e = getenv("GWF_GFA_THREADS")) {
		const int t = atoi(e);
		return t < 1 ? 1 : (t > 64 ? 64 : t);
	}
	const unsigned hc = std::thread::hardware_concurrency();
	size_t t = std::min<size_t>(hc ? hc : 1, 16);
	t = std::min<size_t>(t, len >> 20);
	return t < 1 ? 1 : (int)t;
}

// false: the caller parses sequentially
bool read_gfa_parallel(const char *text, size_t len, Gfa &g)
{
	const int nt = parse_threads(len);
	if (nt < 2) return false;
	std::vector<const char *> cut((size_t)nt + 1);
	cut[0] = text, cut[(size_t)nt] = text + len;
	for (int t = 1; t < nt; ++t) {
		const char *p = text + len * (size_t)t / (size_t)nt;
		if (p < cut[(size_t)t - 1]) p = cut[(size_t)t - 1];
		const char *nl = (const char *)memchr(p, '\n', (size_t)(text + len - p));
		cut[(size_t)t] = nl ? nl + 1 : text + len;
	}
	g.threads = nt;
	std::vector<Chunk> ch((size_t)nt);
	std::vector<std::thread> th;
	for (int t = 1; t < nt; ++t) th.emplace_back(scan_chunk, cut[(size_t)t], cut[(size_t)t + 1], std::ref(ch[(size_t)t]));
	scan_chunk(cut[0], cut[1], ch[0]);
	for (auto &x : th) x.join();
	size_t ns = 0, nl = 0, name_bytes = 0, seq_bytes = 0;
	for (const Chunk &c : ch) {
		if (c.fasta) return false;
		ns += c.s.size(), nl += c.l.size();
		for (const SRec &r : c.s) name_bytes += r.name.size(), seq_bytes += r.has_seq ? r.seq.size() : 0;
	}
	g.seg.reserve(ns + 16);
	g.arc.reserve(2 * nl + 16);
	g.seq_pool.reserve(seq_bytes + 16);
	g.names.reserve(ns, name_bytes);
	// slots kAhead records ahead, pool entries kNear records ahead
	constexpr size_t kAhead = 16, kNear = 8;
	for (const Chunk &c : ch) {
		size_t is = 0, il = 0;
		for (uint8_t k : c.kind) {
			if (is + kAhead < c.s.size()) g.names.prefetch(c.s[is + kAhead].h);
			if (il + kAhead < c.l.size()) {
				g.names.prefetch(c.l[il + kAhead].hv);
				g.names.prefetch(c.l[il + kAhead].hw);
			}
			if (il + kNear < c.l.size()) {
				g.names.prefetch_entry(c.l[il + kNear].hv);
				g.names.prefetch_entry(c.l[il + kNear].hw);
			}
			if (k == 'S') apply_S(g, c.s[is++]);
			else apply_L(g, c.l[il++]);
		}
	}
	finalize(g);
	return true;
}

// ---------------------------------------------------------------- subgraph (gfa-sub.c:41-272)
struct TNode {
	uint64_t xnd;
	uint32_t v;
	uint32_t in_tree; // reused as the output index after extraction
	bool forced;
};
inline uint32_t tn_n(const TNode *p) { return (uint32_t)(p->xnd << 1 >> 33); }
struct TCmp {
	bool operator()(const TNode *a, const TNode *b) const
	{
		return a->xnd < b->xnd || (a->xnd == b->xnd && a->v < b->v);
	}
};

struct Sub {
	std::vector<uint32_t> v;   // oriented GFA vertex of output vertex j
	std::vector<int32_t> off, n;
	std::vector<uint64_t> a;   // new target << 32 | arc index in g.arc
};

void sub_from(const Gfa &g, uint32_t v0, int32_t max_dist, Sub &sub)
{
	// one node per oriented vertex at most: nodes live in a vector indexed by vertex, `made` says
	// which exist (the reference keeps them in a hash table keyed by vertex)
	const uint32_t nvt = g.n_vtx();
	std::vector<TNode> node(nvt);
	std::vector<uint8_t> made(nvt, 0);
	std::set<TNode *, TCmp> tree;
	std::vector<TNode *> L;
	int32_t orphan_inv = 0;
	auto gen = [&](uint32_t v, uint32_t d) {
		TNode *p = &node[v];
		made[v] = 1;
		p->v = v, p->in_tree = 1, p->forced = false;
		p->xnd = 1ULL << 63 | (uint64_t)g.arc_n(v ^ 1) << 32 | d;
		return p;
	};
	auto get = [&](uint32_t v) -> TNode * { return v < nvt && made[v] ? &node[v] : nullptr; };
	if (v0 >= nvt) return;
	TNode *p0 = gen(v0, 0);
	tree.insert(p0);
	while (!tree.empty()) {
		TNode *q = nullptr;
		TNode *r = *tree.begin();
		if (orphan_inv) {
			for (auto it = tree.begin(); it != tree.end(); ++it) {
				TNode *c = get((*it)->v ^ 1);
				if (c && !c->in_tree) {
					--orphan_inv;
					q = *it;
					tree.erase(it);
					break;
				}
			}
		} else if (tn_n(r) > 0) {
			uint32_t rv = r->v ^ 1, nv = g.arc_n(rv), ofs = g.arc_off(rv), i;
			for (i = 0; i < nv; ++i) {
				const Arc &avi = g.arc[ofs + i];
				TNode *k1 = get(avi.w ^ 1), *k2 = get(avi.w);
				if ((!k1 && k2 && !k2->in_tree) || (!k2 && k1 && !k1->in_tree)) continue;
				break;
			}
			if (i < nv) {
				std::vector<TNode *> all(tree.begin(), tree.end());
				tree.clear();
				for (TNode *x : all) x->xnd &= ~(1ULL << 63);
				for (TNode *x : all) tree.insert(x);
			}
		}
		if (!q) {
			q = *tree.begin();
			tree.erase(tree.begin());
		}
		q->forced = (tn_n(q) > 0 || q->xnd >> 63 == 0);
		q->in_tree = 0;
		L.push_back(q);
		if (TNode *c = get(q->v ^ 1))
			if (c->in_tree) ++orphan_inv;
		uint32_t d = (uint32_t)q->xnd;
		uint32_t nv = g.arc_n(q->v), ofs = g.arc_off(q->v);
		for (uint32_t i = 0; i < nv; ++i) {
			const Arc &avi = g.arc[ofs + i];
			int32_t dt = (int32_t)(d + (uint32_t)g.seg[avi.w >> 1].len);
			if (max_dist > 0 && dt > max_dist) continue;
			TNode *c = get(avi.w ^ 1);
			if (c && !c->in_tree && !c->forced) continue;
			TNode *p = get(avi.w);
			if (!p) {
				p = gen(avi.w, (uint32_t)dt);
			} else {
				if (!p->in_tree) continue;
				tree.erase(p);
				if ((uint32_t)dt < (uint32_t)p->xnd) p->xnd = p->xnd >> 32 << 32 | (uint32_t)dt;
			}
			if (tn_n(p) > 0) p->xnd -= 1ULL << 32;
			tree.insert(p);
		}
	}
	for (size_t j = 0; j < L.size(); ++j) L[j]->in_tree = (uint32_t)j;
	sub.v.resize(L.size());
	sub.off.resize(L.size());
	sub.n.resize(L.size());
	sub.a.clear();
	for (size_t j = 0; j < L.size(); ++j) {
		size_t o0 = sub.a.size();
		uint32_t nv = g.arc_n(L[j]->v), ofs = g.arc_off(L[j]->v);
		for (uint32_t i = 0; i < nv; ++i) {
			TNode *t = get(g.arc[ofs + i].w);
			if (!t) continue;
			sub.a.push_back((uint64_t)t->in_tree << 32 | (uint64_t)(ofs + i));
		}
		sub.v[j] = L[j]->v;
		sub.off[j] = (int32_t)o0;
		sub.n[j] = (int32_t)(sub.a.size() - o0);
		std::sort(sub.a.begin() + (long)o0, sub.a.end());
	}
}

// IUPAC complement, upper and lower case; every other byte maps to itself (U -> A).
unsigned char comp_base(unsigned char c)
{
	static unsigned char t[256];
	static bool init = false;
	if (!init) {
		for (int i = 0; i < 256; ++i) t[i] = (unsigned char)i;
		const char *pairs[] = {"AT", "CG", "RY", "KM", "BV", "DH"};
		for (const char *p : pairs) {
			t[(unsigned char)p[0]] = (unsigned char)p[1], t[(unsigned char)p[1]] = (unsigned char)p[0];
			t[(unsigned char)tolower(p[0])] = (unsigned char)tolower(p[1]);
			t[(unsigned char)tolower(p[1])] = (unsigned char)tolower(p[0]);
		}
		t[(unsigned char)'U'] = 'A', t[(unsigned char)'u'] = 'a';
		init = true;
	}
	return t[c];
}

gwf_graph_t *to_gwf(const Gfa &gfa, uint32_t v0) // main.cu:294-345
{
	Sub sub;
	sub_from(gfa, v0, 1 << 30, sub);
	gwf_graph_t *g = (gwf_graph_t *)calloc(1, sizeof(gwf_graph_t));
	g->n_vtx = (uint32_t)sub.v.size();
	g->n_arc = (uint32_t)sub.a.size();
	g->len = (uint32_t *)malloc(sizeof(uint32_t) * (g->n_vtx ? g->n_vtx : 1));
	g->src = (uint32_t *)malloc(sizeof(uint32_t) * (g->n_vtx ? g->n_vtx : 1));
	g->seq = (char **)calloc(g->n_vtx ? g->n_vtx : 1, sizeof(char *));
	g->arc = (gwf_arc_t *)calloc(g->n_arc ? g->n_arc : 1, sizeof(gwf_arc_t));
	bool bad = false;
	uint32_t k = 0;
	for (uint32_t i = 0; i < g->n_vtx; ++i) {
		uint32_t v = sub.v[i];
		const Seg &s = gfa.seg[v >> 1];
		uint32_t len = (uint32_t)s.len;
		g->len[i] = len;
		g->src[i] = v;
		g->seq[i] = (char *)malloc(len + 1);
		if (!s.has_seq || s.seq_len < len) bad = true;
		const char *sq = gfa.seq(s);
		const uint32_t have = s.seq_len < len ? s.seq_len : len;
		char *out = g->seq[i];
		if (v & 1) {
			for (uint32_t j = 0; j < len; ++j) {
				const size_t p = (size_t)len - j - 1;
				out[j] = p < s.seq_len ? (char)comp_base((unsigned char)sq[p]) : 'N';
			}
		} else {
			memcpy(out, sq, have);
			memset(out + have, 'N', len - have);
		}
		g->seq[i][len] = 0;
		for (int32_t l = 0; l < sub.n[i]; ++l) {
			uint64_t a = sub.a[(size_t)(sub.off[i] + l)];
			g->arc[k].a = (uint64_t)i << 32 | (a >> 32);
			g->arc[k].o = gfa.arc[(uint32_t)a].ow;
			++k;
		}
	}
	if (bad) gwf_set_error("GFA segment without a sequence (or shorter than LN) on the walk; 'N' used");
	return g;
}

// The parsed graph from start_seg on, as a gwf_graph_t.
gwf_graph_t *finish(Gfa &gfa, const char *start_seg)
{
	if (gfa.seg.empty()) {
		gwf_set_error("GFA has no segments");
		return nullptr;
	}
	uint32_t v0 = 0;
	if (start_seg) {
		// "name", or "name+" / "name-" for a strand: the reference starts on the forward strand
		// only (main.cu:404 leaves the orientation as a TODO)
		uint32_t strand = 0;
		std::string name(start_seg);
		int64_t sid = gfa.find_seg(name);
		if (sid < 0 && name.size() > 1 && (name.back() == '+' || name.back() == '-')) {
			strand = name.back() == '-' ? 1 : 0;
			name.pop_back();
			sid = gfa.find_seg(name);
		}
		if (sid < 0) {
			gwf_set_error("start segment not found");
			return nullptr;
		}
		v0 = (uint32_t)sid << 1 | strand;
	}
	return to_gwf(gfa, v0);
}

gwf_graph_t *load_text(const char *text, size_t len, const char *start_seg)
{
	Gfa gfa;
	if (!read_gfa_parallel(text, len, gfa)) {
		gfa = Gfa();
		LineSource src;
		src.mem = text, src.mem_len = (int64_t)len;
		read_gfa(src, gfa);
	}
	return finish(gfa, start_seg);
}

} // namespace

unsigned char gwf_comp_base(unsigned char c) { return comp_base(c); }

// The whole (decompressed) file in one malloc'd buffer; realloc grows it without filling it.
// "-" or NULL is standard input. Returns NULL (and sets the error) on failure.
char *gwf_read_file(const char *path, size_t *len)
{
	gzFile fp = path && strcmp(path, "-") ? gzopen(path, "r") : gzdopen(0, "r");
	if (!fp) {
		gwf_set_error("cannot open input file");
		return nullptr;
	}
	gzbuffer(fp, 1 << 20);
	size_t cap = 1 << 24, n = 0;
	char *text = (char *)malloc(cap);
	for (; text;) {
		if (cap - n < (1u << 22)) {
			char *t2 = (char *)realloc(text, cap * 2);
			if (!t2) {
				free(text), text = nullptr;
				break;
			}
			text = t2, cap *= 2;
		}
		const int r = gzread(fp, text + n, (unsigned)std::min<size_t>(cap - n, 1u << 30));
		if (r <= 0) break;
		n += (size_t)r;
	}
	gzclose(fp);
	if (!text) {
		gwf_set_error("out of host memory reading the input file");
		return nullptr;
	}
	*len = n;
	return text;
}

extern "C" gwf_graph_t *gwf_gfa_load(const char *path, const char *start_seg)
{
	size_t n = 0;
	char *text = gwf_read_file(path, &n);
	if (!text) return nullptr;
	gwf_graph_t *g = load_text(text, n, start_seg);
	free(text);
	return g;
}

extern "C" gwf_graph_t *gwf_gfa_load_mem(const char *text, int64_t len, const char *start_seg)
{
	if (!text || len < 0) {
		gwf_set_error("null GFA text");
		return nullptr;
	}
	return load_text(text, (size_t)len, start_seg);
}

extern "C" void gwf_graph_free(gwf_graph_t *g)
{
	if (!g) return;
	gwf_cleanup(g);
	for (uint32_t i = 0; i < g->n_vtx; ++i) free(g->seq[i]);
	free(g->len), free(g->src), free(g->seq), free(g->arc);
	free(g);
}

namespace {
int n_digits(int64_t x)
{
	uint64_t u = x < 0 ? (uint64_t)(-(x + 1)) + 1 : (uint64_t)x;
	int n = x < 0 ? 2 : 1;
	while (u >= 10) u /= 10, ++n;
	return n;
}

char *put_int(char *p, int64_t x)
{
	char tmp[24];
	int n = 0;
	uint64_t u = x < 0 ? (uint64_t)(-(x + 1)) + 1 : (uint64_t)x;
	do {
		tmp[n++] = (char)('0' + u % 10);
		u /= 10;
	} while (u);
	if (x < 0) *p++ = '-';
	while (n) *p++ = tmp[--n];
	return p;
}

char *put_str(char *p, const char *s, size_t n)
{
	memcpy(p, s, n);
	return p + n;
}

// the gwf_graph_print text (main.cu:354-359): "S\t<i>\t<seq>\tLN:i:<len>" per vertex, then
// "L\t<v>\t+\t<w>\t+\t<o>M" per arc
int64_t dump_size(const gwf_graph_t *g)
{
	int64_t n = 0;
	for (uint32_t i = 0; i < g->n_vtx; ++i)
		n += 2 + n_digits((int)i) + 1 + (int64_t)strlen(g->seq[i]) + 6 + n_digits((int)g->len[i]) + 1;
	for (uint32_t i = 0; i < g->n_arc; ++i)
		n += 2 + n_digits((int)(uint32_t)(g->arc[i].a >> 32)) + 3 + n_digits((int)(uint32_t)g->arc[i].a) + 3 +
		     n_digits(g->arc[i].o) + 2;
	return n;
}

void dump_into(const gwf_graph_t *g, char *p)
{
	for (uint32_t i = 0; i < g->n_vtx; ++i) {
		p = put_str(p, "S\t", 2);
		p = put_int(p, (int)i);
		*p++ = '\t';
		p = put_str(p, g->seq[i], strlen(g->seq[i]));
		p = put_str(p, "\tLN:i:", 6);
		p = put_int(p, (int)g->len[i]);
		*p++ = '\n';
	}
	for (uint32_t i = 0; i < g->n_arc; ++i) {
		p = put_str(p, "L\t", 2);
		p = put_int(p, (int)(uint32_t)(g->arc[i].a >> 32));
		p = put_str(p, "\t+\t", 3);
		p = put_int(p, (int)(uint32_t)g->arc[i].a);
		p = put_str(p, "\t+\t", 3);
		p = put_int(p, g->arc[i].o);
		p = put_str(p, "M\n", 2);
	}
}
} // namespace

extern "C" int64_t gwf_graph_dump(const gwf_graph_t *g, char *buf, int64_t cap)
{
	const int64_t n = dump_size(g);
	if (!buf || cap <= 0) return n;
	if (cap > n) {
		dump_into(g, buf);
		buf[n] = 0;
	} else {
		std::vector<char> tmp((size_t)n);
		dump_into(g, tmp.data());
		memcpy(buf, tmp.data(), (size_t)cap);
	}
	return n;
}
