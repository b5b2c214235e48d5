// synth.cpp — seeded synthetic variation graphs and error-bearing reads (gwfa_synth.h).
// PRNG: xoshiro256** seeded through splitmix64 (both public-domain published generators,
// written here from their definitions).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gwfa_synth.h"

namespace {

struct Rng {
	uint64_t s[4];
	explicit Rng(uint64_t seed)
	{
		uint64_t x = seed;
		for (int i = 0; i < 4; ++i) {
			x += 0x9e3779b97f4a7c15ULL;
			uint64_t z = x;
			z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
			z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
			s[i] = z ^ (z >> 31);
		}
	}
	static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
	uint64_t next()
	{
		uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
		s[2] ^= s[0], s[3] ^= s[1], s[1] ^= s[2], s[0] ^= s[3];
		s[2] ^= t, s[3] = rotl(s[3], 45);
		return r;
	}
	double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
	uint32_t below(uint32_t n) { return (uint32_t)(uniform() * n); }
	double normal()
	{
		double u1 = uniform(), u2 = uniform();
		if (u1 < 1e-300) u1 = 1e-300;
		return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
	}
};

const char kBase[4] = {'A', 'C', 'G', 'T'};

struct Graph {
	std::vector<std::string> seg;
	std::vector<std::vector<uint32_t>> out;
	std::vector<uint32_t> backbone; // origin candidates
	std::vector<std::pair<uint32_t, uint32_t>> links;

	uint32_t add(std::string s, bool bb)
	{
		seg.push_back(std::move(s));
		out.emplace_back();
		if (bb) backbone.push_back((uint32_t)seg.size() - 1);
		return (uint32_t)seg.size() - 1;
	}
	void link(uint32_t a, uint32_t b)
	{
		out[a].push_back(b);
		links.emplace_back(a, b);
	}
};

struct Reads {
	std::string seqs;
	std::vector<int64_t> offs;
	std::vector<int32_t> lens, origin;
	std::vector<float> err;
};

Graph *make_graph(int64_t L, int32_t every, double p_snp, int32_t indel_max, int32_t sv_every,
                  int32_t sv_min, int32_t sv_max, uint64_t seed)
{
	Rng rng(seed);
	std::string B((size_t)L, 'A');
	for (int64_t i = 0; i < L; ++i) B[(size_t)i] = kBase[rng.next() >> 62];
	struct Ev { int64_t pos; int type; int64_t len; }; // 0 SNP, 1 INS, 2 DEL
	std::vector<Ev> ev;
	int64_t sv_next = sv_every > 0 ? sv_every : -1, sv_block_end = -1;
	int64_t margin = (int64_t)(sv_every > 0 && sv_max > indel_max ? sv_max : indel_max) + 2;
	for (int64_t p = every; p + margin < L; p += every) {
		if (sv_next > 0 && p >= sv_next) {
			int64_t len = sv_min + (int64_t)rng.below((uint32_t)(sv_max - sv_min + 1));
			int type = (rng.next() >> 63) ? 1 : 2;
			ev.push_back({p, type, len});
			if (type == 2) sv_block_end = p + len;
			sv_next += sv_every;
			continue;
		}
		if (p <= sv_block_end + 1) continue;
		if (rng.uniform() < p_snp)
			ev.push_back({p, 0, 1});
		else {
			int64_t len = 1 + (int64_t)rng.below((uint32_t)indel_max);
			ev.push_back({p, (rng.next() >> 63) ? 1 : 2, len});
		}
	}
	Graph *g = new Graph;
	std::vector<uint32_t> tails;
	int64_t cur = 0;
	auto connect = [&](uint32_t to) {
		for (uint32_t t : tails) g->link(t, to);
	};
	for (const Ev &e : ev) {
		if (e.pos < cur + 1) continue; // keep one backbone base between events
		uint32_t bb = g->add(B.substr((size_t)cur, (size_t)(e.pos - cur)), true);
		connect(bb);
		tails.assign(1, bb);
		if (e.type == 0) {
			char ref = B[(size_t)e.pos], alt;
			do alt = kBase[rng.next() >> 62]; while (alt == ref);
			uint32_t r = g->add(std::string(1, ref), false), a = g->add(std::string(1, alt), false);
			g->link(bb, r), g->link(bb, a);
			tails.assign({r, a});
			cur = e.pos + 1;
		} else if (e.type == 1) {
			std::string ins((size_t)e.len, 'A');
			for (auto &c : ins) c = kBase[rng.next() >> 62];
			uint32_t s = g->add(ins, false);
			g->link(bb, s);
			tails.assign({bb, s});
			cur = e.pos;
		} else {
			uint32_t s = g->add(B.substr((size_t)e.pos, (size_t)e.len), false);
			g->link(bb, s);
			tails.assign({bb, s});
			cur = e.pos + e.len;
		}
	}
	uint32_t last = g->add(B.substr((size_t)cur), true);
	connect(last);
	return g;
}

Reads *make_reads(const Graph &g, int32_t n, int32_t kind, double a, double b, int32_t lmin,
                  int32_t lmax, double emin, double emax, uint64_t seed)
{
	Rng rng(seed);
	Reads *R = new Reads;
	R->offs.reserve((size_t)n), R->lens.reserve((size_t)n);
	std::string truth, read;
	for (int32_t i = 0; i < n; ++i) {
		int64_t L;
		if (kind == 1) L = (int64_t)std::llround(a * std::exp(b * rng.normal()));
		else if (kind == 2) L = (int64_t)std::llround(a + (b - a) * rng.uniform());
		else L = (int64_t)a;
		if (L < lmin) L = lmin;
		if (L > lmax) L = lmax;
		double e = emin + (emax - emin) * rng.uniform();
		uint32_t origin = 0;
		for (int attempt = 0;; ++attempt) {
			origin = g.backbone[rng.below((uint32_t)g.backbone.size())];
			truth.clear();
			uint32_t v = origin;
			for (;;) {
				const std::string &s = g.seg[v];
				truth.append(s, 0, (size_t)std::min<int64_t>((int64_t)s.size(), L - (int64_t)truth.size()));
				if ((int64_t)truth.size() >= L || g.out[v].empty()) break;
				v = g.out[v][rng.below((uint32_t)g.out[v].size())];
			}
			if ((int64_t)truth.size() >= L || attempt > 1000) break;
		}
		read.clear();
		for (char c : truth) {
			if (rng.uniform() < e) {
				double r = rng.uniform();
				if (r < 0.6) {
					char x;
					do x = kBase[rng.next() >> 62]; while (x == c);
					read.push_back(x);
				} else if (r < 0.8) {
					read.push_back(kBase[rng.next() >> 62]);
					read.push_back(c);
				} // else: deletion
			} else
				read.push_back(c);
		}
		if (read.empty()) read.push_back(truth.empty() ? 'A' : truth[0]);
		R->offs.push_back((int64_t)R->seqs.size());
		R->lens.push_back((int32_t)read.size());
		R->origin.push_back((int32_t)origin);
		R->err.push_back((float)e);
		R->seqs += read;
	}
	return R;
}

} // namespace

extern "C" {

void *gwf_synth_graph_new(int64_t backbone_len, int32_t site_every, double p_snp, int32_t indel_max,
                          int32_t sv_every, int32_t sv_min, int32_t sv_max, uint64_t seed)
{
	if (backbone_len < 2 || site_every < 2 || indel_max < 1 || indel_max >= site_every) return nullptr;
	if (sv_every > 0 && (sv_min < 1 || sv_max < sv_min)) return nullptr;
	return make_graph(backbone_len, site_every, p_snp, indel_max, sv_every, sv_min, sv_max, seed);
}

void gwf_synth_graph_free(void *g) { delete (Graph *)g; }

int32_t gwf_synth_graph_nseg(void *g) { return (int32_t)((Graph *)g)->seg.size(); }

int64_t gwf_synth_graph_gfa(void *gp, char *buf, int64_t cap)
{
	const Graph &g = *(Graph *)gp;
	std::string out = "H\tVN:Z:1.0\n";
	char tmp[64];
	for (size_t i = 0; i < g.seg.size(); ++i) {
		snprintf(tmp, sizeof tmp, "S\ts%zu\t", i + 1);
		out += tmp;
		out += g.seg[i];
		out += '\n';
	}
	for (const auto &l : g.links) {
		snprintf(tmp, sizeof tmp, "L\ts%u\t+\ts%u\t+\t0M\n", l.first + 1, l.second + 1);
		out += tmp;
	}
	if (buf && cap > 0) memcpy(buf, out.data(), (size_t)std::min<int64_t>(cap, (int64_t)out.size()));
	return (int64_t)out.size();
}

void *gwf_synth_reads_new(void *g, int32_t n, int32_t len_kind, double len_a, double len_b,
                          int32_t len_min, int32_t len_max, double err_min, double err_max,
                          uint64_t seed)
{
	if (!g || n < 0) return nullptr;
	return make_reads(*(Graph *)g, n, len_kind, len_a, len_b, len_min, len_max, err_min, err_max, seed);
}

int64_t gwf_synth_reads_bytes(void *r) { return (int64_t)((Reads *)r)->seqs.size(); }

void gwf_synth_reads_copy(void *rp, char *seqs, int64_t *offs, int32_t *lens, int32_t *origin, float *err)
{
	const Reads &r = *(Reads *)rp;
	if (seqs) memcpy(seqs, r.seqs.data(), r.seqs.size());
	if (offs) memcpy(offs, r.offs.data(), r.offs.size() * sizeof(int64_t));
	if (lens) memcpy(lens, r.lens.data(), r.lens.size() * sizeof(int32_t));
	if (origin) memcpy(origin, r.origin.data(), r.origin.size() * sizeof(int32_t));
	if (err) memcpy(err, r.err.data(), r.err.size() * sizeof(float));
}

void gwf_synth_reads_free(void *r) { delete (Reads *)r; }
}
