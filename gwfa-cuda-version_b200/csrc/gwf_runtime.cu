// gwf_runtime.cu — host side of libgwfa_b200: the C ABI declared in include/gwfa.h.
//
// gwf_ed_index builds the reference's host CSR (main.cu:246-270) and a device-resident copy of
// the graph: vertex lengths, base offsets, 2-bit packed and raw sequences, CSR arcs. Batches run
// on one stream: reads are copied once, packed on the device, aligned by the plain or the
// persistent kernel, and reads whose arena overflowed are re-run at the next arena size class.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <unordered_map>
#include <vector>

#include "../../include/gwfa.h"
#include "gwf_cigar.cuh"
#include "gwf_group.cuh"
#include "gwf_kernels.cuh"
#include "gwf_runtime.h"
#include "gwfa_internal.h"

using namespace gwfb;

// ------------------------------------------------------------------ errors
static thread_local char t_err[1024];

void gwf_set_error(const char *msg) { snprintf(t_err, sizeof t_err, "%s", msg); }
void gwf_set_errorf(const char *fmt, ...)
{
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(t_err, sizeof t_err, fmt, ap);
	va_end(ap);
}
extern "C" const char *gwf_last_error(void) { return t_err; }
extern "C" const char *gwf_version(void) { return "gwfa-b200 0.1 (sm_100a)"; }

#define CK(call)                                                                                    \
	do {                                                                                            \
		cudaError_t e_ = (call);                                                                    \
		if (e_ != cudaSuccess) {                                                                    \
			gwf_set_errorf("%s failed: %s", #call, cudaGetErrorString(e_));                        \
			return GWF_E_CUDA;                                                                      \
		}                                                                                           \
	} while (0)

// ------------------------------------------------------------------ buffers
int DBuf::ensure(size_t n)
{
	if (n <= cap) return 0;
	if (p) cudaFree(p);
	p = nullptr, cap = 0;
	size_t want = n + n / 4 + 256;
	if (cudaMalloc(&p, want) != cudaSuccess) {
		p = nullptr;
		cudaGetLastError();
		gwf_set_errorf("device allocation of %zu bytes failed", want);
		return GWF_E_NOMEM;
	}
	cap = want;
	return 0;
}
void DBuf::release()
{
	if (p) cudaFree(p);
	p = nullptr, cap = 0;
}

int HBuf::ensure(size_t n)
{
	if (n <= cap) return 0;
	if (p) cudaFreeHost(p);
	p = nullptr, cap = 0;
	size_t want = n + n / 4 + 256;
	if (cudaMallocHost(&p, want) != cudaSuccess) {
		p = nullptr;
		cudaGetLastError();
		gwf_set_errorf("pinned allocation of %zu bytes failed", want);
		return GWF_E_NOMEM;
	}
	cap = want;
	return 0;
}
void HBuf::release()
{
	if (p) cudaFreeHost(p);
	p = nullptr, cap = 0;
}

// ------------------------------------------------------------------ device selection
int gwf_select_device(int want, int *dev_out)
{
	int n = 0;
	cudaError_t e = cudaGetDeviceCount(&n);
	if (e != cudaSuccess || n == 0) {
		cudaGetLastError();
		gwf_set_errorf("no usable CUDA device: %s", e == cudaSuccess ? "none found" : cudaGetErrorString(e));
		return GWF_E_CUDA;
	}
	int dev = want;
	if (dev < 0) CK(cudaGetDevice(&dev));
	if (dev >= n) {
		gwf_set_error("device ordinal out of range");
		return GWF_E_BAD_INPUT;
	}
	cudaDeviceProp prop;
	CK(cudaGetDeviceProperties(&prop, dev));
	if (prop.major != 10) {
		gwf_set_errorf("device %d is sm_%d%d; this library is built for sm_100a (B200) only", dev,
		               prop.major, prop.minor);
		return GWF_E_CUDA;
	}
	CK(cudaSetDevice(dev));
	*dev_out = dev;
	return 0;
}

// ------------------------------------------------------------------ device graphs
static std::mutex g_graph_mu;
static std::unordered_map<const gwf_graph_t *, GraphDev *> g_graphs;

DevGraph GraphDev::view() const
{
	DevGraph v;
	v.len = (const uint32_t *)len.p;
	v.base = (const uint64_t *)base.p;
	v.pk = (const uint64_t *)pk.p;
	v.raw = (const uint8_t *)raw.p;
	v.arc_off = (const uint32_t *)arc_off.p;
	v.arc = (const uint2 *)arc.p;
	v.arc_key = (const uint32_t *)arc_key.p;
	v.n_vtx = n_vtx;
	v.pure = pure;
	return v;
}

GraphDev::~GraphDev()
{
	int cur = -1;
	cudaGetDevice(&cur);
	if (device >= 0) cudaSetDevice(device);
	len.release(), base.release(), pk.release(), raw.release(), arc_off.release(), arc.release();
	arc_key.release();
	if (cur >= 0) cudaSetDevice(cur);
}

GraphDev *gwf_find_graph(const gwf_graph_t *g)
{
	std::lock_guard<std::mutex> lk(g_graph_mu);
	auto it = g_graphs.find(g);
	return it == g_graphs.end() ? nullptr : it->second;
}

static uint8_t code2(uint8_t c) { return (uint8_t)((c >> 1) & 3); } // A0 C1 T2 G3

static int upload_graph(const gwf_graph_t *g, GraphDev *G)
{
	const uint32_t nv = g->n_vtx;
	std::vector<uint32_t> len(nv);
	std::vector<uint64_t> base(nv);
	uint64_t tot = 0;
	for (uint32_t v = 0; v < nv; ++v) len[v] = g->len[v], base[v] = tot, tot += g->len[v];
	const size_t nw = (size_t)((tot + 31) / 32 + 2);
	std::vector<uint64_t> pk(nw, 0);
	std::vector<uint8_t> raw((size_t)tot + 16, 0);
	int pure = 1;
	for (uint32_t v = 0; v < nv; ++v) {
		const char *s = g->seq[v];
		for (uint32_t j = 0; j < len[v]; ++j) {
			const uint8_t c = (uint8_t)s[j];
			const uint64_t p = base[v] + j;
			raw[(size_t)p] = c;
			if (c != 'A' && c != 'C' && c != 'G' && c != 'T') pure = 0;
			pk[(size_t)(p >> 5)] |= (uint64_t)code2(c) << (2 * (p & 31));
		}
	}
	std::vector<uint32_t> off(nv + 1, 0);
	for (uint32_t e = 0; e < g->n_arc; ++e) off[(uint32_t)(g->arc[e].a >> 32) + 1]++;
	for (uint32_t v = 0; v < nv; ++v) off[v + 1] += off[v];
	std::vector<uint2> arc(g->n_arc ? g->n_arc : 1);
	for (uint32_t e = 0; e < g->n_arc; ++e) arc[e] = make_uint2((uint32_t)g->arc[e].a, (uint32_t)g->arc[e].o);
	// Arrival keys. The reference keys an arrival by (target w, query position) (gwf-ed.cu:1196),
	// which names one graph position when every arc into w enters it at the same offset. Where the
	// arcs into w carry different overlaps, the arcs entering w at one offset share an entry id of
	// their own (>= n_vtx), so that arrivals at different offsets of w stay distinct.
	std::vector<int32_t> first(nv, -1);
	std::vector<uint8_t> mixed(nv, 0);
	bool any_mixed = false;
	for (uint32_t e = 0; e < g->n_arc; ++e) {
		const uint32_t w = (uint32_t)g->arc[e].a;
		if (first[w] < 0) first[w] = g->arc[e].o;
		else if (first[w] != g->arc[e].o) mixed[w] = 1, any_mixed = true;
	}
	std::vector<uint32_t> key;
	if (any_mixed) {
		if ((uint64_t)nv + g->n_arc >= 0xffffffffULL) {
			gwf_set_error("gwf_ed_index: too many vertices and arcs for the arrival keys");
			return GWF_E_BAD_GRAPH;
		}
		std::vector<std::pair<uint64_t, uint32_t>> t;
		key.resize(g->n_arc);
		for (uint32_t e = 0; e < g->n_arc; ++e) {
			const uint32_t w = (uint32_t)g->arc[e].a;
			key[e] = w;
			if (mixed[w]) t.push_back({(uint64_t)w << 32 | (uint32_t)g->arc[e].o, e});
		}
		std::sort(t.begin(), t.end());
		uint32_t next = nv;
		for (size_t i = 0; i < t.size(); ++i) {
			if (i > 0 && t[i].first != t[i - 1].first) ++next;
			key[t[i].second] = next;
		}
	}
	G->n_vtx = nv, G->n_arc = g->n_arc, G->pure = pure, G->total_len = tot;
	G->dens_milli = (int32_t)std::max<uint64_t>(1, (uint64_t)nv * 1000 / std::max<uint64_t>(1, tot));
	int rc;
	if ((rc = G->len.ensure(sizeof(uint32_t) * std::max<size_t>(nv, 1)))) return rc;
	if ((rc = G->base.ensure(sizeof(uint64_t) * std::max<size_t>(nv, 1)))) return rc;
	if ((rc = G->pk.ensure(sizeof(uint64_t) * nw))) return rc;
	if ((rc = G->raw.ensure(raw.size()))) return rc;
	if ((rc = G->arc_off.ensure(sizeof(uint32_t) * (nv + 1)))) return rc;
	if ((rc = G->arc.ensure(sizeof(uint2) * arc.size()))) return rc;
	CK(cudaMemcpy(G->len.p, len.data(), sizeof(uint32_t) * nv, cudaMemcpyHostToDevice));
	CK(cudaMemcpy(G->base.p, base.data(), sizeof(uint64_t) * nv, cudaMemcpyHostToDevice));
	CK(cudaMemcpy(G->pk.p, pk.data(), sizeof(uint64_t) * nw, cudaMemcpyHostToDevice));
	CK(cudaMemcpy(G->raw.p, raw.data(), raw.size(), cudaMemcpyHostToDevice));
	CK(cudaMemcpy(G->arc_off.p, off.data(), sizeof(uint32_t) * (nv + 1), cudaMemcpyHostToDevice));
	CK(cudaMemcpy(G->arc.p, arc.data(), sizeof(uint2) * arc.size(), cudaMemcpyHostToDevice));
	if (any_mixed) {
		if ((rc = G->arc_key.ensure(sizeof(uint32_t) * key.size()))) return rc;
		CK(cudaMemcpy(G->arc_key.p, key.data(), sizeof(uint32_t) * key.size(), cudaMemcpyHostToDevice));
	}
	return 0;
}

extern "C" void gwf_ed_index(gwf_graph_t *g)
{
	if (!g) {
		gwf_set_error("gwf_ed_index: null graph");
		return;
	}
	// host CSR, as the reference (main.cu:246-270): arcs sorted by a, aux[v] = first << 32 | n
	std::stable_sort(g->arc, g->arc + g->n_arc,
	                 [](const gwf_arc_t &x, const gwf_arc_t &y) { return x.a < y.a; });
	free(g->aux);
	g->aux = (uint64_t *)calloc(g->n_vtx ? g->n_vtx : 1, sizeof(uint64_t));
	for (uint32_t st = 0, i = 1; i <= g->n_arc; ++i)
		if (i == g->n_arc || g->arc[i].a >> 32 != g->arc[st].a >> 32) {
			const uint32_t v = (uint32_t)(g->arc[st].a >> 32);
			if (v < g->n_vtx) g->aux[v] = (uint64_t)st << 32 | (i - st);
			st = i;
		}
	// the device path needs well-formed input
	for (uint32_t v = 0; v < g->n_vtx; ++v)
		if (g->len[v] == 0 || !g->seq || !g->seq[v]) {
			gwf_set_errorf("gwf_ed_index: vertex %u has no sequence", v);
			return;
		}
	for (uint32_t e = 0; e < g->n_arc; ++e) {
		const uint32_t s = (uint32_t)(g->arc[e].a >> 32), w = (uint32_t)g->arc[e].a;
		if (s >= g->n_vtx || w >= g->n_vtx || g->arc[e].o < 0 || (uint32_t)g->arc[e].o >= g->len[w]) {
			gwf_set_errorf("gwf_ed_index: arc %u (%u -> %u, overlap %d) is out of range", e, s, w,
			               g->arc[e].o);
			return;
		}
	}
	int dev;
	if (gwf_select_device(-1, &dev)) return; // host CSR stays usable; error recorded
	GraphDev *G = new GraphDev;
	G->device = dev;
	if (upload_graph(g, G)) {
		delete G;
		return;
	}
	std::lock_guard<std::mutex> lk(g_graph_mu);
	auto it = g_graphs.find(g);
	if (it != g_graphs.end()) delete it->second;
	g_graphs[g] = G;
}

extern "C" void gwf_cleanup(gwf_graph_t *g)
{
	if (!g) return;
	free(g->aux);
	g->aux = 0;
	GraphDev *G = nullptr;
	{
		std::lock_guard<std::mutex> lk(g_graph_mu);
		auto it = g_graphs.find(g);
		if (it != g_graphs.end()) G = it->second, g_graphs.erase(it);
	}
	delete G;
}

// ------------------------------------------------------------------ engine
Engine::~Engine()
{
	cudaSetDevice(device);
	for (DBuf *b : {&pk_off, &order, &head, &retry_list, &retry_n, &ws, &slot_off, &w_out})
		b->release();
	for (HBuf *b : {&h_small, &h_stage}) b->release();
	for (cudaEvent_t e : stage_ev)
		if (e) cudaEventDestroy(e);
	if (stream) cudaStreamDestroy(stream);
	if (ev0) cudaEventDestroy(ev0);
	if (ev1) cudaEventDestroy(ev1);
}

static std::mutex g_engine_mu;
static std::unordered_map<int, Engine *> g_engines;

Engine *gwf_engine(int dev)
{
	std::lock_guard<std::mutex> lk(g_engine_mu);
	auto it = g_engines.find(dev);
	if (it != g_engines.end()) return it->second;
	Engine *E = new Engine;
	E->device = dev;
	cudaSetDevice(dev);
	if (cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) != cudaSuccess ||
	    cudaEventCreate(&E->ev0) != cudaSuccess || cudaEventCreate(&E->ev1) != cudaSuccess ||
	    cudaEventCreateWithFlags(&E->stage_ev[0], cudaEventDisableTiming) != cudaSuccess ||
	    cudaEventCreateWithFlags(&E->stage_ev[1], cudaEventDisableTiming) != cudaSuccess) {
		cudaGetLastError();
		gwf_set_error("stream/event creation failed");
		delete E;
		return nullptr;
	}
	cudaDeviceGetAttribute(&E->sm_count, cudaDevAttrMultiProcessorCount, dev);
	{
		size_t fr = 0, tot = 0;
		cudaMemGetInfo(&fr, &tot);
		E->mem_budget = (int64_t)(fr / 2);
	}
	int occ = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_align_persistent<false>, 256, 0);
	E->persistent_ctas_per_sm = occ > 0 ? occ : 1;
	occ = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_align_classes, 256, 0);
	E->classes_ctas_per_sm = occ > 0 ? occ : 1;
	g_engines[dev] = E;
	return E;
}

// ------------------------------------------------------------------ batches
void Batch::release()
{
	for (DBuf *b : {&raw, &raw_off, &ql, &v0, &pk, &pk_off, &pure, &dist, &status, &steps, &order_ql, &order_cls})
		b->release();
	cls_key = ~0ULL, cls_gen = ~0ULL;
	h_meta.release();
	if (gexec) cudaGraphExecDestroy(gexec), gexec = nullptr;
}

// Copies n reads (host, concatenated) into the batch's device buffers; computes host-side
// layout (packed offsets, cost order).
// Host-to-device copy on the engine's stream. A page-locked source goes to the DMA engine as
// it is; a pageable one of more than 1 MiB passes through two pinned 8 MiB chunks in turn, so
// that filling one chunk overlaps the transfer of the other.
static const int kWarpsPerCtaPack = 8; // warps per CTA of the per-read helper kernels

static int upload(Engine &E, void *dst, const void *src, size_t n)
{
	cudaPointerAttributes at;
	const bool pinned = cudaPointerGetAttributes(&at, src) == cudaSuccess && at.type == cudaMemoryTypeHost;
	cudaGetLastError();
	if (pinned || n <= ((size_t)1 << 20)) {
		CK(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, E.stream));
		return 0;
	}
	const size_t chunk = (size_t)8 << 20;
	int rc;
	if ((rc = E.h_stage.ensure(2 * chunk))) return rc;
	for (size_t off = 0, i = 0; off < n; off += chunk, ++i) {
		const size_t b = i & 1, len = std::min(chunk, n - off);
		CK(cudaEventSynchronize(E.stage_ev[b])); // the DMA that last read this chunk, if any
		char *stage = (char *)E.h_stage.p + b * chunk;
		memcpy(stage, (const char *)src + off, len);
		CK(cudaMemcpyAsync((char *)dst + off, stage, len, cudaMemcpyHostToDevice, E.stream));
		CK(cudaEventRecord(E.stage_ev[b], E.stream));
	}
	return 0;
}

int gwf_batch_load(Engine &E, Batch &B, int32_t n_in, const char *seqs, const int64_t *offs,
                   const int32_t *ql_in, const int32_t *v0, int32_t v1, bool both)
{
	// with both strands the batch holds 2 n reads: read n + i is the reverse complement of read
	// i, made on the device, with the same v0
	const int32_t n = both ? 2 * n_in : n_in;
	if (both && n_in > INT32_MAX / 2) return GWF_E_BAD_INPUT;
	B.n = n, B.n_in = n_in, B.both = both, B.v1 = v1;
	++B.generation;
	B.h_ql.assign(ql_in, ql_in + n_in);
	if (both) B.h_ql.insert(B.h_ql.end(), ql_in, ql_in + n_in);
	const int32_t *ql = B.h_ql.data();
	int64_t lo = 0, hi = 0;
	if (n_in > 0) {
		lo = offs[0], hi = offs[0];
		for (int32_t i = 0; i < n_in; ++i) {
			if (ql[i] < 0) return GWF_E_BAD_INPUT;
			lo = std::min(lo, offs[i]);
			hi = std::max(hi, offs[i] + ql[i]);
		}
	}
	const int64_t span = hi - lo, rc_base = span + 16; // the reverse complements after the reads
	// pinned metadata: raw offsets and packed offsets (int64), queue order (int32)
	int rc;
	if ((rc = B.h_meta.ensure(20 * (size_t)n + 64))) return rc;
	int64_t *h_raw_off = (int64_t *)B.h_meta.p, *h_pk_off = h_raw_off + n;
	int32_t *h_order = (int32_t *)(h_pk_off + n);
	for (int32_t i = 0; i < n_in; ++i) h_raw_off[i] = offs[i] - lo;
	if (both)
		for (int32_t i = 0; i < n_in; ++i) h_raw_off[n_in + i] = rc_base + offs[i] - lo;
	int64_t words = 0;
	for (int32_t i = 0; i < n; ++i) h_pk_off[i] = words, words += (ql[i] + 31) / 32 + 2;
	B.pk_words = words;
	// persistent queue: longest reads first (LPT scheduling on a cost ~ length estimate), as a
	// counting sort over 64-base length buckets
	B.max_ql = 0;
	for (int32_t i = 0; i < n; ++i) B.max_ql = std::max(B.max_ql, ql[i]);
	{
		double w[GWF_TUNE_NBUCKETS] = {0};
		for (int32_t i = 0; i < n; ++i) w[gwf_tune_bucket(ql[i])] += (double)ql[i] * (double)ql[i];
		B.dom_bucket = (int32_t)(std::max_element(w, w + GWF_TUNE_NBUCKETS) - w);
	}
	{
		const int32_t nb = (B.max_ql >> 6) + 1;
		std::vector<int32_t> cnt((size_t)nb + 1, 0);
		for (int32_t i = 0; i < n; ++i) cnt[(size_t)(nb - 1 - (ql[i] >> 6)) + 1]++;
		for (int32_t b = 0; b < nb; ++b) cnt[(size_t)b + 1] += cnt[(size_t)b];
		for (int32_t i = 0; i < n; ++i) h_order[cnt[(size_t)(nb - 1 - (ql[i] >> 6))]++] = i;
	}
	const size_t nraw = (size_t)(both ? 2 * rc_base : rc_base);
	if ((rc = B.raw.ensure(nraw)) || (rc = B.raw_off.ensure(8 * (size_t)n + 8)) ||
	    (rc = B.ql.ensure(4 * (size_t)n + 4)) || (rc = B.v0.ensure(4 * (size_t)n + 4)) ||
	    (rc = B.pk.ensure(8 * (size_t)words + 8)) || (rc = B.pk_off.ensure(8 * (size_t)n + 8)) ||
	    (rc = B.pure.ensure((size_t)n + 8)) || (rc = B.dist.ensure(4 * (size_t)n + 4)) ||
	    (rc = B.status.ensure(4 * (size_t)n + 4)) || (rc = B.steps.ensure(4 * (size_t)n + 4)) ||
	    (rc = B.order_ql.ensure(4 * (size_t)n + 4)))
		return rc;
	cudaStream_t s = E.stream;
	if (n > 0) {
		if ((rc = upload(E, B.raw.p, seqs + lo, (size_t)span))) return rc;
		CK(cudaMemsetAsync((char *)B.raw.p + span, 0, 16, s));
		CK(cudaMemcpyAsync(B.raw_off.p, h_raw_off, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
		if ((rc = upload(E, B.ql.p, ql_in, 4 * (size_t)n_in)) || (rc = upload(E, B.v0.p, v0, 4 * (size_t)n_in)))
			return rc;
		if (both) {
			CK(cudaMemcpyAsync((int32_t *)B.ql.p + n_in, B.ql.p, 4 * (size_t)n_in, cudaMemcpyDeviceToDevice, s));
			CK(cudaMemcpyAsync((int32_t *)B.v0.p + n_in, B.v0.p, 4 * (size_t)n_in, cudaMemcpyDeviceToDevice, s));
			CK(cudaMemsetAsync((char *)B.raw.p + rc_base + span, 0, 16, s));
			const int ctas = (n_in + kWarpsPerCtaPack - 1) / kWarpsPerCtaPack;
			k_revcomp_reads<<<ctas, 32 * kWarpsPerCtaPack, 0, s>>>((uint8_t *)B.raw.p, (const int64_t *)B.raw_off.p,
			                                                      (const int32_t *)B.ql.p, n_in);
			CK(cudaGetLastError());
		}
		CK(cudaMemcpyAsync(B.pk_off.p, h_pk_off, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
		CK(cudaMemcpyAsync(B.order_ql.p, h_order, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
	}
	return 0;
}

// Both strands: read i's result from its two strands (i and n_in + i). The smaller distance
// wins, the read itself on a tie; a strand that did not finish (a non-OK status) makes the read's
// status that status and its distance -1.
static void combine_strands(int32_t n_in, const int32_t *d2, const int32_t *s2, int32_t *dist, int32_t *status,
                            int32_t *strand)
{
	for (int32_t i = 0; i < n_in; ++i) {
		const int32_t df = d2[i], dr = d2[n_in + i], sf = s2[i], sr = s2[n_in + i];
		int32_t d = -1, st = GWF_OK, k = -1;
		if (sf != GWF_OK || sr != GWF_OK) st = sf != GWF_OK ? sf : sr;
		else if (df >= 0 && (dr < 0 || df <= dr)) d = df, k = 0;
		else if (dr >= 0) d = dr, k = 1;
		if (dist) dist[i] = d;
		if (status) status[i] = st;
		if (strand) strand[i] = k;
	}
}

static DevReads reads_view(const Batch &B)
{
	DevReads r;
	r.pk = (const uint64_t *)B.pk.p;
	r.pk_off = (const int64_t *)B.pk_off.p;
	r.raw = (const uint8_t *)B.raw.p;
	r.raw_off = (const int64_t *)B.raw_off.p;
	r.ql = (const int32_t *)B.ql.p;
	r.v0 = (const int32_t *)B.v0.p;
	r.pure = (const uint8_t *)B.pure.p;
	r.v1 = B.v1;
	r.n = B.n;
	return r;
}

static KParams base_params(Engine &E, const GraphDev &G, Batch &B, int32_t flags)
{
	KParams p;
	memset(&p, 0, sizeof p);
	p.g = G.view();
	p.r = reads_view(B);
	p.dens_milli = G.dens_milli;
	p.flags = flags;
	p.dist = (int32_t *)B.dist.p;
	p.status = (int32_t *)B.status.p;
	p.retry_list = (int32_t *)E.retry_list.p;
	p.retry_n = (int32_t *)E.retry_n.p;
	p.steps_out = (int32_t *)B.steps.p;
	p.w_out = nullptr;
	return p;
}

static const int kWarpsPerCta = 8;
static const int kMaxLevel = 3;

// Grid and arena of a persistent launch over n_order reads with arenas sized for ql_cap: as many
// warps as the grid holds (at most one per read), fewer when the arenas would not fit the budget.
struct PersistPlan {
	int ctas = 0;
	int64_t slot = 0;
};

static int plan_persistent(Engine &E, int32_t n_order, int32_t ql_cap, int32_t level, int ctas_per_sm,
                           int32_t dens_milli, PersistPlan *pl)
{
	const Caps c = caps_for(ql_cap, level, dens_milli);
	const int64_t slot = ws_layout(c).total;
	int64_t warps = (int64_t)E.sm_count * ctas_per_sm * kWarpsPerCta;
	const int64_t need_warps = (n_order + 0LL);
	if (warps > need_warps) warps = std::max<int64_t>(kWarpsPerCta, ((need_warps + kWarpsPerCta - 1) / kWarpsPerCta) * kWarpsPerCta);
	// keep arenas within a budget of the device memory: half the memory that was free when the
	// engine was created, or what the arena already holds if that is more
	const int64_t budget = std::max<int64_t>(E.mem_budget, (int64_t)E.ws.cap);
	while (warps > kWarpsPerCta && warps * slot > budget) warps -= kWarpsPerCta;
	if (warps * slot > budget) {
		gwf_set_errorf("arena of %lld bytes per warp does not fit the device", (long long)slot);
		return GWF_E_NOMEM;
	}
	int rc;
	if ((rc = E.ws.ensure((size_t)(warps * slot)))) return rc;
	if ((rc = E.head.ensure(16))) return rc;
	pl->ctas = (int)(warps / kWarpsPerCta);
	pl->slot = slot;
	return 0;
}

static int enqueue_persistent(Engine &E, KParams p, const PersistPlan &pl, const int32_t *d_order,
                              int32_t n_order, int32_t ql_cap, int32_t level)
{
	CK(cudaMemsetAsync(E.head.p, 0, 4, E.stream));
	p.order = d_order;
	p.n_order = n_order;
	p.head = (int32_t *)E.head.p;
	p.ws = (uint8_t *)E.ws.p;
	p.slot_bytes = pl.slot;
	p.level = level;
	p.ql_cap = ql_cap;
	if (p.max_lag > 0) k_align_persistent<true><<<pl.ctas, 32 * kWarpsPerCta, 0, E.stream>>>(p);
	else k_align_persistent<false><<<pl.ctas, 32 * kWarpsPerCta, 0, E.stream>>>(p);
	CK(cudaGetLastError());
	return 0;
}

// Persistent launch over the reads listed in d_order (device), arenas sized for ql_cap.
static int launch_persistent(Engine &E, KParams p, const int32_t *d_order, int32_t n_order,
                             int32_t ql_cap, int32_t level, int ctas_per_sm, int *launches)
{
	PersistPlan pl;
	int rc;
	if ((rc = plan_persistent(E, n_order, ql_cap, level, ctas_per_sm, p.dens_milli, &pl))) return rc;
	if ((rc = enqueue_persistent(E, p, pl, d_order, n_order, ql_cap, level))) return rc;
	++*launches;
	return 0;
}

// Plain launch: one warp per read in queue order, per-read arenas (split in chunks when the
// arenas of all reads do not fit).
static int launch_plain(Engine &E, KParams p, Batch &B, int *launches)
{
	const int64_t budget = std::max<int64_t>(E.mem_budget, (int64_t)E.ws.cap);
	int32_t start = 0;
	std::vector<int64_t> offs;
	while (start < B.n) {
		offs.clear();
		int64_t used = 0;
		int32_t end = start;
		while (end < B.n) {
			const int64_t sz = ws_layout(caps_for(B.h_ql[(size_t)end], 0, p.dens_milli)).total;
			if (used + sz > budget && end > start) break;
			offs.push_back(used);
			used += sz;
			++end;
		}
		int rc;
		if ((rc = E.ws.ensure((size_t)used))) return rc;
		if ((rc = E.slot_off.ensure(8 * offs.size()))) return rc;
		if ((rc = E.order.ensure(4 * (size_t)(end - start)))) return rc;
		std::vector<int32_t> ord((size_t)(end - start));
		std::iota(ord.begin(), ord.end(), start);
		CK(cudaMemcpyAsync(E.slot_off.p, offs.data(), 8 * offs.size(), cudaMemcpyHostToDevice, E.stream));
		CK(cudaMemcpyAsync(E.order.p, ord.data(), 4 * ord.size(), cudaMemcpyHostToDevice, E.stream));
		p.order = (const int32_t *)E.order.p;
		p.n_order = end - start;
		p.ws = (uint8_t *)E.ws.p;
		p.slot_off = (const int64_t *)E.slot_off.p;
		p.level = 0;
		const int ctas = (p.n_order + kWarpsPerCta - 1) / kWarpsPerCta;
		if (p.max_lag > 0) k_align_plain<true><<<ctas, 32 * kWarpsPerCta, 0, E.stream>>>(p);
		else k_align_plain<false><<<ctas, 32 * kWarpsPerCta, 0, E.stream>>>(p);
		CK(cudaGetLastError());
		++*launches;
		if (end < B.n) CK(cudaStreamSynchronize(E.stream)); // arenas are reused by the next chunk
		start = end;
	}
	return 0;
}

static int enqueue_pack(Engine &E, Batch &B)
{
	const int ctas = (B.n + kWarpsPerCta - 1) / kWarpsPerCta;
	k_pack_reads<<<ctas, 32 * kWarpsPerCta, 0, E.stream>>>(
	    (const uint8_t *)B.raw.p, (const int64_t *)B.raw_off.p, (const int32_t *)B.ql.p,
	    (const int64_t *)B.pk_off.p, (uint64_t *)B.pk.p, (uint8_t *)B.pure.p, B.n);
	CK(cudaGetLastError());
	return 0;
}

// ---- read classes: reads aligned by groups of 2, 4 or 8 warps
//
// Each read gets a number of warps: the caller's forced value, the tuned value of its length
// bucket (GWF_MODE_AUTO), or by default its share of the batch's work. The default takes a read's
// cost as ql^2 (the wavefront work grows with the length times the score, and the score with the
// length) and the warp slots of the persistent grid as the workers: a read that costs more than
// an even share of the batch per warp slot would finish after the rest, so it gets up to 8 warps,
// as many as its cost is shares (rounded up to a power of two); a read whose arena would make the
// live arenas too large gets more warps too (arena_nw). A batch that fills the device with
// reads of similar cost keeps one warp per read, the most efficient; a small batch or the longest
// reads of a mixed one get groups, which finish each read sooner. The reads of one count form a
// class; classes run longest reads first (8, 4, 2, then 1 warp per read), each class's queue
// ordered longest read first. One launch of k_align_classes runs all classes.
static const int32_t kClassNw[4] = {8, 4, 2, 1};

static int32_t share_nw(double cost, double share)
{
	if (!(cost > share)) return 1;
	const double r = cost / share;
	return r > 4 ? 8 : r > 2 ? 4 : 2;
}

// Live arenas: the persistent kernel slows down sharply once the arenas of all its warp slots
// together pass ~16 GiB (long reads on dense graphs, whose arrival sets are tens of MB per read,
// accessed at random): 6,000 reads of 0.5-20 kbp on the 5 Mbp graph align at 1,368 reads/s with
// one warp per read (120 GB of arenas, cut to the memory budget) and 3,161 with eight. A read
// whose one-warp arenas over every slot would pass that gets enough warps per read to stay below.
// The rule applies to batches of fewer than kArenaRuleReadsPerSlot reads per warp slot, where the
// longest reads set the batch's end; with more, the queue keeps every warp busy and one warp per
// read is the faster shape (20,000 reads of 10 kbp on the 5 Mbp graph, 4.2 per slot: 8,046 reads/s
// with one warp per read against 6,858 with the four that the rule gave them).
static const double kLiveArenaBytes = 16.0 * (1LL << 30);
static const double kArenaRuleReadsPerSlot = 3.0;

static int32_t arena_nw(int32_t ql, int32_t dens_milli, int64_t slots)
{
	const double bytes = (double)ws_layout(caps_for(ql, 0, dens_milli)).total * (double)slots;
	return bytes <= kLiveArenaBytes ? 1 : bytes <= 2 * kLiveArenaBytes ? 2 : bytes <= 4 * kLiveArenaBytes ? 4 : 8;
}

// The shortest read lengths (up to max_ql + 1) from which arena_nw gives 2, 4 and 8 warps: the
// arena grows with the length, so a binary search per level replaces a layout per read.
static void arena_nw_lengths(int32_t max_ql, int32_t dens_milli, int64_t slots, int32_t from[3])
{
	for (int lv = 0; lv < 3; ++lv) {
		const int32_t want = 2 << lv;
		int32_t lo = 1, hi = max_ql + 1; // first length in [lo, hi] with arena_nw >= want
		while (lo < hi) {
			const int32_t mid = lo + (hi - lo) / 2;
			if (arena_nw(mid, dens_milli, slots) >= want) hi = mid;
			else lo = mid + 1;
		}
		from[lv] = lo;
	}
}

// Class layout of the batch for the per-bucket warp counts nw_b (0 = by the read's share of the
// batch's work over `slots` warp slots); uploads the class queues when the layout changed.
static int plan_classes(Engine &E, Batch &B, const int32_t *nw_b, int64_t slots, int32_t dens_milli)
{
	// the layout depends on the batch contents (generation), the warp slots, the graph density
	// and the bucket counts
	uint64_t key = (uint64_t)(uint32_t)slots << 20 | (uint64_t)(uint32_t)dens_milli << 40;
	for (int b = 0; b < GWF_TUNE_NBUCKETS; ++b) key |= (uint64_t)(nw_b[b] & 15) << (4 * b);
	if (key == B.cls_key && B.cls_gen == B.generation) return 0;
	double total = 0;
	for (int32_t i = 0; i < B.n; ++i) total += (double)B.h_ql[(size_t)i] * (double)B.h_ql[(size_t)i];
	const double share = total / (double)std::max<int64_t>(1, slots);
	int32_t from[3] = {INT32_MAX, INT32_MAX, INT32_MAX}; // lengths from which the arena rule gives 2, 4, 8
	if ((double)B.n < kArenaRuleReadsPerSlot * (double)std::max<int64_t>(1, slots))
		arena_nw_lengths(B.max_ql, dens_milli, slots, from);
	int32_t cnt[4] = {0, 0, 0, 0}, cap[4] = {0, 0, 0, 0};
	std::vector<uint8_t> cls((size_t)B.n);
	for (int32_t i = 0; i < B.n; ++i) {
		const int32_t q = B.h_ql[(size_t)i];
		int32_t nw = nw_b[gwf_tune_bucket(q)];
		if (nw <= 0)
			nw = std::max(share_nw((double)q * (double)q, share), q >= from[2] ? 8 : q >= from[1] ? 4 : q >= from[0] ? 2 : 1);
		int k = 3;
		for (int j = 0; j < 4; ++j)
			if (kClassNw[j] == nw) k = j;
		cls[(size_t)i] = (uint8_t)k, ++cnt[k], cap[k] = std::max(cap[k], q);
	}
	// each class longest read first: counting sort over 64-base length buckets
	std::vector<int32_t> order((size_t)B.n);
	int32_t start[4], pos = 0;
	for (int k = 0; k < 4; ++k) start[k] = pos, pos += cnt[k];
	const int32_t nb = (B.max_ql >> 6) + 1;
	std::vector<int32_t> c2((size_t)(4 * nb + 1), 0);
	for (int32_t i = 0; i < B.n; ++i)
		c2[(size_t)(cls[(size_t)i] * nb + (nb - 1 - (B.h_ql[(size_t)i] >> 6))) + 1]++;
	for (size_t b = 0; b + 1 < c2.size(); ++b) c2[b + 1] += c2[b];
	for (int32_t i = 0; i < B.n; ++i)
		order[(size_t)c2[(size_t)(cls[(size_t)i] * nb + (nb - 1 - (B.h_ql[(size_t)i] >> 6)))]++] = i;
	B.cls_n = 0;
	for (int k = 0; k < 4; ++k)
		if (cnt[k] > 0) {
			const int j = B.cls_n++;
			B.cls_nw[j] = kClassNw[k], B.cls_cnt[j] = cnt[k], B.cls_cap[j] = cap[k], B.cls_start[j] = start[k];
		}
	B.cls_key = key, B.cls_gen = B.generation;
	if (B.cls_n == 1 && B.cls_nw[0] == 1) return 0; // one warp per read: the plain persistent queue
	int rc;
	if ((rc = B.order_cls.ensure(4 * (size_t)B.n + 4))) return rc;
	CK(cudaMemcpyAsync(B.order_cls.p, order.data(), 4 * (size_t)B.n, cudaMemcpyHostToDevice, E.stream));
	CK(cudaStreamSynchronize(E.stream)); // the host order vector goes out of scope
	return 0;
}

// Grid and arena of a class launch: a CTA holds, for the class that needs most, 8 / nw group
// arenas sized for the class's longest read; as many CTAs as the budget and the reads allow.
struct ClassLaunch {
	ClassParams cp;
	int ctas = 0;
};

static int plan_class_launch(Engine &E, const Batch &B, int ctas_per_sm, int32_t dens_milli, ClassLaunch *cl)
{
	ClassParams &cp = cl->cp;
	memset(&cp, 0, sizeof cp);
	int64_t need_ctas = 0;
	cp.cta_bytes = 0;
	for (int j = 0; j < B.cls_n; ++j) {
		const int groups = 8 / B.cls_nw[j];
		cp.order[j] = (const int32_t *)B.order_cls.p + B.cls_start[j];
		cp.n[j] = B.cls_cnt[j], cp.nw[j] = B.cls_nw[j], cp.ql_cap[j] = B.cls_cap[j];
		cp.slot[j] = ws_layout(caps_for(B.cls_cap[j], 0, dens_milli)).total;
		cp.cta_bytes = std::max<int64_t>(cp.cta_bytes, groups * cp.slot[j]);
		need_ctas = std::max<int64_t>(need_ctas, ((int64_t)B.cls_cnt[j] + groups - 1) / groups);
	}
	cp.n_cls = B.cls_n;
	int64_t ctas = std::min<int64_t>((int64_t)E.sm_count * ctas_per_sm, std::max<int64_t>(1, need_ctas));
	const int64_t budget = std::max<int64_t>(E.mem_budget, (int64_t)E.ws.cap);
	while (ctas > 1 && ctas * cp.cta_bytes > budget) --ctas;
	if (ctas * cp.cta_bytes > budget) {
		gwf_set_errorf("arena of %lld bytes per CTA does not fit the device", (long long)cp.cta_bytes);
		return GWF_E_NOMEM;
	}
	int rc;
	if ((rc = E.ws.ensure((size_t)(ctas * cp.cta_bytes)))) return rc;
	if ((rc = E.head.ensure(16))) return rc;
	cp.head = (int32_t *)E.head.p;
	cl->ctas = (int)ctas;
	return 0;
}

static int enqueue_classes(Engine &E, KParams p, const ClassLaunch &cl)
{
	CK(cudaMemsetAsync(E.head.p, 0, 16, E.stream));
	p.ws = (uint8_t *)E.ws.p;
	p.level = 0;
	k_align_classes<<<cl.ctas, 32 * kWarpsPerCta, 0, E.stream>>>(p, cl.cp);
	CK(cudaGetLastError());
	return 0;
}

// Level-0 sequence of the persistent form as one CUDA graph: pack, clear the overflow count,
// persistent kernel, copy the overflow count to the host. Captured once per batch contents and
// launch shape, replayed on every run.
static int launch_level0_graph(Engine &E, Batch &B, const KParams &p, int ctas_per_sm, bool classes)
{
	PersistPlan pl;
	ClassLaunch cl;
	int rc;
	if (classes) {
		if ((rc = plan_class_launch(E, B, ctas_per_sm, p.dens_milli, &cl))) return rc;
		pl.ctas = cl.ctas, pl.slot = cl.cp.cta_bytes;
	} else if ((rc = plan_persistent(E, B.n, B.max_ql, 0, ctas_per_sm, p.dens_milli, &pl)))
		return rc;
	const uint64_t key[9] = {B.generation, (uint64_t)(uintptr_t)E.ws.p, (uint64_t)pl.slot, (uint64_t)pl.ctas,
	                         (uint64_t)(uint32_t)p.flags | (uint64_t)(uint32_t)p.max_lag << 32,
	                         (uint64_t)(uintptr_t)E.retry_n.p,
	                         (uint64_t)(uintptr_t)E.h_small.p, (uint64_t)(uintptr_t)E.retry_list.p,
	                         classes ? B.cls_key ^ B.cls_gen << 40 : ~0ULL};
	if (!B.gexec || memcmp(key, B.gkey, sizeof key) != 0) {
		if (B.gexec) cudaGraphExecDestroy(B.gexec), B.gexec = nullptr;
		CK(cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeThreadLocal));
		int erc = enqueue_pack(E, B);
		if (!erc && cudaMemsetAsync(E.retry_n.p, 0, 4, E.stream) != cudaSuccess) erc = GWF_E_CUDA;
		if (!erc) erc = classes ? enqueue_classes(E, p, cl)
		                        : enqueue_persistent(E, p, pl, (const int32_t *)B.order_ql.p, B.n, B.max_ql, 0);
		if (!erc && cudaMemcpyAsync(E.h_small.p, E.retry_n.p, 4, cudaMemcpyDeviceToHost, E.stream) != cudaSuccess)
			erc = GWF_E_CUDA;
		cudaGraph_t graph = nullptr;
		const cudaError_t ce = cudaStreamEndCapture(E.stream, &graph);
		if (erc || ce != cudaSuccess) {
			if (graph) cudaGraphDestroy(graph);
			cudaGetLastError();
			gwf_set_error("capturing the batch launch sequence failed");
			return erc ? erc : GWF_E_CUDA;
		}
		const cudaError_t ie = cudaGraphInstantiate(&B.gexec, graph, 0);
		cudaGraphDestroy(graph);
		if (ie != cudaSuccess) {
			B.gexec = nullptr;
			cudaGetLastError();
			gwf_set_errorf("instantiating the batch graph failed: %s", cudaGetErrorString(ie));
			return GWF_E_CUDA;
		}
		memcpy(B.gkey, key, sizeof key);
	}
	CK(cudaGraphLaunch(B.gexec, E.stream));
	return 0;
}

int gwf_batch_exec(Engine &E, const GraphDev &G, Batch &B, int32_t mode, int32_t flags,
                   int ctas_per_sm, float *ms, int *launches_out, int use_graph, int32_t max_lag,
                   int32_t warps_per_read)
{
	int launches = 0, rc;
	if (B.n == 0) {
		if (ms) *ms = 0;
		if (launches_out) *launches_out = 0;
		return 0;
	}
	if ((rc = E.retry_list.ensure(4 * (size_t)B.n + 4)) || (rc = E.retry_n.ensure(16)) ||
	    (rc = E.h_small.ensure(4 * (size_t)B.n + 64)))
		return rc;
	KParams p = base_params(E, G, B, flags);
	p.max_lag = max_lag > 0 ? max_lag : 0;
	// warps per read of each length bucket (persistent form): forced, tuned (GWF_MODE_AUTO), or
	// 0: by the read's share of the batch's work (plan_classes)
	int32_t nw_b[GWF_TUNE_NBUCKETS];
	for (int b = 0; b < GWF_TUNE_NBUCKETS; ++b) {
		int32_t nw = warps_per_read > 0 ? warps_per_read : 0;
		if (!nw && mode == GWF_MODE_AUTO) nw = gwf_tune_lookup_nw(E.device, b);
		nw_b[b] = nw;
	}
	if (mode == GWF_MODE_AUTO && ctas_per_sm <= 0) { // autotuned shape for the dominant length bucket
		int32_t f = 0, c = 0;
		if (gwf_tune_lookup(E.device, B.dom_bucket, &f, &c)) mode = f, ctas_per_sm = c;
	}
	bool classes = false;
	if (mode != GWF_MODE_PLAIN) {
		const int64_t slots = (int64_t)E.sm_count * E.persistent_ctas_per_sm * kWarpsPerCta;
		if ((rc = plan_classes(E, B, nw_b, slots, G.dens_milli))) return rc;
		classes = B.cls_n > 1 || B.cls_nw[0] > 1;
	}
	if (ctas_per_sm <= 0) ctas_per_sm = classes ? E.classes_ctas_per_sm : E.persistent_ctas_per_sm;
	bool count_copied = false;
	CK(cudaEventRecord(E.ev0, E.stream));
	if (use_graph && mode != GWF_MODE_PLAIN) {
		if ((rc = launch_level0_graph(E, B, p, ctas_per_sm, classes))) return rc;
		launches += 2;
		count_copied = true;
	} else {
		if ((rc = enqueue_pack(E, B))) return rc;
		++launches;
		CK(cudaMemsetAsync(E.retry_n.p, 0, 4, E.stream));
		if (mode == GWF_MODE_PLAIN) rc = launch_plain(E, p, B, &launches);
		else if (classes) {
			ClassLaunch cl;
			if (!(rc = plan_class_launch(E, B, ctas_per_sm, p.dens_milli, &cl)) && !(rc = enqueue_classes(E, p, cl)))
				++launches;
		} else
			rc = launch_persistent(E, p, (const int32_t *)B.order_ql.p, B.n, B.max_ql, 0, ctas_per_sm, &launches);
		if (rc) return rc;
	}
	// re-run arena overflows at larger size classes
	for (int level = 1; level <= kMaxLevel; ++level) {
		int32_t nr = 0;
		if (!count_copied) CK(cudaMemcpyAsync(E.h_small.p, E.retry_n.p, 4, cudaMemcpyDeviceToHost, E.stream));
		count_copied = false;
		CK(cudaStreamSynchronize(E.stream));
		nr = *(int32_t *)E.h_small.p;
		if (nr == 0) break;
		std::vector<int32_t> ids((size_t)nr);
		CK(cudaMemcpyAsync(E.h_small.p, E.retry_list.p, 4 * (size_t)nr, cudaMemcpyDeviceToHost, E.stream));
		CK(cudaStreamSynchronize(E.stream));
		memcpy(ids.data(), E.h_small.p, 4 * (size_t)nr);
		int32_t cap = 0;
		for (int32_t r : ids) cap = std::max(cap, B.h_ql[(size_t)r]);
		std::sort(ids.begin(), ids.end(), [&](int32_t x, int32_t y) { return B.h_ql[(size_t)x] > B.h_ql[(size_t)y]; });
		if ((rc = E.order.ensure(4 * (size_t)nr))) return rc;
		CK(cudaMemcpyAsync(E.order.p, ids.data(), 4 * (size_t)nr, cudaMemcpyHostToDevice, E.stream));
		CK(cudaMemsetAsync(E.retry_n.p, 0, 4, E.stream));
		KParams q = p;
		if (level == kMaxLevel) q.retry_list = nullptr; // last class: keep GWF_E_CAPACITY
		if ((rc = launch_persistent(E, q, (const int32_t *)E.order.p, nr, cap, level,
		                            std::min(ctas_per_sm, E.persistent_ctas_per_sm), &launches)))
			return rc;
	}
	CK(cudaEventRecord(E.ev1, E.stream));
	CK(cudaEventSynchronize(E.ev1));
	if (ms) CK(cudaEventElapsedTime(ms, E.ev0, E.ev1));
	if (launches_out) *launches_out = launches;
	return 0;
}

int gwf_batch_fetch(Engine &E, Batch &B, int32_t *dist, int32_t *status, int32_t *strand)
{
	if (B.n == 0) return 0;
	// through the pinned metadata buffer (its upload has completed: the stream is in order)
	int rc;
	if ((rc = B.h_meta.ensure(8 * (size_t)B.n + 64))) return rc;
	int32_t *hd = (int32_t *)B.h_meta.p, *hs = hd + B.n;
	if (dist || B.both) CK(cudaMemcpyAsync(hd, B.dist.p, 4 * (size_t)B.n, cudaMemcpyDeviceToHost, E.stream));
	if (status || B.both) CK(cudaMemcpyAsync(hs, B.status.p, 4 * (size_t)B.n, cudaMemcpyDeviceToHost, E.stream));
	CK(cudaStreamSynchronize(E.stream));
	if (B.both) {
		combine_strands(B.n_in, hd, hs, dist, status, strand);
		return 0;
	}
	if (dist) memcpy(dist, hd, 4 * (size_t)B.n);
	if (status) memcpy(status, hs, 4 * (size_t)B.n);
	if (strand)
		for (int32_t i = 0; i < B.n; ++i) strand[i] = hd[i] >= 0 ? 0 : -1;
	return 0;
}

// Launches the persistent kernel with parameters built by the caller (gwf_ed_batch_noalloc).
cudaError_t gwf_launch_persistent(const KParams &p, int ctas, int threads, cudaStream_t s)
{
	if (p.max_lag > 0) k_align_persistent<true><<<ctas, threads, 0, s>>>(p);
	else k_align_persistent<false><<<ctas, threads, 0, s>>>(p);
	return cudaGetLastError();
}

cudaError_t gwf_launch_serve(const SrvParams &p, int ctas, int threads, cudaStream_t s, int warps_per_read)
{
	switch (warps_per_read) {
	case 2: k_serve_grp<2><<<ctas, threads, 0, s>>>(p); break;
	case 4: k_serve_grp<4><<<ctas, threads, 0, s>>>(p); break;
	case 8: k_serve_grp<8><<<ctas, threads, 0, s>>>(p); break;
	default: k_serve<<<ctas, threads, 0, s>>>(p); break;
	}
	return cudaGetLastError();
}

int gwf_serve_ctas_per_sm(int warps_per_read)
{
	int occ = 0;
	cudaError_t e;
	switch (warps_per_read) {
	case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_serve_grp<2>, 256, 0); break;
	case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_serve_grp<4>, 256, 0); break;
	case 8: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_serve_grp<8>, 256, 0); break;
	default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_serve, 256, 0); break;
	}
	if (e != cudaSuccess) {
		cudaGetLastError();
		return 1;
	}
	return occ > 0 ? occ : 1;
}

// ------------------------------------------------------------------ public batch entry points
static std::mutex g_batch_mu; // batch calls are serialised (one engine per device)
std::mutex &gwf_batch_mutex() { return g_batch_mu; }
static std::unordered_map<int, Batch *> g_scratch_batches;

static int prepare(const gwf_graph_t *g, const gwf_batch_opts_t *opt, GraphDev **G, Engine **E)
{
	if (!g) {
		gwf_set_error("null graph");
		return GWF_E_BAD_INPUT;
	}
	*G = gwf_find_graph(g);
	if (!*G) {
		gwf_set_error("graph not indexed on a device: call gwf_ed_index first");
		return GWF_E_NOT_INDEXED;
	}
	if (opt && opt->warps_per_read != 0 && opt->warps_per_read != 1 && opt->warps_per_read != 2 &&
	    opt->warps_per_read != 4 && opt->warps_per_read != 8) {
		gwf_set_error("warps_per_read must be 0, 1, 2, 4 or 8");
		return GWF_E_BAD_INPUT;
	}
	int dev;
	int rc = gwf_select_device((*G)->device, &dev);
	if (rc) return rc;
	*E = gwf_engine(dev);
	return *E ? 0 : GWF_E_CUDA;
}

// strand output of the gwf_ed_batch_concat call in progress on this thread (gwf_ed_batch_strand)
static thread_local int32_t *t_strand_out = nullptr;

extern "C" int gwf_ed_batch_concat(const gwf_graph_t *g, int32_t n, const char *seqs,
                                   const int64_t *offs, const int32_t *ql, const int32_t *v0,
                                   int32_t v1, uint32_t max_lag, int32_t *dist, int32_t *status,
                                   const gwf_batch_opts_t *opt)
{
	// max_lag is ignored, as in the reference (gwf-ed.cu:1286-1287), unless GWF_F_MAX_LAG is set
	if (n < 0 || (n > 0 && (!seqs || !offs || !ql || !v0 || !dist))) {
		gwf_set_error("bad batch arguments");
		return GWF_E_BAD_INPUT;
	}
	GraphDev *G;
	Engine *E;
	int rc = prepare(g, opt, &G, &E);
	if (rc) return rc;
	if (v1 >= 0 && (uint32_t)v1 >= G->n_vtx) {
		gwf_set_error("v1 out of range");
		return GWF_E_BAD_INPUT;
	}
	std::lock_guard<std::mutex> lk(g_batch_mu);
	Batch *&B = g_scratch_batches[E->device];
	if (!B) B = new Batch;
	const int32_t flags = opt ? opt->flags : 0;
	if ((rc = gwf_batch_load(*E, *B, n, seqs, offs, ql, v0, v1, (flags & GWF_F_BOTH_STRANDS) != 0))) return rc;
	const int32_t mode = opt ? opt->mode : GWF_MODE_AUTO;
	const int32_t cps = opt ? opt->ctas_per_sm : 0;
	const int32_t lag = (flags & GWF_F_MAX_LAG) ? (int32_t)std::min<uint32_t>(max_lag, INT32_MAX) : 0;
	if ((rc = gwf_batch_exec(*E, *G, *B, mode, flags, cps, nullptr, nullptr, opt ? opt->use_graph : 0, lag,
	                         opt ? opt->warps_per_read : 0)))
		return rc;
	std::vector<int32_t> st;
	if (!status) st.resize((size_t)n), status = st.data();
	return gwf_batch_fetch(*E, *B, dist, status, t_strand_out);
}

extern "C" int gwf_ed_batch_strand(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs,
                                   const int32_t *ql, const int32_t *v0, int32_t v1, uint32_t max_lag,
                                   int32_t *dist, int32_t *status, int32_t *strand, const gwf_batch_opts_t *opt)
{
	if (n > 0 && !strand) {
		gwf_set_error("gwf_ed_batch_strand: null strand array");
		return GWF_E_BAD_INPUT;
	}
	gwf_batch_opts_t o;
	if (opt) o = *opt;
	else memset(&o, 0, sizeof o);
	o.flags |= GWF_F_BOTH_STRANDS;
	t_strand_out = strand;
	const int rc = gwf_ed_batch_concat(g, n, seqs, offs, ql, v0, v1, max_lag, dist, status, &o);
	t_strand_out = nullptr;
	return rc;
}

extern "C" int gwf_ed_batch(const gwf_graph_t *g, int32_t n, const char *const *q, const int32_t *ql,
                            const int32_t *v0, int32_t v1, uint32_t max_lag, int32_t *dist,
                            int32_t *status, const gwf_batch_opts_t *opt)
{
	if (n < 0 || (n > 0 && (!q || !ql || !v0 || !dist))) {
		gwf_set_error("bad batch arguments");
		return GWF_E_BAD_INPUT;
	}
	std::vector<int64_t> offs((size_t)n);
	int64_t tot = 0;
	for (int32_t i = 0; i < n; ++i) {
		if (ql[i] < 0 || (ql[i] > 0 && !q[i])) {
			gwf_set_error("bad read");
			return GWF_E_BAD_INPUT;
		}
		offs[(size_t)i] = tot, tot += ql[i];
	}
	std::vector<char> cat((size_t)tot + 1);
	for (int32_t i = 0; i < n; ++i) memcpy(cat.data() + offs[(size_t)i], q[i], (size_t)ql[i]);
	return gwf_ed_batch_concat(g, n, cat.data(), offs.data(), ql, v0, v1, max_lag, dist, status, opt);
}

extern "C" int32_t gwf_ed(void *km, const gwf_graph_t *g, int32_t ql, const char *q, int32_t v0,
                          int32_t v1, uint32_t max_lag, int32_t traceback)
{
	(void)km; // kalloc.c is empty in the reference
	if (traceback != 0) {
		gwf_set_error("traceback is not implemented by the reference path");
		return GWF_E_UNSUPPORTED;
	}
	if (!g || !q || ql <= 0) {
		gwf_set_error("gwf_ed: empty or null query");
		return GWF_E_BAD_INPUT;
	}
	if (v0 < 0 || (uint32_t)v0 >= g->n_vtx || (v1 >= 0 && (uint32_t)v1 >= g->n_vtx)) {
		gwf_set_error("gwf_ed: v0/v1 out of range");
		return GWF_E_BAD_INPUT;
	}
	int64_t off = 0;
	int32_t dist = -1, status = 0;
	gwf_batch_opts_t opt;
	memset(&opt, 0, sizeof opt);
	opt.mode = GWF_MODE_PERSISTENT;
	int rc = gwf_ed_batch_concat(g, 1, q, &off, &ql, &v0, v1, max_lag, &dist, &status, &opt);
	if (rc) return rc;
	if (status != GWF_OK) return status;
	return dist;
}

// ------------------------------------------------------------------ traceback batches
struct TraceBufs { // per-device path and CIGAR outputs of gwf_ed_batch_align
	DBuf end_off, path_n, path_v, path_arc, cigar_n, cigar, order, slot_off;
};
static std::unordered_map<int, TraceBufs *> g_trace_bufs;

// Traceback launches over the reads in ids at one arena class: one warp per read with the plain
// form's per-read arenas (the trace arrays after the alignment arrays), in chunks that fit the
// budget.
static int launch_trace(Engine &E, KParams p, Batch &B, const std::vector<int32_t> &ids, int level, int *launches)
{
	const int64_t budget = std::max<int64_t>(E.mem_budget, (int64_t)E.ws.cap);
	size_t start = 0;
	std::vector<int64_t> offs;
	while (start < ids.size()) {
		offs.clear();
		int64_t used = 0;
		size_t end = start;
		while (end < ids.size()) {
			const Caps c = caps_for(B.h_ql[(size_t)ids[end]], level, p.dens_milli);
			const int64_t sz = tr_layout(c, ws_layout(c).total).total;
			if (used + sz > budget && end > start) break;
			offs.push_back(used);
			used += sz;
			++end;
		}
		int rc;
		if ((rc = E.ws.ensure((size_t)used))) return rc;
		if ((rc = E.slot_off.ensure(8 * offs.size()))) return rc;
		if ((rc = E.order.ensure(4 * (end - start)))) return rc;
		CK(cudaMemcpyAsync(E.slot_off.p, offs.data(), 8 * offs.size(), cudaMemcpyHostToDevice, E.stream));
		CK(cudaMemcpyAsync(E.order.p, ids.data() + start, 4 * (end - start), cudaMemcpyHostToDevice, E.stream));
		p.order = (const int32_t *)E.order.p;
		p.n_order = (int32_t)(end - start);
		p.ws = (uint8_t *)E.ws.p;
		p.slot_off = (const int64_t *)E.slot_off.p;
		p.level = level;
		const int ctas = (p.n_order + kWarpsPerCta - 1) / kWarpsPerCta;
		k_align_trace<<<ctas, 32 * kWarpsPerCta, 0, E.stream>>>(p);
		CK(cudaGetLastError());
		++*launches;
		// arenas, offsets and order are reused by the next chunk (the copies above are from
		// pageable memory, staged before they return)
		CK(cudaStreamSynchronize(E.stream));
		start = end;
	}
	return 0;
}

// CIGAR launches over the reads whose path is complete: one warp per read, arenas sized from the
// read's length and distance, in chunks that fit the budget. Reads whose wavefront table alone
// would pass the budget (or 2 GiB) get cigar_n = -1.
static int launch_cigar(Engine &E, const GraphDev &G, Batch &B, TraceBufs &T, const int32_t *h_dist,
                        const int32_t *h_status, const int32_t *h_path_n, int32_t max_nv, int32_t max_ops,
                        int *launches)
{
	const int64_t budget = std::max<int64_t>(E.mem_budget, (int64_t)E.ws.cap);
	const int64_t per_read_cap = std::min<int64_t>(budget, 2LL << 30);
	std::vector<int32_t> ids;
	for (int32_t r = 0; r < B.n; ++r) {
		const bool want = h_status[r] == GWF_OK && h_dist[r] >= 0 && h_path_n[r] >= 1 && h_path_n[r] <= max_nv;
		if (want && cigar_arena_bytes(B.h_ql[(size_t)r], h_dist[r]) <= per_read_cap) ids.push_back(r);
	}
	CK(cudaMemsetAsync(T.cigar_n.p, 0xff, 4 * (size_t)B.n, E.stream)); // -1 for the reads left out
	CigarParams p;
	memset(&p, 0, sizeof p);
	p.g = G.view();
	p.r = reads_view(B);
	p.max_nv = max_nv, p.max_ops = max_ops;
	p.dist = (const int32_t *)B.dist.p;
	p.status = (const int32_t *)B.status.p;
	p.end_off = (const int32_t *)T.end_off.p;
	p.path_n = (const int32_t *)T.path_n.p;
	p.path_v = (const int32_t *)T.path_v.p;
	p.path_arc = (const int32_t *)T.path_arc.p;
	p.cigar_n = (int32_t *)T.cigar_n.p;
	p.cigar = (uint32_t *)T.cigar.p;
	size_t start = 0;
	std::vector<int64_t> offs;
	while (start < ids.size()) {
		offs.clear();
		int64_t used = 0;
		size_t end = start;
		while (end < ids.size()) {
			const int64_t sz = cigar_arena_bytes(B.h_ql[(size_t)ids[end]], h_dist[ids[end]]);
			if (used + sz > budget && end > start) break;
			offs.push_back(used);
			used += sz;
			++end;
		}
		int rc;
		if ((rc = E.ws.ensure((size_t)std::max<int64_t>(used, 16)))) return rc;
		if ((rc = T.slot_off.ensure(8 * offs.size()))) return rc;
		if ((rc = T.order.ensure(4 * (end - start)))) return rc;
		CK(cudaMemcpyAsync(T.slot_off.p, offs.data(), 8 * offs.size(), cudaMemcpyHostToDevice, E.stream));
		CK(cudaMemcpyAsync(T.order.p, ids.data() + start, 4 * (end - start), cudaMemcpyHostToDevice, E.stream));
		p.order = (const int32_t *)T.order.p;
		p.n_order = (int32_t)(end - start);
		p.ws = (uint8_t *)E.ws.p;
		p.slot_off = (const int64_t *)T.slot_off.p;
		const int ctas = (p.n_order + kWarpsPerCta - 1) / kWarpsPerCta;
		k_cigar<<<ctas, 32 * kWarpsPerCta, 0, E.stream>>>(p);
		CK(cudaGetLastError());
		++*launches;
		CK(cudaStreamSynchronize(E.stream)); // arenas and offsets are reused by the next chunk
		start = end;
	}
	// the memset above is on a non-blocking stream: done before the caller copies cigar_n back,
	// also when no read was launched
	CK(cudaStreamSynchronize(E.stream));
	return 0;
}

extern "C" int gwf_ed_batch_align(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs,
                                  const int32_t *ql, const int32_t *v0, int32_t v1, int32_t flags,
                                  int32_t max_nv, int32_t max_ops, int32_t *dist, int32_t *status,
                                  int32_t *end_off, int32_t *path_n, int32_t *path_v, int32_t *path_arc,
                                  int32_t *cigar_n, uint32_t *cigar)
{
	if (flags & GWF_F_BOTH_STRANDS) {
		gwf_set_error("traceback of both strands is not supported: align the reverse complement as its own read");
		return GWF_E_UNSUPPORTED;
	}
	if (n < 0 || max_nv < 0 || max_ops < 0 ||
	    (n > 0 && (!seqs || !offs || !ql || !v0 || !dist || !status || !end_off || !path_n ||
	               (max_nv > 0 && (!path_v || !path_arc)) || (max_ops > 0 && (!cigar_n || !cigar))))) {
		gwf_set_error("bad batch arguments");
		return GWF_E_BAD_INPUT;
	}
	GraphDev *G;
	Engine *E;
	int rc = prepare(g, nullptr, &G, &E);
	if (rc) return rc;
	if (v1 >= 0 && (uint32_t)v1 >= G->n_vtx) {
		gwf_set_error("v1 out of range");
		return GWF_E_BAD_INPUT;
	}
	if (n == 0) return 0;
	std::lock_guard<std::mutex> lk(g_batch_mu);
	Batch *&B = g_scratch_batches[E->device];
	if (!B) B = new Batch;
	TraceBufs *&T = g_trace_bufs[E->device];
	if (!T) T = new TraceBufs;
	const size_t cells = (size_t)n * (size_t)std::max(max_nv, 1);
	const size_t ops = (size_t)n * (size_t)std::max(max_ops, 1);
	if ((rc = gwf_batch_load(*E, *B, n, seqs, offs, ql, v0, v1))) return rc;
	if ((rc = T->end_off.ensure(4 * (size_t)n)) || (rc = T->path_n.ensure(4 * (size_t)n)) ||
	    (rc = T->path_v.ensure(4 * cells)) || (rc = T->path_arc.ensure(4 * cells)) ||
	    (max_ops > 0 && ((rc = T->cigar_n.ensure(4 * (size_t)n)) || (rc = T->cigar.ensure(4 * ops)))) ||
	    (rc = E->retry_list.ensure(4 * (size_t)n + 4)) || (rc = E->retry_n.ensure(16)) ||
	    (rc = E->h_small.ensure(4 * (size_t)n + 64)))
		return rc;
	KParams p = base_params(*E, *G, *B, flags);
	p.end_off = (int32_t *)T->end_off.p;
	p.path_n = (int32_t *)T->path_n.p;
	p.path_v = (int32_t *)T->path_v.p;
	p.path_arc = (int32_t *)T->path_arc.p;
	p.max_nv = max_nv;
	int launches = 0;
	if ((rc = enqueue_pack(*E, *B))) return rc;
	std::vector<int32_t> ids((size_t)n);
	std::iota(ids.begin(), ids.end(), 0);
	for (int level = 0; level <= kMaxLevel && !ids.empty(); ++level) {
		CK(cudaMemsetAsync(E->retry_n.p, 0, 4, E->stream));
		KParams q = p;
		if (level == kMaxLevel) q.retry_list = nullptr; // last class: keep GWF_E_CAPACITY
		if ((rc = launch_trace(*E, q, *B, ids, level, &launches))) return rc;
		CK(cudaMemcpyAsync(E->h_small.p, E->retry_n.p, 4, cudaMemcpyDeviceToHost, E->stream));
		CK(cudaStreamSynchronize(E->stream));
		const int32_t nr = level == kMaxLevel ? 0 : *(int32_t *)E->h_small.p;
		ids.resize((size_t)nr);
		if (nr == 0) break;
		CK(cudaMemcpyAsync(E->h_small.p, E->retry_list.p, 4 * (size_t)nr, cudaMemcpyDeviceToHost, E->stream));
		CK(cudaStreamSynchronize(E->stream));
		memcpy(ids.data(), E->h_small.p, 4 * (size_t)nr);
		std::sort(ids.begin(), ids.end());
	}
	if ((rc = gwf_batch_fetch(*E, *B, dist, status))) return rc;
	CK(cudaMemcpy(end_off, T->end_off.p, 4 * (size_t)n, cudaMemcpyDeviceToHost));
	CK(cudaMemcpy(path_n, T->path_n.p, 4 * (size_t)n, cudaMemcpyDeviceToHost));
	if (max_nv > 0) {
		CK(cudaMemcpy(path_v, T->path_v.p, 4 * cells, cudaMemcpyDeviceToHost));
		CK(cudaMemcpy(path_arc, T->path_arc.p, 4 * cells, cudaMemcpyDeviceToHost));
	}
	if (max_ops > 0) {
		if ((rc = launch_cigar(*E, *G, *B, *T, dist, status, path_n, max_nv, max_ops, &launches))) return rc;
		CK(cudaMemcpy(cigar_n, T->cigar_n.p, 4 * (size_t)n, cudaMemcpyDeviceToHost));
		CK(cudaMemcpy(cigar, T->cigar.p, 4 * ops, cudaMemcpyDeviceToHost));
	}
	return 0;
}

extern "C" int gwf_ed_batch_path(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs,
                                 const int32_t *ql, const int32_t *v0, int32_t v1, int32_t flags,
                                 int32_t max_nv, int32_t *dist, int32_t *status, int32_t *end_off,
                                 int32_t *path_n, int32_t *path_v, int32_t *path_arc)
{
	return gwf_ed_batch_align(g, n, seqs, offs, ql, v0, v1, flags, max_nv, 0, dist, status, end_off, path_n,
	                          path_v, path_arc, nullptr, nullptr);
}

// ------------------------------------------------------------------ resident batches
struct gwf_batch_s {
	const gwf_graph_t *g;
	Batch B;
	int launches = 0;
};

extern "C" gwf_batch_t *gwf_batch_create(const gwf_graph_t *g, int32_t n, const char *seqs,
                                         const int64_t *offs, const int32_t *ql, const int32_t *v0,
                                         int32_t v1, const gwf_batch_opts_t *opt)
{
	GraphDev *G;
	Engine *E;
	if (prepare(g, opt, &G, &E)) return nullptr;
	if (n < 0 || (n > 0 && (!seqs || !offs || !ql || !v0))) {
		gwf_set_error("bad batch arguments");
		return nullptr;
	}
	gwf_batch_s *b = new gwf_batch_s;
	b->g = g;
	std::lock_guard<std::mutex> lk(g_batch_mu);
	const bool both = opt && (opt->flags & GWF_F_BOTH_STRANDS);
	if (gwf_batch_load(*E, b->B, n, seqs, offs, ql, v0, v1, both) || cudaStreamSynchronize(E->stream) != cudaSuccess) {
		b->B.release();
		delete b;
		return nullptr;
	}
	return b;
}

extern "C" int gwf_batch_run(gwf_batch_t *b, const gwf_batch_opts_t *opt, float *kernel_ms)
{
	if (!b) return GWF_E_BAD_INPUT;
	GraphDev *G;
	Engine *E;
	int rc = prepare(b->g, opt, &G, &E);
	if (rc) return rc;
	std::lock_guard<std::mutex> lk(g_batch_mu);
	return gwf_batch_exec(*E, *G, b->B, opt ? opt->mode : GWF_MODE_AUTO, opt ? opt->flags : 0,
	                      opt ? opt->ctas_per_sm : 0, kernel_ms, &b->launches, opt ? opt->use_graph : 0, 0,
	                      opt ? opt->warps_per_read : 0);
}

extern "C" int gwf_batch_results(gwf_batch_t *b, int32_t *dist, int32_t *status)
{
	if (!b) return GWF_E_BAD_INPUT;
	GraphDev *G;
	Engine *E;
	int rc = prepare(b->g, nullptr, &G, &E);
	if (rc) return rc;
	std::lock_guard<std::mutex> lk(g_batch_mu);
	return gwf_batch_fetch(*E, b->B, dist, status);
}

extern "C" int32_t gwf_batch_launches(const gwf_batch_t *b) { return b ? b->launches : 0; }

extern "C" int gwf_batch_steps(gwf_batch_t *b, int32_t *steps)
{
	if (!b || !steps) return GWF_E_BAD_INPUT;
	GraphDev *G;
	Engine *E;
	int rc = prepare(b->g, nullptr, &G, &E);
	if (rc) return rc;
	std::lock_guard<std::mutex> lk(g_batch_mu);
	if (b->B.n == 0) return 0;
	// with both strands: the read's own strand (the first n_in entries)
	CK(cudaMemcpyAsync(steps, b->B.steps.p, 4 * (size_t)b->B.n_in, cudaMemcpyDeviceToHost, E->stream));
	CK(cudaStreamSynchronize(E->stream));
	return 0;
}

extern "C" void gwf_batch_destroy(gwf_batch_t *b)
{
	if (!b) return;
	b->B.release();
	delete b;
}

extern "C" void *gwf_pinned_alloc(int64_t bytes)
{
	void *p = nullptr;
	if (bytes <= 0 || cudaMallocHost(&p, (size_t)bytes) != cudaSuccess) {
		cudaGetLastError();
		gwf_set_error("pinned allocation failed");
		return nullptr;
	}
	return p;
}

extern "C" void gwf_pinned_free(void *p)
{
	if (p) cudaFreeHost(p);
}
