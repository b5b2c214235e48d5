// ref_harness.cu — TEST INFRASTRUCTURE ONLY. Runs the reference's own device routine gwf_ed
// (gwf-ed.cu:1292, compiled from the reference sources by oracle/Makefile) on reads that each
// carry their own start vertex v0. The reference driver's kernel hard-codes v0 = 0
// (main.cu:217); everything else follows the reference driver:
//   graph     gfa_read + gwf_gfa2gwf(first segment) + gwf_ed_index  (main.cu:396-415)
//   device    deep copy of the graph                                 (main.cu:415-452)
//   arenas    per-read caps and byte sizes                           (main.cu:498-517)
//   carve     pointer order inside one read's arena                  (main.cu:179-214)
//   streams   16 streams, 90% of free memory, greedy packing,
//             memset + copies + launch + result copy per launch      (main.cu:539-735)
// Usage: gwf-ref-harness <graph.gfa> <reads.fa> <v0.txt|-> [n_streams]
// stdout: one distance per read; stderr: one JSON line with the timing.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <string>
#include <vector>

#include "gfa-priv.h"
#include "gfa.h"
#include "gwfa.h"

gwf_graph_t *gwf_gfa2gwf(const gfa_t *gfa, uint32_t v0); // main.cu:294 (C++ linkage)

#define CK(x)                                                                                  \
	do {                                                                                       \
		cudaError_t e_ = (x);                                                                  \
		if (e_ != cudaSuccess) {                                                               \
			fprintf(stderr, "%s: %s (%s:%d)\n", #x, cudaGetErrorString(e_), __FILE__, __LINE__); \
			exit(2);                                                                           \
		}                                                                                      \
	} while (0)

static double now_s()
{
	timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + ts.tv_nsec * 1e-9;
}

__launch_bounds__(32, 1) __global__ void harness_kernel(char *arena, const size_t *arena_off,
                                                        const gwf_edbuf_t *bufs, const char *seqs,
                                                        const size_t *seq_off, const int32_t *qlen,
                                                        const int32_t *v0, const gwf_graph_t *g,
                                                        int32_t *scores, int n)
{
	__shared__ uint64_t diag_shared[64];
	const int r = blockIdx.x;
	if (r >= n) return;
	gwf_edbuf_t b = bufs[r];
	char *p = arena + arena_off[r];
	b.a_buf.vd = (uint64_t *)p, p += b.max_a * sizeof(uint64_t);
	b.a_buf.k = (int32_t *)p, p += b.max_a * sizeof(int32_t);
	b.a_buf.xo = (uint32_t *)p, p += b.max_a * sizeof(uint32_t);
	b.A = (gwf_diag_t *)p, p += b.max_A * sizeof(gwf_diag_t);
	b.B = (gwf_diag_t *)p, p += b.max_B * sizeof(gwf_diag_t);
	b.ooo = (gwf_diag_t *)p, p += b.max_ooo * sizeof(gwf_diag_t);
	b.intv.vd0 = (uint64_t *)p, p += b.max_intv * sizeof(uint64_t);
	b.intv.vd1 = (uint64_t *)p, p += b.max_intv * sizeof(uint64_t);
	b.tmp.vd0 = (uint64_t *)p, p += b.max_tmp * sizeof(uint64_t);
	b.tmp.vd1 = (uint64_t *)p, p += b.max_tmp * sizeof(uint64_t);
	b.swap.vd0 = (uint64_t *)p, p += b.max_swap * sizeof(uint64_t);
	b.swap.vd1 = (uint64_t *)p, p += b.max_swap * sizeof(uint64_t);
	b.ha = (uint64_t *)p;
	scores[r] = gwf_ed(g, qlen[r], seqs + seq_off[r], v0[r], -1, 0, &b, diag_shared);
}

static uint32_t npow2(uint32_t x)
{
	if (x == 0) return 0;
	--x;
	x |= x >> 1, x |= x >> 2, x |= x >> 4, x |= x >> 8, x |= x >> 16;
	return x + 1;
}

static size_t al64(size_t x) { return (x + 63) & ~(size_t)63; }

int main(int argc, char **argv)
{
	if (argc < 4) {
		fprintf(stderr, "usage: gwf-ref-harness <graph.gfa> <reads.fa> <v0.txt|-> [n_streams]\n");
		return 1;
	}
	int n_streams = argc > 4 ? atoi(argv[4]) : 16;
	gfa_t *gfa = gfa_read(argv[1]);
	if (!gfa) return 1;
	gwf_graph_t *g = gwf_gfa2gwf(gfa, 0);
	gwf_ed_index(g);

	// reads (FASTA, one or more sequence lines per record)
	std::vector<std::string> reads;
	{
		FILE *fp = fopen(argv[2], "r");
		if (!fp) return 1;
		char *line = nullptr;
		size_t cap = 0;
		ssize_t l;
		while ((l = getline(&line, &cap, fp)) >= 0) {
			while (l > 0 && (line[l - 1] == '\n' || line[l - 1] == '\r')) line[--l] = 0;
			if (line[0] == '>') reads.emplace_back();
			else if (!reads.empty()) reads.back() += line;
		}
		free(line);
		fclose(fp);
	}
	const size_t n = reads.size();
	std::vector<int32_t> v0(n, 0);
	if (strcmp(argv[3], "-")) {
		FILE *fp = fopen(argv[3], "r");
		if (!fp) return 1;
		for (size_t i = 0; i < n; ++i)
			if (fscanf(fp, "%d", &v0[i]) != 1) return 1;
		fclose(fp);
	}

	// device graph (main.cu:415-452)
	gwf_graph_t gh = *g, *gd = nullptr;
	CK(cudaMalloc(&gd, sizeof(gwf_graph_t)));
	CK(cudaMalloc(&gh.len, g->n_vtx * sizeof(uint32_t)));
	CK(cudaMemcpy(gh.len, g->len, g->n_vtx * sizeof(uint32_t), cudaMemcpyHostToDevice));
	CK(cudaMalloc(&gh.src, g->n_vtx * sizeof(uint32_t)));
	CK(cudaMemcpy(gh.src, g->src, g->n_vtx * sizeof(uint32_t), cudaMemcpyHostToDevice));
	CK(cudaMalloc(&gh.arc, (g->n_arc ? g->n_arc : 1) * sizeof(gwf_arc_t)));
	CK(cudaMemcpy(gh.arc, g->arc, g->n_arc * sizeof(gwf_arc_t), cudaMemcpyHostToDevice));
	CK(cudaMalloc(&gh.aux, g->n_vtx * sizeof(uint64_t)));
	CK(cudaMemcpy(gh.aux, g->aux, g->n_vtx * sizeof(uint64_t), cudaMemcpyHostToDevice));
	std::vector<char *> sp(g->n_vtx);
	for (uint32_t i = 0; i < g->n_vtx; ++i) {
		size_t len = strlen(g->seq[i]) + 1;
		CK(cudaMalloc(&sp[i], len));
		CK(cudaMemcpy(sp[i], g->seq[i], len, cudaMemcpyHostToDevice));
	}
	char **seqd;
	CK(cudaMalloc(&seqd, g->n_vtx * sizeof(char *)));
	CK(cudaMemcpy(seqd, sp.data(), g->n_vtx * sizeof(char *), cudaMemcpyHostToDevice));
	gh.seq = seqd;
	CK(cudaMemcpy(gd, &gh, sizeof(gwf_graph_t), cudaMemcpyHostToDevice));

	// per-read arena sizes (main.cu:498-517)
	std::vector<gwf_edbuf_t> bufs(n);
	std::vector<size_t> bytes(n), seq_off(n);
	std::vector<int32_t> qlen(n);
	std::string all;
	for (size_t i = 0; i < n; ++i) {
		const size_t l = reads[i].size();
		gwf_edbuf_t &b = bufs[i];
		memset(&b, 0, sizeof b);
		b.max_a = (uint32_t)(((4 * l * 0.1) + 1) * 4);
		b.max_B = 3 * b.max_a + 1;
		b.max_A = b.max_intv = b.max_swap = b.max_a;
		b.max_tmp = b.max_ooo = b.max_B;
		b.ha_mask = npow2((uint32_t)l * 32) - 1;
		size_t s = (size_t)b.max_a * (8 + 4 + 4) + (size_t)(b.max_A + b.max_B + b.max_ooo) * sizeof(gwf_diag_t);
		s += ((size_t)b.max_intv * 2 + (size_t)b.max_tmp * 2 + (size_t)b.max_swap * 2) * sizeof(uint64_t);
		s += ((size_t)b.ha_mask + 1) * sizeof(uint64_t);
		bytes[i] = s;
		qlen[i] = (int32_t)l;
		seq_off[i] = all.size();
		all += reads[i];
		all.push_back(0);
	}

	// streams and pools (main.cu:539-588)
	size_t fr, tot;
	CK(cudaMemGetInfo(&fr, &tot));
	const size_t pool = fr * 90 / 100;
	if (n_streams < 1) n_streams = 1;
	if ((size_t)n_streams > n) n_streams = (int)(n ? n : 1);
	size_t max_one = 0;
	for (size_t i = 0; i < n; ++i) max_one = std::max(max_one, al64(bytes[i]) + al64(qlen[i] + 1) + 7 * 64 + sizeof(gwf_edbuf_t));
	while (n_streams > 1 && pool / n_streams < max_one) --n_streams;
	const size_t cap = pool / n_streams;
	std::vector<cudaStream_t> st(n_streams);
	std::vector<char *> arena(n_streams);
	for (int s = 0; s < n_streams; ++s) {
		CK(cudaStreamCreate(&st[s]));
		CK(cudaMalloc(&arena[s], cap));
	}
	int32_t *scores_h;
	CK(cudaMallocHost(&scores_h, (n ? n : 1) * sizeof(int32_t)));
	char *all_h;
	CK(cudaMallocHost(&all_h, all.size() + 1));
	memcpy(all_h, all.data(), all.size());
	gwf_edbuf_t *bufs_h;
	CK(cudaMallocHost(&bufs_h, (n ? n : 1) * sizeof(gwf_edbuf_t)));
	memcpy(bufs_h, bufs.data(), n * sizeof(gwf_edbuf_t));
	std::vector<std::vector<size_t>> off_h(n_streams), soff_h(n_streams);
	std::vector<int> busy(n_streams, 0);
	std::vector<size_t *> pin_off(n_streams, nullptr), pin_soff(n_streams, nullptr);

	CK(cudaDeviceSynchronize());
	const double t0 = now_s();
	size_t next = 0, launch = 0;
	while (next < n) {
		const int s = (int)(launch % n_streams);
		if (busy[s]) {
			CK(cudaStreamSynchronize(st[s]));
			busy[s] = 0;
		}
		// greedy packing (main.cu:636-667)
		size_t work = 0, m = 0;
		const size_t sbase = seq_off[next];
		while (next + m < n) {
			const size_t r = next + m;
			const size_t w2 = al64(work) + bytes[r];
			const size_t sb = seq_off[r] + qlen[r] + 1 - sbase;
			const size_t k = m + 1;
			size_t off = al64(w2);
			off = al64(off + sb);
			off = al64(off + k * sizeof(gwf_edbuf_t));
			off = al64(off + k * sizeof(size_t)) + al64(k * sizeof(size_t)) + al64(k * 4) * 3;
			if (off > cap) {
				if (m == 0) {
					fprintf(stderr, "read %zu does not fit\n", r);
					return 2;
				}
				break;
			}
			work = w2, m = k;
		}
		CK(cudaFreeHost(pin_off[s] ? pin_off[s] : nullptr));
		CK(cudaFreeHost(pin_soff[s] ? pin_soff[s] : nullptr));
		CK(cudaMallocHost(&pin_off[s], m * sizeof(size_t)));
		CK(cudaMallocHost(&pin_soff[s], m * sizeof(size_t)));
		size_t w = 0;
		for (size_t j = 0; j < m; ++j) {
			w = al64(w);
			pin_off[s][j] = w;
			w += bytes[next + j];
			pin_soff[s][j] = seq_off[next + j] - sbase;
		}
		const size_t sbytes = seq_off[next + m - 1] + qlen[next + m - 1] + 1 - sbase;
		char *base = arena[s];
		size_t o = 0;
		char *work_d = base + o;
		o = al64(o + work);
		char *seq_d = base + o;
		o = al64(o + sbytes);
		gwf_edbuf_t *buf_d = (gwf_edbuf_t *)(base + o);
		o = al64(o + m * sizeof(gwf_edbuf_t));
		size_t *off_d = (size_t *)(base + o);
		o = al64(o + m * sizeof(size_t));
		size_t *soff_d = (size_t *)(base + o);
		o = al64(o + m * sizeof(size_t));
		int32_t *ql_d = (int32_t *)(base + o);
		o = al64(o + m * 4);
		int32_t *v0_d = (int32_t *)(base + o);
		o = al64(o + m * 4);
		int32_t *sc_d = (int32_t *)(base + o);
		CK(cudaMemsetAsync(work_d, 0, work, st[s]));
		CK(cudaMemcpyAsync(buf_d, bufs_h + next, m * sizeof(gwf_edbuf_t), cudaMemcpyHostToDevice, st[s]));
		CK(cudaMemcpyAsync(off_d, pin_off[s], m * sizeof(size_t), cudaMemcpyHostToDevice, st[s]));
		CK(cudaMemcpyAsync(soff_d, pin_soff[s], m * sizeof(size_t), cudaMemcpyHostToDevice, st[s]));
		CK(cudaMemcpyAsync(ql_d, qlen.data() + next, m * 4, cudaMemcpyHostToDevice, st[s]));
		CK(cudaMemcpyAsync(v0_d, v0.data() + next, m * 4, cudaMemcpyHostToDevice, st[s]));
		CK(cudaMemcpyAsync(seq_d, all_h + sbase, sbytes, cudaMemcpyHostToDevice, st[s]));
		harness_kernel<<<(unsigned)m, 32, 0, st[s]>>>(work_d, off_d, buf_d, seq_d, soff_d, ql_d, v0_d, gd, sc_d, (int)m);
		CK(cudaGetLastError());
		CK(cudaMemcpyAsync(scores_h + next, sc_d, m * 4, cudaMemcpyDeviceToHost, st[s]));
		busy[s] = 1;
		next += m;
		++launch;
	}
	for (int s = 0; s < n_streams; ++s) CK(cudaStreamSynchronize(st[s]));
	const double el = now_s() - t0;
	for (size_t i = 0; i < n; ++i) printf("%d\n", scores_h[i]);
	size_t tb = 0;
	for (size_t i = 0; i < n; ++i) tb += qlen[i];
	fprintf(stderr, "{\"reads\": %zu, \"bases\": %zu, \"seconds\": %.6f, \"reads_per_s\": %.3f, \"launches\": %zu, \"streams\": %d}\n",
	        n, tb, el, el > 0 ? n / el : 0.0, launch, n_streams);
	return 0;
}
