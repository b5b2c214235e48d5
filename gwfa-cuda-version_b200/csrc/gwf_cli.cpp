// gwf_cli.cpp — gwf-b200, a command-line driver with the interface of the reference's gwf-test
// (main.cu:360-750): the same options and arguments, one edit distance per read on stdout, in
// input order. The alignment runs through the library's batch entry point on the device.
//
//   gwf-b200 [-p] [-s STR] [-l INT [-P]] [-m persistent|plain] [-x] [-t | -b] <target.gfa> <query.fa|fq[.gz]>
//
//   -p   print the graph (gwf_graph_print format) and exit     (main.cu:382-387, 354-359)
//   -s   starting segment name [first]; a trailing + or - picks the strand (main.cu:399-407)
//   -l   max lag; accepted and ignored, as in the reference     (main.cu:371, 377)
//   -P   apply -l: lag pruning (GWF_F_MAX_LAG; no reference counterpart); -t does not prune
//   -m   execution form [persistent]
//   -x   exact start state (GWF_F_EXACT_START)
//   -t   traceback: after each distance, the end offset, the vertex path and the CIGAR of the
//        read against the path's text (no reference counterpart; the reference's traceback
//        argument is unused, README.md:117-118)
//   -b   both strands: each read and its reverse complement; prints the smaller distance and
//        + (the read as given) or - (its reverse complement) (GWF_F_BOTH_STRANDS; the reference
//        aligns the read as given only, main.cu:370, 404)
//
// Every read is aligned from offset 0 of the start segment (vertex 0 of the converted graph),
// as the reference kernel does (main.cu:217). Timing and counts go to stderr.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gwfa.h"

namespace {

void usage()
{
	fprintf(stderr, "Usage: gwf-b200 [options] <target.gfa> <query.fa>\n");
	fprintf(stderr, "Options:\n");
	fprintf(stderr, "  -l INT    max lag behind the furthest wavefront; ignored unless -P [0]\n");
	fprintf(stderr, "  -P        apply -l: prune states more than -l bases behind the furthest (not with -t)\n");
	fprintf(stderr, "  -s STR    starting segment name, + or - appended for the strand [first, +]\n");
	fprintf(stderr, "  -p        output GFA in the forward strand\n");
	fprintf(stderr, "  -m STR    execution form: persistent or plain [persistent]\n");
	fprintf(stderr, "  -x        exact start state (no reference start-state rule)\n");
	fprintf(stderr, "  -t        traceback: print distance, end offset, vertex path and CIGAR per read\n");
	fprintf(stderr, "  -b        both strands: print distance and + or - (the read or its reverse complement)\n");
}

} // namespace

int main(int argc, char *argv[])
{
	bool print_graph = false, exact = false, trace = false, prune = false, both = false;
	const char *sname = nullptr;
	int32_t mode = GWF_MODE_PERSISTENT;
	uint32_t max_lag = 0;
	int i = 1;
	for (; i < argc && argv[i][0] == '-' && argv[i][1]; ++i) {
		const char *a = argv[i];
		if (!strcmp(a, "-p")) print_graph = true;
		else if (!strcmp(a, "-x")) exact = true;
		else if (!strcmp(a, "-t")) trace = true;
		else if (!strcmp(a, "-P")) prune = true;
		else if (!strcmp(a, "-b")) both = true;
		else if (!strcmp(a, "-s") && i + 1 < argc) sname = argv[++i];
		else if (!strcmp(a, "-l") && i + 1 < argc) max_lag = (uint32_t)atoi(argv[++i]);
		else if (!strcmp(a, "-m") && i + 1 < argc) {
			const char *m = argv[++i];
			if (!strcmp(m, "plain")) mode = GWF_MODE_PLAIN;
			else if (!strcmp(m, "persistent")) mode = GWF_MODE_PERSISTENT;
			else {
				usage();
				return 1;
			}
		} else {
			usage();
			return 1;
		}
	}
	if ((!print_graph && argc - i < 2) || (print_graph && argc - i < 1) || (both && trace)) {
		usage();
		return 1;
	}
	// the reads load on a second thread while the graph loads (the error text is per thread)
	gwf_reads_t *rs = nullptr;
	std::string reads_err;
	std::thread reader;
	if (!print_graph)
		reader = std::thread([&] {
			rs = gwf_reads_load(argv[i + 1]);
			if (!rs) reads_err = gwf_last_error();
		});
	gwf_graph_t *g = gwf_gfa_load(argv[i], sname);
	if (reader.joinable()) reader.join();
	if (!g) {
		fprintf(stderr, "ERROR: %s\n", gwf_last_error());
		gwf_reads_free(rs);
		return 1;
	}
	if (print_graph) {
		const int64_t n = gwf_graph_dump(g, nullptr, 0);
		std::vector<char> text((size_t)n + 1);
		gwf_graph_dump(g, text.data(), n + 1);
		fwrite(text.data(), 1, (size_t)n, stdout);
		gwf_graph_free(g);
		return 0;
	}
	// the reads, concatenated, through the library's reader (FASTA/FASTQ, plain or gzip)
	if (!rs) {
		fprintf(stderr, "ERROR: cannot read %s: %s\n", argv[i + 1], reads_err.c_str());
		gwf_graph_free(g);
		return 1;
	}
	const char *cat = rs->seqs;
	const std::vector<int64_t> offs(rs->offs, rs->offs + rs->n);
	const std::vector<int32_t> lens(rs->lens, rs->lens + rs->n);
	const int32_t n = rs->n;
	fprintf(stderr, "[gwf-b200] %d reads, %lld bases, %u vertices, %u arcs\n", n, (long long)rs->n_bases, g->n_vtx,
	        g->n_arc);
	gwf_ed_index(g);
	std::vector<int32_t> v0((size_t)n, 0), dist((size_t)n, -1), status((size_t)n, 0), strand((size_t)n, -1);
	gwf_batch_opts_t opt;
	memset(&opt, 0, sizeof opt);
	opt.mode = mode;
	opt.flags = (exact ? GWF_F_EXACT_START : 0) | (prune ? GWF_F_MAX_LAG : 0);
	const auto t0 = std::chrono::steady_clock::now();
	std::vector<std::string> paths;
	int rc = 0;
	if (trace) {
		// chunks of reads; rows of max_nv vertices and max_ops CIGAR runs, widened (one more
		// pass) for a chunk whose paths or CIGARs are longer
		paths.resize((size_t)n);
		const int32_t chunk = 8192;
		static const char kOp[16] = {'M', 'I', 'D', '?', '?', '?', '?', '=', 'X', '?', '?', '?', '?', '?', '?', '?'};
		for (int32_t c0 = 0; c0 < n && !rc; c0 += chunk) {
			const int32_t m = std::min(chunk, n - c0);
			int32_t max_nv = 256, max_ops = 512;
			std::vector<int32_t> eo((size_t)m), pn((size_t)m), cn((size_t)m), pv, pa;
			std::vector<uint32_t> cg;
			for (int pass = 0; pass < 2 && !rc; ++pass) {
				pv.assign((size_t)m * (size_t)max_nv, 0), pa.assign((size_t)m * (size_t)max_nv, 0);
				cg.assign((size_t)m * (size_t)max_ops, 0);
				rc = gwf_ed_batch_align(g, m, cat, offs.data() + c0, lens.data() + c0, v0.data() + c0, -1,
				                        opt.flags, max_nv, max_ops, dist.data() + c0, status.data() + c0, eo.data(),
				                        pn.data(), pv.data(), pa.data(), cn.data(), cg.data());
				const int32_t need_nv = m ? *std::max_element(pn.begin(), pn.end()) : 0;
				const int32_t need_ops = m ? *std::max_element(cn.begin(), cn.end()) : 0;
				if (need_nv <= max_nv && need_ops <= max_ops) break;
				max_nv = std::max(max_nv, need_nv), max_ops = std::max(max_ops, need_ops);
			}
			for (int32_t j = 0; j < m && !rc; ++j) {
				std::string &o = paths[(size_t)(c0 + j)];
				o = "\t" + std::to_string(eo[(size_t)j]) + "\t";
				for (int32_t k = 0; k < pn[(size_t)j] && k < max_nv; ++k) {
					if (k) o += ',';
					o += std::to_string(pv[(size_t)j * max_nv + k]);
				}
				o += '\t';
				if (cn[(size_t)j] < 0 || cn[(size_t)j] > max_ops) o += '*';
				for (int32_t k = 0; k >= 0 && k < cn[(size_t)j] && k < max_ops; ++k) {
					const uint32_t x = cg[(size_t)j * max_ops + k];
					o += std::to_string(x >> 4);
					o += kOp[x & 15];
				}
			}
		}
	} else if (n > 0 && both) {
		rc = gwf_ed_batch_strand(g, n, cat, offs.data(), lens.data(), v0.data(), -1, max_lag, dist.data(),
		                         status.data(), strand.data(), &opt);
	} else if (n > 0) {
		rc = gwf_ed_batch_concat(g, n, cat, offs.data(), lens.data(), v0.data(), -1, max_lag, dist.data(),
		                         status.data(), &opt);
	}
	const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	if (rc) {
		fprintf(stderr, "ERROR: batch alignment failed (%d): %s\n", rc, gwf_last_error());
		gwf_reads_free(rs);
		gwf_graph_free(g);
		return 1;
	}
	int32_t bad = 0;
	for (int32_t j = 0; j < n; ++j) {
		if (trace) printf("%d%s\n", dist[(size_t)j], paths[(size_t)j].c_str());
		else if (both) printf("%d\t%c\n", dist[(size_t)j], strand[(size_t)j] == 1 ? '-' : strand[(size_t)j] == 0 ? '+' : '*');
		else printf("%d\n", dist[(size_t)j]);
		if (status[(size_t)j] != GWF_OK) ++bad;
	}
	fprintf(stderr, "[gwf-b200] aligned in %.6f s (%d reads with a per-read error status)\n", el, bad);
	gwf_reads_free(rs);
	gwf_graph_free(g);
	return bad ? 2 : 0;
}
