// reads_loader.cpp — FASTA/FASTQ input of the read sets, plain or gzip, into one concatenated
// buffer in file order (the layout gwf_ed_batch_concat takes). The reference reads its FASTA file
// twice, once to size and once to copy (main.cu:459-534); here the file is read once into memory.
//
// FASTA: a '>' line starts a record, and the following lines, without their line ends, are its
// sequence; lines before the first header are ignored. The text is cut at record starts into one
// chunk per core, the chunks are parsed on threads, and each copies its sequences into its place
// in the output. FASTQ (the first record starts with '@'): four-line records, parsed on one
// thread. A record with no sequence lines is a read of length 0.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string_view>
#include <thread>
#include <vector>

#include "../../include/gwfa.h"
#include "gwfa_internal.h"

namespace {

struct Part {                // the reads of one chunk
	std::vector<char> bytes; // sequences, back to back
	std::vector<int32_t> lens;
	std::vector<int64_t> off; // this chunk's offsets, relative to bytes
};

// FASTA records in [b, e); b is a record start or the start of the text.
void parse_fasta(const char *b, const char *e, Part &p)
{
	p.bytes.reserve((size_t)(e - b)); // the sequences are at most the chunk: no regrowth copies
	bool in_rec = false;
	int64_t cur = 0;
	while (b < e) {
		const char *nl = (const char *)memchr(b, '\n', (size_t)(e - b));
		const char *le = nl ? nl : e;
		std::string_view line(b, (size_t)(le - b));
		b = nl ? nl + 1 : e;
		if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
		if (!line.empty() && line[0] == '>') {
			if (in_rec) p.lens.push_back((int32_t)((int64_t)p.bytes.size() - cur));
			in_rec = true;
			cur = (int64_t)p.bytes.size();
			p.off.push_back(cur);
		} else if (in_rec) {
			p.bytes.insert(p.bytes.end(), line.begin(), line.end());
		}
	}
	if (in_rec) p.lens.push_back((int32_t)((int64_t)p.bytes.size() - cur));
}

// FASTQ records: '@' header, sequence, '+' line, qualities.
void parse_fastq(const char *b, const char *e, Part &p)
{
	p.bytes.reserve((size_t)(e - b) / 2);
	int state = 0; // 0 header, 1 sequence, 2 plus line, 3 qualities
	while (b < e) {
		const char *nl = (const char *)memchr(b, '\n', (size_t)(e - b));
		const char *le = nl ? nl : e;
		std::string_view line(b, (size_t)(le - b));
		b = nl ? nl + 1 : e;
		if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
		if (state == 0) {
			if (!line.empty() && line[0] == '@') state = 1;
		} else if (state == 1) {
			p.off.push_back((int64_t)p.bytes.size());
			p.lens.push_back((int32_t)line.size());
			p.bytes.insert(p.bytes.end(), line.begin(), line.end());
			state = 2;
		} else if (state == 2) {
			state = 3;
		} else {
			state = 0;
		}
	}
}

// Threads for a text of len bytes: GWF_READS_THREADS if set, else one per core with at least
// 4 MiB each, at most 16.
int read_threads(size_t len)
{
	if (const char *e = getenv("GWF_READS_THREADS")) {
		const int t = atoi(e);
		return t < 1 ? 1 : (t > 64 ? 64 : t);
	}
	const unsigned hc = std::thread::hardware_concurrency();
	size_t t = std::min<size_t>(hc ? hc : 1, 16);
	t = std::min<size_t>(t, len >> 22);
	return t < 1 ? 1 : (int)t;
}

// First byte of the first line at or after p that starts with c (or e).
const char *next_line_starting(const char *p, const char *e, char c, const char *text)
{
	if (p > text && p[-1] != '\n') {
		const char *nl = (const char *)memchr(p, '\n', (size_t)(e - p));
		p = nl ? nl + 1 : e;
	}
	while (p < e && *p != c) {
		const char *nl = (const char *)memchr(p, '\n', (size_t)(e - p));
		p = nl ? nl + 1 : e;
	}
	return p;
}

} // namespace

extern "C" gwf_reads_t *gwf_reads_load(const char *path)
{
	size_t len = 0;
	char *text = gwf_read_file(path, &len);
	if (!text) return nullptr;
	const char *b = text, *e = text + len;
	// FASTQ when the first line that is not empty starts with '@'
	const char *first = b;
	while (first < e && (*first == '\n' || *first == '\r')) ++first;
	const bool fastq = first < e && *first == '@';
	std::vector<Part> parts;
	if (fastq) {
		parts.resize(1);
		parse_fastq(b, e, parts[0]);
	} else {
		const int nt = read_threads(len);
		std::vector<const char *> cut((size_t)nt + 1);
		cut[0] = b, cut[(size_t)nt] = e;
		for (int t = 1; t < nt; ++t) {
			const char *p = std::max(cut[(size_t)t - 1], b + len * (size_t)t / (size_t)nt);
			cut[(size_t)t] = next_line_starting(p, e, '>', text);
		}
		parts.resize((size_t)nt);
		std::vector<std::thread> th;
		for (int t = 1; t < nt; ++t)
			th.emplace_back(parse_fasta, cut[(size_t)t], cut[(size_t)t + 1], std::ref(parts[(size_t)t]));
		parse_fasta(cut[0], cut[1], parts[0]);
		for (auto &x : th) x.join();
	}
	free(text);
	int64_t n = 0, bases = 0;
	std::vector<int64_t> base_of((size_t)parts.size()), first_of((size_t)parts.size());
	for (size_t k = 0; k < parts.size(); ++k) {
		first_of[k] = n, base_of[k] = bases;
		n += (int64_t)parts[k].lens.size(), bases += (int64_t)parts[k].bytes.size();
	}
	if (n > INT32_MAX) {
		gwf_set_error("more than 2^31 - 1 reads");
		return nullptr;
	}
	gwf_reads_t *r = (gwf_reads_t *)calloc(1, sizeof(gwf_reads_t));
	if (r) {
		r->n = (int32_t)n, r->n_bases = bases;
		r->seqs = (char *)malloc((size_t)bases + 16);
		r->offs = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
		r->lens = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
	}
	if (!r || !r->seqs || !r->offs || !r->lens) {
		gwf_reads_free(r);
		gwf_set_error("out of host memory for the reads");
		return nullptr;
	}
	memset(r->seqs + bases, 0, 16);
	auto place = [&](size_t k) {
		const Part &p = parts[k];
		if (!p.bytes.empty()) memcpy(r->seqs + base_of[k], p.bytes.data(), p.bytes.size());
		for (size_t i = 0; i < p.lens.size(); ++i) {
			r->offs[first_of[k] + (int64_t)i] = base_of[k] + p.off[i];
			r->lens[first_of[k] + (int64_t)i] = p.lens[i];
		}
	};
	std::vector<std::thread> th;
	for (size_t k = 1; k < parts.size(); ++k) th.emplace_back(place, k);
	if (!parts.empty()) place(0);
	for (auto &x : th) x.join();
	return r;
}

extern "C" void gwf_reads_free(gwf_reads_t *r)
{
	if (!r) return;
	free(r->seqs), free(r->offs), free(r->lens);
	free(r);
}
