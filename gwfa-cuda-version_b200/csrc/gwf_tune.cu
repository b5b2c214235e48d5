// gwf_tune.cu — autotuner of the batch launch shape, per read-length bucket.
//
// The cost of a read grows with ql^2 x error, and the arena a warp needs grows with ql, so the
// best launch shape depends on the lengths in a batch. gwf_tune times, on the caller's own reads
// and separately for each length bucket, the persistent form with 1, 2, 4 and 8 warps per read at
// every CTAs-per-SM count up to the occupancy limit, and the plain form, and keeps the fastest
// per bucket in a per-device table. A batch run with mode GWF_MODE_AUTO then aligns each read
// with the warps per read of its own bucket (one launch, read classes longest first) and takes
// the form and CTAs per SM of the bucket that carries most of its work (sum of ql^2). The table
// can be written to and read from a small JSON file, so a tuned setting survives the process.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gwfa.h"
#include "gwf_runtime.h"
#include "gwfa_internal.h"

namespace {

const int32_t kBucketMax[GWF_TUNE_NBUCKETS] = {1500, 3000, 6000, 12000, INT32_MAX};
constexpr int kMaxDevices = 64;

struct TuneEntry {
	int32_t valid = 0, form = 0, cps = 0, nw = 1;
	float rps = 0;
};

std::mutex g_tune_mu;
TuneEntry g_tune[kMaxDevices][GWF_TUNE_NBUCKETS];

int device_or_current(int device)
{
	if (device >= 0) return device;
	int d = 0;
	if (cudaGetDevice(&d) != cudaSuccess) {
		cudaGetLastError();
		d = 0;
	}
	return d;
}

const char *form_name(int32_t f) { return f == GWF_MODE_PLAIN ? "plain" : "persistent"; }

} // namespace

int gwf_tune_bucket(int32_t ql)
{
	for (int b = 0; b < GWF_TUNE_NBUCKETS; ++b)
		if (ql < kBucketMax[b] || b == GWF_TUNE_NBUCKETS - 1) return b;
	return GWF_TUNE_NBUCKETS - 1;
}

int gwf_tune_lookup_nw(int device, int32_t bucket)
{
	if (device < 0 || device >= kMaxDevices || bucket < 0 || bucket >= GWF_TUNE_NBUCKETS) return 0;
	std::lock_guard<std::mutex> lk(g_tune_mu);
	const TuneEntry &e = g_tune[device][bucket];
	return e.valid && e.form != GWF_MODE_PLAIN ? e.nw : 0;
}

int gwf_tune_lookup(int device, int32_t bucket, int32_t *form, int32_t *ctas_per_sm)
{
	if (device < 0 || device >= kMaxDevices || bucket < 0 || bucket >= GWF_TUNE_NBUCKETS) return 0;
	std::lock_guard<std::mutex> lk(g_tune_mu);
	const TuneEntry &e = g_tune[device][bucket];
	if (!e.valid) return 0;
	*form = e.form, *ctas_per_sm = e.cps;
	return 1;
}

static int write_json(const char *path, int device)
{
	FILE *f = fopen(path, "w");
	if (!f) {
		gwf_set_errorf("gwf_tune: cannot write %s", path);
		return GWF_E_BAD_INPUT;
	}
	cudaDeviceProp prop;
	memset(&prop, 0, sizeof prop);
	if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) cudaGetLastError();
	fprintf(f, "{\"version\": 1, \"device\": %d, \"name\": \"%s\", \"sm_count\": %d, \"buckets\": [", device,
	        prop.name, prop.multiProcessorCount);
	bool first = true;
	for (int b = 0; b < GWF_TUNE_NBUCKETS; ++b) {
		const TuneEntry &e = g_tune[device][b];
		if (!e.valid) continue;
		fprintf(f,
		        "%s\n  {\"bucket\": %d, \"ql_max\": %d, \"form\": \"%s\", \"ctas_per_sm\": %d, \"reads_per_s\": %.1f, "
		        "\"warps_per_read\": %d}",
		        first ? "" : ",", b, kBucketMax[b] == INT32_MAX ? -1 : kBucketMax[b], form_name(e.form), e.cps,
		        (double)e.rps, e.nw);
		first = false;
	}
	fprintf(f, "\n]}\n");
	fclose(f);
	return 0;
}

extern "C" int gwf_tune(const gwf_graph_t *g, int32_t n, const char *seqs, const int64_t *offs,
                        const int32_t *ql, const int32_t *v0, int32_t v1, int32_t max_reads_per_bucket,
                        const char *json_path)
{
	if (!g || n <= 0 || !seqs || !offs || !ql || !v0) {
		gwf_set_error("gwf_tune: bad arguments");
		return GWF_E_BAD_INPUT;
	}
	GraphDev *G = gwf_find_graph(g);
	if (!G) {
		gwf_set_error("gwf_tune: graph not indexed on a device");
		return GWF_E_NOT_INDEXED;
	}
	int dev;
	int rc = gwf_select_device(G->device, &dev);
	if (rc) return rc;
	if (dev >= kMaxDevices) return GWF_E_UNSUPPORTED;
	Engine *E = gwf_engine(dev);
	if (!E) return GWF_E_CUDA;
	if (max_reads_per_bucket <= 0) max_reads_per_bucket = 8192;
	std::vector<std::vector<int32_t>> members(GWF_TUNE_NBUCKETS);
	for (int32_t i = 0; i < n; ++i) {
		if (ql[i] <= 0) continue;
		members[(size_t)gwf_tune_bucket(ql[i])].push_back(i);
	}
	std::lock_guard<std::mutex> blk(gwf_batch_mutex());
	for (int b = 0; b < GWF_TUNE_NBUCKETS; ++b) {
		const std::vector<int32_t> &m = members[(size_t)b];
		if (m.empty()) continue;
		// evenly spread sample of the bucket
		const int32_t k = std::min<int32_t>((int32_t)m.size(), max_reads_per_bucket);
		std::vector<int64_t> so((size_t)k);
		std::vector<int32_t> sq((size_t)k), sv((size_t)k);
		for (int32_t j = 0; j < k; ++j) {
			const int32_t i = m[(size_t)((int64_t)j * (int64_t)m.size() / k)];
			so[(size_t)j] = offs[i], sq[(size_t)j] = ql[i], sv[(size_t)j] = v0[i];
		}
		Batch B;
		if ((rc = gwf_batch_load(*E, B, k, seqs, so.data(), sq.data(), sv.data(), v1))) {
			B.release();
			return rc;
		}
		TuneEntry best;
		struct Cand {
			int32_t form, cps, nw;
		};
		std::vector<Cand> cand;
		for (int nw : {1, 2, 4, 8}) {
			const int occ = nw == 1 ? E->persistent_ctas_per_sm : E->classes_ctas_per_sm;
			for (int c = 1; c <= occ; ++c) cand.push_back({GWF_MODE_PERSISTENT, c, nw});
		}
		cand.push_back({GWF_MODE_PLAIN, 0, 1});
		for (const Cand &fc : cand) {
			float best_ms = 0;
			for (int rep = 0; rep < 3; ++rep) { // one warm-up, then the faster of two timed runs
				float ms = 0;
				if ((rc = gwf_batch_exec(*E, *G, B, fc.form, 0, fc.cps, &ms, nullptr, 0, 0, fc.nw))) {
					B.release();
					return rc;
				}
				if (rep == 1 || (rep == 2 && ms < best_ms)) best_ms = ms;
			}
			const float rps = best_ms > 0 ? (float)k / (best_ms / 1000.0f) : 0.0f;
			if (!best.valid || rps > best.rps)
				best.valid = 1, best.form = fc.form, best.cps = fc.cps, best.nw = fc.nw, best.rps = rps;
		}
		B.release();
		std::lock_guard<std::mutex> lk(g_tune_mu);
		g_tune[dev][b] = best;
	}
	if (json_path) {
		std::lock_guard<std::mutex> lk(g_tune_mu);
		return write_json(json_path, dev);
	}
	return 0;
}

extern "C" int gwf_tune_load(const char *json_path, int32_t device)
{
	if (!json_path) return GWF_E_BAD_INPUT;
	FILE *f = fopen(json_path, "r");
	if (!f) {
		gwf_set_errorf("gwf_tune_load: cannot read %s", json_path);
		return GWF_E_BAD_INPUT;
	}
	std::string text;
	char buf[4096];
	size_t got;
	while ((got = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
	fclose(f);
	const int dev = device_or_current(device);
	if (dev >= kMaxDevices) return GWF_E_UNSUPPORTED;
	TuneEntry table[GWF_TUNE_NBUCKETS];
	int n_read = 0;
	for (size_t pos = text.find("{\"bucket\""); pos != std::string::npos; pos = text.find("{\"bucket\"", pos + 1)) {
		int b = -1, qmax = 0, cps = 0;
		char form[32] = {0};
		double rps = 0;
		if (sscanf(text.c_str() + pos,
		           "{\"bucket\": %d, \"ql_max\": %d, \"form\": \"%31[a-z]\", \"ctas_per_sm\": %d, \"reads_per_s\": %lf",
		           &b, &qmax, form, &cps, &rps) != 5 ||
		    b < 0 || b >= GWF_TUNE_NBUCKETS || cps < 0 || cps > 64) {
			gwf_set_errorf("gwf_tune_load: bad entry in %s", json_path);
			return GWF_E_BAD_INPUT;
		}
		TuneEntry &e = table[b];
		e.valid = 1;
		e.form = strcmp(form, "plain") == 0 ? GWF_MODE_PLAIN : GWF_MODE_PERSISTENT;
		e.cps = e.form == GWF_MODE_PLAIN ? 0 : std::max(1, cps);
		e.rps = (float)rps;
		// warps per read (absent in tables written before the field existed: one warp)
		e.nw = 1;
		const size_t end = text.find('}', pos);
		const size_t at = text.find("\"warps_per_read\":", pos);
		if (at != std::string::npos && at < end) {
			int nw = 1;
			if (sscanf(text.c_str() + at, "\"warps_per_read\": %d", &nw) != 1 || (nw != 1 && nw != 2 && nw != 4 && nw != 8)) {
				gwf_set_errorf("gwf_tune_load: bad warps_per_read in %s", json_path);
				return GWF_E_BAD_INPUT;
			}
			e.nw = e.form == GWF_MODE_PLAIN ? 1 : nw;
		}
		++n_read;
	}
	if (n_read == 0) {
		gwf_set_errorf("gwf_tune_load: no entries in %s", json_path);
		return GWF_E_BAD_INPUT;
	}
	std::lock_guard<std::mutex> lk(g_tune_mu);
	for (int b = 0; b < GWF_TUNE_NBUCKETS; ++b) g_tune[dev][b] = table[b];
	return 0;
}

extern "C" int gwf_tune_get(int32_t device, int32_t bucket, int32_t *form, int32_t *ctas_per_sm,
                            float *reads_per_s)
{
	const int dev = device_or_current(device);
	if (dev >= kMaxDevices || bucket < 0 || bucket >= GWF_TUNE_NBUCKETS) return GWF_E_BAD_INPUT;
	std::lock_guard<std::mutex> lk(g_tune_mu);
	const TuneEntry &e = g_tune[dev][bucket];
	if (form) *form = e.form;
	if (ctas_per_sm) *ctas_per_sm = e.cps;
	if (reads_per_s) *reads_per_s = e.rps;
	return e.valid;
}

extern "C" int gwf_tune_get_shape(int32_t device, int32_t bucket, int32_t *form, int32_t *ctas_per_sm,
                                  int32_t *warps_per_read, float *reads_per_s)
{
	const int rc = gwf_tune_get(device, bucket, form, ctas_per_sm, reads_per_s);
	if (rc < 0) return rc;
	if (warps_per_read) {
		std::lock_guard<std::mutex> lk(g_tune_mu);
		*warps_per_read = g_tune[device_or_current(device)][bucket].nw;
	}
	return rc;
}

extern "C" void gwf_tune_clear(int32_t device)
{
	const int dev = device_or_current(device);
	if (dev >= kMaxDevices) return;
	std::lock_guard<std::mutex> lk(g_tune_mu);
	for (int b = 0; b < GWF_TUNE_NBUCKETS; ++b) g_tune[dev][b] = TuneEntry();
}
