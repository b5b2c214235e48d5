// gwf_serve.cu — continuous-batching request loop on a device-resident graph.
//
// Requests (1..n reads each) queue in FIFO order. K lanes, each a host thread with its own CUDA
// stream and warp arenas, take as many queued requests as their share of the arena budget
// admits and run them through the persistent kernel. While one lane's launch is on the GPU the
// others admit newly arrived requests, so work from different requests overlaps on the device.
// A request is complete when every read has a distance or a per-read error status; its submit,
// admit and completion times are kept for latency percentiles.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gwfa.h"
#include "gwf_runtime.h"
#include "gwfa_internal.h"

namespace {

double now_s()
{
	return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
	int64_t id;
	int32_t n, v1;
	std::vector<char> seqs;
	std::vector<int64_t> offs;
	std::vector<int32_t> ql, v0, dist, status;
	double t_submit = 0, t_admit = 0, t_done = 0;
	bool done = false;
	int32_t error = 0;
};

} // namespace

struct gwf_srv_s {
	const gwf_graph_t *g = nullptr;
	GraphDev *G = nullptr;
	int device = 0;
	int32_t flags = 0;
	int64_t budget = 0;
	int32_t max_reads = 0;
	std::mutex mu;
	std::condition_variable cv_work, cv_done;
	std::deque<std::shared_ptr<Request>> pending;
	std::unordered_map<int64_t, std::shared_ptr<Request>> all;
	int64_t next_id = 0;
	bool stop = false;
	std::vector<std::thread> lanes;
	std::vector<Engine *> engines;
};

static void lane_main(gwf_srv_s *S, int lane_id)
{
	cudaSetDevice(S->device);
	Engine *E = S->engines[(size_t)lane_id];
	Batch B;
	const int64_t lane_budget = S->budget / (int64_t)S->engines.size();
	for (;;) {
		std::vector<std::shared_ptr<Request>> take;
		{
			std::unique_lock<std::mutex> lk(S->mu);
			S->cv_work.wait(lk, [&] { return S->stop || !S->pending.empty(); });
			if (S->stop && S->pending.empty()) break;
			int32_t reads = 0, qmax = 0;
			while (!S->pending.empty()) {
				auto &r = S->pending.front();
				int32_t rq = 0;
				for (int32_t x : r->ql) rq = std::max(rq, x);
				const int32_t nq = std::max(qmax, rq);
				// arena estimate: one warp per read, arenas sized for the longest read
				const int64_t need = (int64_t)(reads + r->n) *
				                     gwfb::ws_layout(gwfb::caps_for(nq, 0, S->G->dens_milli)).total;
				if (!take.empty() && (need > lane_budget || reads + r->n > S->max_reads)) break;
				reads += r->n, qmax = nq;
				take.push_back(r);
				S->pending.pop_front();
			}
		}
		const double t_admit = now_s();
		// concatenate the admitted requests into one batch
		int32_t n = 0;
		int64_t bytes = 0;
		for (auto &r : take) n += r->n, bytes += (int64_t)r->seqs.size();
		std::vector<char> seqs((size_t)bytes + 1);
		std::vector<int64_t> offs((size_t)n);
		std::vector<int32_t> ql((size_t)n), v0((size_t)n), dist((size_t)n), status((size_t)n);
		int32_t v1 = take.empty() ? -1 : take[0]->v1;
		bool mixed_v1 = false;
		{
			int64_t o = 0;
			int32_t i = 0;
			for (auto &r : take) {
				r->t_admit = t_admit;
				if (r->v1 != v1) mixed_v1 = true;
				memcpy(seqs.data() + o, r->seqs.data(), r->seqs.size());
				for (int32_t j = 0; j < r->n; ++j, ++i)
					offs[(size_t)i] = o + r->offs[(size_t)j], ql[(size_t)i] = r->ql[(size_t)j],
					v0[(size_t)i] = r->v0[(size_t)j];
				o += (int64_t)r->seqs.size();
			}
		}
		int rc = 0;
		if (mixed_v1) {
			// requests with different v1 run one after the other
			int32_t i = 0;
			for (auto &r : take) {
				rc = gwf_batch_load(*E, B, r->n, r->seqs.data(), r->offs.data(), r->ql.data(), r->v0.data(), r->v1);
				if (!rc) rc = gwf_batch_exec(*E, *S->G, B, GWF_MODE_PERSISTENT, S->flags, 0, nullptr, nullptr);
				if (!rc) rc = gwf_batch_fetch(*E, B, dist.data() + i, status.data() + i);
				if (rc) break;
				i += r->n;
			}
		} else {
			rc = gwf_batch_load(*E, B, n, seqs.data(), offs.data(), ql.data(), v0.data(), v1);
			if (!rc) rc = gwf_batch_exec(*E, *S->G, B, GWF_MODE_PERSISTENT, S->flags, 0, nullptr, nullptr);
			if (!rc) rc = gwf_batch_fetch(*E, B, dist.data(), status.data());
		}
		const double t_done = now_s();
		{
			std::lock_guard<std::mutex> lk(S->mu);
			int32_t i = 0;
			for (auto &r : take) {
				r->dist.assign(dist.begin() + i, dist.begin() + i + r->n);
				r->status.assign(status.begin() + i, status.begin() + i + r->n);
				if (rc) std::fill(r->status.begin(), r->status.end(), rc);
				r->error = rc;
				r->t_done = t_done;
				r->done = true;
				i += r->n;
			}
		}
		S->cv_done.notify_all();
	}
	B.release();
}

extern "C" gwf_srv_t *gwf_srv_create(const gwf_graph_t *g, const gwf_srv_opts_t *opt)
{
	GraphDev *G = g ? gwf_find_graph(g) : nullptr;
	if (!G) {
		gwf_set_error("gwf_srv_create: graph not indexed on a device");
		return nullptr;
	}
	int dev;
	if (gwf_select_device(G->device, &dev)) return nullptr;
	gwf_srv_s *S = new gwf_srv_s;
	S->g = g, S->G = G, S->device = dev;
	S->flags = opt ? opt->flags : 0;
	size_t fr = 0, tot = 0;
	cudaMemGetInfo(&fr, &tot);
	S->budget = opt && opt->arena_budget_bytes > 0 ? opt->arena_budget_bytes : (int64_t)(fr / 4);
	S->max_reads = opt && opt->max_inflight_reads > 0 ? opt->max_inflight_reads : 65536;
	const int n_lanes = 4;
	for (int i = 0; i < n_lanes; ++i) {
		Engine *E = new Engine;
		E->device = dev;
		if (cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) != cudaSuccess ||
		    cudaEventCreate(&E->ev0) != cudaSuccess || cudaEventCreate(&E->ev1) != cudaSuccess) {
			cudaGetLastError();
			gwf_set_error("gwf_srv_create: stream creation failed");
			delete E;
			break;
		}
		cudaDeviceGetAttribute(&E->sm_count, cudaDevAttrMultiProcessorCount, dev);
		Engine *ref = gwf_engine(dev);
		E->persistent_ctas_per_sm = ref ? ref->persistent_ctas_per_sm : 1;
		E->mem_budget = ref ? ref->mem_budget / n_lanes : ((int64_t)1 << 30);
		S->engines.push_back(E);
	}
	if (S->engines.empty()) {
		delete S;
		return nullptr;
	}
	for (int i = 0; i < (int)S->engines.size(); ++i) S->lanes.emplace_back(lane_main, S, i);
	return S;
}

extern "C" int64_t gwf_srv_submit(gwf_srv_t *S, int32_t n, const char *seqs, const int64_t *offs,
                                  const int32_t *ql, const int32_t *v0, int32_t v1)
{
	if (!S || n <= 0 || !seqs || !offs || !ql || !v0) {
		gwf_set_error("gwf_srv_submit: bad arguments");
		return GWF_E_BAD_INPUT;
	}
	if (v1 >= 0 && (uint32_t)v1 >= S->G->n_vtx) {
		gwf_set_error("gwf_srv_submit: v1 out of range");
		return GWF_E_BAD_INPUT;
	}
	auto r = std::make_shared<Request>();
	r->n = n, r->v1 = v1;
	int64_t tot = 0;
	r->offs.resize((size_t)n);
	for (int32_t i = 0; i < n; ++i) {
		if (ql[i] < 0) {
			gwf_set_error("gwf_srv_submit: negative read length");
			return GWF_E_BAD_INPUT;
		}
		r->offs[(size_t)i] = tot, tot += ql[i];
	}
	r->seqs.resize((size_t)tot + 1);
	for (int32_t i = 0; i < n; ++i) memcpy(r->seqs.data() + r->offs[(size_t)i], seqs + offs[i], (size_t)ql[i]);
	r->ql.assign(ql, ql + n);
	r->v0.assign(v0, v0 + n);
	r->t_submit = now_s();
	{
		std::lock_guard<std::mutex> lk(S->mu);
		if (S->stop) return GWF_E_BUSY;
		r->id = S->next_id++;
		S->all[r->id] = r;
		S->pending.push_back(r);
	}
	S->cv_work.notify_one();
	return r->id;
}

static int fill(const Request &r, int32_t *dist, int32_t *status)
{
	if (dist) memcpy(dist, r.dist.data(), sizeof(int32_t) * (size_t)r.n);
	if (status) memcpy(status, r.status.data(), sizeof(int32_t) * (size_t)r.n);
	return 1;
}

extern "C" int gwf_srv_poll(gwf_srv_t *S, int64_t req, int32_t *dist, int32_t *status)
{
	if (!S) return GWF_E_BAD_INPUT;
	std::lock_guard<std::mutex> lk(S->mu);
	auto it = S->all.find(req);
	if (it == S->all.end()) return GWF_E_BAD_INPUT;
	if (!it->second->done) return 0;
	return fill(*it->second, dist, status);
}

extern "C" int gwf_srv_wait(gwf_srv_t *S, int64_t req, int32_t *dist, int32_t *status, double timeout_s)
{
	if (!S) return GWF_E_BAD_INPUT;
	std::unique_lock<std::mutex> lk(S->mu);
	auto it = S->all.find(req);
	if (it == S->all.end()) return GWF_E_BAD_INPUT;
	auto r = it->second;
	if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r->done; }))
		return GWF_E_TIMEOUT;
	return fill(*r, dist, status);
}

extern "C" int gwf_srv_times(gwf_srv_t *S, int64_t req, double *t_submit, double *t_admit, double *t_done)
{
	if (!S) return GWF_E_BAD_INPUT;
	std::lock_guard<std::mutex> lk(S->mu);
	auto it = S->all.find(req);
	if (it == S->all.end() || !it->second->done) return GWF_E_BAD_INPUT;
	if (t_submit) *t_submit = it->second->t_submit;
	if (t_admit) *t_admit = it->second->t_admit;
	if (t_done) *t_done = it->second->t_done;
	return 0;
}

extern "C" void gwf_srv_destroy(gwf_srv_t *S)
{
	if (!S) return;
	{
		std::lock_guard<std::mutex> lk(S->mu);
		S->stop = true;
	}
	S->cv_work.notify_all();
	for (auto &t : S->lanes) t.join();
	for (Engine *E : S->engines) delete E;
	delete S;
}
