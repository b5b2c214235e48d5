// gwf_serve.cu — continuous-batching request loop on a device-resident graph.
//
// One resident kernel (k_serve) runs on the device; its warps pull single reads from a queue in
// device memory. A host pump thread does everything else:
//   * admission: reads of queued requests are admitted in FIFO order while a slot is free and the
//     arena pool (a fixed device-memory budget) has room for the read's wavefront arena, sized for
//     its own length; the read's bases are copied into its arena and its queue entry published;
//   * completion: the kernel writes one record per read into host-mapped memory; the pump frees
//     the arena and the slot, and completes a request when its last read is done;
//   * retry: a read that overflows its arena comes back with GWF_E_CAPACITY and is queued again
//     in a 4x larger arena (up to three times), ahead of new reads;
//   * liveness: the kernel closes as a whole a few milliseconds after the queue runs dry with no
//     warp busy; the pump relaunches it when positions are queued and it has ended.
// Reads that arrive while others are on the device therefore start as soon as a warp and arena
// memory are free, and results do not depend on what else is in flight.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gwfa.h"
#define GWF_KERNELS_DECL_ONLY
#include "gwf_kernels.cuh"
#include "gwf_runtime.h"
#include "gwfa_internal.h"

using gwfb::SrvDone;
using gwfb::SrvEntry;

namespace {

double now_s()
{
	return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

constexpr int kMaxLevel = 3;         // arena classes 1x, 4x, 16x, 64x, as the batch path
constexpr int64_t kIdleNs = 5000000; // 5 ms
constexpr int64_t kMaxIdleNs = 120LL * 1000000000LL;

// Best-fit allocator over [0, cap) in 256-byte units, with coalescing.
class Pool {
public:
	void init(int64_t cap)
	{
		cap_ = cap & ~255LL;
		by_off_.clear(), by_size_.clear();
		if (cap_ > 0) insert(0, cap_);
		used_ = 0;
	}
	int64_t alloc(int64_t bytes)
	{
		bytes = (bytes + 255) & ~255LL;
		auto it = by_size_.lower_bound({bytes, -1});
		if (it == by_size_.end()) return -1;
		const int64_t off = it->second, sz = it->first;
		erase(off, sz);
		if (sz > bytes) insert(off + bytes, sz - bytes);
		used_ += bytes;
		return off;
	}
	void release(int64_t off, int64_t bytes)
	{
		bytes = (bytes + 255) & ~255LL;
		used_ -= bytes;
		auto nx = by_off_.lower_bound(off);
		if (nx != by_off_.end() && nx->first == off + bytes) {
			const int64_t s = nx->second;
			erase(nx->first, s);
			bytes += s;
		}
		auto pv = by_off_.lower_bound(off);
		if (pv != by_off_.begin()) {
			--pv;
			if (pv->first + pv->second == off) {
				const int64_t o = pv->first, s = pv->second;
				erase(o, s);
				off = o, bytes += s;
			}
		}
		insert(off, bytes);
	}
	int64_t used() const { return used_; }
	int64_t cap() const { return cap_; }

private:
	void insert(int64_t off, int64_t sz) { by_off_[off] = sz, by_size_.insert({sz, off}); }
	void erase(int64_t off, int64_t sz) { by_off_.erase(off), by_size_.erase({sz, off}); }
	std::map<int64_t, int64_t> by_off_;
	std::set<std::pair<int64_t, int64_t>> by_size_;
	int64_t cap_ = 0, used_ = 0;
};

struct Request {
	int64_t id = 0;
	int32_t n = 0, v1 = -1;
	int32_t n_in = 0; // the caller's reads; with both strands n = 2 n_in (reverse complements after)
	std::vector<char> seqs;
	std::vector<int64_t> offs;
	std::vector<int32_t> ql, v0, dist, status;
	int32_t next_read = 0, n_done = 0;
	double t_submit = 0, t_admit = 0, t_done = 0;
	bool done = false;
};

struct Slot {
	std::shared_ptr<Request> r;
	int32_t read = 0, level = 0;
	int64_t off = -1, bytes = 0;
};

} // namespace

struct gwf_srv_s {
	const gwf_graph_t *g = nullptr;
	GraphDev *G = nullptr;
	int device = 0, sm_count = 0, ctas = 0;
	int32_t flags = 0, max_lag = 0, nw = 1; // nw: warps that align one read together
	int64_t budget = 0;
	uint32_t qcap = 0, ccap = 0;
	int cq_shift = 0;
	cudaStream_t kstream = nullptr, fstream = nullptr;
	cudaEvent_t kdone = nullptr;
	bool kernel_running = false;
	// device memory: arena pool, queue ring, control words
	DBuf pool_mem, q_mem, ctl;
	// host memory: completion ring + error word (mapped), queue mirror + control values (pinned)
	void *mapped = nullptr, *pinned = nullptr;
	volatile SrvDone *cq = nullptr;
	volatile int32_t *err = nullptr;
	SrvDone *cq_dev = nullptr;
	int32_t *err_dev = nullptr;
	SrvEntry *h_q = nullptr;
	unsigned long long *h_tail = nullptr, *h_head = nullptr;
	int32_t *h_stop = nullptr;
	char *stage = nullptr; // pinned staging of read bases on their way to the arenas
	int64_t stage_cap = 0;
	Pool pool;
	std::vector<Slot> slots;
	std::vector<int32_t> free_slots;
	std::deque<int32_t> retry;
	std::deque<std::shared_ptr<Request>> pending;
	std::unordered_map<int64_t, std::shared_ptr<Request>> all;
	uint64_t q_pos = 0, cq_pos = 0;
	int64_t in_flight = 0;
	std::mutex mu;
	std::condition_variable cv_work, cv_done;
	bool stop = false;
	int fatal = 0;
	int64_t next_id = 0;
	std::thread pump;
	int64_t launches = 0, retries = 0;
};

namespace {

// control words: the ones every idle warp polls share one 128-byte line, the ones that busy
// warps update sit on lines of their own
unsigned long long *q_tail_dev(gwf_srv_s *S) { return (unsigned long long *)S->ctl.p; }
unsigned long long *q_head_dev(gwf_srv_s *S) { return (unsigned long long *)S->ctl.p + 1; }
int32_t *stop_dev(gwf_srv_s *S) { return (int32_t *)((unsigned long long *)S->ctl.p + 2); }
unsigned long long *cq_tail_dev(gwf_srv_s *S) { return (unsigned long long *)((char *)S->ctl.p + 128); }
int32_t *busy_dev(gwf_srv_s *S) { return (int32_t *)((char *)S->ctl.p + 256); }

int64_t arena_bytes(const gwf_srv_s *S, int32_t ql, int32_t level)
{
	const gwfb::Caps c = gwfb::caps_for(ql, level, S->G->dens_milli);
	return gwfb::srv_al256(gwfb::srv_qbytes(ql) + gwfb::ws_layout(c).total);
}

// Called with S->mu held.
void finish_read(gwf_srv_s *S, const std::shared_ptr<Request> &r, int32_t i, int32_t dist, int32_t st)
{
	r->dist[(size_t)i] = st == 0 ? dist : -1;
	r->status[(size_t)i] = st;
	if (++r->n_done == r->n) {
		r->t_done = now_s();
		r->done = true;
		S->cv_done.notify_all();
	}
}

void release_slot(gwf_srv_s *S, int32_t tag)
{
	Slot &sl = S->slots[(size_t)tag];
	sl.r.reset();
	sl.off = -1;
	S->free_slots.push_back(tag);
	--S->in_flight;
}

// Fails every read that has not completed (device error). Called with S->mu held.
void fail_all(gwf_srv_s *S, int32_t code)
{
	S->fatal = code;
	for (size_t t = 0; t < S->slots.size(); ++t)
		if (S->slots[t].r) finish_read(S, S->slots[t].r, S->slots[t].read, -1, code);
	for (auto &r : S->pending)
		while (r->next_read < r->n) finish_read(S, r, r->next_read++, -1, code);
	S->pending.clear();
	S->retry.clear();
}

// Drains completion records. Called with S->mu held; returns the number consumed.
int drain(gwf_srv_s *S)
{
	int n = 0;
	for (;;) {
		volatile SrvDone *d = S->cq + (S->cq_pos & (S->ccap - 1));
		if (d->gen != (int32_t)((S->cq_pos >> S->cq_shift) + 1)) break;
		std::atomic_thread_fence(std::memory_order_acquire);
		const int32_t tag = d->tag, dist = d->dist, st = d->status;
		++S->cq_pos, ++n;
		if (tag < 0 || (size_t)tag >= S->slots.size() || !S->slots[(size_t)tag].r) {
			fail_all(S, GWF_E_CUDA);
			gwf_set_error("gwf_srv: completion record for an unknown slot");
			return n;
		}
		Slot &sl = S->slots[(size_t)tag];
		S->pool.release(sl.off, sl.bytes);
		sl.off = -1;
		if (st == GWF_E_CAPACITY && sl.level < kMaxLevel) {
			++sl.level;
			++S->retries;
			S->retry.push_back(tag); // keeps its slot; re-admitted with a larger arena
			continue;
		}
		finish_read(S, sl.r, sl.read, dist, st);
		release_slot(S, tag);
	}
	return n;
}

// Admits retries, then new reads, while slots and arena memory last; copies their bases and
// publishes their queue entries. Called with S->mu held; returns the number published.
int admit(gwf_srv_s *S)
{
	std::vector<int32_t> batch;
	const uint64_t first = S->q_pos;
	auto place = [&](int32_t tag) -> int {
		Slot &sl = S->slots[(size_t)tag];
		const int32_t ql = sl.r->ql[(size_t)sl.read];
		const int64_t bytes = arena_bytes(S, ql, sl.level);
		if (bytes > S->pool.cap()) return -1; // can never fit
		const int64_t off = S->pool.alloc(bytes);
		if (off < 0) return 0;
		sl.off = off, sl.bytes = bytes;
		return 1;
	};
	while (!S->retry.empty()) {
		const int32_t tag = S->retry.front();
		const int rc = place(tag);
		if (rc == 0) break;
		S->retry.pop_front();
		if (rc < 0) {
			Slot &sl = S->slots[(size_t)tag];
			finish_read(S, sl.r, sl.read, -1, GWF_E_CAPACITY);
			release_slot(S, tag);
			continue;
		}
		batch.push_back(tag);
	}
	while (S->retry.empty() && !S->pending.empty() && !S->free_slots.empty()) {
		auto r = S->pending.front();
		const int32_t i = r->next_read;
		if (r->ql[(size_t)i] <= 0) {
			finish_read(S, r, i, -1, GWF_E_BAD_INPUT);
		} else {
			const int32_t tag = S->free_slots.back();
			Slot &sl = S->slots[(size_t)tag];
			sl.r = r, sl.read = i, sl.level = 0;
			const int rc = place(tag);
			if (rc == 0) {
				sl.r.reset();
				break; // wait for arena memory
			}
			S->free_slots.pop_back();
			++S->in_flight;
			if (rc < 0) {
				finish_read(S, r, i, -1, GWF_E_CAPACITY);
				release_slot(S, tag);
			} else {
				batch.push_back(tag);
			}
		}
		if (r->t_admit == 0) r->t_admit = now_s();
		if (++r->next_read == r->n) S->pending.pop_front();
	}
	if (batch.empty()) return 0;
	int64_t staged = 0;
	for (int32_t tag : batch) {
		const Slot &sl = S->slots[(size_t)tag];
		const Request &r = *sl.r;
		const int32_t ql = r.ql[(size_t)sl.read];
		uint8_t *raw = (uint8_t *)S->pool_mem.p + sl.off + 256 + gwfb::srv_pk_bytes(ql);
		const char *src = r.seqs.data() + r.offs[(size_t)sl.read];
		if (ql <= S->stage_cap) { // through pinned staging: an asynchronous DMA
			if (staged + ql > S->stage_cap) {
				if (cudaStreamSynchronize(S->fstream) != cudaSuccess) return -1;
				staged = 0;
			}
			memcpy(S->stage + staged, src, (size_t)ql);
			src = S->stage + staged;
			staged += (ql + 15) & ~15;
		}
		if (cudaMemcpyAsync(raw, src, (size_t)ql, cudaMemcpyHostToDevice, S->fstream) != cudaSuccess) return -1;
		SrvEntry &e = S->h_q[S->q_pos & (S->qcap - 1)];
		memset(&e, 0, sizeof e);
		e.seq = (uint32_t)(S->q_pos + 1);
		e.tag = tag;
		e.arena_off = sl.off;
		e.arena_bytes = sl.bytes;
		e.ql = ql;
		e.v0 = r.v0[(size_t)sl.read];
		e.v1 = r.v1;
		e.level = sl.level;
		++S->q_pos;
	}
	// queue entries (two copies when the range wraps), then the tail that publishes them
	const uint64_t mask = S->qcap - 1;
	for (uint64_t p = first; p < S->q_pos;) {
		const uint64_t i = p & mask;
		const uint64_t n = std::min<uint64_t>(S->q_pos - p, S->qcap - i);
		if (cudaMemcpyAsync((SrvEntry *)S->q_mem.p + i, S->h_q + i, n * sizeof(SrvEntry), cudaMemcpyHostToDevice,
		                    S->fstream) != cudaSuccess)
			return -1;
		p += n;
	}
	*S->h_tail = S->q_pos;
	if (cudaMemcpyAsync(q_tail_dev(S), S->h_tail, 8, cudaMemcpyHostToDevice, S->fstream) != cudaSuccess ||
	    cudaStreamSynchronize(S->fstream) != cudaSuccess) // pinned sources are reused next round
		return -1;
	return (int)batch.size();
}

int launch(gwf_srv_s *S)
{
	// the previous kernel left q_head marked closed: clear the mark (nothing runs on the device)
	unsigned long long head = 0;
	if (cudaMemcpy(&head, q_head_dev(S), 8, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
	if (head & gwfb::SRV_CLOSED) {
		*S->h_head = head & ~gwfb::SRV_CLOSED;
		if (cudaMemcpyAsync(q_head_dev(S), S->h_head, 8, cudaMemcpyHostToDevice, S->kstream) != cudaSuccess)
			return -1;
	}
	gwfb::SrvParams p;
	memset(&p, 0, sizeof p);
	p.g = S->G->view();
	p.q = (const SrvEntry *)S->q_mem.p;
	p.q_tail = q_tail_dev(S);
	p.q_head = q_head_dev(S);
	p.stop = stop_dev(S);
	p.busy = busy_dev(S);
	p.cq_tail = cq_tail_dev(S);
	p.cq = S->cq_dev;
	p.err = S->err_dev;
	p.arena = (uint8_t *)S->pool_mem.p;
	p.qmask = S->qcap - 1;
	p.cmask = S->ccap - 1;
	p.cq_shift = S->cq_shift;
	p.dens_milli = S->G->dens_milli;
	p.flags = S->flags;
	p.max_lag = S->max_lag;
	p.idle_ns = kIdleNs;
	p.max_idle_ns = kMaxIdleNs;
	if (gwf_launch_serve(p, S->ctas, 256, S->kstream, S->nw) != cudaSuccess) return -1;
	if (cudaEventRecord(S->kdone, S->kstream) != cudaSuccess) return -1;
	S->kernel_running = true;
	++S->launches;
	return 0;
}

void pump_main(gwf_srv_s *S)
{
	cudaSetDevice(S->device);
	std::unique_lock<std::mutex> lk(S->mu);
	for (;;) {
		int progress = 0;
		if (!S->fatal) {
			progress += drain(S);
			if (*S->err) {
				fail_all(S, GWF_E_CUDA);
				gwf_set_error("gwf_srv: device queue error");
			}
		}
		if (!S->fatal) {
			const int a = admit(S);
			if (a < 0) {
				cudaGetLastError();
				fail_all(S, GWF_E_CUDA);
				gwf_set_error("gwf_srv: copy to the device failed");
			}
			progress += a > 0 ? a : 0;
		}
		if (!S->fatal && S->kernel_running) {
			const cudaError_t e = cudaEventQuery(S->kdone);
			if (e == cudaSuccess) {
				S->kernel_running = false;
				progress += drain(S); // every claimed read has its record now
			} else if (e != cudaErrorNotReady) {
				cudaGetLastError();
				fail_all(S, GWF_E_CUDA);
				gwf_set_errorf("gwf_srv: kernel failed: %s", cudaGetErrorString(e));
			}
		}
		if (!S->fatal && !S->kernel_running && S->q_pos > S->cq_pos) {
			if (launch(S)) {
				cudaGetLastError();
				fail_all(S, GWF_E_CUDA);
				gwf_set_error("gwf_srv: kernel launch failed");
			}
		}
		const bool idle = S->pending.empty() && S->in_flight == 0;
		if (S->stop && (idle || S->fatal)) break;
		if (!progress) S->cv_work.wait_for(lk, std::chrono::microseconds(idle ? 2000 : 50));
	}
	lk.unlock();
	// end the kernel: idle warps see the stop word at their next poll
	*S->h_stop = 1;
	cudaMemcpyAsync(stop_dev(S), S->h_stop, 4, cudaMemcpyHostToDevice, S->fstream);
	cudaStreamSynchronize(S->fstream);
	cudaStreamSynchronize(S->kstream);
	cudaGetLastError();
}

void destroy_resources(gwf_srv_s *S)
{
	if (S->kstream) cudaStreamDestroy(S->kstream);
	if (S->fstream) cudaStreamDestroy(S->fstream);
	if (S->kdone) cudaEventDestroy(S->kdone);
	S->pool_mem.release(), S->q_mem.release(), S->ctl.release();
	if (S->mapped) cudaFreeHost(S->mapped);
	if (S->pinned) cudaFreeHost(S->pinned);
	cudaGetLastError();
}

uint32_t pow2_at_least(int64_t x)
{
	uint32_t p = 1;
	while ((int64_t)p < x && p < (1u << 30)) p <<= 1;
	return p;
}

} // namespace

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
	// serving is latency-first: a request waits for its slowest read, so by default each read gets
	// a group of 8 warps (p99 at 70% of peak: 0.79 s against 4.66 s with one warp, on reads of
	// 0.5-20 kbp on the 5 Mbp graph; peak 2,666 against 1,222 reads/s)
	S->nw = opt && opt->warps_per_read > 0 ? opt->warps_per_read : 8;
	if (S->nw != 1 && S->nw != 2 && S->nw != 4 && S->nw != 8) {
		gwf_set_error("gwf_srv_create: warps_per_read must be 0, 1, 2, 4 or 8");
		delete S;
		return nullptr;
	}
	S->max_lag = opt && (opt->flags & GWF_F_MAX_LAG) && opt->max_lag > 0 ? opt->max_lag : 0;
	size_t fr = 0, tot = 0;
	cudaMemGetInfo(&fr, &tot);
	S->budget = opt && opt->arena_budget_bytes > 0 ? opt->arena_budget_bytes : (int64_t)(fr / 4);
	const int32_t max_reads = opt && opt->max_inflight_reads > 0 ? opt->max_inflight_reads : 16384;
	S->qcap = pow2_at_least(2LL * max_reads);
	S->ccap = S->qcap;
	while ((1u << S->cq_shift) < S->ccap) ++S->cq_shift;
	cudaDeviceGetAttribute(&S->sm_count, cudaDevAttrMultiProcessorCount, dev);
	S->ctas = S->sm_count * gwf_serve_ctas_per_sm(S->nw);
	bool ok = cudaStreamCreateWithFlags(&S->kstream, cudaStreamNonBlocking) == cudaSuccess &&
	          cudaStreamCreateWithFlags(&S->fstream, cudaStreamNonBlocking) == cudaSuccess &&
	          cudaEventCreateWithFlags(&S->kdone, cudaEventDisableTiming) == cudaSuccess;
	ok = ok && S->pool_mem.ensure((size_t)S->budget) == 0 && S->q_mem.ensure(sizeof(SrvEntry) * S->qcap) == 0 &&
	     S->ctl.ensure(384) == 0;
	const size_t mapped_bytes = sizeof(SrvDone) * S->ccap + 256;
	S->stage_cap = 64LL << 20;
	const size_t pinned_bytes = sizeof(SrvEntry) * S->qcap + 256 + (size_t)S->stage_cap;
	ok = ok && cudaHostAlloc(&S->mapped, mapped_bytes, cudaHostAllocMapped) == cudaSuccess;
	ok = ok && cudaHostAlloc(&S->pinned, pinned_bytes, cudaHostAllocDefault) == cudaSuccess;
	if (ok) {
		memset(S->mapped, 0, mapped_bytes);
		memset(S->pinned, 0, pinned_bytes);
		void *dp = nullptr;
		ok = cudaHostGetDevicePointer(&dp, S->mapped, 0) == cudaSuccess;
		S->cq = (volatile SrvDone *)S->mapped;
		S->err = (volatile int32_t *)((char *)S->mapped + sizeof(SrvDone) * S->ccap);
		S->cq_dev = (SrvDone *)dp;
		S->err_dev = (int32_t *)((char *)dp + sizeof(SrvDone) * S->ccap);
		S->h_q = (SrvEntry *)S->pinned;
		S->h_tail = (unsigned long long *)((char *)S->pinned + sizeof(SrvEntry) * S->qcap);
		S->h_head = S->h_tail + 1;
		S->h_stop = (int32_t *)(S->h_tail + 2);
		S->stage = (char *)S->pinned + sizeof(SrvEntry) * S->qcap + 256;
	}
	ok = ok && cudaMemsetAsync(S->ctl.p, 0, 384, S->fstream) == cudaSuccess &&
	     cudaStreamSynchronize(S->fstream) == cudaSuccess;
	if (!ok) {
		cudaGetLastError();
		gwf_set_errorf("gwf_srv_create: device set-up failed (arena budget %lld bytes)", (long long)S->budget);
		destroy_resources(S);
		delete S;
		return nullptr;
	}
	S->pool.init(S->budget);
	S->slots.resize((size_t)max_reads);
	for (int32_t t = max_reads - 1; t >= 0; --t) S->free_slots.push_back(t);
	S->pump = std::thread(pump_main, S);
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
	const bool both = (S->flags & GWF_F_BOTH_STRANDS) != 0;
	if (both && n > INT32_MAX / 2) {
		gwf_set_error("gwf_srv_submit: too many reads");
		return GWF_E_BAD_INPUT;
	}
	r->n_in = n, r->n = both ? 2 * n : n, r->v1 = v1;
	int64_t tot = 0;
	r->offs.resize((size_t)r->n);
	for (int32_t i = 0; i < n; ++i) {
		if (ql[i] < 0) {
			gwf_set_error("gwf_srv_submit: negative read length");
			return GWF_E_BAD_INPUT;
		}
		if (v0[i] < 0 || (uint32_t)v0[i] >= S->G->n_vtx) {
			gwf_set_error("gwf_srv_submit: v0 out of range");
			return GWF_E_BAD_INPUT;
		}
		r->offs[(size_t)i] = tot, tot += ql[i];
	}
	r->seqs.resize((size_t)(both ? 2 * tot : tot) + 16);
	for (int32_t i = 0; i < n; ++i) memcpy(r->seqs.data() + r->offs[(size_t)i], seqs + offs[i], (size_t)ql[i]);
	r->ql.assign(ql, ql + n);
	r->v0.assign(v0, v0 + n);
	if (both) { // read n + i: the reverse complement of read i, from the same v0
		for (int32_t i = 0; i < n; ++i) {
			r->offs[(size_t)(n + i)] = tot + r->offs[(size_t)i];
			const char *src = r->seqs.data() + r->offs[(size_t)i];
			char *dst = r->seqs.data() + r->offs[(size_t)(n + i)];
			for (int32_t j = 0; j < ql[i]; ++j) dst[ql[i] - 1 - j] = (char)gwf_comp_base((unsigned char)src[j]);
		}
		r->ql.insert(r->ql.end(), ql, ql + n);
		r->v0.insert(r->v0.end(), v0, v0 + n);
	}
	r->dist.assign((size_t)r->n, -1);
	r->status.assign((size_t)r->n, 0);
	r->t_submit = now_s();
	{
		std::lock_guard<std::mutex> lk(S->mu);
		if (S->stop) return GWF_E_BUSY;
		if (S->fatal) {
			gwf_set_error("gwf_srv_submit: the server stopped after a device error");
			return S->fatal;
		}
		r->id = S->next_id++;
		S->all[r->id] = r;
		S->pending.push_back(r);
	}
	S->cv_work.notify_one();
	return r->id;
}

// Results of a finished request. With both strands, read i's two strands (i and n_in + i) give
// the smaller distance (the read itself on a tie) and the strand; a strand with a non-OK status
// makes the read's status that status and its distance -1 (as gwf_ed_batch_strand).
static int fill(const Request &r, int32_t *dist, int32_t *status, int32_t *strand = nullptr)
{
	if (r.n == r.n_in) {
		if (dist) memcpy(dist, r.dist.data(), sizeof(int32_t) * (size_t)r.n);
		if (status) memcpy(status, r.status.data(), sizeof(int32_t) * (size_t)r.n);
		if (strand)
			for (int32_t i = 0; i < r.n; ++i) strand[i] = r.dist[(size_t)i] >= 0 ? 0 : -1;
		return 1;
	}
	for (int32_t i = 0; i < r.n_in; ++i) {
		const int32_t df = r.dist[(size_t)i], dr = r.dist[(size_t)(r.n_in + i)];
		const int32_t sf = r.status[(size_t)i], sr = r.status[(size_t)(r.n_in + i)];
		int32_t d = -1, st = GWF_OK, k = -1;
		if (sf != GWF_OK || sr != GWF_OK) st = sf != GWF_OK ? sf : sr;
		else if (df >= 0 && (dr < 0 || df <= dr)) d = df, k = 0;
		else if (dr >= 0) d = dr, k = 1;
		if (dist) dist[i] = d;
		if (status) status[i] = st;
		if (strand) strand[i] = k;
	}
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

extern "C" int gwf_srv_strand(gwf_srv_t *S, int64_t req, int32_t *strand)
{
	if (!S || !strand) return GWF_E_BAD_INPUT;
	std::lock_guard<std::mutex> lk(S->mu);
	auto it = S->all.find(req);
	if (it == S->all.end() || !it->second->done) return GWF_E_BAD_INPUT;
	return fill(*it->second, nullptr, nullptr, strand) == 1 ? 0 : GWF_E_BAD_INPUT;
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

extern "C" int gwf_srv_stats(gwf_srv_t *S, int64_t *out, int32_t n_out)
{
	if (!S || (n_out > 0 && !out)) return GWF_E_BAD_INPUT;
	std::lock_guard<std::mutex> lk(S->mu);
	const int64_t v[GWF_SRV_NSTATS] = {S->launches, S->retries, S->pool.used(), (int64_t)S->q_pos,
	                                   (int64_t)S->cq_pos, S->in_flight, (int64_t)S->pending.size(),
	                                   S->kernel_running ? 1 : 0};
	for (int32_t i = 0; i < n_out && i < GWF_SRV_NSTATS; ++i) out[i] = v[i];
	return GWF_SRV_NSTATS;
}

extern "C" void gwf_srv_destroy(gwf_srv_t *S)
{
	if (!S) return;
	{
		std::lock_guard<std::mutex> lk(S->mu);
		S->stop = true;
	}
	S->cv_work.notify_all();
	if (S->pump.joinable()) S->pump.join();
	destroy_resources(S);
	delete S;
}
