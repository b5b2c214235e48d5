// gwf_runtime.h — internal host structures of libgwfa_b200 (device graphs, engines, batches).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/gwfa.h"
#include "gwf_device.cuh"

struct DBuf { // grow-only device buffer
	void *p = nullptr;
	size_t cap = 0;
	int ensure(size_t n);
	void release();
};

struct HBuf { // grow-only pinned host buffer
	void *p = nullptr;
	size_t cap = 0;
	int ensure(size_t n);
	void release();
};

struct GraphDev { // device-resident copy of one gwf_graph_t
	int device = -1;
	uint32_t n_vtx = 0, n_arc = 0;
	int32_t pure = 0, dens_milli = 1;
	uint64_t total_len = 0;
	DBuf len, base, pk, raw, arc_off, arc;
	DBuf arc_key; // entry id per arc, only when some vertex's in-arcs carry different overlaps
	gwfb::DevGraph view() const;
	~GraphDev();
};

struct Engine { // per-device launch state: stream, events, warp arenas
	int device = 0;
	int sm_count = 0;
	int persistent_ctas_per_sm = 1;
	int classes_ctas_per_sm = 1;
	int64_t mem_budget = 0; // device bytes the arenas may take
	cudaStream_t stream = nullptr;
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
	DBuf pk_off, order, head, retry_list, retry_n, ws, slot_off, w_out;
	HBuf h_small;
	HBuf h_stage;                              // two pinned chunks for pageable uploads
	cudaEvent_t stage_ev[2] = {nullptr, nullptr};
	~Engine();
};

struct Batch { // reads resident on the device
	int32_t n = 0, v1 = -1, max_ql = 0;
	int32_t n_in = 0;   // the caller's reads; n = 2 n_in with both strands (reverse complements after)
	bool both = false;
	int64_t pk_words = 0;
	uint64_t generation = 0;          // bumped by every load (graph key)
	int32_t dom_bucket = 0;           // length bucket with the largest sum of ql^2 (autotuner)
	cudaGraphExec_t gexec = nullptr;  // captured level-0 sequence of the persistent form
	uint64_t gkey[9] = {};
	std::vector<int32_t> h_ql;
	HBuf h_meta; // pinned: raw offsets, packed offsets, queue order; results on the way back
	DBuf raw, raw_off, ql, v0, pk, pk_off, pure, dist, status, steps, order_ql;
	// read classes of the persistent form (reads aligned by groups of warps), cached per layout
	DBuf order_cls;
	uint64_t cls_key = ~0ULL, cls_gen = ~0ULL; // layout key and the batch generation it was made for
	int32_t cls_n = 0, cls_nw[4] = {}, cls_cnt[4] = {}, cls_cap[4] = {}, cls_start[4] = {};
	void release();
};

GraphDev *gwf_find_graph(const gwf_graph_t *g);
Engine *gwf_engine(int dev);
int gwf_select_device(int want, int *dev_out);
int gwf_batch_load(Engine &E, Batch &B, int32_t n, const char *seqs, const int64_t *offs,
                   const int32_t *ql, const int32_t *v0, int32_t v1, bool both = false);
int gwf_batch_exec(Engine &E, const GraphDev &G, Batch &B, int32_t mode, int32_t flags,
                   int ctas_per_sm, float *ms, int *launches_out, int use_graph = 0, int32_t max_lag = 0,
                   int32_t warps_per_read = 0);
int gwf_batch_fetch(Engine &E, Batch &B, int32_t *dist, int32_t *status, int32_t *strand = nullptr);
namespace gwfb {
struct KParams;
struct SrvParams;
}
cudaError_t gwf_launch_persistent(const gwfb::KParams &p, int ctas, int threads, cudaStream_t s);
cudaError_t gwf_launch_serve(const gwfb::SrvParams &p, int ctas, int threads, cudaStream_t s,
                             int warps_per_read = 1);
int gwf_serve_ctas_per_sm(int warps_per_read = 1);

#include <mutex>
std::mutex &gwf_batch_mutex();   // serialises batch calls (one engine per device)
int gwf_tune_bucket(int32_t ql); // autotuner length bucket of a read
int gwf_tune_lookup(int device, int32_t bucket, int32_t *form, int32_t *ctas_per_sm);
int gwf_tune_lookup_nw(int device, int32_t bucket); // tuned warps per read, 0 = none
