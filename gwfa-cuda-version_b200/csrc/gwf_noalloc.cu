// gwf_noalloc.cu — gwf_ed_batch_noalloc: the batch alignment for callers that must not allocate.
//
// Some callers cannot call cudaMalloc at alignment time. Examples are a framework whose caching
// allocator owns the whole device heap, and a latency-bound serving loop where cudaMalloc's
// implicit device synchronisation is not acceptable. This entry point allocates nothing: the
// caller passes device buffers for the reads and the results, and the warp arenas, the queue
// head and two small index tables live in one file-scope device array of fixed size
// (kScratchBytes below). Every GPU that loads the library holds that array until the process
// exits. Reads are compared byte by byte (no packed copy is made), and an arena overflow is
// reported per read as GWF_E_CAPACITY: there is no larger arena to retry in.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/gwfa.h"
#define GWF_KERNELS_DECL_ONLY // KParams only: the kernels are compiled in gwf_runtime.cu
#include "gwf_kernels.cuh"
#include "gwf_runtime.h"
#include "gwfa_internal.h"

using namespace gwfb;

namespace {

constexpr int32_t kMaxReads = GWF_NOALLOC_MAX_READS;
constexpr int32_t kMaxQl = GWF_NOALLOC_MAX_QL;
constexpr int64_t kScratchBytes = GWF_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;
constexpr int kWarpsPerCta = 8;

// layout of the scratch array
constexpr int64_t kOffHead = 0;                                   // int32 queue head
constexpr int64_t kOffOrder = 256;                                // int32[kMaxReads]: 0, 1, 2, ...
constexpr int64_t kOffZero = kOffOrder + 4LL * kMaxReads;         // int64[kMaxReads] of zeros
constexpr int64_t kOffArena = (kOffZero + 8LL * kMaxReads + 255) & ~255LL;
static_assert(kOffArena < kScratchBytes, "scratch too small for its index tables");

} // namespace

static __device__ __align__(256) uint8_t g_noalloc_scratch[kScratchBytes];

__global__ void k_noalloc_init(uint8_t *scratch)
{
	int32_t *order = (int32_t *)(scratch + kOffOrder);
	int64_t *zero = (int64_t *)(scratch + kOffZero);
	for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kMaxReads; i += gridDim.x * blockDim.x)
		order[i] = i, zero[i] = 0;
}

// Per-device set-up: the device address of the scratch array (host code must not use the
// symbol itself, which is a host-side stand-in) and the index tables. Runs on the first call
// made on each device, with that device current.
static std::mutex g_noalloc_mu;
static uint8_t *g_noalloc_ptr[kMaxDevices];

static int noalloc_setup(int dev, cudaStream_t stream, uint8_t **out)
{
	std::lock_guard<std::mutex> lk(g_noalloc_mu);
	if (!g_noalloc_ptr[dev]) {
		void *ptr = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
		if (e != cudaSuccess) {
			gwf_set_errorf("gwf_ed_batch_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
			return GWF_E_CUDA;
		}
		k_noalloc_init<<<64, 256, 0, stream>>>((uint8_t *)ptr);
		e = cudaGetLastError();
		// the tables must be written before any call, from any thread or stream, reads them
		if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
		if (e != cudaSuccess) {
			gwf_set_errorf("gwf_ed_batch_noalloc: set-up kernel failed: %s", cudaGetErrorString(e));
			return GWF_E_CUDA;
		}
		g_noalloc_ptr[dev] = (uint8_t *)ptr;
	}
	*out = g_noalloc_ptr[dev];
	return 0;
}

extern "C" int gwf_ed_batch_noalloc(const gwf_graph_t *g, int32_t n, int32_t max_ql,
                                    const char *d_seqs, const int64_t *d_offs, const int32_t *d_ql,
                                    const int32_t *d_v0, int32_t v1, int32_t *d_dist,
                                    int32_t *d_status, int32_t flags, void *stream)
{
	if (n < 0 || n > kMaxReads) {
		gwf_set_errorf("gwf_ed_batch_noalloc: %d reads exceed the fixed limit of %d per call", n, kMaxReads);
		return GWF_E_CAPACITY;
	}
	if (max_ql > kMaxQl) {
		gwf_set_errorf("gwf_ed_batch_noalloc: reads of %d bases exceed the fixed limit of %d", max_ql, kMaxQl);
		return GWF_E_CAPACITY;
	}
	if (flags & ~GWF_F_EXACT_START) {
		gwf_set_error("gwf_ed_batch_noalloc: only GWF_F_EXACT_START is honoured (no lag pruning here)");
		return GWF_E_BAD_INPUT;
	}
	if (n == 0) return 0;
	if (!g || !d_seqs || !d_offs || !d_ql || !d_v0 || !d_dist || !d_status || max_ql <= 0) {
		gwf_set_error("gwf_ed_batch_noalloc: null pointer or empty reads");
		return GWF_E_BAD_INPUT;
	}
	if (((uintptr_t)d_seqs & 7) != 0) {
		gwf_set_error("gwf_ed_batch_noalloc: the read buffer must be 8-byte aligned");
		return GWF_E_BAD_INPUT;
	}
	GraphDev *G = gwf_find_graph(g);
	if (!G) {
		gwf_set_error("gwf_ed_batch_noalloc: graph not indexed on a device (call gwf_ed_index first)");
		return GWF_E_NOT_INDEXED;
	}
	if (v1 >= 0 && (uint32_t)v1 >= G->n_vtx) {
		gwf_set_error("gwf_ed_batch_noalloc: v1 out of range");
		return GWF_E_BAD_INPUT;
	}
	int dev = -1;
	if (cudaGetDevice(&dev) != cudaSuccess || dev != G->device || dev >= kMaxDevices) {
		cudaGetLastError();
		gwf_set_error("gwf_ed_batch_noalloc: the graph's device must be the current device");
		return GWF_E_CUDA;
	}
	cudaStream_t s = (cudaStream_t)stream;
	uint8_t *scratch = nullptr;
	int rc = noalloc_setup(dev, s, &scratch);
	if (rc) return rc;

	const Caps c = caps_for(kMaxQl, 0, G->dens_milli);
	const int64_t slot = ws_layout(c).total;
	// warps that the scratch holds, at most two CTAs per SM, and no more CTAs than the reads need;
	// a CTA's warps that find the queue empty leave at once
	int64_t warps = (kScratchBytes - kOffArena) / slot;
	int sms = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	warps = warps < (int64_t)sms * 2 * kWarpsPerCta ? warps : (int64_t)sms * 2 * kWarpsPerCta;
	const int64_t need = ((int64_t)n + kWarpsPerCta - 1) / kWarpsPerCta * kWarpsPerCta;
	warps = warps < need ? warps : need;
	warps = (warps / kWarpsPerCta) * kWarpsPerCta;
	if (warps < kWarpsPerCta) {
		gwf_set_errorf("gwf_ed_batch_noalloc: one warp arena (%lld bytes for this graph) does not fit the "
		               "%lld-byte scratch", (long long)slot * kWarpsPerCta, (long long)kScratchBytes);
		return GWF_E_CAPACITY;
	}
	// the queue head is the only state a call must start from zero (hash tables are cleared
	// per read by the kernel)
	cudaError_t e = cudaMemsetAsync(scratch + kOffHead, 0, sizeof(int32_t), s);
	if (e != cudaSuccess) {
		gwf_set_errorf("gwf_ed_batch_noalloc: %s", cudaGetErrorString(e));
		return GWF_E_CUDA;
	}
	KParams p;
	memset(&p, 0, sizeof p);
	p.g = G->view();
	p.g.pure = 0; // byte compares only: no packed copy of the reads
	p.r.raw = (const uint8_t *)d_seqs;
	p.r.raw_off = d_offs;
	p.r.ql = d_ql;
	p.r.v0 = d_v0;
	p.r.pk = nullptr;
	p.r.pk_off = (const int64_t *)(scratch + kOffZero);
	p.r.pure = nullptr;
	p.r.v1 = v1;
	p.r.n = n;
	p.order = (const int32_t *)(scratch + kOffOrder);
	p.n_order = n;
	p.head = (int32_t *)(scratch + kOffHead);
	p.ws = scratch + kOffArena;
	p.slot_bytes = slot;
	p.level = 0;
	p.dens_milli = G->dens_milli;
	p.ql_cap = kMaxQl;
	p.flags = flags;
	p.dist = d_dist;
	p.status = d_status;
	e = gwf_launch_persistent(p, (int)(warps / kWarpsPerCta), 32 * kWarpsPerCta, s);
	if (e != cudaSuccess) {
		gwf_set_errorf("gwf_ed_batch_noalloc: launch failed: %s", cudaGetErrorString(e));
		return GWF_E_CUDA;
	}
	return 0;
}
