// lg_pagerank.cu - PageRank, pull direction, FP64, over a snapshot's in-CSR.
//
// Reference: ll_b_pagerank_pull_ext<Graph,double>::run
// (benchmark/benchmarks/pagerank.h:98-182): pr0 = 1/N (N = max_nodes),
// then `max` times  pr'[t] = (1-d)/N + d * sum_{w in in(t)} pr[w]/out_degree(w),
// dangling mass dropped.
//
// One launch per iteration.  Instead of gathering pr[w] and out_degree(w)
// per edge (two dependent random loads in the reference), each iteration
// writes contrib'[t] = pr'[t] / out_degree(t) next to the rank, so an edge
// costs one coalesced 4-byte id load and one 8-byte gather.  The division is
// the one the reference performs per edge, so the gathered values are
// bit-identical; only the summation order differs (FP64, well within 1e-12).
//
// Work split per launch:
//   * hub CTAs: vertices with >= kHubSlots slots are cut into kHubChunk-slot
//     chunks, one CTA each; the last CTA of a hub (threadfence + counter)
//     adds the partials in chunk order, so results are deterministic;
//   * group warps: every other vertex, 32 consecutive vertices per warp,
//     walked with warp_expand and a segmented warp sum.
#include "lg_device.cuh"

namespace lg {

struct PrArgs {
	SnapCsr in;
	const uint32_t* outdeg;
	const double* contrib;
	double* contrib_next;
	double* pr_out;            // written when non-null (last iteration)
	double base;               // (1 - d) / N
	double d;
	const uint32_t* hubs;
	const uint32_t* hub_chunk_off;
	uint32_t n_hubs;
	uint32_t n_hub_chunks;
	double* hub_partial;
	uint32_t* hub_done;
};

constexpr int kPrThreads = 256;
constexpr int kPrWarps = kPrThreads / 32;

__device__ __forceinline__ void pr_finish(const PrArgs& a, uint32_t v, double s) {
	double pr = __dadd_rn(a.base, __dmul_rn(a.d, s));
	uint32_t dg = __ldg(a.outdeg + v);
	a.contrib_next[v] = dg ? pr / (double)dg : 0.0;
	if (a.pr_out) a.pr_out[v] = pr;
}

// Deterministic CTA sum (fixed shuffle tree, then warp sums in order).
__device__ __forceinline__ double block_sum(double x, double* red) {
	for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	if (lane == 0) red[w] = x;
	__syncthreads();
	double s = 0;
	if (threadIdx.x == 0)
		for (int i = 0; i < kPrWarps; i++) s += red[i];
	return s;
}

__global__ void __launch_bounds__(kPrThreads)
pr_pull_step(PrArgs a) {
	__shared__ double acc[kPrWarps][32];
	__shared__ uint2 hfr[LG_MAX_LEVELS];
	__shared__ uint32_t hstart[LG_MAX_LEVELS + 1];
	__shared__ double red[kPrWarps];
	__shared__ int last;

	if (blockIdx.x < a.n_hub_chunks) {
		// ---- one chunk of a hub vertex ----
		const uint32_t c = blockIdx.x;
		uint32_t lo = 0, hi = a.n_hubs;
		while (hi - lo > 1) {
			uint32_t mid = (lo + hi) >> 1;
			if (__ldg(a.hub_chunk_off + mid) <= c) lo = mid; else hi = mid;
		}
		const uint32_t h = lo, v = __ldg(a.hubs + h);
		const uint32_t j = c - __ldg(a.hub_chunk_off + h);
		const uint32_t nch = __ldg(a.hub_chunk_off + h + 1) - __ldg(a.hub_chunk_off + h);
		const uint32_t f0 = __ldg(a.in.frag_off + v);
		const uint32_t nf = __ldg(a.in.frag_off + v + 1) - f0;
		if (threadIdx.x == 0) {
			uint32_t s = 0;
			for (uint32_t f = 0; f < nf; f++) {
				uint2 fr = a.in.frags[f0 + f];
				hfr[f] = fr;
				hstart[f] = s;
				s += frag_len(fr);
			}
			hstart[nf] = s;
		}
		__syncthreads();
		const uint32_t total = hstart[nf];
		const uint32_t k0 = j * kHubChunk;
		const uint32_t k1 = min(total, k0 + kHubChunk);
		double x = 0.0;
		uint32_t f = 0;
		for (uint32_t k = k0 + threadIdx.x; k < k1; k += kPrThreads) {
			while (hstart[f + 1] <= k) f++;
			uint2 fr = hfr[f];
			uint32_t lv = frag_level(fr), ix = fr.x + (k - hstart[f]);
			if (!slot_deleted(a.in.lt, lv, ix))
				x += __ldg(a.contrib + __ldg(a.in.lt->ids[lv] + ix));
		}
		double s = block_sum(x, red);
		if (threadIdx.x == 0) {
			a.hub_partial[c] = s;
			__threadfence();
			uint32_t prev = atomicAdd(a.hub_done + h, 1u);
			last = (prev == nch - 1);
		}
		__syncthreads();
		if (last && threadIdx.x == 0) {
			__threadfence();
			const uint32_t c0 = __ldg(a.hub_chunk_off + h);
			double t = 0.0;
			for (uint32_t i = 0; i < nch; i++) t += __ldcg(a.hub_partial + c0 + i);
			pr_finish(a, v, t);
			a.hub_done[h] = 0;
		}
		return;
	}

	// ---- 32 consecutive vertices per warp ----
	const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
	const uint64_t v64 = ((uint64_t)(blockIdx.x - a.n_hub_chunks) * kPrWarps + w) * 32 + lane;
	const bool valid = v64 < a.in.V;
	const uint32_t v = (uint32_t)v64;
	uint32_t f0 = 0, cnt = 0;
	if (valid) cnt = vertex_slots(a.in, v, &f0);
	const bool hub = cnt >= kHubSlots;
	if (hub) cnt = 0;
	acc[w][lane] = 0.0;
	__syncwarp();
	warp_expand(a.in, cnt, f0,
		[&](bool act, uint32_t o, uint32_t nbr, uint32_t, uint32_t) {
			double x = act ? __ldg(a.contrib + nbr) : 0.0;
			bool tail;
			double s = warp_segsum(x, o, &tail);
			if (tail) acc[w][o] += s;
			__syncwarp();
		});
	if (valid && !hub) pr_finish(a, v, acc[w][lane]);
}

__global__ void pr_init(const uint32_t* outdeg, uint64_t V, double pr0,
		double* contrib, double* pr_out) {
	uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	uint32_t dg = outdeg[v];
	contrib[v] = dg ? pr0 / (double)dg : 0.0;
	if (pr_out) pr_out[v] = pr0;
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_pagerank_pull(lg_snapshot* sn, int iterations,
		double damping, double* ranks) {
	clear_error();
	if (!sn || !ranks) return set_error(LG_EINVAL, "null argument");
	if (!(damping > 0.0 && damping < 1.0))
		return set_error(LG_EINVAL, "damping must be in (0, 1)");
	if (iterations < 0) return set_error(LG_EINVAL, "iterations must be >= 0");
	if (!sn->in.present)
		return set_error(LG_ESTATE, "pull PageRank needs the in-CSR (reverse edges)");
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	const double N = (double)V;
	const double pr0 = 1.0 / N;
	const double base = (1.0 - damping) / N;

	DevBuf* sc = s->scratch;
	LG_TRY(sc[0].reserve(V * sizeof(double)));
	LG_TRY(sc[1].reserve(V * sizeof(double)));
	LG_TRY(sc[2].reserve(std::max<uint32_t>(sn->in.n_hub_chunks, 1) * sizeof(double)));
	LG_TRY(sc[3].reserve(std::max<uint32_t>(sn->in.n_hubs, 1) * sizeof(uint32_t)));
	LG_CUDA(cudaMemsetAsync(sc[3].p, 0, std::max<uint32_t>(sn->in.n_hubs, 1) * 4, st),
			"memset");
	const bool dev_out = is_device_pointer(ranks);
	double* pr_buf = ranks;
	if (!dev_out) {
		LG_TRY(sc[4].reserve(V * sizeof(double)));
		pr_buf = sc[4].as<double>();
	}
	pr_init<<<grid_for(V, 256), 256, 0, st>>>(sn->out.deg.as<uint32_t>(), V, pr0,
			sc[0].as<double>(), iterations == 0 ? pr_buf : nullptr);
	LG_CUDA(cudaGetLastError(), "pr_init");
	s->launches++;

	PrArgs a;
	a.in = sn->view(1);
	a.outdeg = sn->out.deg.as<uint32_t>();
	a.base = base;
	a.d = damping;
	a.hubs = sn->in.hubs.as<uint32_t>();
	a.hub_chunk_off = sn->in.hub_chunk_off.as<uint32_t>();
	a.n_hubs = sn->in.n_hubs;
	a.n_hub_chunks = sn->in.n_hub_chunks;
	a.hub_partial = sc[2].as<double>();
	a.hub_done = sc[3].as<uint32_t>();
	const uint64_t groups = (V + kPrThreads - 1) / kPrThreads;
	const uint64_t grid = groups + a.n_hub_chunks;
	if (grid > 0x7fffffffull) return set_error(LG_ENOTSUP, "graph too large for one launch");
	for (int it = 0; it < iterations; it++) {
		a.contrib = sc[it & 1].as<double>();
		a.contrib_next = sc[(it + 1) & 1].as<double>();
		a.pr_out = (it == iterations - 1) ? pr_buf : nullptr;
		pr_pull_step<<<(unsigned)grid, kPrThreads, 0, st>>>(a);
	}
	LG_CUDA(cudaGetLastError(), "pr_pull_step");
	s->launches += iterations;
	if (!dev_out) {
		LG_TRY(copy_out(s, ranks, pr_buf, V * sizeof(double)));
		LG_CUDA(cudaStreamSynchronize(st), "pagerank");
	}
	return LG_OK;
}
