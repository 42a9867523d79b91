// lg_pagerank.cu - PageRank, pull direction, FP64, over a snapshot's in-CSR.
//
// Reference: ll_b_pagerank_pull_ext<Graph,double>::run
// (benchmark/benchmarks/pagerank.h:98-182): pr0 = 1/N (N = max_nodes),
// then `max` times  pr'[t] = (1-d)/N + d * sum_{w in in(t)} pr[w]/out_degree(w),
// dangling mass dropped.
//
// Instead of gathering pr[w] and out_degree(w) per edge (two dependent random
// loads in the reference), each iteration writes contrib'[t] = pr'[t] /
// out_degree(t), so an edge costs one 4-byte id load and one 8-byte gather.
// The division is the one the reference performs per edge, so the gathered
// values are bit-identical; a vertex's sum is taken in the reference's
// iteration order except where it is split across blocks (FP64, well within
// 1e-12 in every case).
//
// Work split: the in-CSR slot space of all vertices (vertex order, each
// vertex's fragments newest first) is cut into blocks of kPrRange slots, one
// CTA each.  Phase 1 streams the block's slots: every thread takes
// kPrPerThread slots, finds each slot's fragment by binary search in a
// shared-memory table of the block's fragments, and issues all its id,
// deletion-word and contrib loads before using any of them, so a CTA keeps
// 2048 gathers in flight.  The values land in shared memory.  Phase 2 sums
// each vertex's values from shared memory (one thread per short vertex, a
// warp per long one).  A vertex whose slots straddle blocks leaves one
// partial per block (carry_first: it began before the block, carry_last: it
// runs past its end) and pr_fixup adds them in block order, so results are
// deterministic.
#include "lg_device.cuh"
#include "lg_expand.cuh"

#include <mutex>

namespace lg {

constexpr int kPrThreads = 128;
constexpr int kPrPerThread = 8;
constexpr uint32_t kPrRange = kPrThreads * kPrPerThread;        // 1024 slots
static_assert(kPrRange == kBlockSlots, "range_lb is computed for kBlockSlots");
constexpr uint32_t kPrMaxFrags = kPrRange + 2 * LG_MAX_LEVELS;   // fragments touching a block
constexpr uint32_t kPrLong = 64;       // entries with more slots are reduced by a warp

struct PrArgs {
	SnapCsr in;
	const uint32_t* pos;       // V + 1 in-CSR slot prefix
	const uint32_t* range_lb;  // nranges + 1 block entry bounds
	uint32_t total;            // pos[V]
	uint32_t nranges;
	const uint32_t* outdeg;
	const double* contrib;
	double* contrib_next;
	double* pr_out;            // written when non-null (last iteration)
	double base;               // (1 - d) / N
	double d;
	double* carry_first;       // per block
	double* carry_last;        // per block
};

__device__ __forceinline__ void pr_finish(const PrArgs& a, uint32_t v, double s) {
	const double pr = __dadd_rn(a.base, __dmul_rn(a.d, s));
	const uint32_t dg = __ldg(a.outdeg + v);
	a.contrib_next[v] = dg ? pr / (double)dg : 0.0;
	if (a.pr_out) a.pr_out[v] = pr;
}

__device__ __forceinline__ void pr_emit(const PrArgs& a, uint32_t r, uint32_t ra, uint32_t rb,
		uint32_t e, uint32_t start, uint32_t end, double s) {
	if (start < ra) a.carry_first[r] = s;          // began before the block
	else if (end > rb) a.carry_last[r] = s;        // runs past its end
	else pr_finish(a, e, s);
}

__global__ void __launch_bounds__(kPrThreads)
pr_pull_step(PrArgs a) {
	__shared__ double vals[kPrRange];
	__shared__ uint2 ftab[kPrMaxFrags];
	__shared__ uint32_t fstart[kPrMaxFrags + 1];
	__shared__ uint32_t fidx[kPrRange];
	__shared__ uint32_t longs[kPrRange / kPrLong + 2];
	__shared__ uint32_t sh_eb, sh_ee, sh_nlong;
	__shared__ uint32_t wsum[kPrThreads / 32];
	const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
	const uint32_t r = blockIdx.x;
	const bool last_range = r == a.nranges - 1;
	const uint32_t ra = r * kPrRange;
	const uint32_t rb = last_range ? a.total : min(a.total, ra + kPrRange);
	const uint32_t V = (uint32_t)a.in.V;
	if (tid == 0) {
		// entries of the block: those starting in [ra, rb), plus the one
		// straddling ra (precomputed lower bounds, see block_lower_bounds)
		uint32_t eb = __ldg(a.range_lb + r);
		if (eb > 0 && (eb == V || __ldg(a.pos + eb) > ra)) eb--;
		sh_eb = eb;
		sh_ee = last_range ? V : __ldg(a.range_lb + r + 1);
		sh_nlong = 0;
	}
	__syncthreads();
	const uint32_t eb = sh_eb, ee = sh_ee;

	// fragment table of the block's entries, with absolute virtual starts
	const uint32_t f_begin = __ldg(a.in.frag_off + eb);
	uint32_t nf = (ee > eb) ? __ldg(a.in.frag_off + ee) - f_begin : 0;
	if (nf > kPrMaxFrags) nf = kPrMaxFrags;   // cannot happen: fragments are non-empty
	const uint32_t vbase = __ldg(a.pos + eb);
	// nf <= kPrMaxFrags: every fragment of an entry inside the block has a
	// slot in the block, and only the two end entries add others
	uint32_t carry = 0;
	for (uint32_t c0 = 0; c0 < nf; c0 += kPrThreads) {
		const uint32_t i = c0 + tid;
		uint32_t len = 0;
		if (i < nf) { const uint2 fr = a.in.frags[f_begin + i]; ftab[i] = fr; len = frag_len(fr); }
		// block exclusive scan of len
		uint32_t x = len;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
			if (lane >= (uint32_t)o) x += t;
		}
		if (lane == 31) wsum[wid] = x;
		__syncthreads();
		uint32_t before = carry;
		for (uint32_t w2 = 0; w2 < wid; w2++) before += wsum[w2];
		if (i < nf) fstart[i] = vbase + before + x - len;
		uint32_t tot = 0;
		for (uint32_t w2 = 0; w2 < kPrThreads / 32; w2++) tot += wsum[w2];
		carry += tot;
		__syncthreads();
	}
	if (tid == 0) fstart[nf] = vbase + carry;
	// slot -> fragment map: each fragment marks the first block slot it
	// covers (the last of the fragments starting at or before ra marks slot
	// 0), then an inclusive max-scan over the block's slots spreads the marks
	for (uint32_t k = tid; k < kPrRange; k += kPrThreads) fidx[k] = 0;
	__syncthreads();
	for (uint32_t i = tid; i < nf; i += kPrThreads) {
		const uint32_t st = fstart[i];
		if (st < rb) atomicMax(&fidx[st > ra ? st - ra : 0], i);
	}
	__syncthreads();
	{
		// thread t scans slots [8t, 8t + 8) serially, then a block scan of
		// the thread maxima carries the mark across threads
		uint32_t m = 0, loc[kPrPerThread];
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++) {
			m = max(m, fidx[tid * kPrPerThread + u]);
			loc[u] = m;
		}
		uint32_t x = m;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
			if (lane >= (uint32_t)o) x = max(x, t);
		}
		if (lane == 31) wsum[wid] = x;
		__syncthreads();
		uint32_t before = __shfl_up_sync(0xffffffffu, x, 1);
		if (lane == 0) before = 0;
		for (uint32_t w2 = 0; w2 < wid; w2++) before = max(before, wsum[w2]);
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++)
			fidx[tid * kPrPerThread + u] = max(before, loc[u]);
	}
	__syncthreads();

	// phase 1: stream the block's slots into shared memory, slot
	// ra + u * kPrThreads + tid for thread tid (coalesced id loads); all
	// loads of a thread are issued before any value is used
	{
		const LevelTab* lt = a.in.lt;
		uint32_t id[kPrPerThread], dw[kPrPerThread], bit[kPrPerThread];
		bool in[kPrPerThread];
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++) {
			const uint32_t k = u * kPrThreads + tid;
			const uint32_t s = ra + k;
			in[u] = s < rb && nf > 0;
			id[u] = 0; dw[u] = 0; bit[u] = 0;
			if (in[u]) {
				const uint32_t f = fidx[k];
				const uint2 fr = ftab[f];
				const uint32_t idx = fr.x + (s - fstart[f]);
				const uint32_t lv = frag_level(fr);
				id[u] = __ldg(lt->ids[lv] + idx);
				dw[u] = __ldg(lt->del[lv] + (idx >> 5));
				bit[u] = idx & 31u;
			}
		}
		double x[kPrPerThread];
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++)
			x[u] = (in[u] && !((dw[u] >> bit[u]) & 1u)) ? __ldg(a.contrib + id[u]) : 0.0;
#pragma unroll
		for (int u = 0; u < kPrPerThread; u++) vals[u * kPrThreads + tid] = x[u];
	}
	__syncthreads();

	// phase 2: per-entry sums (short entries by one thread, in slot order)
	for (uint32_t e = eb + tid; e < ee; e += kPrThreads) {
		const uint32_t start = __ldg(a.pos + e), end = __ldg(a.pos + e + 1);
		const uint32_t s0 = max(start, ra), s1 = min(end, rb);
		if (s1 > s0 + kPrLong) {
			const uint32_t q = atomicAdd(&sh_nlong, 1u);
			longs[q] = e;
			continue;
		}
		double s = 0.0;
		for (uint32_t k = s0; k < s1; k++) s += vals[k - ra];
		pr_emit(a, r, ra, rb, e, start, end, s);
	}
	__syncthreads();
	// long entries: one warp each, fixed lane stride and tree order
	for (uint32_t q = wid; q < sh_nlong; q += kPrThreads / 32) {
		const uint32_t e = longs[q];
		const uint32_t start = __ldg(a.pos + e), end = __ldg(a.pos + e + 1);
		const uint32_t s0 = max(start, ra), s1 = min(end, rb);
		double s = 0.0;
		for (uint32_t k = s0 + lane; k < s1; k += 32) s += vals[k - ra];
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if (lane == 0) pr_emit(a, r, ra, rb, e, start, end, s);
	}
}

// Vertices straddling block boundaries: the thread of boundary q handles the
// vertex that starts in block q-1 and crosses q*kPrRange.
__global__ void pr_fixup(PrArgs a) {
	const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1;
	if (q >= a.nranges) return;
	const uint32_t s = (uint32_t)q * kPrRange;
	// last entry e with pos[e] <= s (pos[0] = 0 <= s)
	uint32_t lo = 0, hi = (uint32_t)a.in.V;
	while (lo < hi) {
		const uint32_t mid = (lo + hi + 1) >> 1;
		if (__ldg(a.pos + mid) <= s) lo = mid; else hi = mid - 1;
	}
	const uint32_t e = lo;
	if (e >= a.in.V) return;
	const uint32_t start = __ldg(a.pos + e), end = __ldg(a.pos + e + 1);
	if (!(start < s && start >= s - kPrRange && end > s)) return;
	const uint32_t r2 = (end - 1) / kPrRange;
	double t = __ldcg(a.carry_last + (q - 1));
	for (uint32_t x = (uint32_t)q; x <= r2; x++) t += __ldcg(a.carry_first + x);
	pr_finish(a, e, t);
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

	PrArgs a;
	a.in = sn->view(1);
	a.pos = sn->in.slot_off.as<uint32_t>();
	a.range_lb = sn->in.range_lb.as<uint32_t>();
	a.total = (uint32_t)sn->in.n_frag_slots;
	a.nranges = (uint32_t)std::max<uint64_t>(1, (a.total + kPrRange - 1) / kPrRange);
	a.outdeg = sn->out.deg.as<uint32_t>();
	a.base = base;
	a.d = damping;

	DevBuf* sc = s->scratch;
	LG_TRY(sc[0].reserve(V * sizeof(double)));
	LG_TRY(sc[1].reserve(V * sizeof(double)));
	LG_TRY(sc[2].reserve(2ull * a.nranges * sizeof(double)));
	a.carry_first = sc[2].as<double>();
	a.carry_last = a.carry_first + a.nranges;
	const bool dev_out = is_device_pointer(ranks);
	double* pr_buf = ranks;
	if (!dev_out) {
		LG_TRY(sc[4].reserve(V * sizeof(double)));
		pr_buf = sc[4].as<double>();
	}
	pr_init<<<grid_for(V, 256), 256, 0, st>>>(a.outdeg, V, pr0, sc[0].as<double>(),
			iterations == 0 ? pr_buf : nullptr);
	LG_CUDA(cudaGetLastError(), "pr_init");
	s->launches++;
	const unsigned fix_blocks = grid_for(a.nranges, 256);
	for (int it = 0; it < iterations; it++) {
		a.contrib = sc[it & 1].as<double>();
		a.contrib_next = sc[(it + 1) & 1].as<double>();
		a.pr_out = (it == iterations - 1) ? pr_buf : nullptr;
		pr_pull_step<<<a.nranges, kPrThreads, 0, st>>>(a);
		if (a.nranges > 1) pr_fixup<<<fix_blocks, 256, 0, st>>>(a);
	}
	LG_CUDA(cudaGetLastError(), "pr_pull_step");
	s->launches += (uint64_t)iterations * (a.nranges > 1 ? 2 : 1);
	if (!dev_out) {
		LG_TRY(copy_out(s, ranks, pr_buf, V * sizeof(double)));
		LG_CUDA(cudaStreamSynchronize(st), "pagerank");
	}
	return LG_OK;
}

// ---------------------------------------------------------------------------
// PageRank without device allocation.
//
// lg_pagerank_pull keeps its per-iteration vectors in store-owned scratch
// that it grows with cudaMalloc.  Some callers cannot have the library
// allocate: a thread that is capturing work into a CUDA graph (cudaMalloc
// and cudaFree are not allowed while its stream is being captured), or a
// process whose device memory is already handed out to another allocator,
// where a new cudaMalloc can fail or stall on a device-wide synchronisation.
// For them this variant runs the same kernels on a fixed scratch area that
// is part of the library image: LG_NOALLOC_SCRATCH_BYTES of device memory,
// reserved on every GPU that loads the library, until the process exits.
// ---------------------------------------------------------------------------

namespace lg {

static __device__ __align__(256) unsigned char g_noalloc_scratch[LG_NOALLOC_SCRATCH_BYTES];

} // namespace lg

extern "C" lg_status lg_pagerank_pull_noalloc(lg_snapshot* sn, int iterations,
		double damping, double* ranks) {
	clear_error();
	if (!sn || !ranks) return set_error(LG_EINVAL, "null argument");
	if (!(damping > 0.0 && damping < 1.0))
		return set_error(LG_EINVAL, "damping must be in (0, 1)");
	if (iterations < 0) return set_error(LG_EINVAL, "iterations must be >= 0");
	if (!sn->in.present)
		return set_error(LG_ESTATE, "pull PageRank needs the in-CSR (reverse edges)");
	lg_store* s = sn->store;
	const uint64_t V = sn->V;
	const uint64_t total = sn->in.n_frag_slots;
	const uint64_t nranges = std::max<uint64_t>(1, (total + kPrRange - 1) / kPrRange);
	// contrib (two vectors), the result staged for host outputs, carries
	const uint64_t need = 3 * V * sizeof(double) + 2 * nranges * sizeof(double);
	if (need > LG_NOALLOC_SCRATCH_BYTES)
		return set_error(LG_EINVAL, "graph needs %llu scratch bytes, more than the %llu "
				"this entry point has (24 B per vertex + 16 B per %u in-CSR slots)",
				(unsigned long long)need, (unsigned long long)LG_NOALLOC_SCRATCH_BYTES,
				kPrRange);
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	// Device address of the scratch array, looked up once per device with
	// that device current (host code must not use the symbol itself).
	static std::mutex mu;
	static void* scratch_of[LG_NOALLOC_MAX_DEVICES] = {};
	if (s->device < 0 || s->device >= LG_NOALLOC_MAX_DEVICES)
		return set_error(LG_ENOTSUP, "device ordinal %d beyond %d", s->device,
				LG_NOALLOC_MAX_DEVICES);
	void* base = nullptr;
	{
		std::lock_guard<std::mutex> lk(mu);
		if (!scratch_of[s->device]) {
			void* p = nullptr;
			LG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
			scratch_of[s->device] = p;
		}
		base = scratch_of[s->device];
	}
	cudaStream_t st = s->stream;
	double* c0 = (double*)base;
	double* c1 = c0 + V;
	double* staged = c1 + V;
	double* carries = staged + V;

	PrArgs a;
	a.in = sn->view(1);
	a.pos = sn->in.slot_off.as<uint32_t>();
	a.range_lb = sn->in.range_lb.as<uint32_t>();
	a.total = (uint32_t)total;
	a.nranges = (uint32_t)nranges;
	a.outdeg = sn->out.deg.as<uint32_t>();
	a.base = (1.0 - damping) / (double)V;
	a.d = damping;
	a.carry_first = carries;
	a.carry_last = carries + nranges;
	const bool dev_out = is_device_pointer(ranks);
	double* pr_buf = dev_out ? ranks : staged;
	pr_init<<<grid_for(V, 256), 256, 0, st>>>(a.outdeg, V, 1.0 / (double)V, c0,
			iterations == 0 ? pr_buf : nullptr);
	for (int it = 0; it < iterations; it++) {
		a.contrib = (it & 1) ? c1 : c0;
		a.contrib_next = (it & 1) ? c0 : c1;
		a.pr_out = (it == iterations - 1) ? pr_buf : nullptr;
		pr_pull_step<<<a.nranges, kPrThreads, 0, st>>>(a);
		if (a.nranges > 1) pr_fixup<<<grid_for(a.nranges, 256), 256, 0, st>>>(a);
	}
	LG_CUDA(cudaGetLastError(), "pagerank noalloc");
	s->launches += 1 + (uint64_t)iterations * (a.nranges > 1 ? 2 : 1);
	if (!dev_out) {
		LG_CUDA(cudaMemcpyAsync(ranks, pr_buf, V * sizeof(double), cudaMemcpyDeviceToHost, st),
				"copy result");
		s->d2h_bytes += V * sizeof(double);
		LG_CUDA(cudaStreamSynchronize(st), "pagerank noalloc");
	}
	return LG_OK;
}
