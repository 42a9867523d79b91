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
// values are bit-identical; only the summation order differs (FP64, well
// within 1e-12).
//
// Work split (lg_expand.cuh): the in-CSR slot space of all vertices, in
// vertex order, is cut into ranges of kPrRange slots, one warp per range.  A
// vertex whose slots straddle range boundaries leaves one partial sum per
// range (carry_first: it began before the range, carry_last: it runs past
// the end) and pr_fixup adds those partials in range order, so every result
// is deterministic.
#include "lg_device.cuh"
#include "lg_expand.cuh"

namespace lg {

constexpr uint32_t kPrRange = 2048;
constexpr int kPrThreads = 256;
constexpr int kPrWarps = kPrThreads / 32;

struct PrArgs {
	SnapCsr in;
	const uint32_t* pos;       // V + 1 in-CSR slot prefix
	uint32_t total;            // pos[V]
	uint32_t nranges;
	const uint32_t* outdeg;
	const double* contrib;
	double* contrib_next;
	double* pr_out;            // written when non-null (last iteration)
	double base;               // (1 - d) / N
	double d;
	double* carry_first;       // per range
	double* carry_last;        // per range
};

__device__ __forceinline__ void pr_finish(const PrArgs& a, uint32_t v, double s) {
	const double pr = __dadd_rn(a.base, __dmul_rn(a.d, s));
	const uint32_t dg = __ldg(a.outdeg + v);
	a.contrib_next[v] = dg ? pr / (double)dg : 0.0;
	if (a.pr_out) a.pr_out[v] = pr;
}

// Sum of contrib over `n` slots of a vertex's fragment chain, starting `off`
// slots into it, by one lane in iteration order (4 loads in flight).
__device__ __forceinline__ double lane_sum(const PrArgs& a, uint32_t f, uint32_t off,
		uint32_t n) {
	const LevelTab* lt = a.in.lt;
	uint2 fr = a.in.frags[f];
	while (off >= frag_len(fr)) { off -= frag_len(fr); fr = a.in.frags[++f]; }
	double s = 0.0;
	while (n > 0) {
		const uint32_t lv = frag_level(fr);
		const uint32_t base = fr.x + off;
		const uint32_t m = min(frag_len(fr) - off, n);
		const uint32_t* ids = lt->ids[lv] + base;
		const uint32_t* del = lt->del[lv];
		uint32_t i = 0;
		for (; i + 4 <= m; i += 4) {
			uint32_t id[4], dw[4];
#pragma unroll
			for (int u = 0; u < 4; u++) {
				id[u] = __ldg(ids + i + u);
				dw[u] = __ldg(del + ((base + i + u) >> 5));
			}
			double x[4];
#pragma unroll
			for (int u = 0; u < 4; u++)
				x[u] = ((dw[u] >> ((base + i + u) & 31)) & 1u) ? 0.0 : __ldg(a.contrib + id[u]);
#pragma unroll
			for (int u = 0; u < 4; u++) s += x[u];
		}
		for (; i < m; i++) {
			const uint32_t dw = __ldg(del + ((base + i) >> 5));
			if (!((dw >> ((base + i) & 31)) & 1u)) s += __ldg(a.contrib + __ldg(ids + i));
		}
		n -= m;
		off = 0;
		if (n) fr = a.in.frags[++f];
	}
	return s;
}

// Sum over `n` slots of one vertex (starting `off` slots in) by the whole
// warp: lane i takes slots i, i + 32, ..., then a fixed tree reduction.
__device__ __forceinline__ double warp_sum(const PrArgs& a, uint32_t f, uint32_t off,
		uint32_t n) {
	const uint32_t lane = threadIdx.x & 31u;
	const LevelTab* lt = a.in.lt;
	uint2 fr = a.in.frags[f];
	while (off >= frag_len(fr)) { off -= frag_len(fr); fr = a.in.frags[++f]; }
	double s = 0.0;
	while (n > 0) {
		const uint32_t lv = frag_level(fr);
		const uint32_t base = fr.x + off;
		const uint32_t m = min(frag_len(fr) - off, n);
		const uint32_t* ids = lt->ids[lv] + base;
		const uint32_t* del = lt->del[lv];
		for (uint32_t i0 = 0; i0 < m; i0 += 32 * kUnroll) {
			uint32_t id[kUnroll];
			bool live[kUnroll];
#pragma unroll
			for (int u = 0; u < kUnroll; u++) {
				const uint32_t i = i0 + u * 32 + lane;
				live[u] = i < m;
				id[u] = 0;
				if (live[u]) {
					const uint32_t dw = __ldg(del + ((base + i) >> 5));
					id[u] = __ldg(ids + i);
					live[u] = !((dw >> ((base + i) & 31)) & 1u);
				}
			}
#pragma unroll
			for (int u = 0; u < kUnroll; u++) if (live[u]) s += __ldg(a.contrib + id[u]);
		}
		n -= m;
		off = 0;
		if (n) fr = a.in.frags[++f];
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	return s;
}

// One warp per range of kPrRange slots.  Entries (vertices) with fewer than
// 32 slots in the range are summed by their own lane, sequentially in
// iteration order; longer ones by the whole warp.
__global__ void __launch_bounds__(kPrThreads)
pr_pull_step(PrArgs a) {
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
	const uint64_t r64 = (uint64_t)blockIdx.x * kPrWarps + wid;
	if (r64 >= a.nranges) return;
	const uint32_t r = (uint32_t)r64;
	const bool last_range = r == a.nranges - 1;
	const uint32_t ra = r * kPrRange;
	const uint32_t rb = last_range ? a.total : min(a.total, ra + kPrRange);
	uint32_t e_begin, e_end;
	range_entries(a.pos, (uint32_t)a.in.V, ra, rb, last_range, &e_begin, &e_end);
	for (uint32_t ew = e_begin; ew < e_end; ew += 32) {
		const Window w = load_window(a.in, nullptr, a.pos, ew, e_end, ra, rb);
		const uint32_t span = w.s1 - w.s0;
		const bool longe = w.valid && span >= 32;
		double s = 0.0;
		if (w.valid && !longe && span > 0) s = lane_sum(a, w.f0, w.s0 - w.start, span);
		for (unsigned m = __ballot_sync(0xffffffffu, longe); m; m &= m - 1) {
			const int t = __ffs(m) - 1;
			const uint32_t f0 = __shfl_sync(0xffffffffu, w.f0, t);
			const uint32_t off = __shfl_sync(0xffffffffu, w.s0 - w.start, t);
			const uint32_t n = __shfl_sync(0xffffffffu, span, t);
			const double ws = warp_sum(a, f0, off, n);
			if ((int)lane == t) s = ws;
		}
		if (w.valid) {
			const uint32_t end = __ldg(a.pos + w.e + 1);
			if (w.start < ra) a.carry_first[r] = s;        // began before the range
			else if (end > rb) a.carry_last[r] = s;        // runs past its end
			else pr_finish(a, w.v, s);
		}
	}
}

// Vertices straddling range boundaries: the thread of boundary q handles the
// vertex that starts in range q-1 and crosses q*kPrRange.
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
	const unsigned blocks = grid_for(a.nranges, kPrWarps);
	const unsigned fix_blocks = grid_for(a.nranges, 256);
	for (int it = 0; it < iterations; it++) {
		a.contrib = sc[it & 1].as<double>();
		a.contrib_next = sc[(it + 1) & 1].as<double>();
		a.pr_out = (it == iterations - 1) ? pr_buf : nullptr;
		pr_pull_step<<<blocks, kPrThreads, 0, st>>>(a);
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
