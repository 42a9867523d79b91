// lg_ppr.cu - personalized PageRank for K seeds at once, as an N x K block.
//
// The reference has no personalized variant; this is the pull iteration of
// ll_b_pagerank_pull_ext::run (benchmark/benchmarks/pagerank.h:120-169) with
// the uniform teleport (1-d)/N replaced, per column k, by (1-d) on seed_k:
//   x0[:, k] = e_seed_k,   x'[t, k] = (1-d) [t == seed_k] + d * sum_{w in in(t)} x[w, k] / out_degree(w)
// for a fixed number of iterations, dangling mass dropped as in the reference.
//
// Layout: row-major V x K doubles, so one in-edge (w -> t) reads the
// contiguous K-wide row of w; lane j of a warp owns columns j, j+32, ...
// Work is split like PageRank (lg_expand.cuh): warps take fixed ranges of
// the in-CSR slot space; inside a chunk the 32 edges are handled one after
// another by the whole warp (the edge id is loaded once for K columns).
// Rows of vertices that straddle ranges are combined in range order by
// ppr_fixup.  The K columns are processed in passes of a K-tile (a multiple
// of 32, LG_TUNE_PPR_KTILE): a pass runs every iteration on its columns, so a
// smaller tile re-reads the edge ids once more per pass but keeps the gathered
// rows of a pass narrower.  The slots per warp range are LG_TUNE_PPR_RANGE.  Every snapshot's iterations are captured into one CUDA graph
// and launched once.
#include "lg_device.cuh"
#include "lg_expand.cuh"
#include "lg_tune.h"

#include <algorithm>
#include <vector>

namespace lg {

constexpr int kPprThreads = 256;
constexpr uint32_t kNoSeed = 0xffffffffu;

struct PprArgs {
	SnapCsr in;
	const uint32_t* pos;
	uint32_t total;
	uint32_t nranges;
	const uint32_t* outdeg;
	const double* y;          // x / out_degree of the previous iteration
	double* y_next;
	double* x_out;            // written on the last iteration (or null)
	double d;
	double tele;              // 1 - d
	const uint32_t* seed_first;   // V: first index into seed_col, or kNoSeed
	const uint2* seed_col;        // (vertex, column) sorted by vertex
	uint32_t n_seeds;
	double* carry_first;      // nranges x K
	double* carry_last;       // nranges x K
	uint32_t K;               // row length of y / x / carries
	uint32_t col0;            // first column of this pass (a K-tile of CPL * 32 columns)
	uint32_t range;           // virtual slots per warp range
};

template <int CPL>
__device__ __forceinline__ void ppr_finish(const PprArgs& a, uint32_t v, const double* s) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t dg = __ldg(a.outdeg + v);
	const uint32_t sf = __ldg(a.seed_first + v);
#pragma unroll
	for (int i = 0; i < CPL; i++) {
		const uint32_t c = a.col0 + lane + 32 * i;
		double t = 0.0;
		if (sf != kNoSeed)
			for (uint32_t q = sf; q < a.n_seeds && a.seed_col[q].x == v; q++)
				if (a.seed_col[q].y == c) t = a.tele;
		const double x = __dadd_rn(t, __dmul_rn(a.d, s[i]));
		a.y_next[(uint64_t)v * a.K + c] = dg ? x / (double)dg : 0.0;
		if (a.x_out) a.x_out[(uint64_t)v * a.K + c] = x;
	}
}

template <int CPL>
__global__ void __launch_bounds__(kPprThreads)
ppr_step(PprArgs a) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t r64 = (uint64_t)blockIdx.x * (kPprThreads / 32) + (threadIdx.x >> 5);
	if (r64 >= a.nranges) return;
	const uint32_t r = (uint32_t)r64;
	const bool last_range = r == a.nranges - 1;
	const uint32_t ra = r * a.range;
	const uint32_t rb = last_range ? a.total : min(a.total, ra + a.range);
	uint32_t e_begin, e_end;
	range_entries(a.pos, (uint32_t)a.in.V, ra, rb, last_range, &e_begin, &e_end);
	const LevelTab* lt = a.in.lt;
	for (uint32_t ew = e_begin; ew < e_end; ew += 32) {
		const Window w = load_window(a.in, nullptr, a.pos, ew, e_end, ra, rb);
		const uint32_t my_end = w.valid ? __ldg(a.pos + w.e + 1) : 0;
		double acc[CPL];
#pragma unroll
		for (int i = 0; i < CPL; i++) acc[i] = 0.0;
		int cur = -1;
		auto flush = [&](int o) {
			const uint32_t st = __shfl_sync(0xffffffffu, w.start, o);
			const uint32_t en = __shfl_sync(0xffffffffu, my_end, o);
			const uint32_t v = __shfl_sync(0xffffffffu, w.v, o);
			if (st < ra) {
#pragma unroll
				for (int i = 0; i < CPL; i++) a.carry_first[(uint64_t)r * a.K + a.col0 + lane + 32 * i] = acc[i];
			} else if (en > rb) {
#pragma unroll
				for (int i = 0; i < CPL; i++) a.carry_last[(uint64_t)r * a.K + a.col0 + lane + 32 * i] = acc[i];
			} else {
				ppr_finish<CPL>(a, v, acc);
			}
#pragma unroll
			for (int i = 0; i < CPL; i++) acc[i] = 0.0;
		};
		for (uint32_t base = w.lo; base < w.hi; base += 32) {
			const uint32_t k = base + lane;
			uint32_t own, lv, idx, nb = 0;
			locate_slot(a.in, w, k, &own, &lv, &idx);
			bool act = k < w.hi;
			if (act) {
				const uint32_t word = __ldg(lt->del[lv] + (idx >> 5));
				nb = __ldg(lt->ids[lv] + idx);
				act = !((word >> (idx & 31)) & 1u);
			}
			const unsigned inside = __ballot_sync(0xffffffffu, k < w.hi);
			for (unsigned m = inside; m; m &= m - 1) {
				const int t = __ffs(m) - 1;
				const int o = (int)__shfl_sync(0xffffffffu, own, t);
				const uint32_t src = __shfl_sync(0xffffffffu, nb, t);
				const bool live = __shfl_sync(0xffffffffu, act, t);
				if (o != cur) {
					if (cur >= 0) flush(cur);
					cur = o;
				}
				if (live) {
					const double* row = a.y + (uint64_t)src * a.K + a.col0;
#pragma unroll
					for (int i = 0; i < CPL; i++) acc[i] += __ldg(row + lane + 32 * i);
				}
			}
		}
		if (cur >= 0) flush(cur);
		// entries without slots in the snapshot: teleport term only
		unsigned empty = __ballot_sync(0xffffffffu, w.valid && w.s0 == w.s1);
		for (; empty; empty &= empty - 1) {
			const int o = __ffs(empty) - 1;
			const uint32_t v = __shfl_sync(0xffffffffu, w.v, o);
			double z[CPL];
#pragma unroll
			for (int i = 0; i < CPL; i++) z[i] = 0.0;
			ppr_finish<CPL>(a, v, z);
		}
	}
}

// One warp per range boundary: the vertex that starts in range q-1 and
// crosses q * range sums its carried rows in range order.
template <int CPL>
__global__ void ppr_fixup(PprArgs a) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t q = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5) + 1;
	if (q >= a.nranges) return;
	const uint32_t s = (uint32_t)q * a.range;
	uint32_t lo = 0, hi = (uint32_t)a.in.V;
	while (lo < hi) {
		const uint32_t mid = (lo + hi + 1) >> 1;
		if (__ldg(a.pos + mid) <= s) lo = mid; else hi = mid - 1;
	}
	const uint32_t e = lo;
	if (e >= a.in.V) return;
	const uint32_t start = __ldg(a.pos + e), end = __ldg(a.pos + e + 1);
	if (!(start < s && start >= s - a.range && end > s)) return;
	const uint32_t r2 = (end - 1) / a.range;
	const uint32_t c0 = a.col0 + lane;
	double t[CPL];
#pragma unroll
	for (int i = 0; i < CPL; i++) t[i] = __ldcg(a.carry_last + (uint64_t)(q - 1) * a.K + c0 + 32 * i);
	for (uint32_t x = (uint32_t)q; x <= r2; x++)
#pragma unroll
		for (int i = 0; i < CPL; i++) t[i] += __ldcg(a.carry_first + (uint64_t)x * a.K + c0 + 32 * i);
	ppr_finish<CPL>(a, e, t);
}

__global__ void ppr_seed_init(const uint2* seed_col, uint32_t n, const uint32_t* outdeg,
		uint32_t K, double* y) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint32_t v = seed_col[i].x, c = seed_col[i].y;
	const uint32_t dg = outdeg[v];
	y[(uint64_t)v * K + c] = dg ? 1.0 / (double)dg : 0.0;
}

__global__ void ppr_seed_x(const uint2* seed_col, uint32_t n, uint32_t K, double* x) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) x[(uint64_t)seed_col[i].x * K + seed_col[i].y] = 1.0;
}

template <int CPL>
void launch_ppr_iteration(const PprArgs& a, cudaStream_t st) {
	ppr_step<CPL><<<grid_for(a.nranges, kPprThreads / 32), kPprThreads, 0, st>>>(a);
	if (a.nranges > 1) ppr_fixup<CPL><<<grid_for(a.nranges, 8), 256, 0, st>>>(a);
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_ppr(lg_snapshot* const* snaps, int n_snaps, const int64_t* seeds,
		int K, int iterations, double damping, double* out) {
	clear_error();
	if (!snaps || n_snaps <= 0 || !seeds || !out) return set_error(LG_EINVAL, "null argument");
	if (K <= 0 || K > 256 || K % 32 != 0)
		return set_error(LG_ENOTSUP, "K must be a multiple of 32 in [32, 256]");
	if (!(damping > 0.0 && damping < 1.0)) return set_error(LG_EINVAL, "damping must be in (0, 1)");
	if (iterations < 0) return set_error(LG_EINVAL, "iterations must be >= 0");
	lg_store* s = snaps[0]->store;
	const uint64_t V = snaps[0]->V;
	for (int i = 0; i < n_snaps; i++) {
		if (!snaps[i] || snaps[i]->store != s || snaps[i]->V != V)
			return set_error(LG_EINVAL, "snapshots must share the store and max_nodes");
		if (!snaps[i]->in.present) return set_error(LG_ESTATE, "PPR needs the in-CSR");
	}
	for (int k = 0; k < K; k++)
		if (seeds[k] < 0 || (uint64_t)seeds[k] >= V)
			return set_error(LG_EINVAL, "seed %lld out of range", (long long)seeds[k]);
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;

	// seeds sorted by vertex -> (vertex, column) pairs and a per-vertex index
	std::vector<uint2> sc(K);
	for (int k = 0; k < K; k++) sc[k] = make_uint2((uint32_t)seeds[k], (uint32_t)k);
	std::sort(sc.begin(), sc.end(), [](uint2 x, uint2 y) { return x.x < y.x || (x.x == y.x && x.y < y.y); });
	std::vector<std::pair<uint32_t, uint32_t>> firsts;
	for (int k = 0; k < K; k++)
		if (k == 0 || sc[k].x != sc[k - 1].x) firsts.push_back({sc[k].x, (uint32_t)k});

	const uint64_t row = (uint64_t)K * 8;
	// the store's scratch (kept for the next call, contents not preserved)
	DevBuf* yb = s->scratch;         // scratch[0], [1]: the two V x K blocks
	DevBuf& carry = s->scratch[2];
	DevBuf& seedb = s->scratch[3];
	DevBuf& firstb = s->scratch[4];
	DevBuf& resb = s->scratch[5];
	LG_TRY(yb[0].reserve(V * row));
	LG_TRY(yb[1].reserve(V * row));
	LG_TRY(seedb.reserve(K * sizeof(uint2)));
	LG_TRY(firstb.reserve(V * 4));
	// launch parameters: columns per pass (a multiple of 32 dividing K) and
	// slots per warp range
	int ktile = (int)tune_value(s->device, LG_TUNE_PPR_KTILE);
	ktile = std::min(K, std::max(32, ktile - ktile % 32));
	while (K % ktile) ktile -= 32;
	const uint32_t range = (uint32_t)tune_value(s->device, LG_TUNE_PPR_RANGE);
	uint32_t maxr = 1;
	for (int i = 0; i < n_snaps; i++)
		maxr = std::max<uint32_t>(maxr, (uint32_t)((snaps[i]->in.n_frag_slots + range - 1) / range));
	LG_TRY(carry.reserve(2ull * maxr * row));
	const bool dev_out = is_device_pointer(out);
	double* res = out;
	if (!dev_out) { LG_TRY(resb.reserve((uint64_t)n_snaps * V * row)); res = resb.as<double>(); }
	LG_CUDA(cudaMemcpyAsync(seedb.p, sc.data(), K * sizeof(uint2), cudaMemcpyHostToDevice, st), "h2d");
	LG_CUDA(cudaMemsetAsync(firstb.p, 0xff, V * 4, st), "memset");
	for (auto& f : firsts)
		LG_CUDA(cudaMemcpyAsync(firstb.as<uint32_t>() + f.first, &f.second, 4,
				cudaMemcpyHostToDevice, st), "h2d");
	s->h2d_bytes += K * sizeof(uint2) + firsts.size() * 4;
	LG_CUDA(cudaStreamSynchronize(st), "ppr setup");

	// capture every snapshot's iterations into one graph
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	LG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture");
	uint64_t launches = 0;
	cudaError_t cap = cudaSuccess;     // first error while capturing; the capture
	                                   // is ended on every path below
	for (int i = 0; i < n_snaps; i++) {
		lg_snapshot* sn = snaps[i];
		PprArgs a;
		a.in = sn->view(1);
		a.pos = sn->in.slot_off.as<uint32_t>();
		a.total = (uint32_t)sn->in.n_frag_slots;
		a.range = range;
		a.nranges = (uint32_t)std::max<uint64_t>(1, (a.total + range - 1) / range);
		a.outdeg = sn->out.deg.as<uint32_t>();
		a.d = damping;
		a.tele = 1.0 - damping;
		a.seed_first = firstb.as<uint32_t>();
		a.seed_col = seedb.as<uint2>();
		a.n_seeds = (uint32_t)K;
		a.carry_first = carry.as<double>();
		a.carry_last = carry.as<double>() + (uint64_t)a.nranges * K;
		a.K = (uint32_t)K;
		double* xo = res + (uint64_t)i * V * K;
		if (cap == cudaSuccess) cap = cudaMemsetAsync(yb[0].p, 0, V * row, st);
		ppr_seed_init<<<grid_for(K, 256), 256, 0, st>>>(seedb.as<uint2>(), K, a.outdeg, K,
				yb[0].as<double>());
		launches++;
		if (iterations == 0) {
			if (cap == cudaSuccess) cap = cudaMemsetAsync(xo, 0, V * row, st);
			ppr_seed_x<<<grid_for(K, 256), 256, 0, st>>>(seedb.as<uint2>(), K, K, xo);
			launches++;
		}
		// column tiles are independent: each runs all iterations on its columns
		for (int c0 = 0; c0 < K; c0 += ktile) {
			a.col0 = (uint32_t)c0;
			for (int it = 0; it < iterations; it++) {
				a.y = yb[it & 1].as<double>();
				a.y_next = yb[(it + 1) & 1].as<double>();
				a.x_out = (it == iterations - 1) ? xo : nullptr;
				switch (ktile / 32) {
				case 1: launch_ppr_iteration<1>(a, st); break;
				case 2: launch_ppr_iteration<2>(a, st); break;
				case 3: launch_ppr_iteration<3>(a, st); break;
				case 4: launch_ppr_iteration<4>(a, st); break;
				case 5: launch_ppr_iteration<5>(a, st); break;
				case 6: launch_ppr_iteration<6>(a, st); break;
				case 7: launch_ppr_iteration<7>(a, st); break;
				default: launch_ppr_iteration<8>(a, st); break;
				}
				launches += a.nranges > 1 ? 2 : 1;
			}
		}
	}
	if (cap == cudaSuccess) cap = cudaGetLastError();
	cudaError_t ce = cudaStreamEndCapture(st, &graph);
	if (cap != cudaSuccess || ce != cudaSuccess) {
		if (graph) cudaGraphDestroy(graph);
		return cuda_status(cap != cudaSuccess ? cap : ce, "graph capture");
	}
	ce = cudaGraphInstantiate(&exec, graph, 0);
	if (ce != cudaSuccess) { cudaGraphDestroy(graph); return cuda_status(ce, "graph instantiate"); }
	ce = cudaGraphLaunch(exec, st);
	if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
	cudaGraphExecDestroy(exec);
	cudaGraphDestroy(graph);
	if (ce != cudaSuccess) return cuda_status(ce, "ppr graph");
	s->launches += launches;
	if (!dev_out) {
		LG_TRY(copy_out(s, out, res, (uint64_t)n_snaps * V * row));
		LG_CUDA(cudaStreamSynchronize(st), "ppr");
	}
	return LG_OK;
}
