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
// values are bit-identical; only the order in which a vertex's values are
// added differs from the reference's left-to-right loop (FP64, well within
// 1e-12 in every case), and it is fixed, so results are deterministic.
//
// lg_pagerank_pull runs every iteration over the snapshot's live
// in-adjacency flattened into one CSR (lg_flat.cuh: ids in iteration order,
// head bits where a vertex's in-edges begin, the rows with in-edges): the
// snapshot's own when lg_snapshot_flatten made one, else one built for the
// call in store scratch.
//
// pr_flat_step is the flat sweep of lg_flat_sweep.cuh with the PageRank op:
// each warp takes a tile of kFlatTile consecutive edges, 8 per lane, issues
// the tile's id loads and gathers up front, adds each lane's values serially
// and joins the lanes with one segmented warp scan keyed by the head bits; a
// vertex that runs past a tile boundary leaves partials (carry_first,
// carry_last) that pr_flat_fixup adds.  No block barriers: each warp stages
// its finished row sums in its own shared memory.  Vertices without
// in-edges have the constant rank (1-d)/N after the first iteration and are
// written once (pr_empty_rows).
//
// lg_pagerank_pull_noalloc cannot hold the E-sized flat array, so it walks
// the fragments directly every iteration (pr_pull_step, one CTA per 1024
// virtual slots, values staged in shared memory).
#include "lg_flat_sweep.cuh"
#include "lg_tune.h"

#include <mutex>

namespace lg {

constexpr uint32_t kPrLong = 64;       // entries with more slots are reduced by a warp

// ---------------------------------------------------------------------------
// Iterations over the flat array
// ---------------------------------------------------------------------------

// One PageRank iteration as a flat sweep (lg_flat_sweep.cuh): an edge's value
// is the gathered contribution of its source; a row's sum s gives
// pr = (1-d)/N + d*s and the next contribution pr / out_degree.
struct PrOp {
	static constexpr bool kResidual = false;
	const uint32_t* nz_rows;   // R
	const uint32_t* nz_outdeg; // R: out-degree of nz_rows[k]
	const double* contrib;
	double* contrib_next;
	double* pr_out;            // written when non-null (last iteration)
	double base;               // (1 - d) / N
	double d;
	__device__ __forceinline__ bool skip() const { return false; }
	__device__ __forceinline__ void values(uint32_t, const uint32_t (&id)[kFlatPerLane],
			double (&x)[kFlatPerLane]) const {
#pragma unroll
		for (int i = 0; i < kFlatPerLane; i++)
			x[i] = id[i] != kNoId ? __ldg(contrib + id[i]) : 0.0;
	}
	__device__ __forceinline__ double finish(uint32_t k, double s) const {
		const uint32_t v = __ldg(nz_rows + k);
		const double pr = __dadd_rn(base, __dmul_rn(d, s));
		const uint32_t dg = __ldg(nz_outdeg + k);
		contrib_next[v] = dg ? pr / (double)dg : 0.0;
		if (pr_out) pr_out[v] = pr;
		return 0.0;
	}
	__device__ __forceinline__ void residual(double) const {}
};

__global__ void __launch_bounds__(kFlatWarps * 32)
pr_flat_step(FlatTiles a, PrOp op) {
	__shared__ double rowsum[kFlatWarps][kFlatTile];
	flat_sweep_tile(a, op, rowsum);
}

// The same with registers capped for 64 resident warps per SM.
__global__ void __launch_bounds__(kFlatWarps * 32, 64 / kFlatWarps)
pr_flat_step_occ8(FlatTiles a, PrOp op) {
	__shared__ double rowsum[kFlatWarps][kFlatTile];
	flat_sweep_tile(a, op, rowsum);
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kFlatLoopWarps * 32, kMinBlocks)
pr_flat_loop(FlatTiles a, PrOp op) {
	__shared__ double rowsum[kFlatLoopWarps][kFlatTile];
	flat_sweep_loop(a, op, rowsum);
}

__global__ void __launch_bounds__(kFixupThreads)
pr_flat_fixup(FlatTiles a, PrOp op) {
	flat_sweep_fixup_body(a, op);
}

// nz_outdeg[k] = out-degree of row k's vertex (rows read it in order).
__global__ void pr_row_degrees(const uint32_t* nz_rows, uint32_t R, const uint32_t* outdeg,
		uint32_t* nz_outdeg) {
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < R) nz_outdeg[k] = __ldg(outdeg + __ldg(nz_rows + k));
}

// Vertices without in-edges: rank pr, contrib pr / out_degree.
__global__ void pr_empty_rows(const uint32_t* flat_off, const uint32_t* outdeg, uint64_t V,
		double pr, double* contrib, double* pr_out) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v >= V) return;
	if (__ldg(flat_off + v + 1) != __ldg(flat_off + v)) return;
	if (contrib) {
		const uint32_t dg = __ldg(outdeg + v);
		contrib[v] = dg ? pr / (double)dg : 0.0;
	}
	if (pr_out) pr_out[v] = pr;
}

// ---------------------------------------------------------------------------
// Fragment-walking iteration (no flat array)
// ---------------------------------------------------------------------------

struct PrArgs {
	SlotSpace sp;
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

// One CTA per block of kMapRange virtual slots.  Phase 1 streams the block's
// slots (slot ra + u * kMapThreads + tid for thread tid, coalesced id loads,
// all loads of a thread issued before any value is used) into shared
// memory; phase 2 sums each vertex's values (one thread per short vertex, a
// warp per long one).  A vertex straddling blocks leaves a partial per block
// that pr_fixup adds in block order.
__global__ void __launch_bounds__(kMapThreads)
pr_pull_step(PrArgs a) {
	__shared__ BlockMap m;
	__shared__ double vals[kMapRange];
	__shared__ uint32_t longs[kMapRange / kPrLong + 2];
	__shared__ uint32_t sh_nlong;
	const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
	const uint32_t r = blockIdx.x, ra = r * kMapRange, rb = block_end(a.sp, r);
	if (tid == 0) sh_nlong = 0;
	map_block(a.sp, r, ra, rb, m);
	const uint32_t eb = m.eb, ee = m.ee;
	{
		const LevelTab* lt = a.sp.g.lt;
		uint32_t id[kMapPerThread], dw[kMapPerThread], bit[kMapPerThread];
		bool in[kMapPerThread];
#pragma unroll
		for (int u = 0; u < kMapPerThread; u++) {
			uint32_t lv = 0, idx = 0;
			in[u] = block_slot(m, ra, rb, u * kMapThreads + tid, &lv, &idx);
			id[u] = 0; dw[u] = 0; bit[u] = 0;
			if (in[u]) {
				id[u] = __ldg(lt->ids[lv] + idx);
				dw[u] = __ldg(lt->del[lv] + (idx >> 5));
				bit[u] = idx & 31u;
			}
		}
		double x[kMapPerThread];
#pragma unroll
		for (int u = 0; u < kMapPerThread; u++)
			x[u] = (in[u] && !((dw[u] >> bit[u]) & 1u)) ? __ldg(a.contrib + id[u]) : 0.0;
#pragma unroll
		for (int u = 0; u < kMapPerThread; u++) vals[u * kMapThreads + tid] = x[u];
	}
	__syncthreads();

	// phase 2: per-entry sums (short entries by one thread, in slot order)
	for (uint32_t e = eb + tid; e < ee; e += kMapThreads) {
		const uint32_t start = __ldg(a.sp.pos + e), end = __ldg(a.sp.pos + e + 1);
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
	for (uint32_t q = wid; q < sh_nlong; q += kMapThreads / 32) {
		const uint32_t e = longs[q];
		const uint32_t start = __ldg(a.sp.pos + e), end = __ldg(a.sp.pos + e + 1);
		const uint32_t s0 = max(start, ra), s1 = min(end, rb);
		double s = 0.0;
		for (uint32_t k = s0 + lane; k < s1; k += 32) s += vals[k - ra];
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if (lane == 0) pr_emit(a, r, ra, rb, e, start, end, s);
	}
}

// Vertices straddling block boundaries: the thread of boundary q handles the
// vertex that starts in block q-1 and crosses q*kMapRange.
__global__ void pr_fixup(PrArgs a) {
	const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1;
	if (q >= a.sp.nranges) return;
	const uint32_t s = (uint32_t)q * kMapRange;
	// last entry e with pos[e] <= s (pos[0] = 0 <= s)
	uint32_t lo = 0, hi = (uint32_t)a.sp.g.V;
	while (lo < hi) {
		const uint32_t mid = (lo + hi + 1) >> 1;
		if (__ldg(a.sp.pos + mid) <= s) lo = mid; else hi = mid - 1;
	}
	const uint32_t e = lo;
	if (e >= a.sp.g.V) return;
	const uint32_t start = __ldg(a.sp.pos + e), end = __ldg(a.sp.pos + e + 1);
	if (!(start < s && start >= s - kMapRange && end > s)) return;
	const uint32_t r2 = (end - 1) / kMapRange;
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

static lg_status check_args(lg_snapshot* sn, int iterations, double damping, double* ranks) {
	if (!sn || !ranks) return set_error(LG_EINVAL, "null argument");
	if (!(damping > 0.0 && damping < 1.0))
		return set_error(LG_EINVAL, "damping must be in (0, 1)");
	if (iterations < 0) return set_error(LG_EINVAL, "iterations must be >= 0");
	if (!sn->in.present)
		return set_error(LG_ESTATE, "pull PageRank needs the in-CSR (reverse edges)");
	return LG_OK;
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_pagerank_pull(lg_snapshot* sn, int iterations,
		double damping, double* ranks) {
	clear_error();
	LG_TRY(check_args(sn, iterations, damping, ranks));
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	if (V == 0) return LG_OK;
	const double N = (double)V;
	const double pr0 = 1.0 / N;
	const double base = (1.0 - damping) / N;
	const unsigned B = 256;
	DevBuf* sc = s->scratch;
	const uint32_t* outdeg = sn->out.deg.as<uint32_t>();

	// flat in-adjacency: the snapshot's own (lg_snapshot_flatten) or one
	// built for this call in store scratch
	FlatCsr* f = sn->flat[1];
	if (!f) {
		if (!s->flat_scratch) s->flat_scratch = new FlatCsr;
		LG_TRY(build_flat(sn, 1, *s->flat_scratch, false));
		f = s->flat_scratch;
	}
	if (!f->has_nz_outdeg) {
		LG_TRY(f->nz_outdeg.reserve(f->rcap() * sizeof(uint32_t)));
		if (f->R > 0) {
			pr_row_degrees<<<grid_for(f->R, B), B, 0, st>>>(f->nz_rows(), (uint32_t)f->R, outdeg,
					f->nz_outdeg.as<uint32_t>());
			LG_CUDA(cudaGetLastError(), "pr_row_degrees");
			s->launches++;
		}
		f->has_nz_outdeg = true;
	}
	const uint32_t ntiles = f->ntiles;
	const uint32_t* flat_off = f->off.as<uint32_t>();

	LG_TRY(sc[0].reserve(V * sizeof(double)));
	LG_TRY(sc[1].reserve(V * sizeof(double)));
	LG_TRY(sc[2].reserve(2ull * std::max<uint32_t>(ntiles, 1) * sizeof(double)));
	const FlatTiles a = flat_tiles(*f, sc[2].as<double>());
	PrOp op;
	op.nz_rows = f->nz_rows();
	op.nz_outdeg = f->nz_outdeg.as<uint32_t>();
	op.base = base;
	op.d = damping;
	const bool dev_out = is_device_pointer(ranks);
	double* pr_buf = ranks;
	if (!dev_out) {
		LG_TRY(sc[4].reserve(V * sizeof(double)));
		pr_buf = sc[4].as<double>();
	}
	double* c0 = sc[0].as<double>();
	double* c1 = sc[1].as<double>();
	pr_init<<<grid_for(V, B), B, 0, st>>>(outdeg, V, pr0, c0, iterations == 0 ? pr_buf : nullptr);
	pr_empty_rows<<<grid_for(V, B), B, 0, st>>>(flat_off, outdeg, V, base, c1, nullptr);
	LG_CUDA(cudaGetLastError(), "pr_init");
	s->launches += 2;
	const unsigned fix_blocks = flat_fixup_blocks(ntiles);   // a thread per tile boundary
	const int ctas = (int)tune_value(s->device, LG_TUNE_PR_CTAS_PER_SM);
	const bool occ8 = tune_value(s->device, LG_TUNE_PR_TILE_OCC) == 8;
	int sms = 148;
	if (ctas > 0) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
	for (int it = 0; it < iterations; it++) {
		op.contrib = (it & 1) ? c1 : c0;
		op.contrib_next = (it & 1) ? c0 : c1;
		op.pr_out = (it == iterations - 1) ? pr_buf : nullptr;
		if (ntiles > 0) {
			launch_flat_sweep(a, op, sms, ctas, st, occ8 ? pr_flat_step_occ8 : pr_flat_step,
					pr_flat_loop<4>, pr_flat_loop<6>, pr_flat_loop<8>);
			s->launches++;
		}
		if (ntiles > 1) {
			pr_flat_fixup<<<fix_blocks, kFixupThreads, 0, st>>>(a, op);
			s->launches++;
		}
		if (it == 0 && iterations > 1) {
			// c0 still holds pr0 / out_degree for vertices without in-edges
			pr_empty_rows<<<grid_for(V, B), B, 0, st>>>(flat_off, outdeg, V, base, c0, nullptr);
			s->launches++;
		}
	}
	if (iterations > 0) {
		pr_empty_rows<<<grid_for(V, B), B, 0, st>>>(flat_off, outdeg, V, base, nullptr, pr_buf);
		s->launches++;
	}
	LG_CUDA(cudaGetLastError(), "pr_flat_step");
	if (!dev_out) {
		LG_TRY(copy_out(s, ranks, pr_buf, V * sizeof(double)));
		LG_CUDA(cudaStreamSynchronize(st), "pagerank");
	}
	return LG_OK;
}

// ---------------------------------------------------------------------------
// The gather floor: pr_flat_step's loads without its sums.
// ---------------------------------------------------------------------------

namespace lg {

// Lane j of the warp owning tile t loads the ids of edges e0 + 8j .. + 7
// (one 32-byte load, evict-first, as pr_flat_step) and gathers x at them;
// the warp's total goes to out[t].
__global__ void __launch_bounds__(kFlatWarps * 32)
pr_gather_floor(const uint32_t* ids, uint32_t E, uint32_t ntiles, const double* x,
		double* out) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t t = blockIdx.x * kFlatWarps + (threadIdx.x >> 5);
	if (t >= ntiles) return;
	const uint32_t eb = t * kFlatTile + lane * kFlatPerLane;
	uint32_t id[kFlatPerLane];
	if (eb + kFlatPerLane <= E) {
		asm("ld.global.cs.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
			: "=r"(id[0]), "=r"(id[1]), "=r"(id[2]), "=r"(id[3]),
			  "=r"(id[4]), "=r"(id[5]), "=r"(id[6]), "=r"(id[7])
			: "l"(ids + eb));
	} else {
#pragma unroll
		for (int i = 0; i < kFlatPerLane; i++) id[i] = eb + i < E ? __ldcs(ids + eb + i) : kNoId;
	}
	double v[kFlatPerLane];
#pragma unroll
	for (int i = 0; i < kFlatPerLane; i++) v[i] = id[i] != kNoId ? __ldg(x + id[i]) : 0.0;
	double s = 0.0;
#pragma unroll
	for (int i = 0; i < kFlatPerLane; i++) s += v[i];
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	if (lane == 0) out[t] = s;
}

__global__ void sum_doubles(const double* a, uint32_t n, double* out) {
	double s = 0.0;
	for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) s += a[i];
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	__shared__ double w[32];
	if ((threadIdx.x & 31u) == 0) w[threadIdx.x >> 5] = s;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (uint32_t i = 0; i < blockDim.x / 32; i++) t += w[i];
		*out = t;
	}
}

} // namespace lg

extern "C" lg_status lg_pagerank_gather_pass(lg_snapshot* sn, int passes, double* checksum) {
	clear_error();
	if (!sn) return set_error(LG_EINVAL, "null snapshot");
	if (passes < 1) return set_error(LG_EINVAL, "passes must be positive");
	FlatCsr* f = sn->flat[1];
	if (!f) return set_error(LG_ESTATE, "flatten the in-CSR first (lg_snapshot_flatten)");
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	DevBuf* sc = s->scratch;
	LG_TRY(sc[0].reserve(V * sizeof(double)));
	LG_TRY(sc[2].reserve((std::max<uint32_t>(f->ntiles, 1) + 1) * sizeof(double)));
	double* x = sc[0].as<double>();
	double* part = sc[2].as<double>();
	pr_init<<<grid_for(V, 256), 256, 0, st>>>(sn->out.deg.as<uint32_t>(), V, 1.0 / (double)V, x,
			nullptr);
	s->launches++;
	if (f->ntiles > 0) {
		for (int p = 0; p < passes; p++)
			pr_gather_floor<<<flat_sweep_blocks(f->ntiles), kFlatWarps * 32, 0, st>>>(
					f->ids.as<uint32_t>(), (uint32_t)f->E, f->ntiles, x, part);
		s->launches += passes;
	}
	LG_CUDA(cudaGetLastError(), "pr_gather_floor");
	if (checksum) {
		if (f->ntiles > 0) {
			sum_doubles<<<1, 1024, 0, st>>>(part, f->ntiles, part + f->ntiles);
			s->launches++;
		} else {
			LG_CUDA(cudaMemsetAsync(part, 0, sizeof(double), st), "memset");
		}
		LG_CUDA(cudaGetLastError(), "sum");
		LG_CUDA(cudaMemcpyAsync(checksum, part + (f->ntiles > 0 ? f->ntiles : 0), sizeof(double),
				cudaMemcpyDeviceToHost, st), "d2h");
		LG_CUDA(cudaStreamSynchronize(st), "gather pass");
		s->d2h_bytes += sizeof(double);
	}
	return LG_OK;
}

// ---------------------------------------------------------------------------
// PageRank without device allocation.
//
// lg_pagerank_pull keeps its per-iteration vectors in store-owned scratch
// that it grows with cudaMalloc.  Some callers cannot have the library
// allocate: a process whose device memory is already handed out to another
// allocator (a framework's caching allocator, a pool sized to the GPU),
// where a new cudaMalloc can fail or stall on a device-wide
// synchronisation, or serving code that allows no allocation after start-up.
// For them this variant runs the fragment-walking kernels on a fixed scratch
// area that is part of the library image: LG_NOALLOC_SCRATCH_BYTES of device
// memory, reserved on every GPU that loads the library, until the process
// exits.
// ---------------------------------------------------------------------------

namespace lg {

static __device__ __align__(256) unsigned char g_noalloc_scratch[LG_NOALLOC_SCRATCH_BYTES];

} // namespace lg

extern "C" lg_status lg_pagerank_pull_noalloc(lg_snapshot* sn, int iterations,
		double damping, double* ranks) {
	clear_error();
	LG_TRY(check_args(sn, iterations, damping, ranks));
	lg_store* s = sn->store;
	const uint64_t V = sn->V;
	const SlotSpace sp = slot_space(sn, 1);
	const uint64_t nranges = sp.nranges;
	// contrib (two vectors), the result staged for host outputs, carries
	const uint64_t need = 3 * V * sizeof(double) + 2 * nranges * sizeof(double);
	if (need > LG_NOALLOC_SCRATCH_BYTES)
		return set_error(LG_EINVAL, "graph needs %llu scratch bytes, more than the %llu "
				"this entry point has (24 B per vertex + 16 B per %u in-CSR slots)",
				(unsigned long long)need, (unsigned long long)LG_NOALLOC_SCRATCH_BYTES,
				kMapRange);
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
	a.sp = sp;
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
		pr_pull_step<<<nranges, kMapThreads, 0, st>>>(a);
		if (nranges > 1) pr_fixup<<<grid_for(nranges, 256), 256, 0, st>>>(a);
	}
	LG_CUDA(cudaGetLastError(), "pagerank noalloc");
	s->launches += 1 + (uint64_t)iterations * (nranges > 1 ? 2 : 1);
	if (!dev_out) {
		LG_CUDA(cudaMemcpyAsync(ranks, pr_buf, V * sizeof(double), cudaMemcpyDeviceToHost, st),
				"copy result");
		s->d2h_bytes += V * sizeof(double);
		LG_CUDA(cudaStreamSynchronize(st), "pagerank noalloc");
	}
	return LG_OK;
}
