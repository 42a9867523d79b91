// lg_tc.cu - triangle counting on the symmetrised snapshot.
//
// Reference: ll_b_triangle_counting_LU (benchmark/benchmarks/
// triangle_counting.h:343-470), run on a graph loaded with -U (both arcs of
// every edge) and flattened to one level: it counts triangles u < v < w with
// all three undirected edges present, each once.  The reference requires a
// single level with sorted adjacency (triangle_counting.h:422-425); here the
// multiversion snapshot is flattened on the device:
//   1. every live arc u->v (u != v) becomes the undirected edge oriented from
//      the lower to the higher rank, rank = (out+in degree, id), a total order
//      that keeps the forward lists of hubs short;
//   2. the keys (a << 32 | b) are radix sorted and de-duplicated, giving the
//      forward lists N+(a) sorted by id;
//   3. every oriented edge (a, b) counts |N+(a) & N+(b)|: each triangle is
//      seen exactly once, at the edge between its two lowest-ranked vertices.
//      Short lists are intersected by one lane, long ones by the warp, both
//      with a binary search per element of the shorter list (merging 32
//      chunks of similar-length lists was measured slower at R-MAT scale 24:
//      890 ms against 552 ms for the whole call).
// The count is an exact integer sum (atomicAdd of per-warp partials).
#include "lg_expand.cuh"
#include "lg_sort.cuh"

namespace lg {

constexpr int kTcThreads = 256;

__device__ __forceinline__ bool rank_less(uint32_t x, uint32_t y, const uint32_t* rk) {
	uint32_t dx = __ldg(rk + x), dy = __ldg(rk + y);
	return dx < dy || (dx == dy && x < y);
}

__global__ void tc_rank(const uint32_t* out_deg, const uint32_t* in_deg, uint64_t V,
		uint32_t* rk) {
	uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v < V) rk[v] = out_deg[v] + (in_deg ? in_deg[v] : 0u);
}

// Every live arc of the out-CSR, over balanced 1024-slot ranges of all
// vertices' slots (pos = the snapshot's slot prefix), becomes an oriented key;
// each warp stages its keys in shared memory and appends kTcStage at a time
// (one counter atomic per batch, not per 32 slots).
constexpr uint32_t kTcRange = 1024;
constexpr uint32_t kTcStage = 256;
__global__ void __launch_bounds__(kTcThreads)
tc_emit(SnapCsr out, const uint32_t* pos, uint32_t total, const uint32_t* rk,
		unsigned long long* keys, unsigned long long* n_keys) {
	__shared__ unsigned long long stage[kTcThreads / 32][kTcStage];
	unsigned long long* sb = stage[threadIdx.x >> 5];
	uint32_t ns = 0;                       // staged keys of this warp (warp-uniform)
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t nranges = (total + kTcRange - 1) / kTcRange;
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	for (uint32_t r = warp; r < nranges; r += nwarps)
	range_for_each(out, nullptr, pos, (uint32_t)out.V, total, nranges, kTcRange, r,
		[&](bool act, uint32_t, uint32_t src, uint32_t nbr, uint32_t, uint32_t) {
			const bool take = act && nbr != src;
			unsigned long long key = 0;
			if (take) {
				uint32_t a = src, b = nbr;
				if (rank_less(b, a, rk)) { a = nbr; b = src; }
				key = ((unsigned long long)a << 32) | b;
			}
			const unsigned m = __ballot_sync(0xffffffffu, take);
			if (m) {
				if (ns + (uint32_t)__popc(m) > kTcStage) {
					__syncwarp();
					unsigned long long base = 0;
					if (lane == 0) base = atomicAdd(n_keys, (unsigned long long)ns);
					base = __shfl_sync(0xffffffffu, base, 0);
					for (uint32_t i = lane; i < ns; i += 32) keys[base + i] = sb[i];
					__syncwarp();
					ns = 0;
				}
				if (take) sb[ns + __popc(m & ((1u << lane) - 1u))] = key;
				ns += __popc(m);
			}
		});
	if (ns) {
		__syncwarp();
		unsigned long long base = 0;
		if (lane == 0) base = atomicAdd(n_keys, (unsigned long long)ns);
		base = __shfl_sync(0xffffffffu, base, 0);
		for (uint32_t i = lane; i < ns; i += 32) keys[base + i] = sb[i];
	}
}

// off[v] = first oriented edge whose source is >= v
__global__ void tc_offsets(const unsigned long long* keys, uint64_t m, uint64_t V,
		uint32_t* off) {
	uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i > m) return;
	uint64_t a = i < m ? (keys[i] >> 32) : V;
	int64_t p = i > 0 ? (int64_t)(keys[i - 1] >> 32) : -1;
	for (int64_t v = p + 1; v <= (int64_t)a && v <= (int64_t)V; v++) off[v] = (uint32_t)i;
}

// adj[i] = target of oriented edge i (the low half of its key): the
// forward lists as 4-byte ids, half the bytes of the keys.
__global__ void tc_targets(const unsigned long long* keys, uint64_t m, uint32_t* adj) {
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
			i += (uint64_t)gridDim.x * blockDim.x)
		adj[i] = (uint32_t)keys[i];
}

__device__ __forceinline__ bool bsearch_u32(const uint32_t* base, uint32_t n, uint32_t x) {
	uint32_t lo = 0, hi = n;
	while (lo < hi) {
		uint32_t mid = (lo + hi) >> 1;
		uint32_t y = __ldg(base + mid);
		if (y < x) lo = mid + 1; else hi = mid;
	}
	return lo < n && __ldg(base + lo) == x;
}

constexpr uint32_t kTcSmall = 16;   // lists this short are intersected by one lane

__global__ void __launch_bounds__(kTcThreads)
tc_count(const unsigned long long* keys, const uint32_t* adj, uint64_t m, const uint32_t* off,
		unsigned long long* total) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t warp = (uint64_t)blockIdx.x * (kTcThreads / 32) + (threadIdx.x >> 5);
	const uint64_t nwarps = (uint64_t)gridDim.x * (kTcThreads / 32);
	unsigned long long c = 0;
	for (uint64_t e0 = warp * 32; e0 < m; e0 += nwarps * 32) {
		const uint64_t e = e0 + lane;
		uint32_t sa = 0, la = 0, sb = 0, lb = 0;
		if (e < m) {
			const unsigned long long k = keys[e];
			const uint32_t a = (uint32_t)(k >> 32), b = (uint32_t)k;
			sa = __ldg(off + a); la = __ldg(off + a + 1) - sa;
			sb = __ldg(off + b); lb = __ldg(off + b + 1) - sb;
			if (la > lb) { uint32_t t = sa; sa = sb; sb = t; t = la; la = lb; lb = t; }
		}
		// (sa, la) is now the shorter list
		const bool small = la <= kTcSmall;
		if (e < m && small)
			for (uint32_t j = 0; j < la; j++)
				c += bsearch_u32(adj + sb, lb, __ldg(adj + sa + j));
		unsigned big = __ballot_sync(0xffffffffu, e < m && !small);
		while (big) {
			const int src = __ffs(big) - 1;
			big &= big - 1;
			const uint32_t s0 = __shfl_sync(0xffffffffu, sa, src);
			const uint32_t n0 = __shfl_sync(0xffffffffu, la, src);
			const uint32_t s1 = __shfl_sync(0xffffffffu, sb, src);
			const uint32_t n1 = __shfl_sync(0xffffffffu, lb, src);
			for (uint32_t j = lane; j < n0; j += 32)
				c += bsearch_u32(adj + s1, n1, __ldg(adj + s0 + j));
		}
	}
	for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
	if (lane == 0 && c) atomicAdd(total, c);
}

} // namespace lg

using namespace lg;

extern "C" lg_status lg_triangle_count(lg_snapshot* sn, lg_tc_result* result) {
	clear_error();
	if (!sn || !result) return set_error(LG_EINVAL, "null argument");
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	const uint64_t E = sn->out.n_edges;
	if (E >= 0xffffffffull) return set_error(LG_ENOTSUP, "more than 2^32-1 live edges");
	DevBuf rank, keys, tmpk, tmpp, counts, scan_tmp, uniq, flags, off, ctr, adj;
	LG_TRY(rank.reserve(V * 4));
	LG_TRY(keys.reserve(std::max<uint64_t>(E, 1) * 8));
	LG_TRY(ctr.reserve(2 * sizeof(unsigned long long)));
	LG_CUDA(cudaMemsetAsync(ctr.p, 0, 2 * sizeof(unsigned long long), st), "memset");
	tc_rank<<<grid_for(V, 256), 256, 0, st>>>(sn->out.deg.as<uint32_t>(),
			sn->in.present ? sn->in.deg.as<uint32_t>() : nullptr, V, rank.as<uint32_t>());
	const SnapCsr out = sn->view(0);
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
	tc_emit<<<(unsigned)sms * 8u, kTcThreads, 0, st>>>(out, sn->out.slot_off.as<uint32_t>(),
			(uint32_t)sn->out.n_frag_slots, rank.as<uint32_t>(), keys.as<unsigned long long>(),
			ctr.as<unsigned long long>());
	LG_CUDA(cudaGetLastError(), "tc_emit");
	s->launches += 2;
	unsigned long long nk = 0;
	LG_CUDA(cudaMemcpyAsync(&nk, ctr.p, 8, cudaMemcpyDeviceToHost, st), "d2h");
	LG_CUDA(cudaStreamSynchronize(st), "tc emit");
	s->d2h_bytes += 8;
	unsigned long long* sorted = nullptr;
	LG_TRY(radix_sort_u64(s, keys.as<unsigned long long>(), nullptr, nk, tmpk, tmpp,
			counts, scan_tmp, &sorted, nullptr));
	LG_TRY(uniq.reserve(std::max<unsigned long long>(nk, 1) * 8));
	uint64_t m = 0;
	LG_TRY(unique_u64(s, sorted, nk, uniq.as<unsigned long long>(), flags, scan_tmp, &m));
	LG_TRY(off.reserve((V + 1) * 4));
	tc_offsets<<<grid_for(m + 1, 256), 256, 0, st>>>(uniq.as<unsigned long long>(), m, V,
			off.as<uint32_t>());
	LG_TRY(adj.reserve(std::max<uint64_t>(m, 1) * 4));
	tc_targets<<<(unsigned)sms * 8u, 256, 0, st>>>(uniq.as<unsigned long long>(), m,
			adj.as<uint32_t>());
	tc_count<<<(unsigned)sms * 16u, kTcThreads, 0, st>>>(uniq.as<unsigned long long>(),
			adj.as<uint32_t>(), m, off.as<uint32_t>(), ctr.as<unsigned long long>() + 1);
	LG_CUDA(cudaGetLastError(), "tc_count");
	s->launches += 3;
	unsigned long long t = 0;
	LG_CUDA(cudaMemcpyAsync(&t, ctr.as<unsigned long long>() + 1, 8, cudaMemcpyDeviceToHost, st), "d2h");
	LG_CUDA(cudaStreamSynchronize(st), "tc");
	s->d2h_bytes += 8;
	result->triangles = (int64_t)t;
	result->undirected_edges = m;
	result->arcs = nk;
	return LG_OK;
}
