// lg_bc.cu - Brandes betweenness centrality from explicit sources, FP64.
//
// Reference: ll_b_bc_random (benchmark/benchmarks/bc_random.h:55-193) over
// ll_bfs_template: per source s, sigma is pushed along down edges
// (level[w] == level[v] + 1, is_down_edge, ll_bfs_template.h:337-351) and
// the reverse sweep, deepest level first, sets
//   delta[v] = sum over down edges v->w of sigma[v] / sigma[w] * (1 + delta[w])
// and BC[v] += delta[v] for v != s (bc_random.h:73-111).  The reference
// accumulates in FP32 and picks sources with rand(); here sources are given
// and everything is FP64.  Sums go through FP64 atomics, so results agree
// with an exact evaluation to ~1e-15 relative, not bit for bit.
//
// lg_bc (plain): one source at a time.  The forward sweep is a top-down BFS
// over balanced frontier ranges that also adds sigma[v] into sigma[w] for
// every down edge; the backward sweep walks each level's out-edges.
//
// lg_bc_batched (lg_msbfs.cu) runs 64 sources per pass on bit masks.
#include "lg_device.cuh"
#include "lg_expand.cuh"

namespace lg {

constexpr int32_t kBcUnreached = LG_UNREACHED;
constexpr uint32_t kBcRange = 1024;
constexpr int kBcThreads = 256;

__device__ __forceinline__ void bc_push(bool take, uint32_t item, uint32_t* list,
		unsigned long long* len) {
	const unsigned m = __ballot_sync(0xffffffffu, take);
	if (!m) return;
	const uint32_t lane = threadIdx.x & 31u;
	const int leader = __ffs(m) - 1;
	unsigned long long base = 0;
	if ((int)lane == leader) base = atomicAdd(len, (unsigned long long)__popc(m));
	base = __shfl_sync(0xffffffffu, base, leader);
	if (take) list[base + __popc(m & ((1u << lane) - 1u))] = item;
}

// ---------------------------------------------------------------------------
// Plain: one source
// ---------------------------------------------------------------------------

__global__ void bc_source_init(int32_t* level, double* sigma, double* delta,
		uint64_t V, uint32_t s, uint32_t* order) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v < V) {
		level[v] = (v == s) ? 0 : kBcUnreached;
		sigma[v] = (v == s) ? 1.0 : 0.0;
		delta[v] = 0.0;
	}
	if (v == 0) order[0] = s;
}

__global__ void __launch_bounds__(kBcThreads)
bc_forward(SnapCsr out, const uint32_t* fr, const uint32_t* pos, uint32_t n,
		uint32_t total, uint32_t nranges, int32_t* level, double* sigma, int32_t k,
		uint32_t* next, unsigned long long* ctr) {
	const uint64_t r = (uint64_t)blockIdx.x * (kBcThreads / 32) + (threadIdx.x >> 5);
	if (r >= nranges) return;
	range_for_each(out, fr, pos, n, total, nranges, kBcRange, (uint32_t)r,
		[&](bool act, uint32_t own, uint32_t v, uint32_t w, uint32_t, uint32_t) {
			bool won = false, down = false;
			if (act) {
				int32_t lw = __ldcg(level + w);
				if (lw == kBcUnreached) {
					won = atomicCAS(level + w, kBcUnreached, k + 1) == kBcUnreached;
					lw = k + 1;   // set by us or by a concurrent parent
				}
				down = lw == k + 1;
			}
			if (down) atomicAdd(sigma + w, __ldcg(sigma + v));
			bc_push(won, w, next, ctr);
		});
}

__global__ void __launch_bounds__(kBcThreads)
bc_backward(SnapCsr out, const uint32_t* fr, const uint32_t* pos, uint32_t n,
		uint32_t total, uint32_t nranges, const int32_t* level, const double* sigma,
		double* delta, int32_t k) {
	const uint64_t r = (uint64_t)blockIdx.x * (kBcThreads / 32) + (threadIdx.x >> 5);
	if (r >= nranges) return;
	range_for_each(out, fr, pos, n, total, nranges, kBcRange, (uint32_t)r,
		[&](bool act, uint32_t own, uint32_t v, uint32_t w, uint32_t, uint32_t) {
			double c = 0.0;
			if (act && __ldcg(level + w) == k + 1)
				c = __ldcg(sigma + v) / __ldcg(sigma + w) * (1.0 + __ldcg(delta + w));
			bool tail;
			const double sum = warp_segsum(c, own, &tail);
			if (tail && sum != 0.0) atomicAdd(delta + v, sum);
		});
}

__global__ void bc_accumulate(const uint32_t* lvl, uint32_t n, const double* delta,
		double* bc) {
	const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) { const uint32_t v = lvl[i]; bc[v] += delta[v]; }
}

} // namespace lg

using namespace lg;

namespace {

lg_status list_offsets(lg_store* s, const SnapCsr& g, const uint32_t* list, uint32_t n,
		DevBuf& cnt, DevBuf& pos, DevBuf& scan_tmp, uint64_t* total) {
	list_slots<<<grid_for(n, 256), 256, 0, s->stream>>>(g, list, n, cnt.as<uint32_t>());
	s->launches += 4;
	s->d2h_bytes += 8;
	return exclusive_scan_u32(cnt.as<uint32_t>(), pos.as<uint32_t>(), n, scan_tmp,
			s->stream, total);
}

lg_status read_u64(lg_store* s, const unsigned long long* d, uint64_t* h) {
	unsigned long long x = 0;
	LG_CUDA(cudaMemcpyAsync(&x, d, 8, cudaMemcpyDeviceToHost, s->stream), "d2h");
	LG_CUDA(cudaStreamSynchronize(s->stream), "bc");
	s->d2h_bytes += 8;
	*h = x;
	return LG_OK;
}

lg_status check_sources(lg_snapshot* sn, const int64_t* sources, int n) {
	if (!sn || (!sources && n > 0)) return set_error(LG_EINVAL, "null argument");
	if (n < 0) return set_error(LG_EINVAL, "negative source count");
	for (int i = 0; i < n; i++)
		if (sources[i] < 0 || (uint64_t)sources[i] >= sn->V)
			return set_error(LG_EINVAL, "source %lld out of range", (long long)sources[i]);
	return LG_OK;
}

} // namespace

extern "C" lg_status lg_bc(lg_snapshot* sn, const int64_t* sources, int n_sources,
		double* bc) {
	clear_error();
	if (!bc) return set_error(LG_EINVAL, "null output");
	LG_TRY(check_sources(sn, sources, n_sources));
	lg_store* s = sn->store;
	LG_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
	cudaStream_t st = s->stream;
	const uint64_t V = sn->V;
	DevBuf level, sigma, delta, order, cnt, pos, scan_tmp, ctrb, bcb;
	LG_TRY(level.reserve(V * 4));
	LG_TRY(sigma.reserve(V * 8));
	LG_TRY(delta.reserve(V * 8));
	LG_TRY(order.reserve(V * 4));
	LG_TRY(cnt.reserve(V * 4));
	LG_TRY(pos.reserve((V + 1) * 4));
	LG_TRY(ctrb.reserve(8));
	const bool dev_out = is_device_pointer(bc);
	double* acc = bc;
	if (!dev_out) { LG_TRY(bcb.reserve(V * 8)); acc = bcb.as<double>(); }
	LG_CUDA(cudaMemsetAsync(acc, 0, V * 8, st), "memset");
	const SnapCsr out = sn->view(0);
	int32_t* lv = level.as<int32_t>();
	double* sg = sigma.as<double>();
	double* dl = delta.as<double>();
	uint32_t* ord = order.as<uint32_t>();
	unsigned long long* ctr = ctrb.as<unsigned long long>();
	std::vector<uint64_t> off;
	for (int i = 0; i < n_sources; i++) {
		const uint32_t src = (uint32_t)sources[i];
		bc_source_init<<<grid_for(V, 256), 256, 0, st>>>(lv, sg, dl, V, src, ord);
		s->launches++;
		off.assign({0, 1});
		for (int32_t k = 0;; k++) {
			const uint64_t b = off[k], n = off[k + 1] - off[k];
			if (n == 0) break;
			uint64_t total = 0;
			LG_TRY(list_offsets(s, out, ord + b, (uint32_t)n, cnt, pos, scan_tmp, &total));
			LG_CUDA(cudaMemsetAsync(ctr, 0, 8, st), "memset");
			const uint32_t nr = (uint32_t)((total + kBcRange - 1) / kBcRange);
			if (nr) {
				bc_forward<<<grid_for(nr, kBcThreads / 32), kBcThreads, 0, st>>>(out, ord + b,
						pos.as<uint32_t>(), (uint32_t)n, (uint32_t)total, nr, lv, sg, k,
						ord + off[k + 1], ctr);
				s->launches++;
			}
			LG_CUDA(cudaGetLastError(), "bc_forward");
			uint64_t produced = 0;
			LG_TRY(read_u64(s, ctr, &produced));
			off.push_back(off[k + 1] + produced);
		}
		// backward: levels D-1 .. 1 (the deepest level has no down edges)
		const int D = (int)off.size() - 2;           // levels 0..D-1 are non-empty
		for (int k = D - 2; k >= 1; k--) {
			const uint64_t b = off[k], n = off[k + 1] - off[k];
			uint64_t total = 0;
			LG_TRY(list_offsets(s, out, ord + b, (uint32_t)n, cnt, pos, scan_tmp, &total));
			const uint32_t nr = (uint32_t)((total + kBcRange - 1) / kBcRange);
			if (nr) {
				bc_backward<<<grid_for(nr, kBcThreads / 32), kBcThreads, 0, st>>>(out, ord + b,
						pos.as<uint32_t>(), (uint32_t)n, (uint32_t)total, nr, lv, sg, dl, k);
				s->launches++;
			}
			bc_accumulate<<<grid_for(n, 256), 256, 0, st>>>(ord + b, (uint32_t)n, dl, acc);
			s->launches++;
			LG_CUDA(cudaGetLastError(), "bc_backward");
		}
	}
	if (!dev_out) LG_TRY(copy_out(s, bc, acc, V * 8));
	LG_CUDA(cudaStreamSynchronize(st), "bc");
	return LG_OK;
}
