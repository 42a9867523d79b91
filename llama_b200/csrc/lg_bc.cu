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
// lg_bc (plain): one source per pass, on the traversal the batched kernel
// uses: the forward sweep is level-synchronous and direction-optimising
// (the same frontier heuristic as lg_bc_batched): a top-down step walks the
// frontier's out-edges in balanced ranges, claims unreached targets and
// adds sigma[v] into sigma[w] along every down edge; a bottom-up step lets
// every unreached vertex sum sigma over its in-neighbours of the current
// level in the flat in-CSR (all of them, so no early exit).  One host read
// per level (the next frontier's size and out-degree sum) drives the loop;
// ranges are sized on the device.  The backward sweep walks each level's
// out-edges, deepest level first.
//
// lg_bc_batched (lg_msbfs.cu) runs 64 sources per pass on bit masks.
#include "lg_expand.cuh"
#include "lg_flat.cuh"

#include <vector>

namespace lg {

constexpr int32_t kBcUnreached = LG_UNREACHED;
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
// Plain: one source per pass
// ---------------------------------------------------------------------------

constexpr uint32_t kBcHeavy = 512;     // in-degree above which a warp serves a vertex
constexpr uint32_t kBcMaxRange = 1024; // largest slot range per warp

// Slots per warp range over `total` slots and `nwarps` warps: the even share
// rounded up to 32, between 32 and kBcMaxRange.
__device__ __forceinline__ uint32_t bc_range(uint32_t total, uint32_t nwarps) {
	uint32_t r = (uint32_t)(((uint64_t)total + nwarps - 1) / nwarps);
	r = (r + 31u) & ~31u;
	return min(max(r, 32u), kBcMaxRange);
}

// queue / ctr bookkeeping: ctr[0] = vertices pushed, ctr[1] = their
// out-degree sum (the direction heuristic's frontier edges)
__device__ __forceinline__ void bc_push_deg(bool take, uint32_t item, uint32_t* list,
		unsigned long long* ctr, const uint32_t* outdeg) {
	bc_push(take, item, list, ctr);
	unsigned long long d = take ? (unsigned long long)__ldg(outdeg + item) : 0ull;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
	if ((threadIdx.x & 31u) == 0 && d) atomicAdd(ctr + 1, d);
}

__global__ void bc_source_init(int32_t* level, double* sigma, double* delta,
		uint64_t V, uint32_t s, uint32_t* order, unsigned long long* ctr,
		const uint32_t* outdeg) {
	const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (v < V) {
		level[v] = (v == s) ? 0 : kBcUnreached;
		sigma[v] = (v == s) ? 1.0 : 0.0;
		delta[v] = 0.0;
	}
	if (v == 0) {
		order[0] = s;
		ctr[0] = 1;
		ctr[1] = __ldg(outdeg + s);
	}
}

// Top-down step from the level-k queue over its out-edges (warp ranges of
// the queue's slot space, sized on the device from pos[n]): an unreached w
// is claimed for level k + 1 and queued; every down edge v -> w adds
// sigma[v] into sigma[w].
__global__ void __launch_bounds__(kBcThreads)
bc_top_down(SnapCsr out, const uint32_t* fr, const uint32_t* pos, uint32_t n,
		int32_t* level, double* sigma, int32_t k, uint32_t* next,
		unsigned long long* ctr, const uint32_t* outdeg) {
	const uint32_t total = __ldg(pos + n);
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	const uint32_t range = bc_range(total, nwarps);
	const uint32_t nranges = (total + range - 1) / range;
	for (uint32_t r = warp; r < nranges; r += nwarps)
		range_for_each(out, fr, pos, n, total, nranges, range, r,
			[&](bool act, uint32_t, uint32_t v, uint32_t w, uint32_t, uint32_t) {
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
				bc_push_deg(won, w, next, ctr, outdeg);
			});
}

// Bottom-up step over the flat in-CSR: every unreached vertex w with at
// most kBcHeavy in-edges sums sigma over its in-neighbours at level k (all
// of them: sigma needs every parent); a non-zero sum puts w at level k + 1.
// Only w's own thread writes w, so no atomics are needed on sigma.
__global__ void __launch_bounds__(kBcThreads)
bc_bottom_up(const uint32_t* off, const uint32_t* ids, uint32_t V, int32_t* level,
		double* sigma, int32_t k, uint32_t* next, unsigned long long* ctr,
		const uint32_t* outdeg) {
	const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
	bool take = false;
	if (w < V && __ldcg(level + w) == kBcUnreached) {
		const uint32_t b = __ldg(off + w), e = __ldg(off + w + 1);
		if (e - b <= kBcHeavy) {
			double s = 0.0;
			for (uint32_t q = b; q < e; q++) {
				const uint32_t v = __ldg(ids + q);
				if (__ldcg(level + v) == k) s += __ldcg(sigma + v);
			}
			if (s != 0.0) {
				sigma[w] = s;
				level[w] = k + 1;
				take = true;
			}
		}
	}
	bc_push_deg(take, w, next, ctr, outdeg);
}

// The same for the vertices with more than kBcHeavy in-edges (hlist): a
// warp per vertex, lanes striding the in-list, sums joined by a fixed tree.
__global__ void __launch_bounds__(kBcThreads)
bc_bottom_up_heavy(const uint32_t* off, const uint32_t* ids, const uint32_t* hlist,
		const unsigned long long* hcount, int32_t* level, double* sigma, int32_t k,
		uint32_t* next, unsigned long long* ctr, const uint32_t* outdeg) {
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t nh = (uint32_t)*hcount;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nh; i += nwarps) {
		const uint32_t w = __ldg(hlist + i);
		if (__ldcg(level + w) != kBcUnreached) continue;   // uniform across the warp
		const uint32_t b = __ldg(off + w), e = __ldg(off + w + 1);
		double s = 0.0;
		for (uint32_t q = b + lane; q < e; q += 32) {
			const uint32_t v = __ldg(ids + q);
			if (__ldcg(level + v) == k) s += __ldcg(sigma + v);
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		const bool take = lane == 0 && s != 0.0;
		if (take) { sigma[w] = s; level[w] = k + 1; }
		bc_push_deg(take, w, next, ctr, outdeg);
	}
}

__global__ void bc_heavy_list(const uint32_t* off, uint32_t V, uint32_t* list,
		unsigned long long* count) {
	const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
	const bool h = v < V && __ldg(off + v + 1) - __ldg(off + v) > kBcHeavy;
	bc_push(h, v, list, count);
}

// Backward step for the level-k queue: delta[v] = sum over down edges v->w
// of sigma[v] / sigma[w] * (1 + delta[w]), summed per v across the warp.
__global__ void __launch_bounds__(kBcThreads)
bc_backward(SnapCsr out, const uint32_t* fr, const uint32_t* pos, uint32_t n,
		const int32_t* level, const double* sigma, double* delta, int32_t k) {
	const uint32_t total = __ldg(pos + n);
	const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
	const uint32_t range = bc_range(total, nwarps);
	const uint32_t nranges = (total + range - 1) / range;
	for (uint32_t r = warp; r < nranges; r += nwarps)
		range_for_each(out, fr, pos, n, total, nranges, range, r,
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
	DevBuf level, sigma, delta, order, cnt, pos, scan_tmp, ctrb, bcb, heavy;
	LG_TRY(level.reserve(V * 4));
	LG_TRY(sigma.reserve(V * 8));
	LG_TRY(delta.reserve(V * 8));
	LG_TRY(order.reserve(V * 4));
	LG_TRY(cnt.reserve(V * 4));
	LG_TRY(pos.reserve((V + 1) * 4));
	LG_TRY(ctrb.reserve(2 * sizeof(unsigned long long)));
	const bool dev_out = is_device_pointer(bc);
	double* acc = bc;
	if (!dev_out) { LG_TRY(bcb.reserve(V * 8)); acc = bcb.as<double>(); }
	LG_CUDA(cudaMemsetAsync(acc, 0, V * 8, st), "memset");
	const FlatCsr* fo = sn->flat[0];
	const SnapCsr out = (fo && fo->has_view) ? fo->view(sn->out.deg.as<uint32_t>()) : sn->view(0);
	const uint32_t* outdeg = sn->out.deg.as<uint32_t>();
	// the bottom-up steps read in-edges: the snapshot's flat in-CSR, or one
	// built for the call
	const FlatCsr* fi = sn->flat[1];
	if (!fi && sn->in.present && n_sources > 0) {
		if (!s->flat_scratch) s->flat_scratch = new FlatCsr;
		LG_TRY(build_flat(sn, 1, *s->flat_scratch, false));
		fi = s->flat_scratch;
	}
	uint32_t* hlist = nullptr;
	unsigned long long* hcount = nullptr;
	if (fi) {
		LG_TRY(heavy.reserve(sizeof(unsigned long long) + std::max<uint64_t>(V, 1) * 4));
		hcount = heavy.as<unsigned long long>();
		hlist = reinterpret_cast<uint32_t*>(hcount + 1);
		LG_CUDA(cudaMemsetAsync(hcount, 0, sizeof(unsigned long long), st), "memset");
		bc_heavy_list<<<grid_for(V, 256), 256, 0, st>>>(fi->off.as<uint32_t>(), (uint32_t)V,
				hlist, hcount);
		s->launches++;
	}
	// the store's pinned words for the per-level counters
	unsigned long long* hc = nullptr;
	LG_TRY(host_words(s, &hc));
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
	const unsigned grid = (unsigned)sms * 8u;
	const double alpha = 14.0, beta = 24.0;
	int32_t* lv = level.as<int32_t>();
	double* sg = sigma.as<double>();
	double* dl = delta.as<double>();
	uint32_t* ord = order.as<uint32_t>();
	unsigned long long* ctr = ctrb.as<unsigned long long>();
	std::vector<uint64_t> off;
	for (int i = 0; i < n_sources; i++) {
		const uint32_t src = (uint32_t)sources[i];
		bc_source_init<<<grid_for(V, 256), 256, 0, st>>>(lv, sg, dl, V, src, ord, ctr, outdeg);
		LG_CUDA(cudaMemcpyAsync(hc, ctr, 2 * sizeof(unsigned long long),
				cudaMemcpyDeviceToHost, st), "d2h");
		LG_CUDA(cudaStreamSynchronize(st), "bc");
		s->launches++;
		off.assign({0, 1});
		uint64_t mf = hc[1];
		uint64_t mu = sn->out.n_edges > mf ? sn->out.n_edges - mf : 0;
		bool top_down = true;
		for (int32_t k = 0;; k++) {
			const uint64_t b = off[k], n = off[k + 1] - off[k];
			if (n == 0) break;
			if (top_down && fi && (double)mf > (double)mu / alpha) top_down = false;
			else if (!top_down && (double)n < (double)V / beta) top_down = true;
			LG_CUDA(cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long), st), "memset");
			uint32_t* nxt = ord + off[k + 1];
			if (top_down) {
				list_slots<<<grid_for(n, 256), 256, 0, st>>>(out, ord + b, (uint32_t)n,
						cnt.as<uint32_t>());
				LG_TRY(exclusive_scan_u32(cnt.as<uint32_t>(), pos.as<uint32_t>(), n, scan_tmp,
						st, nullptr));
				bc_top_down<<<grid, kBcThreads, 0, st>>>(out, ord + b, pos.as<uint32_t>(),
						(uint32_t)n, lv, sg, k, nxt, ctr, outdeg);
				s->launches += 5;
			} else {
				bc_bottom_up<<<grid_for(V, kBcThreads), kBcThreads, 0, st>>>(
						fi->off.as<uint32_t>(), fi->ids.as<uint32_t>(), (uint32_t)V, lv, sg, k,
						nxt, ctr, outdeg);
				bc_bottom_up_heavy<<<grid, kBcThreads, 0, st>>>(fi->off.as<uint32_t>(),
						fi->ids.as<uint32_t>(), hlist, hcount, lv, sg, k, nxt, ctr, outdeg);
				s->launches += 2;
			}
			LG_CUDA(cudaGetLastError(), "bc forward");
			LG_CUDA(cudaMemcpyAsync(hc, ctr, 2 * sizeof(unsigned long long),
					cudaMemcpyDeviceToHost, st), "d2h");
			LG_CUDA(cudaStreamSynchronize(st), "bc");
			s->d2h_bytes += 2 * sizeof(unsigned long long);
			off.push_back(off[k + 1] + hc[0]);
			mf = hc[1];
			mu -= std::min(mu, mf);
		}
		// backward: levels D-2 .. 1 (the deepest level has no down edges,
		// level 0 is the source)
		const int D = (int)off.size() - 2;           // levels 0..D-1 are non-empty
		for (int k = D - 2; k >= 1; k--) {
			const uint64_t b = off[k], n = off[k + 1] - off[k];
			list_slots<<<grid_for(n, 256), 256, 0, st>>>(out, ord + b, (uint32_t)n,
					cnt.as<uint32_t>());
			LG_TRY(exclusive_scan_u32(cnt.as<uint32_t>(), pos.as<uint32_t>(), n, scan_tmp, st,
					nullptr));
			bc_backward<<<grid, kBcThreads, 0, st>>>(out, ord + b, pos.as<uint32_t>(),
					(uint32_t)n, lv, sg, dl, k);
			bc_accumulate<<<grid_for(n, 256), 256, 0, st>>>(ord + b, (uint32_t)n, dl, acc);
			s->launches += 6;
			LG_CUDA(cudaGetLastError(), "bc_backward");
		}
	}
	if (!dev_out) LG_TRY(copy_out(s, bc, acc, V * 8));
	LG_CUDA(cudaStreamSynchronize(st), "bc");
	return LG_OK;
}
